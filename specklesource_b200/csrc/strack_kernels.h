// strack_kernels.h -- launch interface between the C-ABI host code and the
// strack / strackw / cull kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "strack_common.cuh"

namespace sbk {

// The neighbourhood of a complex-match peak, handed from the complex kernel
// to the peak kernel (overSampleC and the gaussPeak1D samples,
// speckleTrack.c:648-709): |c|^2 of the fftshifted 2W x 2W surface around the
// coarse peak (iC, jC).  The oversampled peak lies within two samples of it,
// so the row and column strips hold every sample the two 1-D fits can read.
struct PeakJob {
    int32_t point;
    int32_t iC, jC;       // findCPeak's peak; -1000 when rejected; PJ_NODATA: getPatches failed
    int32_t pad;
    double p1, p2;        // patch powers (cMax normalisation)
    float blk[NFAST][NFAST];        // rows iC-4 .. iC+3, cols jC-4 .. jC+3
    float hs[4][NGAUSS + 3];        // rows iC-2 .. iC+1, cols jC-11 .. jC+9
    float vs[NGAUSS + 3][4];        // rows iC-11 .. iC+9, cols jC-2 .. jC+1
};
constexpr int32_t PJ_NODATA = -2000000;

// Arguments of the peak kernel (one warp per list position).
struct PeakArgs {
    const PeakJob* peak;
    int nList;
    int W;                 // complex window (the surface is 2W x 2W)
    double hanCorr;
    const float2* osD;     // real oversampling table (48 x 8 floats D, 16 phases)
    PointRec* rec;
    FitJob* fit;
};
cudaError_t launch_strack_peak(const PeakArgs& a, int numSM, cudaStream_t st);

// Arguments of the complex stage (one grid point per CTA iteration).
struct CmplxArgs {
    const void* img1;
    const void* img2;
    int nr1, na1, nr2, na2;
    int sampleType, byteOrder;
    const PointPlan* plan;
    const int* list;
    int nList;
    const float* hanning;  // W x W, or nullptr when -noHanning
    double hanCorr;        // 1.5 with Hanning, else 1.0
    const float2* twW;     // W_W^e forward twiddles, W entries
    const float2* tau;     // parity twiddles, W entries
    const float2* osA;     // 48 x 8 oversampling matrix
    const float2* osD;     // real form of it: 48 x 8 floats D, then 16 phases
    float azThresh;
    int checkAzFocus, noComplex;
    int baseOn;
    double Bn, Bp, dBn, dBp, dBnQ, dBpQ, lambda;
    const double* sinThetaD;
    const double* cosThetaD;
    const double* overRange;
    PointRec* rec;
    FitJob* fit;  // one entry per list position
    // interferogram phase correction (phaseCorrectInt); intf null: none
    const uint32_t* intf;  // na x nr (re, im) int16 pairs, one word each
    int intNr, intNa, intNrl, intNal, intMSB;
    int intPs, intPSA, intPSR;  // patch, padded sizes (ps * nal, ps * nrl)
    const float2* twP;          // exp(-2 pi i e / ps), e < ps
    int gauss;                  // -gauss: 2-D Gaussian fit instead of the oversampling
    PeakJob* peak;              // one entry per list position (unused with -gauss)
    // split-BF16 form only
    int* tcErr;                 // set when a bounded wait on the tensor cores gave up
    float* tcDebug;             // non-null: |c|^2 planes of list entry 0 (4 x 64 x 64)
};

// Arguments of an amplitude try (small: s = 1, large: s = LA = 2).
struct AmpArgs {
    const void* img1;
    const void* img2;
    int nr1, na1, nr2, na2;
    int sampleType, byteOrder;
    const PointPlan* plan;
    const int* list;
    int nList;              // list length, or its upper bound when nListDev is set
    const int* nListDev;    // non-null: the list length, read on the device
    int stage;   // 1 small, 2 large
    int s;       // window scale
    int wR, wA, wRa, wAa;
    int nR;      // grid columns (to rebuild i, j from the point index)
    int rStart, aStart, deltaR, deltaA;
    int noComplex;
    float azThresh;
    int checkAzFocus;
    const int* azEff;     // azShift in effect for each point (nullptr: use rec.azset)
    const float2* twWs;   // W_Ws table (Ws = wa*s)
    const float2* tw2Ws;  // W_{2Ws} table
    const float2* tau;    // parity twiddles for Ws
    const float2* osA;
    const float2* osD;    // real form of the oversampling matrix (shared-memory kernel)
    float2* scratch;      // per-CTA workspace
    size_t scratchPerCta; // float2 elements
    PointRec* rec;
    FitJob* fit;
    int gauss;            // -gauss: 2-D Gaussian fit instead of the oversampling
};

bool cmplx_supported(int W);
// thread counts compiled per window: the default and one alternative (0: none)
int cmplx_default_threads(int W);
int cmplx_alt_threads(int W);
// resident CTAs per SM at `threads` (0: the default count)
int cmplx_blocks_per_sm(int W, int threads = 0);
cudaError_t launch_strack_cmplx(int W, const CmplxArgs& a, int nCta, cudaStream_t st, int threads = 0);

// split-BF16 tensor-core form of the complex stage (strack_cmplx_tc.cu)
bool cmplx_tc_supported(int W);
int cmplx_tc_threads();  // threads per CTA of the tensor-core kernel
int cmplx_tc_blocks_per_sm();
cudaError_t launch_strack_cmplx_tc(const CmplxArgs& a, int nCta, cudaStream_t st);

bool amp_supported(int Ws);
size_t amp_scratch_elems(int Ws);
int amp_blocks_per_sm(int Ws);  // resident CTAs per SM of the staged amplitude kernel
int amp_threads(int Ws);
cudaError_t launch_strack_amp(int Ws, const AmpArgs& a, int nCta, cudaStream_t st);

// shared-memory-resident amplitude tries for small windows
bool amps_supported(int Ws);
int amps_blocks_per_sm(int Ws);
cudaError_t launch_strack_amps(int Ws, const AmpArgs& a, int nCta, cudaStream_t st);

}  // namespace sbk
