// capi.cu -- the library's C ABI (include/speckle_b200.h): contexts, device
// buffers, the host-side plan of the strack grid, and the stage sequence.
//
// The serial per-point loop of speckleTrack (Strack/speckleTrack.c:194-338)
// becomes:
//   host  : plan every grid point in raster order (findImage2Pos with its
//           carry-over of r2/a2, maskValue, boundsCheck for the three window
//           sizes) -- cheap scalar work that keeps the reference's sequential
//           semantics exactly;
//   device: complex stage over the points with a complex try, then the small
//           and the large amplitude tries over the points whose replayed
//           control flow reaches them, then one finalize pass.
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <algorithm>
#include <vector>

#include "../../include/speckle_b200.h"
#include "capi_internal.h"
#include "strack_device.cuh"
#include "strack_finalize.h"
#include "partition.h"
#include "strack_fit.h"
#include "strack_kernels.h"

using namespace sbk;

// ---------------------------------------------------------------- context

int sb_ctx_fail(sb_context* c, int code, const char* fmt, ...)
{
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        c->err = buf;
    }
    return code;
}

int sb_ctx_cuda(sb_context* c, cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return SB_OK;
    return sb_ctx_fail(c, SB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

void* sb_ctx_buf(sb_context* c, const char* name, size_t bytes, cudaError_t* err)
{
    DevBuf& b = c->bufs[name];
    if (b.bytes < bytes) {
        // stream-ordered: growing a buffer does not wait for the whole device
        // (cudaFree would), so contexts serving other jobs keep running
        if (b.ptr) cudaFreeAsync(b.ptr, c->stream);
        b.ptr = nullptr;
        b.bytes = 0;
        cudaError_t e = cudaMallocAsync(&b.ptr, bytes > 0 ? bytes : 16, c->stream);
        if (e != cudaSuccess) {
            *err = e;
            return nullptr;
        }
        b.bytes = bytes;
    }
    *err = cudaSuccess;
    return b.ptr;
}

extern "C" int sb_abi_version(void) { return SB_ABI_VERSION; }

extern "C" int sb_context_create(int device, sb_context** out)
{
    if (!out) return SB_ERR_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return SB_ERR_NODEVICE;
    if (device < 0 || device >= n) return SB_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return SB_ERR_NODEVICE;
    sb_context* c = new sb_context();
    c->device = device;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        delete c;
        return SB_ERR_NODEVICE;
    }
    c->numSM = prop.multiProcessorCount;
    c->smMajor = prop.major;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return SB_ERR_CUDA;
    }
    if (cudaStreamCreateWithFlags(&c->copyStream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaStreamDestroy(c->stream);
        delete c;
        return SB_ERR_CUDA;
    }
    for (int k = 0; k < 4; ++k) cudaEventCreate(&c->ev[k]);
    for (int k = 0; k < 16; ++k) cudaEventCreate(&c->sev[k]);
    for (int k = 0; k < SB_MAX_BANDS; ++k) cudaEventCreateWithFlags(&c->chunkEv[k], cudaEventDisableTiming);
    // Load sb_amp_match_noalloc's module (with its fixed workspace) and kernels
    // now, so that entry point never loads code or allocates inside its calls.
    // A failure here only disables that entry point; it reports the error.
    c->noallocPrep = sb_noalloc_prepare();
    if (c->noallocPrep != cudaSuccess) cudaGetLastError();
    *out = c;
    return SB_OK;
}

extern "C" void sb_context_destroy(sb_context* c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    cudaStreamSynchronize(c->copyStream);
    for (auto& kv : c->bufs)
        if (kv.second.ptr) cudaFreeAsync(kv.second.ptr, c->stream);
    cudaStreamSynchronize(c->stream);
    for (auto& kv : c->tables)
        if (kv.second) cudaFree(kv.second);
    for (int k = 0; k < 4; ++k) cudaEventDestroy(c->ev[k]);
    for (int k = 0; k < 16; ++k) cudaEventDestroy(c->sev[k]);
    for (int k = 0; k < SB_MAX_BANDS; ++k) cudaEventDestroy(c->chunkEv[k]);
    cudaStreamDestroy(c->copyStream);
    cudaStreamDestroy(c->stream);
    delete c;
}

extern "C" int sb_set_wait_limit(sb_context* c, int64_t naps)
{
    if (!c) return SB_ERR_ARG;
    if (naps < 0) return sb_ctx_fail(c, SB_ERR_ARG, "wait limit must be >= 0");
    c->waitNaps = (long long)naps;
    return SB_OK;
}

extern "C" int64_t sb_context_device_bytes(const sb_context* c)
{
    if (!c) return 0;
    size_t b = c->tableBytes;
    for (const auto& kv : c->bufs) b += kv.second.bytes;
    return (int64_t)b;
}

extern "C" int sb_context_release(sb_context* c)
{
    if (!c) return SB_ERR_ARG;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return sb_ctx_cuda(c, e, "cudaSetDevice");
    cudaStreamSynchronize(c->stream);
    cudaStreamSynchronize(c->copyStream);
    for (auto& kv : c->bufs)
        if (kv.second.ptr) cudaFreeAsync(kv.second.ptr, c->stream);
    c->bufs.clear();
    e = cudaStreamSynchronize(c->stream);  // the pool returns the memory at this synchronisation
    if (e != cudaSuccess) return sb_ctx_cuda(c, e, "release");
    return SB_OK;
}

extern "C" int sb_set_form(sb_context* c, int form)
{
    if (!c) return SB_ERR_ARG;
    if (form != SB_FORM_FP32 && form != SB_FORM_SPLIT_BF16) return sb_ctx_fail(c, SB_ERR_ARG, "unknown form %d", form);
    c->form = form;
    return SB_OK;
}

extern "C" int sb_last_form(const sb_context* c) { return c ? c->lastForm : SB_FORM_FP32; }

static int win_index(int W)
{
    switch (W) {
    case 16: return 0;
    case 24: return 1;
    case 32: return 2;
    case 48: return 3;
    case 64: return 4;
    default: return -1;
    }
}

extern "C" int sb_set_tuning(sb_context* c, int kernel, int window, int threads, int ctasPerSm)
{
    if (!c) return SB_ERR_ARG;
    c->err.clear();
    if (ctasPerSm < 0) return sb_ctx_fail(c, SB_ERR_ARG, "ctasPerSm must be >= 0");
    const int wi = win_index(window);
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return sb_ctx_cuda(c, e, "cudaSetDevice");
    if (kernel == SB_TUNE_COMPLEX) {
        if (wi < 0) return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "complex window %d has no kernel", window);
        if (threads != 0 && threads != cmplx_default_threads(window) && threads != cmplx_alt_threads(window))
            return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "complex window %d: %d threads not compiled", window, threads);
        const int mx = cmplx_blocks_per_sm(window, threads);
        if (ctasPerSm > mx) return sb_ctx_fail(c, SB_ERR_ARG, "at most %d CTAs per SM at %d threads", mx, threads);
        c->tuneCmplxThreads[wi] = threads;
        c->tuneCmplxCtas[wi] = ctasPerSm;
        return SB_OK;
    }
    if (kernel == SB_TUNE_COMPLEX_TC) {
        if (!cmplx_tc_supported(window) || (threads != 0 && threads != cmplx_tc_threads()))
            return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "split-BF16 complex stage: window 64, %d threads",
                               cmplx_tc_threads());
        const int mx = cmplx_tc_blocks_per_sm();
        if (ctasPerSm > mx) return sb_ctx_fail(c, SB_ERR_ARG, "at most %d CTAs per SM", mx);
        c->tuneTcCtas = ctasPerSm;
        return SB_OK;
    }
    if (kernel == SB_TUNE_AMPLITUDE) {
        if (wi < 0 || !amps_supported(window) || threads != 0)
            return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "shared-memory amplitude try: windows 16-64, default threads");
        const int mx = amps_blocks_per_sm(window);
        if (ctasPerSm > mx) return sb_ctx_fail(c, SB_ERR_ARG, "at most %d CTAs per SM", mx);
        c->tuneAmpsCtas[wi] = ctasPerSm;
        return SB_OK;
    }
    return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "unknown kernel %d", kernel);
}

// Launch shape of the complex stage at window W (tuning table or defaults).
static void complex_shape(const sb_context* c, int W, bool tcForm, int* threads, int* bpsm)
{
    if (tcForm) {
        *threads = cmplx_tc_threads();
        const int mx = cmplx_tc_blocks_per_sm();
        *bpsm = c->tuneTcCtas > 0 && c->tuneTcCtas < mx ? c->tuneTcCtas : mx;
        return;
    }
    const int wi = win_index(W);
    *threads = wi >= 0 ? c->tuneCmplxThreads[wi] : 0;
    const int mx = cmplx_blocks_per_sm(W, *threads);
    const int t = wi >= 0 ? c->tuneCmplxCtas[wi] : 0;
    *bpsm = t > 0 && t < mx ? t : mx;
}

static int amps_ctas(const sb_context* c, int Ws)
{
    const int mx = amps_blocks_per_sm(Ws);
    const int wi = win_index(Ws);
    const int t = wi >= 0 ? c->tuneAmpsCtas[wi] : 0;
    return t > 0 && t < mx ? t : mx;
}

extern "C" const char* sb_last_error(const sb_context* c)
{
    if (!c) return "null context";
    return c->err.c_str();
}

extern "C" int sb_last_timing(const sb_context* c, float ms[4])
{
    if (!c || !ms) return SB_ERR_ARG;
    for (int k = 0; k < 4; ++k) ms[k] = c->timing[k];
    return SB_OK;
}

extern "C" int64_t sb_last_launch_count(const sb_context* c) { return c ? c->launches : 0; }

extern "C" int sb_last_stage_timing(const sb_context* c, float ms[8])
{
    if (!c || !ms) return SB_ERR_ARG;
    for (int k = 0; k < 8; ++k) ms[k] = c->stage[k];
    return SB_OK;
}

// ---------------------------------------------------------------- tables

// Host-computed constant tables (double precision, rounded once to float).
const void* sb_table(sb_context* c, const std::string& key, const std::vector<float2>& host)
{
    auto it = c->tables.find(key);
    if (it != c->tables.end()) return it->second;
    void* d = nullptr;
    if (cudaMalloc(&d, host.size() * sizeof(float2)) != cudaSuccess) return nullptr;
    cudaMemcpy(d, host.data(), host.size() * sizeof(float2), cudaMemcpyHostToDevice);
    c->tables[key] = d;
    c->tableBytes += host.size() * sizeof(float2);
    return d;
}

static const double kPi = 3.14159265358979323846;

const float2* tw_table(sb_context* c, int N)
{
    std::vector<float2> h(N);
    for (int e = 0; e < N; ++e) {
        double ang = -2.0 * kPi * (double)e / (double)N;
        h[e] = make_float2((float)cos(ang), (float)sin(ang));
    }
    return (const float2*)sb_table(c, "tw" + std::to_string(N), h);
}

// tau_1[k'] = +exp(+2 pi i k'/(2W)) for k' < W/2, -exp(...) for k' >= W/2.
const float2* tau_table(sb_context* c, int W)
{
    std::vector<float2> h(W);
    for (int k = 0; k < W; ++k) {
        double ang = 2.0 * kPi * (double)k / (2.0 * W);
        double sgn = (k < W / 2) ? 1.0 : -1.0;
        h[k] = make_float2((float)(sgn * cos(ang)), (float)(sgn * sin(ang)));
    }
    return (const float2*)sb_table(c, "tau" + std::to_string(W), h);
}

// A[n][t] = sum_{f=-4..3} exp(+2 pi i f (n - 12 t)/96), n = 24..71.
const float2* osA_table(sb_context* c)
{
    std::vector<float2> h(OSW * NFAST);
    for (int n = 0; n < OSW; ++n)
        for (int t = 0; t < NFAST; ++t) {
            double re = 0, im = 0;
            const int d = (n + 24) - NOVER * t;
            for (int f = -NFAST / 2; f < NFAST / 2; ++f) {
                double ang = 2.0 * kPi * (double)f * (double)d / (double)(NFAST * NOVER);
                re += cos(ang);
                im += sin(ang);
            }
            h[n * NFAST + t] = make_float2((float)re, (float)im);
        }
    return (const float2*)sb_table(c, "osA", h);
}

// Real form of the oversampling matrix: A[n][t] = p(n) exp(+i pi t/8) D[n][t]
// with |p(n)| = 1 and D[n][t] = 2 sum_{g=1/2..7/2} cos(2 pi g (n + 24 - 12 t)/96);
// stored as the 48 x 8 floats of D followed by the 16 phases exp(i pi s/8).
const float2* osD_table(sb_context* c)
{
    std::vector<float2> h(OSW * NFAST / 2 + 16);
    float* f = reinterpret_cast<float*>(h.data());
    for (int n = 0; n < OSW; ++n)
        for (int t = 0; t < NFAST; ++t) {
            const int d = (n + 24) - NOVER * t;
            double v = 0.0;
            for (int g2 = 1; g2 < NFAST; g2 += 2)  // g = g2 / 2
                v += 2.0 * cos(kPi * (double)g2 * (double)d / (double)(NFAST * NOVER));
            f[n * NFAST + t] = (float)v;
        }
    for (int s = 0; s < 16; ++s)
        h[OSW * NFAST / 2 + s] = make_float2((float)cos(kPi * s / 8.0), (float)sin(kPi * s / 8.0));
    return (const float2*)sb_table(c, "osD", h);
}

// computeHanning (speckleTrack.c:1830-1852), W x W, square windows.
const float* hanning_table(sb_context* c, int W)
{
    std::vector<float2> h((W * W + 1) / 2);
    float* f = reinterpret_cast<float*>(h.data());
    for (int i = 0; i < W / 2; i++) {
        int i1 = W / 2 + i, i2 = W / 2 - i - 1;
        double wi = 0.5 * (1.0 + cos((2.0 * kPi) * (double)i / (double)(W - 1)));
        for (int j = 0; j < W / 2; j++) {
            int j1 = W / 2 + j, j2 = W / 2 - j - 1;
            double wj = 0.5 * (1.0 + cos((2.0 * kPi) * (double)j / (double)(W - 1)));
            float v = (float)(wi * wj);
            f[i1 * W + j1] = v;
            f[i2 * W + j2] = v;
            f[i2 * W + j1] = v;
            f[i1 * W + j2] = v;
        }
    }
    return (const float*)sb_table(c, "han" + std::to_string(W), h);
}

// ---------------------------------------------------------------- planning

static int inBounds(int r1, int a1, int wR, int wA, int sR, int sA)
{
    return (r1 > 0 && (r1 + wR) < sR && a1 > 0 && (a1 + wA) < sA);  // speckleTrack.c:1943-1946
}

// getShifts, speckleTrack.c:1857-1940.
static void getShifts(double range, double azimuth, const sb_offset_grid* o, double* dr, double* da)
{
    float minvalue = (float)((float)-SB_LARGEINT * 0.9);
    range = (range - o->r0) / o->deltaR;
    azimuth = (azimuth - o->a0) / o->deltaA;
    if (range < 0.0 || azimuth < 0.0 || (int)range >= o->nr || (int)azimuth >= o->na) {
        *dr = -SB_LARGEINT;
        *da = -SB_LARGEINT;
        return;
    }
    int j = (int)range, i = (int)azimuth;
    const int nr = o->nr;
    const float *R = o->dr, *A = o->da;
    if (j == (o->nr - 1) || i == (o->na - 1)) {
        *dr = R[(size_t)i * nr + j];
        *da = A[(size_t)i * nr + j];
        if (*dr < minvalue || *da < minvalue) {
            *dr = -SB_LARGEINT;
            *da = -SB_LARGEINT;
        }
        return;
    }
    float t = (float)(range - (double)j), u = (float)(azimuth - (double)i);
    const float* img[2] = {R, A};
    double* outv[2] = {dr, da};
    for (int q = 0; q < 2; ++q) {
        const float* M = img[q];
        float p1 = M[(size_t)i * nr + j], p2 = M[(size_t)i * nr + j + 1];
        float p3 = M[(size_t)(i + 1) * nr + j + 1], p4 = M[(size_t)(i + 1) * nr + j];
        if (p1 <= minvalue || p2 <= minvalue || p3 <= minvalue || p4 <= minvalue) {
            float mx = fmaxf(fmaxf(fmaxf(p1, p2), p3), p4);
            *outv[q] = mx;
            if (*outv[q] < minvalue) {
                *dr = -SB_LARGEINT;
                *da = -SB_LARGEINT;
                return;
            }
        } else {
            *outv[q] = (float)((1.0 - t) * (1.0 - u) * p1 + t * (1.0 - u) * p2 + t * u * p3 + (1.0 - t) * u * p4);
        }
    }
}

// findImage2Pos, speckleTrack.c:810-847 (keeps r2/a2 when the grid has no value).
static void findImage2Pos(const sb_track_params* p, int r1, int a1, int* r2, int* a2)
{
    double aShift = 0, rShift = 0, sc = (double)p->scaleFactor;
    int haveShift = 0;
    if (p->polyShift == 0) {
        getShifts(r1, a1, p->initOffsets, &rShift, &aShift);
        if (rShift > (-SB_LARGEINT + 1))
            haveShift = 1;
        else
            return;
    }
    if (p->polyShift != 0 || haveShift == 0) {
        rShift = p->rShiftPoly[0] + (double)(r1 * sc) * p->rShiftPoly[1] + (double)(a1 * sc) * p->rShiftPoly[2];
        aShift = p->aShiftPoly[0] + (double)(r1 * sc) * p->aShiftPoly[1] + (double)(a1 * sc) * p->aShiftPoly[2];
    }
    rShift /= sc;
    aShift /= sc;
    *r2 = (rShift >= 0) ? r1 + (int)(rShift + 0.5) : r1 + (int)(rShift - 0.5);
    *a2 = (aShift >= 0) ? a1 + (int)(aShift + 0.5) : a1 + (int)(aShift - 0.5);
}

// maskValue, speckleTrack.c:1951-1965.
static int maskValue(const sb_track_params* p, int r1, int a1)
{
    const sb_mask* m = p->mask;
    if (!m) return 1;
    int ia1 = (a1 + p->wA / 2 - m->a0) / m->nal;
    int ir1 = (r1 + p->wR / 2 - m->r0) / m->nrl;
    if (ia1 < 0 || ia1 >= m->na || ir1 < 0 || ir1 >= m->nr) return 0;
    return (int)(signed char)m->mask[(size_t)ia1 * m->nr + ir1];
}

static void plan_strack(const sb_track_params* p, int nr1, int na1, int nr2, int na2, std::vector<PointPlan>& plan,
                        std::vector<int>& clist)
{
    const int nR = p->nR, nA = p->nA;
    plan.resize((size_t)nR * nA);
    clist.clear();
    int r2 = 0, a2 = 0;  // uninitialised in the reference: pinned to 0
    for (int i = 0; i < nA; i++) {
        const int a1 = p->aStart + i * p->deltaA - p->wA / 2;
        for (int j = 0; j < nR; j++) {
            const int r1 = p->rStart + j * p->deltaR - p->wR / 2;
            findImage2Pos(p, r1, a1, &r2, &a2);
            int maskVal = maskValue(p, r1 * p->scaleFactor, a1 * p->scaleFactor);
            maskVal = maskVal < 1 ? maskVal : 1;
            PointPlan pl;
            pl.r1 = r1;
            pl.a1 = a1;
            pl.r2 = r2;
            pl.a2 = a2;
            pl.flags = 0;
            if (maskVal > 0) pl.flags |= PF_MASK;
            if (inBounds(r1, a1, p->wR, p->wA, nr1, na1) && inBounds(r2, a2, p->wR, p->wA, nr2, na2))
                pl.flags |= PF_CBOUND;
            for (int s = 1; s <= 2; ++s) {
                const int a1a = p->aStart + i * p->deltaA - p->wA / 2 * s;
                const int r1a = p->rStart + j * p->deltaR - p->wR / 2 * s;
                const int r2a = r1a + (r2 - r1), a2a = a1a + (a2 - a1);
                if (inBounds(r1a, a1a, p->wRa * s, p->wAa * s, nr1, na1) &&
                    inBounds(r2a, a2a, p->wRa * s, p->wAa * s, nr2, na2))
                    pl.flags |= (s == 1 ? PF_SBOUND : PF_LBOUND);
            }
            const size_t k = (size_t)i * nR + j;
            plan[k] = pl;
            if ((pl.flags & PF_CBOUND) && (pl.flags & PF_MASK) && p->noComplex == 0) clist.push_back((int)k);
        }
    }
}

// ---------------------------------------------------------------- images

// Device view of an input image (uploads host images into a context buffer).
int sb_image_to_device(sb_context* c, const sb_image* im, const char* name, const void** dptr)
{
    const size_t elem = im->sampleType == SB_CFLOAT32 ? 8 : 4;
    const size_t bytes = (size_t)im->nr * (size_t)im->na * elem;
    if (im->onDevice) {
        *dptr = im->data;
        return SB_OK;
    }
    cudaError_t e;
    void* d = sb_ctx_buf(c, name, bytes, &e);
    if (!d) return sb_ctx_cuda(c, e, "cudaMalloc(image)");
    e = cudaMemcpyAsync(d, im->data, bytes, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return sb_ctx_cuda(c, e, "cudaMemcpyAsync(image)");
    *dptr = d;
    return SB_OK;
}

// Banded upload for sb_strack: host images go up in nb azimuth bands on the
// copy stream (band k = rows [k*rows, (k+1)*rows) of each image), and
// chunkEv[k] marks band k of both images resident, so complex matching of the
// points whose windows lie in bands <= k overlaps the copies of later bands.
// Device-resident images are used in place.  rows[i] = 0 for a device image.
struct Bands {
    int nb = 1;
    int rows[2] = {0, 0};
};
static int upload_banded(sb_context* c, const sb_image* im[2], const void* dptr[2], Bands* b)
{
    size_t hostBytes = 0;
    for (int i = 0; i < 2; ++i) {
        const size_t elem = im[i]->sampleType == SB_CFLOAT32 ? 8 : 4;
        if (!im[i]->onDevice) hostBytes += (size_t)im[i]->nr * (size_t)im[i]->na * elem;
    }
    // about 8 MB per band and image, at most SB_MAX_BANDS bands (matching waits for the first)
    size_t nb = hostBytes / ((size_t)16 << 20);
    b->nb = nb < 1 ? 1 : (nb > (size_t)SB_MAX_BANDS ? SB_MAX_BANDS : (int)nb);
    cudaError_t e;
    char* dst[2] = {nullptr, nullptr};
    for (int i = 0; i < 2; ++i) {
        if (im[i]->onDevice) {
            dptr[i] = im[i]->data;
            b->rows[i] = 0;
            continue;
        }
        const size_t elem = im[i]->sampleType == SB_CFLOAT32 ? 8 : 4;
        const size_t bytes = (size_t)im[i]->nr * (size_t)im[i]->na * elem;
        dst[i] = (char*)sb_ctx_buf(c, i == 0 ? "img1" : "img2", bytes, &e);
        if (!dst[i]) return sb_ctx_cuda(c, e, "cudaMalloc(image)");
        dptr[i] = dst[i];
        b->rows[i] = (im[i]->na + b->nb - 1) / b->nb;
    }
    // the copy stream waits for the main stream: the buffers' (stream-ordered)
    // allocation and any work still reading them come first
    cudaEventRecord(c->chunkEv[0], c->stream);
    cudaStreamWaitEvent(c->copyStream, c->chunkEv[0], 0);
    for (int k = 0; k < b->nb; ++k) {
        for (int i = 0; i < 2; ++i) {
            if (!dst[i]) continue;
            const size_t elem = im[i]->sampleType == SB_CFLOAT32 ? 8 : 4;
            const size_t rowBytes = (size_t)im[i]->nr * elem;
            const int r0 = k * b->rows[i];
            const int r1 = (k + 1) * b->rows[i] < im[i]->na ? (k + 1) * b->rows[i] : im[i]->na;
            if (r1 <= r0) continue;
            e = cudaMemcpyAsync(dst[i] + (size_t)r0 * rowBytes, (const char*)im[i]->data + (size_t)r0 * rowBytes,
                                (size_t)(r1 - r0) * rowBytes, cudaMemcpyHostToDevice, c->copyStream);
            if (e != cudaSuccess) return sb_ctx_cuda(c, e, "cudaMemcpyAsync(image band)");
        }
        cudaEventRecord(c->chunkEv[k], c->copyStream);
    }
    return SB_OK;
}

static int check_image(sb_context* c, const sb_image* im)
{
    if (!im || !im->data || im->nr <= 0 || im->na <= 0) return sb_ctx_fail(c, SB_ERR_ARG, "invalid image");
    if (im->sampleType != SB_CFLOAT32 && im->sampleType != SB_CINT16)
        return sb_ctx_fail(c, SB_ERR_ARG, "invalid sampleType %d", im->sampleType);
    if (im->byteOrder != SB_LSB && im->byteOrder != SB_MSB)
        return sb_ctx_fail(c, SB_ERR_ARG, "invalid byteOrder %d", im->byteOrder);
    return SB_OK;
}

// Copies (or aliases) an output grid.
static int out_copy(sb_context* c, void* dst, const void* src, size_t bytes, int onDevice)
{
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                    c->stream);
    return sb_ctx_cuda(c, e, "cudaMemcpyAsync(output)");
}

static FitArgs make_fit_args(const sb_track_params* p, FitJob* fit, int nList, int stage, PointRec* rec)
{
    FitArgs f;
    f.fit = fit;
    f.nList = nList;
    f.nListDev = nullptr;
    f.stage = stage;
    f.wR = p->wR; f.wA = p->wA; f.wRa = p->wRa; f.wAa = p->wAa;
    f.noComplex = p->noComplex;
    f.azThresh = p->azDefocusThresh;
    f.checkAzFocus = p->checkAzFocus;
    f.rec = rec;
    return f;
}

#define CK(call, what)                                               \
    do {                                                             \
        cudaError_t _e = (call);                                     \
        if (_e != cudaSuccess) return sb_ctx_cuda(c, _e, what);      \
    } while (0)

// ---------------------------------------------------------------- strack

extern "C" int sb_strack(sb_context* c, const sb_track_params* p, const sb_image* img1, const sb_image* img2,
                         sb_track_result* out)
{
    if (!c) return SB_ERR_ARG;
    c->err.clear();
    c->launches = 0;
    if (!p || !out) return sb_ctx_fail(c, SB_ERR_ARG, "null params or result");
    int rc;
    if ((rc = check_image(c, img1)) != SB_OK || (rc = check_image(c, img2)) != SB_OK) return rc;
    if (img1->sampleType != img2->sampleType) return sb_ctx_fail(c, SB_ERR_ARG, "images differ in sample type");
    if (img1->byteOrder != img2->byteOrder) return sb_ctx_fail(c, SB_ERR_ARG, "images differ in byte order");
    if (p->nR <= 0 || p->nA <= 0) return sb_ctx_fail(c, SB_ERR_ARG, "empty grid nR=%d nA=%d", p->nR, p->nA);
    if ((int64_t)p->nR * p->nA > (int64_t)1 << 30) return sb_ctx_fail(c, SB_ERR_ARG, "grid too large");
    if (p->scaleFactor <= 0) return sb_ctx_fail(c, SB_ERR_ARG, "scaleFactor must be positive");
    if (p->polyShift == 0 && !p->initOffsets) return sb_ctx_fail(c, SB_ERR_ARG, "polyShift=0 needs initOffsets");
    if (p->mask && (p->mask->nal <= 0 || p->mask->nrl <= 0 || !p->mask->mask))
        return sb_ctx_fail(c, SB_ERR_ARG, "invalid mask");
    if (!out->offR || !out->offA || !out->corr || !out->type)
        return sb_ctx_fail(c, SB_ERR_ARG, "null output grid");
    const int W = p->wR;
    if (p->wR != p->wA) return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "complex window must be square (wr == wa)");
    if (p->noComplex == 0 && !cmplx_supported(W))
        return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "complex window %d not supported", W);
    const int WA = p->wRa;
    if (p->maxTries > 0) {
        if (p->wRa != p->wAa) return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "amplitude window must be square");
        if (!amp_supported(WA)) return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "amplitude window %d not supported", WA);
        if (p->maxTries > 1 && !amp_supported(WA * LA))
            return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "large amplitude window %d not supported", WA * LA);
    }
    // interferogram (initPhaseCorrect, speckleTrack.c:1576-1601): patch of
    // max(wA/nal, wR/nrl, 8) samples, padded to (ps nal) x (ps nrl)
    int intPs = 0;
    if (p->intf && p->noComplex == 0) {
        const sb_interferogram* fi = p->intf;
        if (!fi->data || fi->nr <= 0 || fi->na <= 0 || fi->nrl <= 0 || fi->nal <= 0)
            return sb_ctx_fail(c, SB_ERR_ARG, "invalid interferogram");
        intPs = p->wA / fi->nal > p->wR / fi->nrl ? p->wA / fi->nal : p->wR / fi->nrl;
        intPs = intPs > 8 ? intPs : 8;
        if (intPs * fi->nal < p->wA || intPs * fi->nrl < p->wR)
            return sb_ctx_fail(c, SB_ERR_UNSUPPORTED,
                               "interferogram looks (%d, %d) give a padded patch smaller than the window (the "
                               "reference reads outside it)", fi->nrl, fi->nal);
        if (2 * intPs * intPs > W * (W + 1) || intPs * fi->nal >= 32768 || intPs * fi->nrl >= 32768)
            return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "interferogram patch %d too large for window %d", intPs, W);
    }
    const sb_baseline* bl = p->baseline;
    const int baseOn =
        bl && (bl->Bn != 0 || bl->Bp != 0 || bl->dBn != 0 || bl->dBp != 0 || bl->dBnQ != 0 || bl->dBpQ != 0);
    if (baseOn && (!bl->sinThetaD || !bl->cosThetaD || !bl->overRange))
        return sb_ctx_fail(c, SB_ERR_ARG, "baseline tables missing");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    cudaEventRecord(c->ev[0], c->stream);
    for (int k = 0; k < 8; ++k) c->stage[k] = 0.f;

    // ---- plan: host loop when the initial shift comes from an offset grid
    // (its carry-over of r2/a2 is sequential), device kernel for a polynomial
    const int n = p->nR * p->nA;
    const bool devPlan = p->polyShift != 0;
    std::vector<PointPlan> plan;
    std::vector<int> clist;
    cudaError_t e;
    PointPlan* dplan = (PointPlan*)sb_ctx_buf(c, "plan", sizeof(PointPlan) * n, &e);
    PointRec* drec = (PointRec*)sb_ctx_buf(c, "rec", sizeof(PointRec) * n, &e);
    int* dlist = (int*)sb_ctx_buf(c, "list", sizeof(int) * (n + 1), &e);
    FitJob* dfit = (FitJob*)sb_ctx_buf(c, "fit", sizeof(FitJob) * (n + 1), &e);
    unsigned long long* dstats = (unsigned long long*)sb_ctx_buf(c, "stats", sizeof(unsigned long long) * 8, &e);
    float* dR = (float*)sb_ctx_buf(c, "offR", sizeof(float) * n, &e);
    float* dA = (float*)sb_ctx_buf(c, "offA", sizeof(float) * n, &e);
    float* dC = (float*)sb_ctx_buf(c, "corr", sizeof(float) * n, &e);
    float* dZ = (float*)sb_ctx_buf(c, "azd", sizeof(float) * n, &e);
    uint8_t* dT = (uint8_t*)sb_ctx_buf(c, "type", n, &e);
    int* dlist2 = (int*)sb_ctx_buf(c, "listBands", sizeof(int) * (n + 1), &e);
    int* dkey = (int*)sb_ctx_buf(c, "listKey", sizeof(int) * (n + 1), &e);
    int* dpart = (int*)sb_ctx_buf(c, "partScratch", sizeof(int) * partition_scratch_ints(n, PART_KMAX), &e);
    if (!dplan || !drec || !dlist || !dfit || !dstats || !dR || !dA || !dC || !dZ || !dT || !dlist2 ||
        !dkey || !dpart)
        return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
    // images: banded upload on the copy stream, overlapping the planning and
    // the complex matching of earlier bands
    const sb_image* ims[2] = {img1, img2};
    const void* dimg[2] = {nullptr, nullptr};
    Bands bands;
    if ((rc = upload_banded(c, ims, dimg, &bands)) != SB_OK) return rc;
    const void *d1 = dimg[0], *d2 = dimg[1];
    if (!devPlan) plan_strack(p, img1->nr, img1->na, img2->nr, img2->na, plan, clist);
    int nC = 0;
    if (devPlan) {
        PlanArgs pa;
        memset(&pa, 0, sizeof(pa));
        pa.rStart = p->rStart; pa.aStart = p->aStart; pa.deltaR = p->deltaR; pa.deltaA = p->deltaA;
        pa.nR = p->nR; pa.nA = p->nA;
        pa.wR = p->wR; pa.wA = p->wA; pa.wRa = p->wRa; pa.wAa = p->wAa;
        pa.scaleFactor = p->scaleFactor;
        pa.noComplex = p->noComplex;
        for (int k = 0; k < 3; ++k) {
            pa.rPoly[k] = p->rShiftPoly[k];
            pa.aPoly[k] = p->aShiftPoly[k];
        }
        pa.nr1 = img1->nr; pa.na1 = img1->na; pa.nr2 = img2->nr; pa.na2 = img2->na;
        if (p->mask) {
            const size_t mb = (size_t)p->mask->nr * p->mask->na;
            uint8_t* dm = (uint8_t*)sb_ctx_buf(c, "mask", mb, &e);
            if (!dm) return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
            CK(cudaMemcpyAsync(dm, p->mask->mask, mb, cudaMemcpyHostToDevice, c->stream), "mask");
            pa.mask = dm;
            pa.mR0 = p->mask->r0; pa.mA0 = p->mask->a0; pa.mNr = p->mask->nr; pa.mNa = p->mask->na;
            pa.mNrl = p->mask->nrl; pa.mNal = p->mask->nal;
        }
        // A large grid's complex list is grouped into range strips of image 1
        // (stable, so row-major inside a strip): the patches in flight then
        // read a band of a few hundred columns that stays in L2 while the
        // sweep moves down it, instead of whole image rows.
        const bool strips = n >= 16 * c->numSM && img1->nr >= 8 * SB_BANDS_MAX;
        const int K = strips ? SB_BANDS_MAX : 1;
        pa.stripPx = strips ? (img1->nr + SB_BANDS_MAX - 1) / SB_BANDS_MAX : 0;
        CK(launch_plan_poly(pa, dplan, dkey, c->stream), "plan_poly");
        CK(launch_partition(dkey, nullptr, n, K, dlist, dpart, c->stream), "partition");
        c->launches += 4;
        CK(cudaMemcpyAsync(&nC, dpart + partition_keyoff_at(n, K) + K, sizeof(int), cudaMemcpyDeviceToHost,
                           c->stream),
           "count");
        CK(cudaStreamSynchronize(c->stream), "sync");
    } else {
        CK(cudaMemcpyAsync(dplan, plan.data(), sizeof(PointPlan) * n, cudaMemcpyHostToDevice, c->stream), "plan");
        if (!clist.empty())
            CK(cudaMemcpyAsync(dlist, clist.data(), sizeof(int) * clist.size(), cudaMemcpyHostToDevice, c->stream),
               "list");
        nC = (int)clist.size();
    }
    const double *dSin = nullptr, *dCos = nullptr, *dOver = nullptr;
    if (baseOn) {
        const size_t nb = sizeof(double) * (size_t)img1->nr;
        double* b = (double*)sb_ctx_buf(c, "baseTabs", 3 * nb, &e);
        if (!b) return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
        CK(cudaMemcpyAsync(b, bl->sinThetaD, nb, cudaMemcpyHostToDevice, c->stream), "baseline");
        CK(cudaMemcpyAsync((char*)b + nb, bl->cosThetaD, nb, cudaMemcpyHostToDevice, c->stream), "baseline");
        CK(cudaMemcpyAsync((char*)b + 2 * nb, bl->overRange, nb, cudaMemcpyHostToDevice, c->stream), "baseline");
        dSin = b;
        dCos = (const double*)((char*)b + nb);
        dOver = (const double*)((char*)b + 2 * nb);
    }
    cudaEventRecord(c->ev[1], c->stream);

    // ---- kernels
    CK(launch_rec_init(drec, n, c->stream), "rec_init");
    c->launches++;
    CK(cudaMemsetAsync(dstats, 0, sizeof(unsigned long long) * 8, c->stream), "memset");
    int* tcErrFlag = nullptr;  // set when the split-BF16 form ran
    c->lastForm = SB_FORM_FP32;
    if (nC > 0) {
        CmplxArgs a;
        memset(&a, 0, sizeof(a));
        a.img1 = d1;
        a.img2 = d2;
        a.nr1 = img1->nr; a.na1 = img1->na; a.nr2 = img2->nr; a.na2 = img2->na;
        a.sampleType = img1->sampleType;
        a.byteOrder = img1->byteOrder;
        a.plan = dplan;
        a.list = dlist;
        a.nList = nC;
        a.hanning = p->hanningFlag ? hanning_table(c, W) : nullptr;
        a.hanCorr = p->hanningFlag ? 1.5 : 1.0;
        a.twW = tw_table(c, W);
        a.tau = tau_table(c, W);
        a.osA = osA_table(c);
        a.osD = osD_table(c);
        a.gauss = p->gaussFlag ? 1 : 0;
        a.azThresh = p->azDefocusThresh;
        a.checkAzFocus = p->checkAzFocus;
        a.noComplex = p->noComplex;
        a.baseOn = baseOn;
        if (baseOn) {
            a.Bn = bl->Bn; a.Bp = bl->Bp; a.dBn = bl->dBn; a.dBp = bl->dBp; a.dBnQ = bl->dBnQ; a.dBpQ = bl->dBpQ;
            a.lambda = bl->lambda;
            a.sinThetaD = dSin; a.cosThetaD = dCos; a.overRange = dOver;
        }
        a.rec = drec;
        a.fit = dfit;
        if (p->intf) {
            // phaseCorrectInt: the interferogram on the device, patch geometry
            const sb_interferogram* fi = p->intf;
            const size_t ib = (size_t)fi->nr * fi->na * 4;
            const uint32_t* di = (const uint32_t*)fi->data;
            if (!fi->onDevice) {
                uint32_t* buf = (uint32_t*)sb_ctx_buf(c, "intf", ib, &e);
                if (!buf) return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
                CK(cudaMemcpyAsync(buf, fi->data, ib, cudaMemcpyHostToDevice, c->stream), "interferogram");
                di = buf;
            }
            a.intf = di;
            a.intNr = fi->nr; a.intNa = fi->na; a.intNrl = fi->nrl; a.intNal = fi->nal;
            a.intMSB = fi->byteOrder == SB_MSB;
            a.intPs = intPs;
            a.intPSA = intPs * fi->nal;
            a.intPSR = intPs * fi->nrl;
            a.twP = tw_table(c, intPs);
            if (!a.twP) return sb_ctx_fail(c, SB_ERR_NOMEM, "table allocation failed");
        }
        if (!a.twW || !a.tau || !a.osA || !a.osD || (p->hanningFlag && !a.hanning))
            return sb_ctx_fail(c, SB_ERR_NOMEM, "table allocation failed");
        // the split-BF16 tensor-core form where it applies (see sb_set_form)
        const bool tcForm = c->form == SB_FORM_SPLIT_BF16 && cmplx_tc_supported(W) && !baseOn && !p->intf &&
                            !p->gaussFlag && c->smMajor >= 10;
        c->lastForm = tcForm ? SB_FORM_SPLIT_BF16 : SB_FORM_FP32;
        int* dTcErr = nullptr;
        if (tcForm) {
            dTcErr = (int*)sb_ctx_buf(c, "tcErr", sizeof(int), &e);
            if (!dTcErr) return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
            CK(cudaMemsetAsync(dTcErr, 0, sizeof(int), c->stream), "memset");
            a.tcErr = dTcErr;
            tcErrFlag = dTcErr;
        }
        int cthreads = 0, bpsm = 0;
        complex_shape(c, W, tcForm, &cthreads, &bpsm);
        if (bpsm <= 0) return sb_ctx_fail(c, SB_ERR_CUDA, "complex kernel cannot be resident (W=%d)", W);
        // per-band sub-lists (one band: the list as planned)
        std::vector<int> bandOff(bands.nb + 1, 0);
        bandOff[1] = nC;
        if (bands.nb > 1) {
            CK(launch_band_key(dplan, dlist, nC, W, bands.rows[0], bands.rows[1], bands.nb, dkey, c->stream),
               "band_key");
            CK(launch_partition(dkey, dlist, nC, bands.nb, dlist2, dpart, c->stream), "partition");
            c->launches += 4;
            CK(cudaMemcpyAsync(bandOff.data(), dpart + partition_keyoff_at(nC, bands.nb),
                               sizeof(int) * (bands.nb + 1), cudaMemcpyDeviceToHost, c->stream),
               "offsets");
            CK(cudaStreamSynchronize(c->stream), "sync");
            a.list = dlist2;
        }
        const int nBand = bands.nb > 1 ? bands.nb : 1;
        // peak hand-off buffer: list chunks of at most kPeakChunk patches, each
        // launched as complex kernel + peak kernel (-gauss keeps the fit in
        // the complex kernel)
        constexpr int kPeakChunk = 1 << 19;  // bench.py and serve.py's memory estimate use the same figure
        PeakJob* dpeak = nullptr;
        if (!p->gaussFlag) {
            const size_t pc = nC < kPeakChunk ? (size_t)nC : (size_t)kPeakChunk;
            dpeak = (PeakJob*)sb_ctx_buf(c, "peakjob", pc * sizeof(PeakJob), &e);
            if (!dpeak) return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
        }
        cudaEventRecord(c->sev[0], c->stream);
        for (int k = 0; k < nBand; ++k) {
            if (bandOff[k + 1] == bandOff[k]) continue;
            CK(cudaStreamWaitEvent(c->stream, c->chunkEv[k], 0), "wait band");
            for (int off = bandOff[k]; off < bandOff[k + 1]; off += kPeakChunk) {
                const int cnt = bandOff[k + 1] - off < kPeakChunk ? bandOff[k + 1] - off : kPeakChunk;
                CmplxArgs ak = a;
                ak.list = a.list + off;
                ak.fit = dfit + off;
                ak.nList = cnt;
                ak.peak = dpeak;
                const int nCta = c->numSM * bpsm < cnt ? c->numSM * bpsm : cnt;
                if (tcForm)
                    CK(launch_strack_cmplx_tc(ak, nCta, c->stream), "strack_cmplx_tc");
                else
                    CK(launch_strack_cmplx(W, ak, nCta, c->stream, cthreads), "strack_cmplx");
                c->launches++;
                if (dpeak) {
                    PeakArgs pk;
                    pk.peak = dpeak;
                    pk.nList = cnt;
                    pk.W = W;
                    pk.hanCorr = a.hanCorr;
                    pk.osD = a.osD;
                    pk.rec = drec;
                    pk.fit = dfit + off;
                    CK(launch_strack_peak(pk, c->numSM, c->stream), "strack_peak");
                    c->launches++;
                }
            }
        }
        cudaEventRecord(c->sev[1], c->stream);
        FitArgs f = make_fit_args(p, dfit, a.nList, 0, drec);
        CK(launch_strack_fit(f, c->stream), "strack_fit");
        c->launches++;
        cudaEventRecord(c->sev[2], c->stream);
        c->stage[5] = (float)a.nList;
    }
    // every band resident before the amplitude tries
    CK(cudaStreamWaitEvent(c->stream, c->chunkEv[bands.nb - 1], 0), "wait bands");
    WalkParams w;
    w.wR = p->wR; w.wA = p->wA; w.wRa = p->wRa; w.wAa = p->wAa;
    w.noComplex = p->noComplex;
    w.maxTries = p->maxTries;
    const bool ownAz = (p->wRa == p->wR && p->wAa == p->wA);
    int* dAz = nullptr;
    // The tries run without host round trips: each try's list length stays on
    // the device (kernels launched for the whole grid read it), and the
    // stage timings and the tensor-core wait flag are read after the call.
    int* dStageCnt = (int*)sb_ctx_buf(c, "stageCnt", sizeof(int) * 4, &e);
    if (!dStageCnt) return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
    CK(cudaMemsetAsync(dStageCnt, 0, sizeof(int) * 4, c->stream), "memset");
    bool stageRan[3] = {false, false, false};
    for (int stage = 1; stage <= 2 && stage <= p->maxTries; ++stage) {
        CK(launch_select(dplan, drec, n, w, stage, dkey, c->stream), "select");
        CK(launch_partition(dkey, nullptr, n, 1, dlist, dpart, c->stream), "partition");
        c->launches += 4;
        const int* dCnt = dpart + partition_keyoff_at(n, 1) + 1;
        CK(cudaMemcpyAsync(dStageCnt + stage, dCnt, sizeof(int), cudaMemcpyDeviceToDevice, c->stream), "count");
        const int Ws = WA * (stage == 1 ? 1 : LA);
        // small windows (shared-memory kernel): launched for the whole grid,
        // the list length read on the device; larger windows size a per-CTA
        // workspace by the list, so their length is read back first
        const bool onChip = amps_supported(Ws);
        int cnt = n;
        if (!onChip) {
            CK(cudaMemcpyAsync(&cnt, dCnt, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "count");
            CK(cudaStreamSynchronize(c->stream), "sync");
            if (cnt == 0) continue;
        }
        const bool needFill = !ownAz && !(p->noComplex && stage == 1);
        if (needFill) {
            dAz = (int*)sb_ctx_buf(c, "azEff", sizeof(int) * n, &e);
            if (!dAz) return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
            CK(launch_az_fill(drec, n, dAz, c->stream), "az_fill");
            c->launches++;
        }
        AmpArgs a;
        memset(&a, 0, sizeof(a));
        a.img1 = d1;
        a.img2 = d2;
        a.nr1 = img1->nr; a.na1 = img1->na; a.nr2 = img2->nr; a.na2 = img2->na;
        a.sampleType = img1->sampleType;
        a.byteOrder = img1->byteOrder;
        a.plan = dplan;
        a.list = dlist;
        a.nList = cnt;  // the length, or its upper bound (the grid) when read on the device
        a.nListDev = onChip ? dCnt : nullptr;
        a.stage = stage;
        a.s = stage == 1 ? 1 : LA;
        a.wR = p->wR; a.wA = p->wA; a.wRa = p->wRa; a.wAa = p->wAa;
        a.nR = p->nR;
        a.rStart = p->rStart; a.aStart = p->aStart; a.deltaR = p->deltaR; a.deltaA = p->deltaA;
        a.noComplex = p->noComplex;
        a.azThresh = p->azDefocusThresh;
        a.checkAzFocus = p->checkAzFocus;
        a.azEff = needFill ? dAz : nullptr;
        a.twWs = tw_table(c, Ws);
        a.tw2Ws = tw_table(c, 2 * Ws);
        a.tau = tau_table(c, Ws);
        a.osA = osA_table(c);
        a.osD = osD_table(c);
        a.gauss = p->gaussFlag ? 1 : 0;
        a.rec = drec;
        a.fit = dfit;
        // small windows: everything in shared memory; larger: per-CTA
        // workspace in global memory staged through shared tiles
        int nCta = c->numSM * (onChip ? amps_ctas(c, Ws) : amp_blocks_per_sm(Ws));
        if (nCta > cnt) nCta = cnt;
        if (nCta < 1) return sb_ctx_fail(c, SB_ERR_CUDA, "amplitude kernel cannot be resident (Ws=%d)", Ws);
        if (!onChip) {
            a.scratchPerCta = amp_scratch_elems(Ws);
            a.scratch = (float2*)sb_ctx_buf(c, "ampScratch", sizeof(float2) * a.scratchPerCta * nCta, &e);
        }
        if ((!onChip && !a.scratch) || !a.twWs || !a.tw2Ws || !a.tau || !a.osA || !a.osD)
            return sb_ctx_fail(c, SB_ERR_NOMEM, "amplitude workspace allocation failed");
        cudaEventRecord(c->sev[2 + 2 * stage], c->stream);
        if (onChip)
            CK(launch_strack_amps(Ws, a, nCta, c->stream), "strack_amps");
        else
            CK(launch_strack_amp(Ws, a, nCta, c->stream), "strack_amp");
        c->launches++;
        cudaEventRecord(c->sev[3 + 2 * stage], c->stream);
        FitArgs f = make_fit_args(p, dfit, cnt, stage, drec);
        f.nListDev = onChip ? dCnt : nullptr;
        CK(launch_strack_fit(f, c->stream), "strack_fit");
        c->launches++;
        cudaEventRecord(c->sev[8 + stage], c->stream);
        stageRan[stage] = true;
    }
    CK(launch_finalize(dplan, drec, n, w, p->scaleFactor, dR, dA, dC, dZ, dT, dstats, c->stream), "finalize");
    c->launches++;
    cudaEventRecord(c->ev[2], c->stream);

    // ---- outputs
    if ((rc = out_copy(c, out->offR, dR, sizeof(float) * n, out->onDevice)) != SB_OK) return rc;
    if ((rc = out_copy(c, out->offA, dA, sizeof(float) * n, out->onDevice)) != SB_OK) return rc;
    if ((rc = out_copy(c, out->corr, dC, sizeof(float) * n, out->onDevice)) != SB_OK) return rc;
    if (out->azd && (rc = out_copy(c, out->azd, dZ, sizeof(float) * n, out->onDevice)) != SB_OK) return rc;
    if ((rc = out_copy(c, out->type, dT, n, out->onDevice)) != SB_OK) return rc;
    unsigned long long st[8];
    CK(cudaMemcpyAsync(st, dstats, sizeof(st), cudaMemcpyDeviceToHost, c->stream), "stats");
    int stageCnt[4] = {0, 0, 0, 0}, tcBad = 0;
    CK(cudaMemcpyAsync(stageCnt, dStageCnt, sizeof(stageCnt), cudaMemcpyDeviceToHost, c->stream), "counts");
    if (tcErrFlag) CK(cudaMemcpyAsync(&tcBad, tcErrFlag, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "tcErr");
    cudaEventRecord(c->ev[3], c->stream);
    CK(cudaStreamSynchronize(c->stream), "strack");
    if (tcBad) return sb_ctx_fail(c, SB_ERR_TIMEOUT, "split-BF16 complex stage: a tensor-core wait timed out");
    if (nC > 0) {
        float t0 = 0, t1 = 0;
        cudaEventElapsedTime(&t0, c->sev[0], c->sev[1]);
        cudaEventElapsedTime(&t1, c->sev[1], c->sev[2]);
        c->stage[0] = t0;
        c->stage[3] += t1;
    }
    for (int stage = 1; stage <= 2; ++stage) {
        if (!stageRan[stage]) continue;
        float t0 = 0, t1 = 0;
        cudaEventElapsedTime(&t0, c->sev[2 + 2 * stage], c->sev[3 + 2 * stage]);
        cudaEventElapsedTime(&t1, c->sev[3 + 2 * stage], c->sev[8 + stage]);
        c->stage[stage] = t0;
        c->stage[3] += t1;
        c->stage[5 + stage] = (float)stageCnt[stage];
    }
    out->nComplex = (int64_t)st[0];
    out->nAmp = (int64_t)st[1];
    out->nAmpL = (int64_t)st[2];
    out->nFail = (int64_t)st[3];
    out->nAttempted = (int64_t)n - (int64_t)st[4];
    cudaEventElapsedTime(&c->timing[0], c->ev[0], c->ev[3]);
    cudaEventElapsedTime(&c->timing[1], c->ev[0], c->ev[1]);
    cudaEventElapsedTime(&c->timing[2], c->ev[1], c->ev[2]);
    cudaEventElapsedTime(&c->timing[3], c->ev[2], c->ev[3]);
    {
        float tk = c->timing[2] - c->stage[0] - c->stage[1] - c->stage[2] - c->stage[3];
        c->stage[4] = tk > 0 ? tk : 0.f;
    }
    return SB_OK;
}

// ---------------------------------------------------------------- batched strack
// Many image pairs in one call.  The pairs are ordered by window bucket
// (complex window, amplitude window); both images of every pair are copied
// into two atlases (images stacked along azimuth, one row pitch), so a point's
// windows are addressed like any single pair's and every stage kernel runs
// once per bucket over the points of all pairs in it: one persistent complex
// launch per bucket (and list chunk), one peak and one fit launch, then the
// amplitude tries and the finalize pass per bucket.  Per point the arithmetic
// is that of sb_strack, so each pair's grids equal its own sb_strack result.

namespace {
// Events owned for the duration of one batched call.
struct BatchEvents {
    std::vector<cudaEvent_t> ev;
    bool good = true;
    explicit BatchEvents(int n) : ev((size_t)n, nullptr)
    {
        for (auto& e : ev)
            if (cudaEventCreate(&e) != cudaSuccess) good = false;
    }
    ~BatchEvents()
    {
        for (auto e : ev)
            if (e) cudaEventDestroy(e);
    }
    bool ok() const { return good; }
    cudaEvent_t operator[](int i) const { return ev[(size_t)i]; }
};

struct Bucket {
    int wR, wRa;
    int pFirst, pLast;           // range in the bucket order of the pairs
    int g0, g1;                  // global point range
    int l0, l1;                  // range of the complex list
};
}  // namespace

extern "C" int sb_strack_batch(sb_context* c, int32_t nPairs, const sb_track_params* P, const sb_image* I1,
                               const sb_image* I2, sb_track_result* out)
{
    if (!c) return SB_ERR_ARG;
    c->err.clear();
    c->launches = 0;
    if (nPairs <= 0 || !P || !I1 || !I2 || !out) return sb_ctx_fail(c, SB_ERR_ARG, "empty batch or null arrays");
    const sb_track_params& p0 = P[0];
    int rc;
    int64_t total = 0;
    for (int k = 0; k < nPairs; ++k) {
        const sb_track_params* p = &P[k];
        if ((rc = check_image(c, &I1[k])) != SB_OK || (rc = check_image(c, &I2[k])) != SB_OK) return rc;
        if (I1[k].sampleType != I1[0].sampleType || I2[k].sampleType != I1[0].sampleType ||
            I1[k].byteOrder != I1[0].byteOrder || I2[k].byteOrder != I1[0].byteOrder)
            return sb_ctx_fail(c, SB_ERR_ARG, "pair %d: every image of a batch has the same sample type and byte order",
                               k);
        if (p->nR <= 0 || p->nA <= 0) return sb_ctx_fail(c, SB_ERR_ARG, "pair %d: empty grid", k);
        if (p->scaleFactor <= 0) return sb_ctx_fail(c, SB_ERR_ARG, "pair %d: scaleFactor must be positive", k);
        if (p->polyShift == 0 && !p->initOffsets)
            return sb_ctx_fail(c, SB_ERR_ARG, "pair %d: polyShift=0 needs initOffsets", k);
        if (p->mask && (p->mask->nal <= 0 || p->mask->nrl <= 0 || !p->mask->mask))
            return sb_ctx_fail(c, SB_ERR_ARG, "pair %d: invalid mask", k);
        if (!out[k].offR || !out[k].offA || !out[k].corr || !out[k].type)
            return sb_ctx_fail(c, SB_ERR_ARG, "pair %d: null output grid", k);
        if (p->intf || (p->baseline && (p->baseline->Bn != 0 || p->baseline->Bp != 0 || p->baseline->dBn != 0 ||
                                         p->baseline->dBp != 0 || p->baseline->dBnQ != 0 || p->baseline->dBpQ != 0)))
            return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "pair %d: interferogram or baseline flattening: use sb_strack", k);
        if (p->wR != p->wA || (p->maxTries > 0 && p->wRa != p->wAa))
            return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "pair %d: windows must be square", k);
        if (p->noComplex == 0 && !cmplx_supported(p->wR))
            return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "pair %d: complex window %d not supported", k, p->wR);
        if (p->maxTries > 0 && (!amp_supported(p->wRa) || (p->maxTries > 1 && !amp_supported(p->wRa * LA))))
            return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "pair %d: amplitude window %d not supported", k, p->wRa);
        if (p->noComplex != p0.noComplex || p->hanningFlag != p0.hanningFlag || p->maxTries != p0.maxTries ||
            p->checkAzFocus != p0.checkAzFocus || p->gaussFlag != p0.gaussFlag ||
            p->azDefocusThresh != p0.azDefocusThresh || p->scaleFactor != p0.scaleFactor)
            return sb_ctx_fail(c, SB_ERR_ARG,
                               "pair %d: the flags (noComplex, hanning, tries, checkAzFocus, gauss, azDefocusThresh, "
                               "scaleFactor) must be the same for every pair of a batch", k);
        total += (int64_t)p->nR * p->nA;
    }
    if (total > (int64_t)1 << 30) return sb_ctx_fail(c, SB_ERR_ARG, "batch grid too large");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    cudaEventRecord(c->ev[0], c->stream);
    for (int k = 0; k < 8; ++k) c->stage[k] = 0.f;

    // ---- bucket order and atlases
    std::vector<int> order(nPairs);
    for (int k = 0; k < nPairs; ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [P](int x, int y) {
        return P[x].wR != P[y].wR ? P[x].wR < P[y].wR : P[x].wRa < P[y].wRa;
    });
    const size_t elem = I1[0].sampleType == SB_CFLOAT32 ? 8 : 4;
    int width[2] = {0, 0};
    std::vector<int64_t> rowOff[2] = {std::vector<int64_t>(nPairs), std::vector<int64_t>(nPairs)};
    int64_t height[2] = {0, 0};
    for (int q = 0; q < nPairs; ++q) {
        const int k = order[q];
        const sb_image* im[2] = {&I1[k], &I2[k]};
        for (int i = 0; i < 2; ++i) {
            width[i] = im[i]->nr > width[i] ? im[i]->nr : width[i];
            rowOff[i][k] = height[i];
            height[i] += im[i]->na;
        }
    }
    if (height[0] >= ((int64_t)1 << 31) || height[1] >= ((int64_t)1 << 31))
        return sb_ctx_fail(c, SB_ERR_ARG, "batch images too tall for one atlas");
    cudaError_t e;
    char* atlas[2];
    for (int i = 0; i < 2; ++i) {
        atlas[i] = (char*)sb_ctx_buf(c, i ? "atlas2" : "atlas1", (size_t)width[i] * height[i] * elem, &e);
        if (!atlas[i]) return sb_ctx_cuda(c, e, "cudaMalloc(atlas)");
    }
    for (int k = 0; k < nPairs; ++k) {
        const sb_image* im[2] = {&I1[k], &I2[k]};
        for (int i = 0; i < 2; ++i) {
            const size_t pitch = (size_t)width[i] * elem, rowB = (size_t)im[i]->nr * elem;
            CK(cudaMemcpy2DAsync(atlas[i] + (size_t)rowOff[i][k] * pitch, pitch, im[i]->data, rowB, rowB,
                                 (size_t)im[i]->na, im[i]->onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                 c->stream),
               "atlas copy");
        }
    }
    // ---- plans of every pair, offset into the atlases; complex lists per bucket
    const int n = (int)total;
    std::vector<int> gStart(nPairs);
    std::vector<Bucket> buckets;
    {
        int g = 0;
        for (int q = 0; q < nPairs; ++q) {
            const int k = order[q];
            const sb_track_params* p = &P[k];
            if (buckets.empty() || buckets.back().wR != p->wR || buckets.back().wRa != p->wRa) {
                Bucket b;
                b.wR = p->wR;
                b.wRa = p->wRa;
                b.pFirst = q;
                b.g0 = g;
                buckets.push_back(b);
            }
            gStart[k] = g;
            g += p->nR * p->nA;
            buckets.back().pLast = q + 1;
            buckets.back().g1 = g;
        }
    }
    const int nBk = (int)buckets.size();
    PointPlan* dplan = (PointPlan*)sb_ctx_buf(c, "plan", sizeof(PointPlan) * n, &e);
    PointRec* drec = (PointRec*)sb_ctx_buf(c, "rec", sizeof(PointRec) * n, &e);
    int* dclist = (int*)sb_ctx_buf(c, "clist", sizeof(int) * (n + 1), &e);
    int* dlist = (int*)sb_ctx_buf(c, "list", sizeof(int) * (n + 1), &e);
    int* dpairOf = (int*)sb_ctx_buf(c, "pairOf", sizeof(int) * n, &e);
    FitJob* dfit = (FitJob*)sb_ctx_buf(c, "fit", sizeof(FitJob) * (n + 1), &e);
    unsigned long long* dstats = (unsigned long long*)sb_ctx_buf(c, "stats", sizeof(unsigned long long) * 8 * nPairs, &e);
    float* dR = (float*)sb_ctx_buf(c, "offR", sizeof(float) * n, &e);
    float* dA = (float*)sb_ctx_buf(c, "offA", sizeof(float) * n, &e);
    float* dC = (float*)sb_ctx_buf(c, "corr", sizeof(float) * n, &e);
    float* dZ = (float*)sb_ctx_buf(c, "azd", sizeof(float) * n, &e);
    uint8_t* dT = (uint8_t*)sb_ctx_buf(c, "type", n, &e);
    int* dkey = (int*)sb_ctx_buf(c, "listKey", sizeof(int) * (n + 1), &e);
    int* dpart = (int*)sb_ctx_buf(c, "partScratch", sizeof(int) * partition_scratch_ints(n, PART_KMAX), &e);
    int* dAz = (int*)sb_ctx_buf(c, "azEff", sizeof(int) * n, &e);
    if (!dplan || !drec || !dclist || !dlist || !dpairOf || !dfit || !dstats || !dR || !dA || !dC || !dZ || !dT ||
        !dkey || !dpart || !dAz)
        return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
    // Plans: on the device for a polynomial shift (each complex candidate keyed
    // by its bucket), on the host for an offset grid (its holes carry r2/a2
    // over from point to point); then one ordered partition by bucket gives
    // every bucket's complex list, in point order.  More buckets than the
    // partition takes: every pair planned on the host.
    const bool devBuckets = nBk <= PART_KMAX;
    std::vector<std::vector<PointPlan>> hostPlans;  // alive until the stream has copied them
    std::vector<std::vector<int>> hostKeys, hostPairs;
    std::vector<int> clist;
    for (int bi = 0; bi < nBk; ++bi) {
        for (int q = buckets[bi].pFirst; q < buckets[bi].pLast; ++q) {
            const int k = order[q];
            const sb_track_params* p = &P[k];
            const int m = p->nR * p->nA, g = gStart[k];
            if (devBuckets && p->polyShift != 0) {
                PlanArgs pa;
                memset(&pa, 0, sizeof(pa));
                pa.rStart = p->rStart; pa.aStart = p->aStart; pa.deltaR = p->deltaR; pa.deltaA = p->deltaA;
                pa.nR = p->nR; pa.nA = p->nA;
                pa.wR = p->wR; pa.wA = p->wA; pa.wRa = p->wRa; pa.wAa = p->wAa;
                pa.scaleFactor = p->scaleFactor;
                pa.noComplex = p->noComplex;
                for (int t = 0; t < 3; ++t) {
                    pa.rPoly[t] = p->rShiftPoly[t];
                    pa.aPoly[t] = p->aShiftPoly[t];
                }
                pa.nr1 = I1[k].nr; pa.na1 = I1[k].na; pa.nr2 = I2[k].nr; pa.na2 = I2[k].na;
                if (p->mask) {  // one buffer, reused in stream order
                    const size_t mb = (size_t)p->mask->nr * p->mask->na;
                    uint8_t* dm = (uint8_t*)sb_ctx_buf(c, "mask", mb, &e);
                    if (!dm) return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
                    CK(cudaMemcpyAsync(dm, p->mask->mask, mb, cudaMemcpyHostToDevice, c->stream), "mask");
                    pa.mask = dm;
                    pa.mR0 = p->mask->r0; pa.mA0 = p->mask->a0; pa.mNr = p->mask->nr; pa.mNa = p->mask->na;
                    pa.mNrl = p->mask->nrl; pa.mNal = p->mask->nal;
                }
                pa.a1Off = (int)rowOff[0][k];
                pa.a2Off = (int)rowOff[1][k];
                pa.keyValue = bi;
                pa.pairOf = dpairOf + g;
                pa.pairId = k;
                CK(launch_plan_poly(pa, dplan + g, dkey + g, c->stream), "plan_poly");
                c->launches++;
                continue;
            }
            std::vector<PointPlan> pl;
            std::vector<int> cl;
            plan_strack(p, I1[k].nr, I1[k].na, I2[k].nr, I2[k].na, pl, cl);
            for (PointPlan& x : pl) {
                x.a1 += (int)rowOff[0][k];
                x.a2 += (int)rowOff[1][k];
            }
            if (devBuckets) {
                std::vector<int> key((size_t)m, -1);
                for (int v : cl) key[(size_t)v] = bi;
                hostKeys.push_back(std::move(key));
                CK(cudaMemcpyAsync(dkey + g, hostKeys.back().data(), sizeof(int) * m, cudaMemcpyHostToDevice,
                                   c->stream),
                   "keys");
            } else {
                for (int v : cl) clist.push_back(g + v);
            }
            hostPairs.push_back(std::vector<int>((size_t)m, k));
            CK(cudaMemcpyAsync(dpairOf + g, hostPairs.back().data(), sizeof(int) * m, cudaMemcpyHostToDevice,
                               c->stream),
               "pairOf");
            hostPlans.push_back(std::move(pl));
            CK(cudaMemcpyAsync(dplan + g, hostPlans.back().data(), sizeof(PointPlan) * m, cudaMemcpyHostToDevice,
                               c->stream),
               "plan");
        }
        if (!devBuckets) buckets[bi].l1 = (int)clist.size();
    }
    if (devBuckets) {
        CK(launch_partition(dkey, nullptr, n, nBk, dclist, dpart, c->stream), "partition");
        c->launches += 3;
        std::vector<int> keyOff((size_t)nBk + 1);
        CK(cudaMemcpyAsync(keyOff.data(), dpart + partition_keyoff_at(n, nBk), sizeof(int) * (nBk + 1),
                           cudaMemcpyDeviceToHost, c->stream),
           "offsets");
        CK(cudaStreamSynchronize(c->stream), "sync");
        for (int bi = 0; bi < nBk; ++bi) {
            buckets[bi].l0 = keyOff[(size_t)bi];
            buckets[bi].l1 = keyOff[(size_t)bi + 1];
        }
    } else {
        int l = 0;
        for (int bi = 0; bi < nBk; ++bi) {  // l0 of each bucket: where the previous one ended
            buckets[bi].l0 = l;
            l = buckets[bi].l1;
        }
        if (!clist.empty())
            CK(cudaMemcpyAsync(dclist, clist.data(), sizeof(int) * clist.size(), cudaMemcpyHostToDevice, c->stream),
               "clist");
        CK(cudaStreamSynchronize(c->stream), "sync");
    }
    CK(cudaMemsetAsync(dstats, 0, sizeof(unsigned long long) * 8 * nPairs, c->stream), "memset");
    cudaEventRecord(c->ev[1], c->stream);
    CK(launch_rec_init(drec, n, c->stream), "rec_init");
    c->launches++;

    const int form = c->form;
    // per-bucket complex-stage events and try counts, read after the call
    BatchEvents bev(2 * nBk);
    if (!bev.ok()) return sb_ctx_fail(c, SB_ERR_CUDA, "event creation failed");
    std::vector<char> cmplxRan((size_t)nBk, 0);
    int* dStageCnt = (int*)sb_ctx_buf(c, "stageCnt", sizeof(int) * 3 * nBk, &e);
    if (!dStageCnt) return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
    CK(cudaMemsetAsync(dStageCnt, 0, sizeof(int) * 3 * nBk, c->stream), "memset");
    int* dTcErr = (int*)sb_ctx_buf(c, "tcErr", sizeof(int), &e);
    if (!dTcErr) return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
    CK(cudaMemsetAsync(dTcErr, 0, sizeof(int), c->stream), "memset");
    c->lastForm = SB_FORM_FP32;
    constexpr int kPeakChunk = 1 << 19;
    for (int bi = 0; bi < nBk; ++bi) {
        const Bucket& b = buckets[bi];
        const sb_track_params* p = &P[order[b.pFirst]];  // windows and flags of the bucket
        const int W = p->wR, WA = p->wRa;
        const int nB = b.g1 - b.g0, nC = b.l1 - b.l0;
        // ---- complex stage over the bucket's complex list
        if (nC > 0) {
            CmplxArgs a;
            memset(&a, 0, sizeof(a));
            a.img1 = atlas[0];
            a.img2 = atlas[1];
            a.nr1 = width[0]; a.na1 = (int)height[0]; a.nr2 = width[1]; a.na2 = (int)height[1];
            a.sampleType = I1[0].sampleType;
            a.byteOrder = I1[0].byteOrder;
            a.plan = dplan;
            a.nList = nC;
            a.hanning = p->hanningFlag ? hanning_table(c, W) : nullptr;
            a.hanCorr = p->hanningFlag ? 1.5 : 1.0;
            a.twW = tw_table(c, W);
            a.tau = tau_table(c, W);
            a.osA = osA_table(c);
            a.osD = osD_table(c);
            a.gauss = p->gaussFlag ? 1 : 0;
            a.azThresh = p->azDefocusThresh;
            a.checkAzFocus = p->checkAzFocus;
            a.noComplex = p->noComplex;
            a.rec = drec;
            if (!a.twW || !a.tau || !a.osA || !a.osD || (p->hanningFlag && !a.hanning))
                return sb_ctx_fail(c, SB_ERR_NOMEM, "table allocation failed");
            const bool tcForm = form == SB_FORM_SPLIT_BF16 && cmplx_tc_supported(W) && !p->gaussFlag && c->smMajor >= 10;
            if (tcForm) {
                a.tcErr = dTcErr;
                c->lastForm = SB_FORM_SPLIT_BF16;
            }
            int cthreads = 0, bpsm = 0;
            complex_shape(c, W, tcForm, &cthreads, &bpsm);
            if (bpsm <= 0) return sb_ctx_fail(c, SB_ERR_CUDA, "complex kernel cannot be resident (W=%d)", W);
            PeakJob* dpeak = nullptr;
            if (!p->gaussFlag) {
                const size_t pc = nC < kPeakChunk ? (size_t)nC : (size_t)kPeakChunk;
                dpeak = (PeakJob*)sb_ctx_buf(c, "peakjob", pc * sizeof(PeakJob), &e);
                if (!dpeak) return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
            }
            cudaEventRecord(bev[2 * bi], c->stream);
            for (int off = 0; off < nC; off += kPeakChunk) {
                const int cnt = nC - off < kPeakChunk ? nC - off : kPeakChunk;
                CmplxArgs ak = a;
                ak.list = dclist + b.l0 + off;
                ak.fit = dfit + off;
                ak.nList = cnt;
                ak.peak = dpeak;
                const int nCta = c->numSM * bpsm < cnt ? c->numSM * bpsm : cnt;
                if (tcForm)
                    CK(launch_strack_cmplx_tc(ak, nCta, c->stream), "strack_cmplx_tc");
                else
                    CK(launch_strack_cmplx(W, ak, nCta, c->stream, cthreads), "strack_cmplx");
                c->launches++;
                if (dpeak) {
                    PeakArgs pk;
                    pk.peak = dpeak;
                    pk.nList = cnt;
                    pk.W = W;
                    pk.hanCorr = a.hanCorr;
                    pk.osD = a.osD;
                    pk.rec = drec;
                    pk.fit = dfit + off;
                    CK(launch_strack_peak(pk, c->numSM, c->stream), "strack_peak");
                    c->launches++;
                }
            }
            FitArgs f = make_fit_args(p, dfit, nC, 0, drec);
            CK(launch_strack_fit(f, c->stream), "strack_fit");
            c->launches++;
            cudaEventRecord(bev[2 * bi + 1], c->stream);
            cmplxRan[bi] = 1;
            c->stage[5] += (float)nC;
        }
        // ---- amplitude tries over the bucket's points
        WalkParams w;
        w.wR = p->wR; w.wA = p->wA; w.wRa = p->wRa; w.wAa = p->wAa;
        w.noComplex = p->noComplex;
        w.maxTries = p->maxTries;
        const bool ownAz = (p->wRa == p->wR && p->wAa == p->wA);
        PointPlan* bplan = dplan + b.g0;
        PointRec* brec = drec + b.g0;
        for (int stage = 1; stage <= 2 && stage <= p->maxTries; ++stage) {
            CK(launch_select(bplan, brec, nB, w, stage, dkey, c->stream), "select");
            CK(launch_partition(dkey, nullptr, nB, 1, dlist, dpart, c->stream), "partition");
            c->launches += 4;
            // the try's list length stays on the device (no host round trip)
            const int* dCnt = dpart + partition_keyoff_at(nB, 1) + 1;
            CK(cudaMemcpyAsync(dStageCnt + 3 * bi + stage, dCnt, sizeof(int), cudaMemcpyDeviceToDevice, c->stream),
               "count");
            const int Ws = WA * (stage == 1 ? 1 : LA);
            // as in sb_strack: the length is read back only for the staged kernel
            const bool onChip = amps_supported(Ws);
            int cnt = nB;  // upper bound
            if (!onChip) {
                CK(cudaMemcpyAsync(&cnt, dCnt, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "count");
                CK(cudaStreamSynchronize(c->stream), "sync");
                if (cnt == 0) continue;
            }
            const bool needFill = !ownAz && !(p->noComplex && stage == 1);
            if (needFill) {  // azShift carries over within a pair, from 0 at its first point
                for (int q = b.pFirst; q < b.pLast; ++q) {
                    const int k = order[q];
                    CK(launch_az_fill(drec + gStart[k], P[k].nR * P[k].nA, dAz + (gStart[k] - b.g0), c->stream),
                       "az_fill");
                    c->launches++;
                }
            }
            AmpArgs a;
            memset(&a, 0, sizeof(a));
            a.img1 = atlas[0];
            a.img2 = atlas[1];
            a.nr1 = width[0]; a.na1 = (int)height[0]; a.nr2 = width[1]; a.na2 = (int)height[1];
            a.sampleType = I1[0].sampleType;
            a.byteOrder = I1[0].byteOrder;
            a.plan = bplan;
            a.list = dlist;
            a.nList = cnt;
            a.nListDev = onChip ? dCnt : nullptr;
            a.stage = stage;
            a.s = stage == 1 ? 1 : LA;
            a.wR = p->wR; a.wA = p->wA; a.wRa = p->wRa; a.wAa = p->wAa;
            a.noComplex = p->noComplex;
            a.azThresh = p->azDefocusThresh;
            a.checkAzFocus = p->checkAzFocus;
            a.azEff = needFill ? dAz : nullptr;
            a.twWs = tw_table(c, Ws);
            a.tw2Ws = tw_table(c, 2 * Ws);
            a.tau = tau_table(c, Ws);
            a.osA = osA_table(c);
            a.osD = osD_table(c);
            a.gauss = p->gaussFlag ? 1 : 0;
            a.rec = brec;
            a.fit = dfit;
            int nCta = c->numSM * (onChip ? amps_ctas(c, Ws) : amp_blocks_per_sm(Ws));
            if (nCta > cnt) nCta = cnt;
            if (nCta < 1) return sb_ctx_fail(c, SB_ERR_CUDA, "amplitude kernel cannot be resident (Ws=%d)", Ws);
            if (!onChip) {
                a.scratchPerCta = amp_scratch_elems(Ws);
                a.scratch = (float2*)sb_ctx_buf(c, "ampScratch", sizeof(float2) * a.scratchPerCta * nCta, &e);
            }
            if ((!onChip && !a.scratch) || !a.twWs || !a.tw2Ws || !a.tau || !a.osA || !a.osD)
                return sb_ctx_fail(c, SB_ERR_NOMEM, "amplitude workspace allocation failed");
            if (onChip)
                CK(launch_strack_amps(Ws, a, nCta, c->stream), "strack_amps");
            else
                CK(launch_strack_amp(Ws, a, nCta, c->stream), "strack_amp");
            c->launches++;
            FitArgs f = make_fit_args(p, dfit, cnt, stage, brec);
            f.nListDev = onChip ? dCnt : nullptr;
            CK(launch_strack_fit(f, c->stream), "strack_fit");
            c->launches++;
        }
        CK(launch_finalize(bplan, brec, nB, w, p->scaleFactor, dR + b.g0, dA + b.g0, dC + b.g0, dZ + b.g0, dT + b.g0,
                           dstats, c->stream, dpairOf + b.g0),
           "finalize");
        c->launches++;
    }
    cudaEventRecord(c->ev[2], c->stream);
    // ---- outputs, per pair
    for (int k = 0; k < nPairs; ++k) {
        const size_t g = (size_t)gStart[k], m = (size_t)P[k].nR * P[k].nA;
        const int od = out[k].onDevice;
        if ((rc = out_copy(c, out[k].offR, dR + g, sizeof(float) * m, od)) != SB_OK) return rc;
        if ((rc = out_copy(c, out[k].offA, dA + g, sizeof(float) * m, od)) != SB_OK) return rc;
        if ((rc = out_copy(c, out[k].corr, dC + g, sizeof(float) * m, od)) != SB_OK) return rc;
        if (out[k].azd && (rc = out_copy(c, out[k].azd, dZ + g, sizeof(float) * m, od)) != SB_OK) return rc;
        if ((rc = out_copy(c, out[k].type, dT + g, m, od)) != SB_OK) return rc;
    }
    std::vector<unsigned long long> st((size_t)8 * nPairs);
    CK(cudaMemcpyAsync(st.data(), dstats, sizeof(unsigned long long) * 8 * nPairs, cudaMemcpyDeviceToHost, c->stream),
       "stats");
    int tcBad = 0;
    CK(cudaMemcpyAsync(&tcBad, dTcErr, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "tcErr");
    std::vector<int> stageCnt((size_t)3 * nBk);
    CK(cudaMemcpyAsync(stageCnt.data(), dStageCnt, sizeof(int) * 3 * nBk, cudaMemcpyDeviceToHost, c->stream),
       "counts");
    cudaEventRecord(c->ev[3], c->stream);
    CK(cudaStreamSynchronize(c->stream), "strack_batch");
    for (int bi = 0; bi < nBk; ++bi) {
        if (cmplxRan[bi]) {
            float t0 = 0;
            cudaEventElapsedTime(&t0, bev[2 * bi], bev[2 * bi + 1]);
            c->stage[0] += t0;
        }
        c->stage[6] += (float)stageCnt[(size_t)3 * bi + 1];
        c->stage[7] += (float)stageCnt[(size_t)3 * bi + 2];
    }
    if (tcBad) return sb_ctx_fail(c, SB_ERR_TIMEOUT, "split-BF16 complex stage: a tensor-core wait timed out");
    for (int k = 0; k < nPairs; ++k) {
        const unsigned long long* s = &st[(size_t)8 * k];
        out[k].nComplex = (int64_t)s[0];
        out[k].nAmp = (int64_t)s[1];
        out[k].nAmpL = (int64_t)s[2];
        out[k].nFail = (int64_t)s[3];
        out[k].nAttempted = (int64_t)P[k].nR * P[k].nA - (int64_t)s[4];
    }
    cudaEventElapsedTime(&c->timing[0], c->ev[0], c->ev[3]);
    cudaEventElapsedTime(&c->timing[1], c->ev[0], c->ev[1]);
    cudaEventElapsedTime(&c->timing[2], c->ev[1], c->ev[2]);
    cudaEventElapsedTime(&c->timing[3], c->ev[2], c->ev[3]);
    return SB_OK;
}
