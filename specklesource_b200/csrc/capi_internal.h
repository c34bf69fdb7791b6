// capi_internal.h -- the context object behind sb_context and helpers shared
// by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>

#include "../../include/speckle_b200.h"

struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
};

constexpr int SB_MAX_BANDS = 32;  // equals sbk::SB_BANDS_MAX

struct sb_context {
    int device = 0;
    int numSM = 0;
    int smMajor = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    float timing[4] = {0, 0, 0, 0};
    float stage[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    cudaEvent_t sev[16] = {};  // per-stage event pairs
    cudaStream_t copyStream = nullptr;  // host -> device image bands
    cudaEvent_t chunkEv[SB_MAX_BANDS] = {};  // band k of both images is resident
    int nsev = 0;
    int64_t launches = 0;
    std::string err;
    std::map<std::string, DevBuf> bufs;   // grown on demand, reused across calls
    std::map<std::string, void*> tables;  // constant tables
    size_t tableBytes = 0;                // device bytes of the tables
    cudaError_t noallocPrep = cudaSuccess;  // result of sb_noalloc_prepare at creation
    long long waitNaps = 1LL << 26;  // bounded device waits: 64 ns naps per wait (~4 s)
    int form = SB_FORM_FP32;         // transform form of the complex stage (sb_set_form)
    // launch shapes set by sb_set_tuning (0: the library default); index by
    // window: 16, 24, 32, 48, 64 -> 0..4
    int tuneCmplxThreads[5] = {0, 0, 0, 0, 0};
    int tuneCmplxCtas[5] = {0, 0, 0, 0, 0};
    int tuneTcCtas = 0;
    int tuneAmpsCtas[5] = {0, 0, 0, 0, 0};
    int lastForm = SB_FORM_FP32;     // form the last sb_strack call's complex stage ran
};

int sb_ctx_fail(sb_context* c, int code, const char* fmt, ...);
int sb_ctx_cuda(sb_context* c, cudaError_t e, const char* what);
void* sb_ctx_buf(sb_context* c, const char* name, size_t bytes, cudaError_t* err);
int sb_image_to_device(sb_context* c, const sb_image* im, const char* name, const void** dptr);
const float2* tw_table(sb_context* c, int N);
// Loads the allocation-free entry point's kernels and its file-scope workspace
// on the current device (noalloc.cu).
cudaError_t sb_noalloc_prepare();
