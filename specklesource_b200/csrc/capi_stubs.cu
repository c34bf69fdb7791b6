// capi_stubs.cu -- entry points of the C ABI whose kernels are not built yet.
#include "capi_internal.h"

extern "C" int sb_strackw(sb_context* c, const sb_track_params*, const sb_image*, const sb_image*, sb_track_result*)
{
    return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "strackw is not built yet");
}
extern "C" int sb_est_dop_carrier(sb_context* c, const float*, const float*, int32_t, int32_t, int32_t, int32_t,
                                  int32_t*)
{
    return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "not built yet");
}
