// exp / log / sin for float32 and float64.
//
// NaN inputs propagate quieted (glibc returns x + x / x * x for them). The
// finite-input evaluation calls CUDA's libdevice routines; the correctly
// rounded replacements live in the same functions once they pass the
// exhaustive float32 sweep and the float64 random sweeps in tests/.
#pragma once
#include "ionp_scalar.cuh"

namespace ionp {

__device__ __forceinline__ float cr_expf(float x) { return isnan_f(x) ? quiet_f(x) : expf(x); }
__device__ __forceinline__ float cr_logf(float x) {
    if (isnan_f(x)) return quiet_f(x);
    if (x < 0.0f) return dnan_f();
    return logf(x);
}
__device__ __forceinline__ float cr_sinf(float x) {
    if (isnan_f(x)) return quiet_f(x);
    if (isinf(x)) return dnan_f();
    return sinf(x);
}
__device__ __forceinline__ double cr_exp(double x) { return isnan_d(x) ? quiet_d(x) : exp(x); }
__device__ __forceinline__ double cr_log(double x) {
    if (isnan_d(x)) return quiet_d(x);
    if (x < 0.0) return dnan_d();
    return log(x);
}
__device__ __forceinline__ double cr_sin(double x) {
    if (isnan_d(x)) return quiet_d(x);
    if (isinf(x)) return dnan_d();
    return sin(x);
}

}  // namespace ionp
