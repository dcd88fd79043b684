// Correctly rounded exp / log / sin for float32 and float64.
//
// The reference computes these with the platform libm (glibc on Linux:
// ionp-core/src/ufunc.rs:4237-4367 call f32::exp/ln/sin and f64::...),
// whose float32 results are not always correctly rounded (glibc's expf is
// up to ~0.5000001 ULP off). This engine returns the correctly rounded
// result, which equals glibc's wherever glibc is correctly rounded and is
// within 1 ULP of it elsewhere.
//
// float32: y = the double-precision function at the float argument (CUDA's
// exp/log/sin, documented maximum errors 1 / 1 / 2 ULP in double, i.e. a
// relative error < 2^-51). If y*(1-2^-49) and y*(1+2^-49) round to the same
// float, that float is the correctly rounded result; otherwise (about one
// argument in 10^7) the value is recomputed in double-double (~2^-100) and
// rounded from there.
// float64: double-double evaluation (ionp_dd.cuh) rounded to double.
// NaN arguments propagate quieted; the domain errors return the x86 default
// NaN like glibc.
#pragma once
#include "ionp_scalar.cuh"
#include "ionp_dd.cuh"

namespace ionp {

__device__ __forceinline__ bool round_pins(double y, float* out) {
    const double E = 0x1p-49;
    float a = __double2float_rn(y * (1.0 - E));
    float b = __double2float_rn(y * (1.0 + E));
    *out = a;
    return __float_as_uint(a) == __float_as_uint(b);
}

static __device__ __noinline__ float expf_slow(float x) { return dd::dd_to_float(dd::exp_dd((double)x)); }
static __device__ __noinline__ float logf_slow(float x) { return dd::dd_to_float(dd::log_dd((double)x)); }
static __device__ __noinline__ float sinf_slow(float x) { return dd::dd_to_float(dd::sin_dd((double)x)); }

__device__ __forceinline__ float cr_expf(float x) {
    if (isnan_f(x)) return quiet_f(x);
    if (x > 89.0f) return __uint_as_float(0x7F800000u);
    if (x < -104.0f) return 0.0f;
    float f;
    if (round_pins(exp((double)x), &f)) return f;
    return expf_slow(x);
}
__device__ __forceinline__ float cr_logf(float x) {
    if (isnan_f(x)) return quiet_f(x);
    if (x < 0.0f) return dnan_f();
    if (x == 0.0f) return __uint_as_float(0xFF800000u);
    if (isinf(x)) return x;
    float f;
    if (round_pins(log((double)x), &f)) return f;
    return logf_slow(x);
}
__device__ __forceinline__ float cr_sinf(float x) {
    if (isnan_f(x)) return quiet_f(x);
    if (isinf(x)) return dnan_f();
    float f;
    if (round_pins(sin((double)x), &f)) return f;
    return sinf_slow(x);
}

__device__ __forceinline__ double cr_exp(double x) {
    if (isnan_d(x)) return quiet_d(x);
    if (x > 709.8) return __longlong_as_double(0x7FF0000000000000ll);
    if (x < -745.2) return 0.0;
    return dd::exp_dd(x).hi;
}
__device__ __forceinline__ double cr_log(double x) {
    if (isnan_d(x)) return quiet_d(x);
    if (x < 0.0) return dnan_d();
    if (x == 0.0) return __longlong_as_double((long long)0xFFF0000000000000ull);
    if (isinf(x)) return x;
    return dd::log_dd(x).hi;
}
__device__ __forceinline__ double cr_sin(double x) {
    if (isnan_d(x)) return quiet_d(x);
    if (isinf(x)) return dnan_d();
    if (x == 0.0) return x;
    return dd::sin_dd(x).hi;
}

}  // namespace ionp
