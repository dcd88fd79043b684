// Device-side scalar semantics of anionpy's ufunc engine.
//
// Every function here reproduces, bit for bit, what the reference's Rust CPU
// path computes for one element on an x86-64 host:
//   * IEEE binary ops with x86 SSE NaN rules: a NaN operand propagates
//     quieted (the first NaN operand wins), an invalid op on non-NaN operands
//     gives the x86 default NaN (sign bit set). GPU hardware returns a
//     canonical NaN instead, so NaN results are rebuilt here explicitly.
//   * half::f16 arithmetic = to_f32, f32 op, from_f32 (round to nearest even).
//   * the per-kind scalar op tables of ionp-core/src/ufunc.rs:2170-2575,
//     remainder/fmod (4015-4128) and the buffer casts of
//     ionp-core/src/buffer.rs:64-330.
// All arithmetic uses the explicitly rounded intrinsics (__fadd_rn, ...) and
// the library is built with -fmad=false, so nothing is contracted into FMA.
#pragma once
#include <cstdint>
#include <cuda_fp16.h>

namespace ionp {

enum : int {
    DT_BOOL = 0, DT_I8, DT_I16, DT_I32, DT_I64, DT_U8, DT_U16, DT_U32, DT_U64, DT_F16, DT_F32, DT_F64, DT_COUNT
};

enum : int {
    OP_ADD = 0, OP_SUBTRACT, OP_MULTIPLY, OP_DIVIDE, OP_MAXIMUM, OP_MINIMUM,
    OP_GREATER, OP_GREATER_EQUAL, OP_LESS, OP_LESS_EQUAL, OP_EQUAL, OP_NOT_EQUAL,
    OP_LOGICAL_AND, OP_LOGICAL_OR, OP_LOGICAL_XOR,
    OP_BITWISE_AND, OP_BITWISE_OR, OP_BITWISE_XOR,
    OP_FLOOR_DIVIDE, OP_LEFT_SHIFT, OP_RIGHT_SHIFT,
    OP_REMAINDER = 32, OP_FMOD = 33,
    OP_NEGATIVE = 64, OP_ABSOLUTE = 65, OP_INVERT = 66, OP_LOGICAL_NOT = 67,
    OP_SQRT = 80, OP_EXP = 81, OP_LOG = 82, OP_SIN = 83, OP_COS = 84,
};

// FPE category bits (ionp-core/src/fpe.rs:43-48)
enum : uint32_t { FPE_DIVIDE = 1u, FPE_OVER = 2u, FPE_UNDER = 4u, FPE_INVALID = 8u };

typedef uint16_t h16;  // float16 bits

// ---------------------------------------------------------------------------
// bit helpers, NaN rules
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t fb(float f) { return __float_as_uint(f); }
__device__ __forceinline__ float bf(uint32_t u) { return __uint_as_float(u); }
__device__ __forceinline__ uint64_t db(double d) { return (uint64_t)__double_as_longlong(d); }
__device__ __forceinline__ double bd(uint64_t u) { return __longlong_as_double((long long)u); }

// Sign-bit flips / clears done as integer ops in PTX: the compiler must not
// turn them into floating-point negate/abs, which canonicalise NaN payloads.
__device__ __forceinline__ float neg_bits(float x) {
    uint32_t r;
    asm("xor.b32 %0, %1, 0x80000000;" : "=r"(r) : "r"(__float_as_uint(x)));
    return __uint_as_float(r);
}
__device__ __forceinline__ float abs_bits(float x) {
    uint32_t r;
    asm("and.b32 %0, %1, 0x7FFFFFFF;" : "=r"(r) : "r"(__float_as_uint(x)));
    return __uint_as_float(r);
}
__device__ __forceinline__ double neg_bits(double x) {
    uint64_t r;
    asm("xor.b64 %0, %1, 0x8000000000000000;" : "=l"(r) : "l"((uint64_t)__double_as_longlong(x)));
    return __longlong_as_double((long long)r);
}
__device__ __forceinline__ double abs_bits(double x) {
    uint64_t r;
    asm("and.b64 %0, %1, 0x7FFFFFFFFFFFFFFF;" : "=l"(r) : "l"((uint64_t)__double_as_longlong(x)));
    return __longlong_as_double((long long)r);
}

__device__ __forceinline__ bool isnan_f(float x) { return (fb(x) & 0x7FFFFFFFu) > 0x7F800000u; }
__device__ __forceinline__ bool isnan_d(double x) { return (db(x) & 0x7FFFFFFFFFFFFFFFull) > 0x7FF0000000000000ull; }
__device__ __forceinline__ float quiet_f(float x) { return bf(fb(x) | 0x00400000u); }
__device__ __forceinline__ double quiet_d(double x) { return bd(db(x) | 0x0008000000000000ull); }
__device__ __forceinline__ float dnan_f() { return bf(0xFFC00000u); }
__device__ __forceinline__ double dnan_d() { return bd(0xFFF8000000000000ull); }

__device__ __forceinline__ float nan2(float x, float y) {
    if (isnan_f(x)) return quiet_f(x);
    if (isnan_f(y)) return quiet_f(y);
    return dnan_f();
}
__device__ __forceinline__ double nan2(double x, double y) {
    if (isnan_d(x)) return quiet_d(x);
    if (isnan_d(y)) return quiet_d(y);
    return dnan_d();
}

__device__ __forceinline__ float x_add(float x, float y) { float r = __fadd_rn(x, y); return isnan_f(r) ? nan2(x, y) : r; }
__device__ __forceinline__ float x_sub(float x, float y) { float r = __fsub_rn(x, y); return isnan_f(r) ? nan2(x, y) : r; }
__device__ __forceinline__ float x_mul(float x, float y) { float r = __fmul_rn(x, y); return isnan_f(r) ? nan2(x, y) : r; }
__device__ __forceinline__ float x_div(float x, float y) { float r = __fdiv_rn(x, y); return isnan_f(r) ? nan2(x, y) : r; }
__device__ __forceinline__ double x_add(double x, double y) { double r = __dadd_rn(x, y); return isnan_d(r) ? nan2(x, y) : r; }
__device__ __forceinline__ double x_sub(double x, double y) { double r = __dsub_rn(x, y); return isnan_d(r) ? nan2(x, y) : r; }
__device__ __forceinline__ double x_mul(double x, double y) { double r = __dmul_rn(x, y); return isnan_d(r) ? nan2(x, y) : r; }
__device__ __forceinline__ double x_div(double x, double y) { double r = __ddiv_rn(x, y); return isnan_d(r) ? nan2(x, y) : r; }

__device__ __forceinline__ float x_floor(float x) { return isnan_f(x) ? quiet_f(x) : floorf(x); }
__device__ __forceinline__ double x_floor(double x) { return isnan_d(x) ? quiet_d(x) : floor(x); }
__device__ __forceinline__ float x_sqrt(float x) { return isnan_f(x) ? quiet_f(x) : (x < 0.0f ? dnan_f() : __fsqrt_rn(x)); }
__device__ __forceinline__ double x_sqrt(double x) { return isnan_d(x) ? quiet_d(x) : (x < 0.0 ? dnan_d() : __dsqrt_rn(x)); }

// The common case of fmod, remainder and floor_divide without a branch:
// x finite, 2^-125 <= |y| <= 2^125 and |x / y| below 2^19 (float32) or 2^36
// (float64); quot_fast returns false for every other input, whose outputs
// t and m are then meaningless. p, the quotient from a reciprocal
// approximation scaled up by 2^-20 (2^-38), is at least |x / y| and less
// than |x / y| + 1 in magnitude:
//  float32: rcp.approx is within 1 ulp (2^-23 relative) and the two
//    products round by 2^-24 each, so the relative error of p is inside
//    (2^-20 - 2^-22, 2^-20 + 2^-22), below 2^-19 / |x / y|;
//  float64: the float32 reciprocal of y rounded to float32 is within
//    2^-22.4, one Newton step r1 = r0 + r0 (1 - y r0) squares that to
//    below 2^-44, and the two products round by 2^-53 each.
// So t = trunc(p) is the exact truncated quotient q or q + 1 in magnitude,
// and m = x - t y is exact in one fused multiply-add: it is the true
// remainder when t = q, and the true remainder less y (towards zero, with
// the other sign, never zero) when t is one too large; Sterbenz's lemma
// covers the |x| < |y| case, and otherwise m is a multiple of y's last
// place below |y|.
__device__ __forceinline__ bool quot_fast(float x, float y, float* t, float* m) {
    const uint32_t ax = fb(x) & 0x7FFFFFFFu, ay = fb(y) & 0x7FFFFFFFu;
    float rc;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rc) : "f"(y));
    const float p = __fmul_rn(__fmul_rn(x, rc), 1.0f + 0x1p-20f);
    *t = truncf(p);
    *m = __fmaf_rn(-*t, y, x);
    // 0x01000000 = 2^-125, 0x7E000000 = 2^125
    return (ax < 0x7F800000u) & (ay - 0x01000000u <= 0x7D000000u) & (fabsf(p) < 0x1p19f);
}
__device__ __forceinline__ bool quot_fast(double x, double y, double* t, double* m) {
    const uint64_t ax = db(x) & 0x7FFFFFFFFFFFFFFFull, ay = db(y) & 0x7FFFFFFFFFFFFFFFull;
    float r0f;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r0f) : "f"(__double2float_rn(y)));
    const double r0 = (double)r0f;
    const double r1 = __fma_rn(r0, __fma_rn(-y, r0, 1.0), r0);
    const double p = __dmul_rn(__dmul_rn(x, r1), 1.0 + 0x1p-38);
    *t = trunc(p);
    *m = __fma_rn(-*t, y, x);
    // 0x3820000000000000 = 2^-125, 0x47C0000000000000 = 2^125
    return (ax < 0x7FF0000000000000ull) & (ay - 0x3820000000000000ull <= 0x0FA0000000000000ull) & (fabs(p) < 0x1p36);
}
// glibc fmod semantics (what Rust's float `%` calls): NaN operands propagate,
// fmod(inf, y) and fmod(x, 0) are the default NaN, fmod(x, inf) = x.
// quot_fast's case inline: m, with y added back (x's sign) when t was one
// too large, which is exact. The rest out of line: for quotients below 2^23
// (2^52) q = trunc(fl(x / y)) is again the truncated quotient or one too
// large (rounding is monotone and every integer below 2^24 is
// representable) and the same repair applies; larger quotients take the
// library's fmod.
template <class F> static __device__ __noinline__ F x_fmod_slow(F x, F y) {
    if (isfinite(x) && isfinite(y) && y != (F)0) {
        F q;
        if constexpr (sizeof(F) == 4) q = truncf(__fdiv_rn(x, y));
        else q = trunc(__ddiv_rn(x, y));
        if (fabs(q) < (sizeof(F) == 4 ? (F)0x1p23 : (F)0x1p52)) {
            F r;
            if constexpr (sizeof(F) == 4) r = __fmaf_rn(-q, y, x);
            else r = __fma_rn(-q, y, x);
            if (r != (F)0 && signbit(r) != signbit(x)) r = r + copysign(y, x);
            return r == (F)0 ? copysign((F)0, x) : r;
        }
        if constexpr (sizeof(F) == 4) return fmodf(x, y);
        else return fmod(x, y);
    }
    if (x != x || y != y) return nan2(x, y);
    if (isinf(x) || y == (F)0) {
        if constexpr (sizeof(F) == 4) return dnan_f();
        else return dnan_d();
    }
    return x;  // y infinite, x finite
}
template <class F> __device__ __forceinline__ bool fmod_fast(F x, F y, F* r) {
    F t, m;
    const bool ok = quot_fast(x, y, &t, &m);
    const F v = (m != (F)0 && signbit(m) != signbit(x)) ? m + copysign(y, x) : m;
    *r = v == (F)0 ? copysign((F)0, x) : v;
    return ok;
}
template <class F> __device__ __forceinline__ F x_fmod(F x, F y) {
    F r;
    if (fmod_fast(x, y, &r)) return r;
    return x_fmod_slow(x, y);
}

// ---------------------------------------------------------------------------
// float16 / float32 / float64 conversions (half crate and x86 cvt rules)
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool isnan_h(h16 h) { return (h & 0x7C00u) == 0x7C00u && (h & 0x3FFu); }

__device__ __forceinline__ float h2f(h16 h) {
    if (isnan_h(h)) return bf(((uint32_t)(h & 0x8000u) << 16) | 0x7FC00000u | ((uint32_t)(h & 0x3FFu) << 13));
    return __half2float(__ushort_as_half(h));
}
__device__ __forceinline__ h16 f2h(float f) {
    uint32_t u = fb(f);
    if (isnan_f(f)) return (h16)(((u >> 16) & 0x8000u) | 0x7E00u | ((u >> 13) & 0x3FFu));
    return __half_as_ushort(__float2half_rn(f));
}
// Round-to-nearest-even conversion from double, straight (no f32 step).
__device__ __forceinline__ h16 d2h(double d) {
    uint64_t b = db(d);
    uint32_t sign = (uint32_t)((b >> 48) & 0x8000u);
    uint32_t ex = (uint32_t)((b >> 52) & 0x7FF);
    uint64_t man = b & 0xFFFFFFFFFFFFFull;
    if (ex == 0x7FF) return (h16)(man == 0 ? (sign | 0x7C00u) : (sign | 0x7E00u | (uint32_t)((man >> 42) & 0x3FFu)));
    if (ex == 0) return (h16)sign;
    int e = (int)ex - 1023;
    if (e > 15) return (h16)(sign | 0x7C00u);
    uint64_t m = man | (1ull << 52);
    if (e >= -14) {
        uint64_t q = m >> 42, rem = m & ((1ull << 42) - 1), half = 1ull << 41;
        if (rem > half || (rem == half && (q & 1))) q++;
        uint32_t he = (uint32_t)(e + 15);
        if (q == 2048) { q = 1024; he++; }
        if (he >= 31) return (h16)(sign | 0x7C00u);
        return (h16)(sign | (he << 10) | (uint32_t)(q & 0x3FFu));
    }
    int shift = 28 - e;
    if (shift > 60) return (h16)sign;
    uint64_t q = m >> shift, rem = m & ((1ull << shift) - 1), half = 1ull << (shift - 1);
    if (rem > half || (rem == half && (q & 1))) q++;
    return (h16)(sign | (uint32_t)q);
}
__device__ __forceinline__ double f2d(float f) {
    if (isnan_f(f)) {
        uint32_t u = fb(f);
        return bd(((uint64_t)(u & 0x80000000u) << 32) | 0x7FF8000000000000ull | ((uint64_t)(u & 0x7FFFFFu) << 29));
    }
    return (double)f;
}
__device__ __forceinline__ float d2f(double d) {
    if (isnan_d(d)) {
        uint64_t b = db(d);
        return bf(((uint32_t)(b >> 32) & 0x80000000u) | 0x7FC00000u | (uint32_t)((b >> 29) & 0x7FFFFFu));
    }
    return __double2float_rn(d);
}

// ---------------------------------------------------------------------------
// Casts: the reference's `cast_to` on one element (buffer.rs:64-330)
// ---------------------------------------------------------------------------
template <class I> struct ILim;
template <> struct ILim<int8_t> { static constexpr double lo = -128.0, hi = 127.0; };
template <> struct ILim<int16_t> { static constexpr double lo = -32768.0, hi = 32767.0; };
template <> struct ILim<int32_t> { static constexpr double lo = -2147483648.0, hi = 2147483647.0; };
template <> struct ILim<int64_t> { static constexpr double lo = -9223372036854775808.0, hi = 9223372036854775807.0; };
template <> struct ILim<uint8_t> { static constexpr double lo = 0.0, hi = 255.0; };
template <> struct ILim<uint16_t> { static constexpr double lo = 0.0, hi = 65535.0; };
template <> struct ILim<uint32_t> { static constexpr double lo = 0.0, hi = 4294967295.0; };
template <> struct ILim<uint64_t> { static constexpr double lo = 0.0, hi = 18446744073709551615.0; };

// Rust `x as iN`: saturating, NaN -> 0 (x is an exact double of the source)
template <class I> __device__ __forceinline__ I sat_cast(double x) {
    if (isnan_d(x)) return (I)0;
    if (x <= ILim<I>::lo) return (I)ILim<I>::lo;
    if (x >= ILim<I>::hi) return (I)(sizeof(I) == 8 ? (std::is_signed<I>::value ? (I)0x7FFFFFFFFFFFFFFFll : (I)~0ull) : (I)ILim<I>::hi);
    return (I)x;
}

// Storage type of each dtype code.
template <int D> struct DT;
template <> struct DT<DT_BOOL> { typedef uint8_t T; };
template <> struct DT<DT_I8> { typedef int8_t T; };
template <> struct DT<DT_I16> { typedef int16_t T; };
template <> struct DT<DT_I32> { typedef int32_t T; };
template <> struct DT<DT_I64> { typedef int64_t T; };
template <> struct DT<DT_U8> { typedef uint8_t T; };
template <> struct DT<DT_U16> { typedef uint16_t T; };
template <> struct DT<DT_U32> { typedef uint32_t T; };
template <> struct DT<DT_U64> { typedef uint64_t T; };
template <> struct DT<DT_F16> { typedef h16 T; };
template <> struct DT<DT_F32> { typedef float T; };
template <> struct DT<DT_F64> { typedef double T; };

__host__ __device__ constexpr int dt_size(int d) {
    return d == DT_BOOL || d == DT_I8 || d == DT_U8 ? 1 : d == DT_I16 || d == DT_U16 || d == DT_F16 ? 2
         : d == DT_I32 || d == DT_U32 || d == DT_F32 ? 4 : 8;
}
__host__ __device__ constexpr bool dt_is_float(int d) { return d == DT_F16 || d == DT_F32 || d == DT_F64; }
__host__ __device__ constexpr bool dt_is_sint(int d) { return d >= DT_I8 && d <= DT_I64; }
__host__ __device__ constexpr bool dt_is_uint(int d) { return d >= DT_U8 && d <= DT_U64; }

// cast<SD, DD>: value of dtype SD to dtype DD.
template <int SD, int DD> struct Cast {
    typedef typename DT<SD>::T S;
    typedef typename DT<DD>::T D;
    static __device__ __forceinline__ D go(S x) {
        if constexpr (SD == DD) {
            if constexpr (SD == DT_BOOL) return (D)(x != 0);
            else return x;
        } else if constexpr (SD == DT_BOOL) {
            if constexpr (DD == DT_F16) return (D)(x ? 0x3C00 : 0);
            else if constexpr (DD == DT_F32) return x ? 1.0f : 0.0f;
            else if constexpr (DD == DT_F64) return x ? 1.0 : 0.0;
            else return (D)(x ? 1 : 0);
        } else if constexpr (dt_is_sint(SD) || dt_is_uint(SD)) {
            if constexpr (DD == DT_BOOL) return (D)(x != 0);
            else if constexpr (DD == DT_F16) return d2h((double)x);
            else if constexpr (DD == DT_F32) return (float)x;
            else if constexpr (DD == DT_F64) return (double)x;
            else return (D)x;  // two's complement wrap
        } else {
            // float sources
            if constexpr (DD == DT_BOOL) {
                if constexpr (SD == DT_F16) return (D)((x & 0x7FFFu) != 0);
                else return (D)(x != 0);
            } else if constexpr (DD == DT_F16) {
                if constexpr (SD == DT_F32) return d2h(f2d(x));
                else return d2h(x);
            } else if constexpr (DD == DT_F32) {
                if constexpr (SD == DT_F16) return h2f(x);
                else return d2f(x);
            } else if constexpr (DD == DT_F64) {
                if constexpr (SD == DT_F16) return f2d(h2f(x));
                else return f2d(x);
            } else {
                double v;
                if constexpr (SD == DT_F16) v = (double)h2f(x);
                else v = (double)x;
                if constexpr (DD == DT_I8 || DD == DT_I16 || DD == DT_U8 || DD == DT_U16) return (D)(uint32_t)sat_cast<int32_t>(v);
                else return sat_cast<D>(v);
            }
        }
    }
};

// Runtime-dtype load converted to compute dtype CD (cast-on-load).
template <int CD> __device__ __forceinline__ typename DT<CD>::T load_cast(const void* base, int64_t idx, int sd) {
    switch (sd) {
        case DT_BOOL: return Cast<DT_BOOL, CD>::go(((const uint8_t*)base)[idx]);
        case DT_I8: return Cast<DT_I8, CD>::go(((const int8_t*)base)[idx]);
        case DT_I16: return Cast<DT_I16, CD>::go(((const int16_t*)base)[idx]);
        case DT_I32: return Cast<DT_I32, CD>::go(((const int32_t*)base)[idx]);
        case DT_I64: return Cast<DT_I64, CD>::go(((const int64_t*)base)[idx]);
        case DT_U8: return Cast<DT_U8, CD>::go(((const uint8_t*)base)[idx]);
        case DT_U16: return Cast<DT_U16, CD>::go(((const uint16_t*)base)[idx]);
        case DT_U32: return Cast<DT_U32, CD>::go(((const uint32_t*)base)[idx]);
        case DT_U64: return Cast<DT_U64, CD>::go(((const uint64_t*)base)[idx]);
        case DT_F16: return Cast<DT_F16, CD>::go(((const h16*)base)[idx]);
        case DT_F32: return Cast<DT_F32, CD>::go(((const float*)base)[idx]);
        default: return Cast<DT_F64, CD>::go(((const double*)base)[idx]);
    }
}
// Runtime-dtype store of a value of dtype VD (cast-on-store).
template <int VD> __device__ __forceinline__ void store_cast(void* base, int64_t idx, int dd, typename DT<VD>::T v) {
    switch (dd) {
        case DT_BOOL: ((uint8_t*)base)[idx] = Cast<VD, DT_BOOL>::go(v); break;
        case DT_I8: ((int8_t*)base)[idx] = Cast<VD, DT_I8>::go(v); break;
        case DT_I16: ((int16_t*)base)[idx] = Cast<VD, DT_I16>::go(v); break;
        case DT_I32: ((int32_t*)base)[idx] = Cast<VD, DT_I32>::go(v); break;
        case DT_I64: ((int64_t*)base)[idx] = Cast<VD, DT_I64>::go(v); break;
        case DT_U8: ((uint8_t*)base)[idx] = Cast<VD, DT_U8>::go(v); break;
        case DT_U16: ((uint16_t*)base)[idx] = Cast<VD, DT_U16>::go(v); break;
        case DT_U32: ((uint32_t*)base)[idx] = Cast<VD, DT_U32>::go(v); break;
        case DT_U64: ((uint64_t*)base)[idx] = Cast<VD, DT_U64>::go(v); break;
        case DT_F16: ((h16*)base)[idx] = Cast<VD, DT_F16>::go(v); break;
        case DT_F32: ((float*)base)[idx] = Cast<VD, DT_F32>::go(v); break;
        default: ((double*)base)[idx] = Cast<VD, DT_F64>::go(v); break;
    }
}

// ---------------------------------------------------------------------------
// Float "kind" ops for the generic float algorithms (f32, f64, f16)
// ---------------------------------------------------------------------------
template <int D> struct FOps;
template <> struct FOps<DT_F32> {
    typedef float T;
    static __device__ __forceinline__ T add(T x, T y) { return x_add(x, y); }
    static __device__ __forceinline__ T sub(T x, T y) { return x_sub(x, y); }
    static __device__ __forceinline__ T mul(T x, T y) { return x_mul(x, y); }
    static __device__ __forceinline__ T div(T x, T y) { return x_div(x, y); }
    static __device__ __forceinline__ T rem(T x, T y) { return x_fmod(x, y); }
    static __device__ __forceinline__ T floor_(T x) { return x_floor(x); }
    static __device__ __forceinline__ bool isnan_(T x) { return isnan_f(x); }
    static __device__ __forceinline__ bool isinf_(T x) { return (fb(x) & 0x7FFFFFFFu) == 0x7F800000u; }
    static __device__ __forceinline__ bool isfin(T x) { return (fb(x) & 0x7F800000u) != 0x7F800000u; }
    static __device__ __forceinline__ bool iszero(T x) { return (fb(x) & 0x7FFFFFFFu) == 0; }
    static __device__ __forceinline__ bool neg(T x) { return (fb(x) >> 31) != 0; }
    static __device__ __forceinline__ bool gt(T x, T y) { return x > y; }
    static __device__ __forceinline__ T one() { return 1.0f; }
    static __device__ __forceinline__ T half() { return 0.5f; }
    static __device__ __forceinline__ T nan() { return bf(0x7FC00000u); }
    static __device__ __forceinline__ T negone() { return -1.0f; }
    static __device__ __forceinline__ T copysign0(T s) { return bf(fb(s) & 0x80000000u); }
};
template <> struct FOps<DT_F64> {
    typedef double T;
    static __device__ __forceinline__ T add(T x, T y) { return x_add(x, y); }
    static __device__ __forceinline__ T sub(T x, T y) { return x_sub(x, y); }
    static __device__ __forceinline__ T mul(T x, T y) { return x_mul(x, y); }
    static __device__ __forceinline__ T div(T x, T y) { return x_div(x, y); }
    static __device__ __forceinline__ T rem(T x, T y) { return x_fmod(x, y); }
    static __device__ __forceinline__ T floor_(T x) { return x_floor(x); }
    static __device__ __forceinline__ bool isnan_(T x) { return isnan_d(x); }
    static __device__ __forceinline__ bool isinf_(T x) { return (db(x) & 0x7FFFFFFFFFFFFFFFull) == 0x7FF0000000000000ull; }
    static __device__ __forceinline__ bool isfin(T x) { return (db(x) & 0x7FF0000000000000ull) != 0x7FF0000000000000ull; }
    static __device__ __forceinline__ bool iszero(T x) { return (db(x) & 0x7FFFFFFFFFFFFFFFull) == 0; }
    static __device__ __forceinline__ bool neg(T x) { return (db(x) >> 63) != 0; }
    static __device__ __forceinline__ bool gt(T x, T y) { return x > y; }
    static __device__ __forceinline__ T one() { return 1.0; }
    static __device__ __forceinline__ T half() { return 0.5; }
    static __device__ __forceinline__ T nan() { return bd(0x7FF8000000000000ull); }
    static __device__ __forceinline__ T negone() { return -1.0; }
    static __device__ __forceinline__ T copysign0(T s) { return bd(db(s) & 0x8000000000000000ull); }
};
template <> struct FOps<DT_F16> {
    typedef h16 T;
    static __device__ __forceinline__ T add(T x, T y) { return f2h(x_add(h2f(x), h2f(y))); }
    static __device__ __forceinline__ T sub(T x, T y) { return f2h(x_sub(h2f(x), h2f(y))); }
    static __device__ __forceinline__ T mul(T x, T y) { return f2h(x_mul(h2f(x), h2f(y))); }
    static __device__ __forceinline__ T div(T x, T y) { return f2h(x_div(h2f(x), h2f(y))); }
    static __device__ __forceinline__ T rem(T x, T y) { return f2h(x_fmod(h2f(x), h2f(y))); }
    static __device__ __forceinline__ T floor_(T x) { return f2h(x_floor(h2f(x))); }
    static __device__ __forceinline__ bool isnan_(T x) { return isnan_h(x); }
    static __device__ __forceinline__ bool isinf_(T x) { return (x & 0x7FFFu) == 0x7C00u; }
    static __device__ __forceinline__ bool isfin(T x) { return (x & 0x7C00u) != 0x7C00u; }
    static __device__ __forceinline__ bool iszero(T x) { return (x & 0x7FFFu) == 0; }
    static __device__ __forceinline__ bool neg(T x) { return (x & 0x8000u) != 0; }
    static __device__ __forceinline__ bool gt(T x, T y) { return h2f(x) > h2f(y); }
    static __device__ __forceinline__ T one() { return 0x3C00; }
    static __device__ __forceinline__ T half() { return 0x3800; }
    static __device__ __forceinline__ T nan() { return 0x7E00; }
    static __device__ __forceinline__ T negone() { return 0xBC00; }
    static __device__ __forceinline__ T copysign0(T s) { return (T)(s & 0x8000u); }
};

// float floor_divide in numpy's npy_divmod order (ufunc.rs:2493-2572).
// floor_divide_full is the whole sequence, special values included; it is
// kept out of line so that the unrolled element loops carry only the fast
// path below (its code would otherwise be copied into every unrolled
// element and overflow the instruction cache).
template <int D> static __device__ __noinline__ typename FOps<D>::T floor_divide_full(typename FOps<D>::T x, typename FOps<D>::T y) {
    typedef FOps<D> O;
    typedef typename O::T T;
    if (O::isinf_(x) && O::isfin(y) && !O::iszero(y)) return O::nan();
    if (O::isinf_(y) && O::isfin(x) && !O::iszero(x) && O::neg(x) != O::neg(y)) return O::negone();
    if (O::isfin(x) && O::isfin(y) && !O::iszero(y)) {
        T raw_r = O::rem(x, y);
        T div = O::div(O::sub(x, raw_r), y);
        if (!O::iszero(raw_r) && O::neg(raw_r) != O::neg(y)) div = O::sub(div, O::one());
        if (!O::iszero(div)) {
            T fl = O::floor_(div);
            return O::gt(O::sub(div, fl), O::half()) ? O::add(fl, O::one()) : fl;
        }
        return O::copysign0(O::div(x, y));
    }
    return O::floor_(O::div(x, y));
}
// The one-division path and the special values, out of line. With x, y
// finite, y != 0 and t = trunc(fl(x / y)) (q or q + 1 in magnitude) below
// 2^20 (2^49), x - t*y is exact in one FMA, one repair step makes t the
// exact truncated quotient q and r = fmod(x, y), and npy_divmod's
// (x - r) / y then lies within 1/4 of q, so its floor-and-round gives q
// (q - 1 after the sign fix) exactly; a zero result takes npy_divmod's
// copysign(0, x / y), the sign of x XOR y. Larger quotients take the full
// sequence. The special values take the results floor_divide_full gives
// them, case by case, without a division (a NaN operand: the first NaN,
// quieted; a zero divisor: 0/0 the default NaN, else an infinity of the
// quotient's sign; an infinite dividend: NaN, the default one when the
// divisor is infinite too; an infinite divisor: -1 when x is nonzero with
// the other sign, else a zero of the quotient's sign).
template <int D> static __device__ __noinline__ typename FOps<D>::T floor_divide_slow(typename FOps<D>::T x, typename FOps<D>::T y) {
    typedef FOps<D> O;
    typedef typename O::T T;
    if (O::isfin(x) && O::isfin(y) && !O::iszero(y)) {
        const T t = trunc(O::div(x, y));
        if (fabs(t) < (D == DT_F32 ? (T)0x1p20 : (T)0x1p49)) {
            T r, q = t;
            if constexpr (D == DT_F32) r = __fmaf_rn(-t, y, x);
            else r = __fma_rn(-t, y, x);
            if (!O::iszero(r) && O::neg(r) != O::neg(x)) {
                r = O::add(r, copysign(y, x));
                q = O::sub(q, O::neg(x) == O::neg(y) ? (T)1 : (T)-1);
            }
            if (!O::iszero(r) && O::neg(r) != O::neg(y)) q = O::sub(q, (T)1);
            if (q == (T)0) return (O::neg(x) != O::neg(y)) ? (T)-0.0 : (T)0.0;
            return q;
        }
        return floor_divide_full<D>(x, y);  // a quotient of 2^20 (2^49) or more
    }
    if (O::isnan_(x)) return O::floor_(x);
    if (O::isnan_(y)) return O::floor_(y);
    const bool sq = O::neg(x) != O::neg(y);
    T dn;  // the default NaN of 0/0 and inf/inf
    if constexpr (D == DT_F32) dn = dnan_f(); else dn = dnan_d();
    if (O::iszero(y)) return O::iszero(x) ? dn : (sq ? -(T)INFINITY : (T)INFINITY);
    if (O::isinf_(x)) return O::isinf_(y) ? dn : O::nan();
    if (!O::iszero(x) && sq) return O::negone();
    // a zero with the sign of x XOR y, built from the bits
    if constexpr (D == DT_F32) return bf((fb(x) ^ fb(y)) & 0x80000000u);
    else return bd((db(x) ^ db(y)) & 0x8000000000000000ull);
}
// quot_fast's case inline: npy_divmod's result is then the exact floor of
// x / y. With m = x - t y, the floor is t - 1 exactly when m is nonzero with
// the sign opposite to y's: for a positive quotient that is t one too
// large, and for a negative one a nonzero remainder with t exact; in the
// other two cases (t exact, or one too large in magnitude below a negative
// quotient with a nonzero remainder) it is t. A zero result takes the sign
// of x XOR y. Everything else goes out of line.
template <class T> __device__ __forceinline__ bool floor_divide_fast(T x, T y, T* r) {
    T t, m;
    const bool ok = quot_fast(x, y, &t, &m);
    const T f = (m != (T)0 && signbit(m) != signbit(y)) ? t - (T)1 : t;
    if constexpr (sizeof(T) == 4) *r = f == 0.0f ? bf((fb(x) ^ fb(y)) & 0x80000000u) : f;
    else *r = f == 0.0 ? bd((db(x) ^ db(y)) & 0x8000000000000000ull) : f;
    return ok;
}
template <int D> __device__ __forceinline__ typename FOps<D>::T float_floor_divide(typename FOps<D>::T x, typename FOps<D>::T y) {
    typedef typename FOps<D>::T T;
    if constexpr (D == DT_F32 || D == DT_F64) {
        T r;
        if (floor_divide_fast(x, y, &r)) return r;
        return floor_divide_slow<D>(x, y);
    }
    return floor_divide_full<D>(x, y);
}

// float_max / float_min (ufunc.rs:2402-2436)
template <class F> __device__ __forceinline__ F float_max(F x, F y) {
    if (x != x) return x;
    if (y != y) return y;
    if (x == y) return signbit(x) ? y : x;
    return x > y ? x : y;
}
template <class F> __device__ __forceinline__ F float_min(F x, F y) {
    if (x != x) return x;
    if (y != y) return y;
    if (x == y) return signbit(x) ? x : y;
    return x < y ? x : y;
}
// float_same_f16 Maximum/Minimum (ufunc.rs:2448-2458): first operand on ties
__device__ __forceinline__ h16 h_max(h16 x, h16 y) {
    if (isnan_h(x)) return x;
    if (isnan_h(y)) return y;
    float a = h2f(x), b = h2f(y);
    return (a == b || a > b) ? x : y;
}
__device__ __forceinline__ h16 h_min(h16 x, h16 y) {
    if (isnan_h(x)) return x;
    if (isnan_h(y)) return y;
    float a = h2f(x), b = h2f(y);
    return (a == b || a < b) ? x : y;
}
// float_remainder_f/_f32 (ufunc.rs:4015-4034)
template <class F> __device__ __forceinline__ F float_remainder(F x, F y) {
    F r = x_fmod(x, y);
    if (r == (F)0) return copysign((F)0, y);
    if ((r < (F)0) != (y < (F)0)) return x_add(r, y);
    return r;
}
// its fast path (fmod_fast's pairs: r and y finite, so the add needs no NaN
// rule)
template <class F> __device__ __forceinline__ bool remainder_fast(F x, F y, F* r) {
    F m;
    const bool ok = fmod_fast(x, y, &m);
    *r = m == (F)0 ? copysign((F)0, y) : (((m < (F)0) != (y < (F)0)) ? m + y : m);
    return ok;
}

// ---------------------------------------------------------------------------
// Integer ops (ufunc.rs:2200-2320, 4036-4128)
// ---------------------------------------------------------------------------
template <class I> __device__ __forceinline__ I w_add(I x, I y) { typedef typename std::make_unsigned<I>::type U; return (I)(U)((U)x + (U)y); }
template <class I> __device__ __forceinline__ I w_sub(I x, I y) { typedef typename std::make_unsigned<I>::type U; return (I)(U)((U)x - (U)y); }
template <class I> __device__ __forceinline__ I w_mul(I x, I y) {
    typedef typename std::make_unsigned<I>::type U;
    if constexpr (sizeof(I) < 4) return (I)(U)((uint32_t)(U)x * (uint32_t)(U)y);
    else return (I)(U)((U)x * (U)y);
}
// Truncated quotient of 64-bit magnitudes (uy != 0). A 64-bit division is a
// long emulated sequence on the GPU; this one needs it only for quotients of
// 2^20 or more. Below that, fq = rn(rn(rz(ux) * rcp~(ru(uy))) * (1 - 2^-20)),
// rcp~ the hardware reciprocal approximation (within 2^-22 relative): rz(ux)
// <= ux and ru(uy) >= uy, so fq stays below ux / uy -- the scale by
// (1 - 2^-20) outweighs the approximation and the two roundings -- and
// within a relative 1.5 x 2^-20 of it, so trunc(fq) is the exact quotient or
// at most one or two below; the remainder ux - q uy (no underflow: q uy <=
// ux) then repairs q exactly.
__device__ __forceinline__ uint64_t udiv64_trunc(uint64_t ux, uint64_t uy) {
    if (ux < uy) return 0;
    float rc;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rc) : "f"(__ull2float_ru(uy)));
    const float fq = __fmul_rn(__fmul_rn(__ull2float_rz(ux), rc), 1.0f - 0x1p-20f);
    if (fq < 0x1p20f) {
        uint64_t q = (uint64_t)fq;
        uint64_t r = ux - q * uy;
        if (r >= uy) { ++q; r -= uy; }
        if (r >= uy) ++q;
        return q;
    }
    return ux / uy;
}
template <class I> __device__ __forceinline__ I w_div(I x, I y) {
    if constexpr (std::is_signed<I>::value) { if (y == (I)-1) return w_sub<I>((I)0, x); }
    if constexpr (sizeof(I) == 8) {
        if constexpr (std::is_signed<I>::value) {
            const uint64_t ux = x < 0 ? 0ull - (uint64_t)x : (uint64_t)x;
            const uint64_t uy = y < 0 ? 0ull - (uint64_t)y : (uint64_t)y;
            const uint64_t q = udiv64_trunc(ux, uy);
            return (I)(((x < 0) != (y < 0)) ? 0ull - q : q);
        } else {
            return (I)udiv64_trunc((uint64_t)x, (uint64_t)y);
        }
    }
    return (I)(x / y);
}
template <class I> __device__ __forceinline__ I w_rem(I x, I y) {
    if constexpr (std::is_signed<I>::value) { if (y == (I)-1) return (I)0; }
    return (I)(x % y);
}
template <class I> __device__ __forceinline__ I i_floor_div(I x, I y) {
    if (y == 0) return 0;
    if constexpr (!std::is_signed<I>::value) return (I)(x / y);
    else {
        // one division: r = x - q y (wrapping; also 0 for MIN / -1)
        I q = w_div(x, y), r = w_sub<I>(x, w_mul<I>(q, y));
        if (r != 0 && ((r < 0) != (y < 0))) return w_sub<I>(q, (I)1);
        return q;
    }
}
template <class I> __device__ __forceinline__ I i_remainder(I x, I y) {
    if (y == 0) return 0;
    if constexpr (!std::is_signed<I>::value) return (I)(x % y);
    else {
        I r = w_sub<I>(x, w_mul<I>(w_div(x, y), y));
        if (r != 0 && ((r < 0) != (y < 0))) return w_add(r, y);
        return r;
    }
}
template <class I> __device__ __forceinline__ I i_fmod(I x, I y) { return y == 0 ? (I)0 : w_rem(x, y); }
template <class I> __device__ __forceinline__ I i_shl(I x, I amt) {
    constexpr int B = (int)sizeof(I) * 8;
    if constexpr (std::is_signed<I>::value) { if (amt < 0) return 0; }
    if (amt >= (I)B) return 0;
    typedef typename std::make_unsigned<I>::type U;
    return (I)(U)((U)x << (int)amt);
}
template <class I> __device__ __forceinline__ I i_shr(I x, I amt) {
    constexpr int B = (int)sizeof(I) * 8;
    bool oob = amt >= (I)B;
    if constexpr (std::is_signed<I>::value) oob = oob || amt < 0;
    if (oob) { if constexpr (std::is_signed<I>::value) return x < 0 ? (I)-1 : (I)0; else return (I)0; }
    return (I)(x >> (int)amt);
}

// ---------------------------------------------------------------------------
// The binary op table: compute dtype CD in, result dtype out.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr bool op_is_compare(int op) { return op >= OP_GREATER && op <= OP_NOT_EQUAL; }
__host__ __device__ constexpr bool op_is_logical(int op) { return op >= OP_LOGICAL_AND && op <= OP_LOGICAL_XOR; }

template <int OP, int CD> struct BinOp {
    typedef typename DT<CD>::T T;
    static constexpr int OUT_DT = (op_is_compare(OP) || op_is_logical(OP)) ? DT_BOOL : CD;
    typedef typename DT<OUT_DT>::T R;
    // float floor_divide / remainder / fmod: fast(x, y, &r) is true, with r
    // = apply(x, y), for the pairs of their branch-free fast path, and
    // those pairs raise no FPE flag (the divisor is nonzero)
    static constexpr bool FAST = (CD == DT_F32 || CD == DT_F64) &&
                                 (OP == OP_FLOOR_DIVIDE || OP == OP_REMAINDER || OP == OP_FMOD);
    static __device__ __forceinline__ bool fast(T x, T y, R* r) {
        if constexpr (OP == OP_FLOOR_DIVIDE) return floor_divide_fast(x, y, r);
        else if constexpr (OP == OP_REMAINDER) return remainder_fast(x, y, r);
        else return fmod_fast(x, y, r);
    }
    static __device__ __forceinline__ R apply(T x, T y) {
        if constexpr (op_is_compare(OP)) {
            if constexpr (CD == DT_F16) return cmp(h2f(x), h2f(y));
            else return cmp(x, y);
        } else if constexpr (CD == DT_BOOL) {
            bool a = x != 0, b = y != 0;
            if constexpr (OP == OP_ADD || OP == OP_MAXIMUM || OP == OP_LOGICAL_OR || OP == OP_BITWISE_OR) return (R)(a || b);
            else if constexpr (OP == OP_MULTIPLY || OP == OP_MINIMUM || OP == OP_LOGICAL_AND || OP == OP_BITWISE_AND) return (R)(a && b);
            else return (R)(a != b);
        } else if constexpr (dt_is_sint(CD) || dt_is_uint(CD)) {
            if constexpr (OP == OP_ADD) return w_add(x, y);
            else if constexpr (OP == OP_SUBTRACT) return w_sub(x, y);
            else if constexpr (OP == OP_MULTIPLY) return w_mul(x, y);
            else if constexpr (OP == OP_MAXIMUM) return x > y ? x : y;
            else if constexpr (OP == OP_MINIMUM) return x < y ? x : y;
            else if constexpr (OP == OP_BITWISE_AND) return x & y;
            else if constexpr (OP == OP_BITWISE_OR) return x | y;
            else if constexpr (OP == OP_BITWISE_XOR) return x ^ y;
            else if constexpr (OP == OP_FLOOR_DIVIDE) return i_floor_div(x, y);
            else if constexpr (OP == OP_LEFT_SHIFT) return i_shl(x, y);
            else if constexpr (OP == OP_RIGHT_SHIFT) return i_shr(x, y);
            else if constexpr (OP == OP_REMAINDER) return i_remainder(x, y);
            else if constexpr (OP == OP_FMOD) return i_fmod(x, y);
            else return (R)0;
        } else if constexpr (CD == DT_F16) {
            if constexpr (OP == OP_ADD) return FOps<DT_F16>::add(x, y);
            else if constexpr (OP == OP_SUBTRACT) return FOps<DT_F16>::sub(x, y);
            else if constexpr (OP == OP_MULTIPLY) return FOps<DT_F16>::mul(x, y);
            else if constexpr (OP == OP_DIVIDE) return FOps<DT_F16>::div(x, y);
            else if constexpr (OP == OP_MAXIMUM) return h_max(x, y);
            else if constexpr (OP == OP_MINIMUM) return h_min(x, y);
            else if constexpr (OP == OP_FLOOR_DIVIDE) return float_floor_divide<DT_F16>(x, y);
            else if constexpr (OP == OP_REMAINDER) return f2h(float_remainder(h2f(x), h2f(y)));
            else if constexpr (OP == OP_FMOD) return f2h(x_fmod(h2f(x), h2f(y)));
            else return (R)0;
        } else {
            if constexpr (OP == OP_ADD) return x_add(x, y);
            else if constexpr (OP == OP_SUBTRACT) return x_sub(x, y);
            else if constexpr (OP == OP_MULTIPLY) return x_mul(x, y);
            else if constexpr (OP == OP_DIVIDE) return x_div(x, y);
            else if constexpr (OP == OP_MAXIMUM) return float_max(x, y);
            else if constexpr (OP == OP_MINIMUM) return float_min(x, y);
            else if constexpr (OP == OP_FLOOR_DIVIDE) return float_floor_divide<CD>(x, y);
            else if constexpr (OP == OP_REMAINDER) return float_remainder(x, y);
            else if constexpr (OP == OP_FMOD) return x_fmod(x, y);
            else return (R)0;
        }
    }
    template <class U> static __device__ __forceinline__ R cmp(U x, U y) {
        if constexpr (OP == OP_GREATER) return x > y;
        else if constexpr (OP == OP_GREATER_EQUAL) return x >= y;
        else if constexpr (OP == OP_LESS) return x < y;
        else if constexpr (OP == OP_LESS_EQUAL) return x <= y;
        else if constexpr (OP == OP_EQUAL) return x == y;
        else return x != y;
    }
};

// Post-hoc FPE predicate of one element (fpe.rs:173-300): which detector runs
// for this op and loop dtype.
template <int OP, int CD> struct FpeKind {
    static constexpr int value =
        (OP == OP_DIVIDE || OP == OP_FLOOR_DIVIDE) ? 1 :
        ((OP == OP_REMAINDER || OP == OP_FMOD) && !dt_is_float(CD)) ? 2 :
        (OP == OP_MULTIPLY && dt_is_float(CD)) ? 3 : 0;
};
template <class T> __device__ __forceinline__ bool is_zero_val(T x) { return x == (T)0; }
__device__ __forceinline__ bool is_zero_h(h16 x) { return (x & 0x7FFFu) == 0; }

template <int OP, int CD>
__device__ __forceinline__ uint32_t fpe_bits(typename DT<CD>::T x, typename DT<CD>::T y, typename BinOp<OP, CD>::R r) {
    constexpr int K = FpeKind<OP, CD>::value;
    if constexpr (K == 0) return 0u;
    else {
        bool yz, xz;
        if constexpr (CD == DT_F16) { yz = is_zero_h(y); xz = is_zero_h(x); }
        else if constexpr (CD == DT_BOOL) { yz = y == 0; xz = x == 0; }
        else { yz = y == (typename DT<CD>::T)0; xz = x == (typename DT<CD>::T)0; }
        if constexpr (K == 1) {
            constexpr bool ofl = dt_is_float(BinOp<OP, CD>::OUT_DT);
            return yz ? (FPE_DIVIDE | ((ofl && xz) ? FPE_INVALID : 0u)) : 0u;
        } else if constexpr (K == 2) {
            return yz ? FPE_DIVIDE : 0u;
        } else {
            typedef FOps<CD> O;
            if (!O::isfin(x) || !O::isfin(y) || xz || yz) return 0u;
            if (O::isinf_(r)) return FPE_OVER;
            bool tiny;
            if constexpr (CD == DT_F16) tiny = (r & 0x7C00u) == 0;
            else if constexpr (CD == DT_F32) tiny = (fb(r) & 0x7F800000u) == 0;
            else tiny = (db(r) & 0x7FF0000000000000ull) == 0;
            return tiny ? FPE_UNDER : 0u;
        }
    }
}

}  // namespace ionp
