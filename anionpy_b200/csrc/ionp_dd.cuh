// Double-double arithmetic and high-precision exp / log / sin of a double
// argument, usable from host and device code.
//
// A double-double (dd) is an unevaluated sum hi + lo with |lo| <= ulp(hi)/2,
// giving ~106 significant bits. The building blocks are the classic error-free
// transformations (Knuth's two-sum, Dekker's fast two-sum, and two-product
// through a fused multiply-add), which need round-to-nearest IEEE binary64
// and no contraction of a*b+c into fma except where fma is called explicitly.
//
// Evaluation schemes (all from the mathematics, no library tables):
//   exp : x = k ln2 + r with ln2 carried in three doubles, |r| <= ln2/2, then
//         the Taylor series of e^r in dd to 2^-104, scaled by 2^k;
//   log : x = 2^e m with m in [sqrt(2)/2, sqrt(2)), log m = 2 atanh(s) with
//         s = (m-1)/(m+1) as an odd series in dd, plus e ln2;
//   sin : reduction to r in [-pi/4, pi/4] and a quadrant, by Cody-Waite with
//         pi/2 in three doubles for |x| < 2^20 and by Payne-Hanek with the
//         binary expansion of 2/pi beyond, then the sin or cos series in dd.
// Accuracy is ~2^-100 relative except sin near a multiple of pi/2, where the
// reduction's absolute error (~2^-139 |x|-scaled) dominates.
#pragma once
#include <cmath>
#include <cstdint>

#ifndef __CUDACC__
#ifndef __host__
#define __host__
#define __device__
#endif
#ifndef __forceinline__
#define __forceinline__ inline
#endif
#endif

#include "ionp_constants.h"

namespace ionp {
namespace dd {

struct D2 { double hi, lo; };

__host__ __device__ __forceinline__ double fma_(double a, double b, double c) {
#ifdef __CUDA_ARCH__
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
__host__ __device__ __forceinline__ D2 two_sum(double a, double b) {
    double s = a + b;
    double bb = s - a;
    double e = (a - (s - bb)) + (b - bb);
    return {s, e};
}
__host__ __device__ __forceinline__ D2 fast_two_sum(double a, double b) {
    double s = a + b;
    return {s, b - (s - a)};
}
__host__ __device__ __forceinline__ D2 two_prod(double a, double b) {
    double p = a * b;
    return {p, fma_(a, b, -p)};
}
__host__ __device__ __forceinline__ D2 add(D2 x, D2 y) {
    D2 s = two_sum(x.hi, y.hi);
    D2 t = two_sum(x.lo, y.lo);
    s.lo += t.hi;
    s = fast_two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return fast_two_sum(s.hi, s.lo);
}
__host__ __device__ __forceinline__ D2 add_d(D2 x, double y) {
    D2 s = two_sum(x.hi, y);
    s.lo += x.lo;
    return fast_two_sum(s.hi, s.lo);
}
__host__ __device__ __forceinline__ D2 neg(D2 x) { return {-x.hi, -x.lo}; }
__host__ __device__ __forceinline__ D2 mul(D2 x, D2 y) {
    D2 p = two_prod(x.hi, y.hi);
    p.lo += x.hi * y.lo + x.lo * y.hi;
    return fast_two_sum(p.hi, p.lo);
}
__host__ __device__ __forceinline__ D2 mul_d(D2 x, double y) {
    D2 p = two_prod(x.hi, y);
    p.lo += x.lo * y;
    return fast_two_sum(p.hi, p.lo);
}
__host__ __device__ __forceinline__ D2 div(D2 x, D2 y) {
    double q1 = x.hi / y.hi;
    D2 r = add(x, neg(mul_d(y, q1)));
    double q2 = r.hi / y.hi;
    r = add(r, neg(mul_d(y, q2)));
    double q3 = r.hi / y.hi;
    D2 q = fast_two_sum(q1, q2);
    return add_d(q, q3);
}
__host__ __device__ __forceinline__ D2 div_d(D2 x, double y) {
    double q1 = x.hi / y;
    D2 p = two_prod(q1, y);
    D2 r = two_sum(x.hi, -p.hi);
    r.lo -= p.lo;
    r.lo += x.lo;
    double q2 = (r.hi + r.lo) / y;
    return fast_two_sum(q1, q2);
}

// e^x for finite x with e^x in the double range (callers screen the ends).
__host__ __device__ inline D2 exp_dd(double x) {
    double k = rint(x * 1.4426950408889634);  // x / ln2
    // r = x - k ln2, exact products by two_prod, ln2 in three parts
    D2 p1 = two_prod(k, LN2_1);
    D2 r = two_sum(x, -p1.hi);
    r = add_d(r, -p1.lo);
    D2 p2 = two_prod(k, LN2_2);
    r = add(r, neg(p2));
    r = add_d(r, -k * LN2_3);
    // e^r = sum r^i / i!, |r| <= 0.35: 23 terms reach 2^-104
    D2 term = {1.0, 0.0}, sum = {1.0, 0.0};
    for (int i = 1; i <= 23; ++i) {
        term = div_d(mul(term, r), (double)i);
        sum = add(sum, term);
    }
    // scale by 2^k in two steps so the intermediate stays normal
    int ki = (int)k;
    int k1 = ki / 2, k2 = ki - k1;
    double s1 = ldexp(1.0, k1), s2 = ldexp(1.0, k2);
    return {sum.hi * s1 * s2, sum.lo * s1 * s2};
}

// log x for finite x > 0.
__host__ __device__ inline D2 log_dd(double x) {
    int e;
    double m = frexp(x, &e);  // x = m 2^e, m in [0.5, 1)
    m *= 2.0;
    e -= 1;                    // m in [1, 2)
    if (m > 1.4142135623730951) { m *= 0.5; e += 1; }
    D2 num = two_sum(m, -1.0);
    D2 den = two_sum(m, 1.0);
    D2 s = div(num, den);
    D2 s2 = mul(s, s);
    D2 t = s, sum = s;
    for (int k = 1; k <= 22; ++k) {
        t = mul(t, s2);
        sum = add(sum, div_d(t, (double)(2 * k + 1)));
    }
    sum = {sum.hi * 2.0, sum.lo * 2.0};
    if (e == 0) return sum;
    double ed = (double)e;
    D2 l = two_prod(ed, LN2_1);
    l = add(l, two_prod(ed, LN2_2));
    l = add_d(l, ed * LN2_3);
    return add(l, sum);
}

// 32 bits of the fraction of 2/pi starting at 1-based bit `pos` (bits at
// positions <= 0 are the zeros of the integer part).
__host__ __device__ __forceinline__ uint32_t bits32(int pos) {
    int z = pos - 1;
    if (z + 32 <= 0) return 0u;
    if (z < 0) return two_over_pi_word(0) >> (-z);
    int q = z >> 5, r = z & 31;
    uint64_t v = ((uint64_t)two_over_pi_word(q) << 32) | two_over_pi_word(q + 1);
    return (uint32_t)(v >> (32 - r));
}

// x reduced mod pi/2: r in [-pi/4, pi/4] (dd) and the quadrant (k mod 4).
__host__ __device__ inline D2 reduce_pio2(double ax, int* quadrant) {
    if (ax < 1048576.0) {
        double k = rint(ax * 0.6366197723675814);  // 2/pi
        D2 p1 = two_prod(k, PI_2_1);
        D2 r = two_sum(ax, -p1.hi);
        r = add_d(r, -p1.lo);
        D2 p2 = two_prod(k, PI_2_2);
        r = add(r, neg(p2));
        r = add_d(r, -k * PI_2_3);
        *quadrant = ((int64_t)k) & 3;
        return r;
    }
    // Payne-Hanek: ax = M 2^E (M < 2^53 integer); take the bits of 2/pi from
    // position i0 = E - 1 so that ax * 2/pi mod 4 = 4 * frac(M * 0.b_i0 b_i0+1 ...)
    int ex;
    double mant = frexp(ax, &ex);  // ax = mant 2^ex, mant in [0.5, 1)
    uint64_t M = (uint64_t)ldexp(mant, 53);
    int E = ex - 53;
    int i0 = E - 1;  // 1-based bit position in 2/pi's fraction
    // window W = 9 words of 2/pi starting at bit i0 (zeros before bit 1)
    uint32_t w[9];
    for (int j = 0; j < 9; ++j) w[j] = bits32(i0 + 32 * j);
    // P = M * W, keep the low 288 bits (the fraction of M * F)
    uint32_t m0 = (uint32_t)M, m1 = (uint32_t)(M >> 32);
    uint32_t p[10] = {0};
    // little-endian limbs of W: limb 0 is w[8]
    uint64_t carry = 0;
    for (int t = 0; t < 10; ++t) {
        uint64_t acc = carry;
        uint64_t hi_part = 0;
        int li = t;       // m0 * limb t
        if (li < 9) {
            uint64_t prod = (uint64_t)m0 * w[8 - li];
            acc += (uint32_t)prod;
            hi_part += prod >> 32;
        }
        if (t >= 1 && t - 1 < 9) {
            uint64_t prod = (uint64_t)m1 * w[8 - (t - 1)];
            acc += (uint32_t)prod;
            hi_part += prod >> 32;
        }
        p[t] = (uint32_t)acc;
        carry = (acc >> 32) + hi_part;
    }
    // fraction bits: p[8] (top) .. p[0]; the top two bits are the quadrant
    uint64_t top = ((uint64_t)p[8] << 32) | p[7];
    uint64_t mid = ((uint64_t)p[6] << 32) | p[5];
    int quad = (int)(top >> 62);
    top <<= 2;
    top |= mid >> 62;
    mid <<= 2;
    mid |= (uint64_t)p[4] >> 30;
    // f = top/2^64 + mid/2^128 in [0, 1)
    D2 f = two_sum(ldexp((double)(top >> 11), -53), ldexp((double)(top & 0x7FF), -64));
    f = add_d(f, ldexp((double)(mid >> 11), -117));
    if (f.hi >= 0.5) { f = add_d(f, -1.0); quad = (quad + 1) & 3; }
    D2 pio2 = fast_two_sum(PI_2_1, PI_2_2);
    pio2 = add_d(pio2, PI_2_3);
    *quadrant = quad;
    return mul(f, pio2);
}

__host__ __device__ inline D2 sin_series(D2 r) {
    D2 r2 = mul(r, r);
    D2 term = r, sum = r;
    for (int i = 1; i <= 13; ++i) {
        term = div_d(mul(term, r2), -(double)((2 * i) * (2 * i + 1)));
        sum = add(sum, term);
    }
    return sum;
}
__host__ __device__ inline D2 cos_series(D2 r) {
    D2 r2 = mul(r, r);
    D2 term = {1.0, 0.0}, sum = {1.0, 0.0};
    for (int i = 1; i <= 13; ++i) {
        term = div_d(mul(term, r2), -(double)((2 * i - 1) * (2 * i)));
        sum = add(sum, term);
    }
    return sum;
}
// sin x for finite x.
__host__ __device__ inline D2 sin_dd(double x) {
    double ax = fabs(x);
    int q;
    D2 r = reduce_pio2(ax, &q);
    D2 v = (q & 1) ? cos_series(r) : sin_series(r);
    if (q & 2) v = neg(v);
    if (x < 0) v = neg(v);
    return v;
}

__host__ __device__ __forceinline__ bool is_inf_f(float f) {
#ifdef __CUDA_ARCH__
    return isinf(f);
#else
    return std::isinf(f);
#endif
}
// Correct rounding of hi + lo (|lo| <= ulp(hi)/2) to float.
__host__ __device__ inline float dd_to_float(D2 v) {
    float f = (float)v.hi;
    if (v.lo == 0.0 || is_inf_f(f)) {
        // hi exactly at the overflow midpoint with lo < 0 stays finite
        if (is_inf_f(f) && v.lo < 0 && fabs(v.hi) == 0x1.ffffffp+127) return v.hi > 0 ? 0x1.fffffep+127f : -0x1.fffffep+127f;
        return f;
    }
    double fd = (double)f;
    if (v.hi == fd) return f;
    float g = nextafterf(f, v.hi > fd ? INFINITY : -INFINITY);
    double mid = 0.5 * (fd + (double)g);
    if (v.hi == mid && ((v.lo > 0) == (v.hi > fd))) return g;
    return f;
}

}  // namespace dd
}  // namespace ionp
