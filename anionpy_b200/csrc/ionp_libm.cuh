// exp / log / sin for float32 and float64 that equal the host C library's
// results bit for bit, NaN bits included.
//
// The reference evaluates these ufuncs with Rust's f32::exp/ln/sin and
// f64::exp/ln/sin (ionp-core/src/ufunc.rs:4237-4367), which on Linux call
// the C library: glibc 2.39 on x86-64, resolved to its FMA variants on any
// CPU with FMA and AVX2. This file restates glibc's published algorithms:
//
//   exp32, log32, sin32  sysdeps/ieee754/flt-32/e_expf.c, e_logf.c, s_sinf.c
//                        (table plus a short polynomial evaluated in double)
//   exp64, log64         sysdeps/ieee754/dbl-64/e_exp.c, e_log.c (the same
//                        family, with a double-double-like final sum)
//   sin64                sysdeps/ieee754/dbl-64/s_sin.c, branred.c (sin/cos
//                        of i/128 from a table with Taylor corrections;
//                        Cody-Waite reduction by pi/2 below |x| = 105414350,
//                        24-bit-chunk Payne-Hanek reduction above)
//
// Equal bits need the same constants and the same rounding of every
// intermediate. glibc's compiler fuses a product into the addition that
// uses it when every use of the product is an addition in the same basic
// block (GCC's -ffp-contract=fast); each such fused multiply-add is an
// explicit fma() below and every other operation rounds on its own (the
// CUDA library is built with -fmad=false, the host check with
// -ffp-contract=off). The polynomial coefficients and reduction constants
// are glibc's published ones; the tables are generated by
// gen_libm_tables.py (ionp_libm_tables.h).
//
// The same source compiles for the host (g++), where the tests compare it
// with the C library over every float32 and over random float64 samples.
#pragma once
#include <cstdint>
#include <cstring>
#include <cmath>

#if defined(__CUDACC__)
#define LM_FN __device__ __forceinline__
#define LM_SLOW static __device__ __noinline__
#define LM_TAB static __device__ const
#else
#define LM_FN static inline
#define LM_SLOW static inline
#define LM_TAB static const
#endif

namespace ionp {
namespace lm {

#include "ionp_libm_tables.h"

// ---------------------------------------------------------------- helpers
LM_FN uint32_t fbits(float x) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(x);
#else
    uint32_t u; std::memcpy(&u, &x, 4); return u;
#endif
}
LM_FN float ffrom(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float x; std::memcpy(&x, &u, 4); return x;
#endif
}
LM_FN uint64_t dbits(double x) {
#ifdef __CUDA_ARCH__
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t u; std::memcpy(&u, &x, 8); return u;
#endif
}
LM_FN double dfrom(uint64_t u) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)u);
#else
    double x; std::memcpy(&x, &u, 8); return x;
#endif
}
LM_FN double fmad(double a, double b, double c) {
#ifdef __CUDA_ARCH__
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
template <class T> LM_FN T ld(const T* p) {
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}
// x86 NaN results: an operation on a NaN returns that NaN made quiet
// (payload and sign kept); an invalid operation on non-NaNs returns the
// "default" NaN, which has the sign bit set.
LM_FN float quiet32(float x) { return ffrom(fbits(x) | 0x00400000u); }
LM_FN double quiet64(double x) { return dfrom(dbits(x) | 0x0008000000000000ull); }
LM_FN float dnan32() { return ffrom(0xFFC00000u); }
LM_FN double dnan64() { return dfrom(0xFFF8000000000000ull); }
LM_FN float inf32() { return ffrom(0x7F800000u); }
LM_FN double inf64() { return dfrom(0x7FF0000000000000ull); }

// ------------------------------------------------------------------ exp32
// e^x = 2^(k/32) * 2^(r/32), k = round(32 x / ln 2), |r| <= 1/2; 2^(k/32)
// from the table plus k's integer part added into the exponent bits,
// 2^(r/32) by a cubic. (e_expf.c)
LM_FN float exp32(float x) {
    const double INV = 0x1.71547652b82fep+5;   // 32 / ln 2
    const double SHIFT = 0x1.8p+52;            // round-to-integer shifter
    const double C0 = 0x1.c6af84b912394p-20, C1 = 0x1.ebfce50fac4f3p-13, C2 = 0x1.62e42ff0c52d6p-6;
    const uint32_t ux = fbits(x);
    if (((ux >> 20) & 0x7ff) >= 0x42b) {      // |x| >= 88, inf or NaN
        if (ux == 0xFF800000u) return 0.0f;
        if (((ux >> 20) & 0x7ff) >= 0x7f8) return (ux & 0x7FFFFFu) ? quiet32(x) : x;
        if (x > 0x1.62e42ep6f) return inf32();
        if (x < -0x1.9fe368p6f) return 0.0f;
    }
    const double xd = (double)x;
    double kd = fmad(INV, xd, SHIFT);
    const uint64_t ki = dbits(kd);
    kd -= SHIFT;
    const double r = fmad(INV, xd, -kd);
    const double s = dfrom(ld(&EXPF_TAB[ki & 31]) + (ki << 47));
    const double z = fmad(C0, r, C1);
    const double r2 = r * r;
    double y = fmad(C2, r, 1.0);
    y = fmad(z, r2, y);
    return (float)(y * s);
}

// ------------------------------------------------------------------ log32
// x = 2^k z, z in [0x1.66p-1, 0x1.66p0); log x = k ln2 + log c + log1p(z/c
// - 1) with 1/c and log c from the table of 16 subintervals. (e_logf.c)
LM_FN float log32(float x) {
    const double LN2 = 0x1.62e42fefa39efp-1;
    const double A0 = -0x1.00ea348b88334p-2, A1 = 0x1.5575b0be00b6ap-2, A2 = -0x1.ffffef20a4123p-2;
    uint32_t ix = fbits(x);
    if (ix == 0x3F800000u) return 0.0f;
    if (ix - 0x00800000u >= 0x7F800000u - 0x00800000u) {   // subnormal, 0, negative, inf, NaN
        if ((ix << 1) == 0) return -inf32();
        if (ix == 0x7F800000u) return x;
        if ((ix & 0x80000000u) || (ix << 1) >= 0xFF000000u)
            return ((ix << 1) > 0xFF000000u) ? quiet32(x) : dnan32();
        ix = fbits(x * 0x1p23f) - (23u << 23);
    }
    const uint32_t d = ix - 0x3F330000u;
    const int i = (int)((d >> 19) & 15);
    const int k = (int32_t)d >> 23;
    const double invc = ld(&LOGF_TAB[2 * i]), logc = ld(&LOGF_TAB[2 * i + 1]);
    const double z = (double)ffrom(ix - (d & 0xFF800000u));
    const double r = fmad(z, invc, -1.0);
    const double y0 = fmad((double)k, LN2, logc);
    const double r2 = r * r;
    double y = fmad(A1, r, A2);
    y = fmad(A0, r2, y);
    y = fmad(y, r2, y0 + r);
    return (float)y;
}

// ------------------------------------------------------------------ sin32
// |x| < pi/4: odd polynomial; |x| < 120: x - n pi/2 in double; larger:
// n and the remainder from 96 bits of 2/pi in integer arithmetic. The
// quadrant picks the sin or cos polynomial and its sign. (s_sinf.c,
// sincosf.h)
// sin (n even) or cos (n odd) polynomial of the reduced argument, in the
// operation order of each:
//   sin: fma(x7, fma(x2, S3, S2), fma(x3, S1, x)),  x3 = x x2, x7 = x3 x2
//   cos: fma(x6, fma(x2, C4, C3), fma(x4, C2, fma(x2, C1, C0))),
//        x4 = x2 x2, x6 = x4 x2
// Both have the same shape -- p = fma(x2, A, B), u = y x2, w = u x2,
// fma(w, p, fma(u, K, L)) -- so one body evaluates whichever the lane needs
// with its own coefficients, the same operations on the same operands as
// the polynomial alone (lanes of a warp in different quadrants still run
// one body). flip negates the cos coefficients (the table's second half),
// which is exact.
LM_FN float sin32_poly(double x, double x2, int n, bool flip) {
    const double S1 = -0x1.555545995a603p-3, S2 = 0x1.1107605230bc4p-7, S3 = -0x1.994eb3774cf24p-13;
    const double C0 = 0x1p0, C1 = -0x1.ffffffd0c621cp-2, C2 = 0x1.55553e1068f19p-5,
                 C3 = -0x1.6c087e89a359dp-10, C4 = 0x1.99343027bf8c3p-16;
    const bool c = (n & 1) != 0;
    const double A = c ? (flip ? -C4 : C4) : S3;
    const double B = c ? (flip ? -C3 : C3) : S2;
    const double K = c ? (flip ? -C2 : C2) : S1;
    const double p = fmad(x2, A, B);                 // s1 / c2
    const double u = (c ? x2 : x) * x2;              // x3 / x4
    const double w = u * x2;                          // x7 / x6
    const double c1 = fmad(x2, flip ? -C1 : C1, flip ? -C0 : C0);
    const double v = fmad(u, K, c ? c1 : x);
    return (float)fmad(w, p, v);
}
LM_SLOW double sin32_reduce_large(uint32_t xi, int* np) {
    const unsigned int* w = &TWO_OVER_PI_W[(xi >> 26) & 15];
    const int shift = (xi >> 23) & 7;
    xi = ((xi & 0xFFFFFFu) | 0x800000u) << shift;
    uint64_t r0 = (uint64_t)(uint32_t)(xi * ld(&w[0]));
    const uint64_t r1 = (uint64_t)xi * ld(&w[4]);
    const uint64_t r2 = (uint64_t)xi * ld(&w[8]);
    r0 = (r2 >> 32) | (r0 << 32);
    r0 += r1;
    const uint64_t n = (r0 + (1ull << 61)) >> 62;
    r0 -= n << 62;
    *np = (int)n;
    return (double)(int64_t)r0 * 0x1.921FB54442D18p-62;
}
LM_FN float sin32(float y) {
    const uint32_t ux = fbits(y);
    const uint32_t top = (ux >> 20) & 0x7ff;
    if (top >= 0x42f) {                        // |y| >= 120, inf, NaN
        if (top >= 0x7f8) return (ux & 0x7FFFFFu) ? quiet32(y) : dnan32();
        int n;
        const int sign = (int)(ux >> 31);
        const double x = sin32_reduce_large(ux, &n);
        const int q = n + sign;
        const double s = ((q + 1) & 2) ? -1.0 : 1.0;   // signs {1,-1,-1,1}[q & 3]
        return sin32_poly(x * s, x * x, n, (q & 2) != 0);
    }
    double x = (double)y;
    int n = 0;
    if (top >= 0x3f4) {                        // pi/4 <= |y| < 120: x - n pi/2
        const double r = x * 0x1.45F306DC9C883p+23;   // x * 2/pi * 2^24
        n = ((int32_t)r + 0x800000) >> 24;
        x = fmad(-(double)n, 0x1.921FB54442D18p0, x);
    }
    const double s = ((n + 1) & 2) ? -1.0 : 1.0;
    const float r = sin32_poly(x * s, x * x, n, (n & 2) != 0);
    return top < 0x398 ? y : r;                // |y| < 2^-12: y itself
}

// ------------------------------------------------------------------ cos32
// The same reductions and polynomials as sin32 (s_cosf.c, sincosf.h): below
// pi/4 the cos polynomial (1 below 2^-12); above, quadrant n + 1 of the
// reduced argument, the sign and table half from n (and the input's sign
// for the large reduction, which works on |y|).
LM_FN float cos32(float y) {
    const uint32_t ux = fbits(y);
    const uint32_t top = (ux >> 20) & 0x7ff;
    if (top >= 0x42f) {                        // |y| >= 120, inf, NaN
        if (top >= 0x7f8) return (ux & 0x7FFFFFu) ? quiet32(y) : dnan32();
        int n;
        const int sign = (int)(ux >> 31);
        const double x = sin32_reduce_large(ux, &n);
        const int q = n + sign;
        const double s = ((q + 1) & 2) ? -1.0 : 1.0;   // signs {1,-1,-1,1}[q & 3]
        return sin32_poly(x * s, x * x, n ^ 1, (q & 2) != 0);
    }
    double x = (double)y;
    if (top < 0x3f4) {                         // |y| < pi/4
        if (top < 0x398) return 1.0f;          // |y| < 2^-12
        return sin32_poly(x, x * x, 1, false);
    }
    const double r = x * 0x1.45F306DC9C883p+23;       // x * 2/pi * 2^24
    const int n = ((int32_t)r + 0x800000) >> 24;
    x = fmad(-(double)n, 0x1.921FB54442D18p0, x);
    const double s = ((n + 1) & 2) ? -1.0 : 1.0;
    return sin32_poly(x * s, x * x, n ^ 1, (n & 2) != 0);
}

// ------------------------------------------------------------------ exp64
// e^x = 2^(k/128) e^r, x = k ln2/128 + r; 2^(k/128) = H (1 + t) from the
// table, e^r - 1 by a quintic; result scale + scale * tmp. Results near
// overflow or in the subnormal range take the rescaled path. (e_exp.c)
LM_SLOW double exp64_special(double tmp, uint64_t sbits, uint64_t ki) {
    if ((ki & 0x80000000ull) == 0) {           // k > 0: scale may overflow
        sbits -= 1009ull << 52;
        const double scale = dfrom(sbits);
        return 0x1p1009 * fmad(scale, tmp, scale);
    }
    sbits += 1022ull << 52;                    // k < 0: subnormal range
    const double scale = dfrom(sbits);
    const double st = scale * tmp;             // not fused: a second use sits in the branch below
    double y = scale + st;
    if (y < 1.0) {
        double lo = (scale - y) + st;
        const double hi = 1.0 + y;
        lo = ((1.0 - hi) + y) + lo;
        y = (hi + lo) - 1.0;
        if (y == 0.0) y = 0.0;
    }
    return 0x1p-1022 * y;
}
LM_FN double exp64(double x) {
    const double INV = 0x1.71547652b82fep0 * 128, SHIFT = 0x1.8p52;
    const double NL2HI = -0x1.62e42fefa0000p-8, NL2LO = -0x1.cf79abc9e3b3ap-47;
    const double C2 = 0x1.ffffffffffdbdp-2, C3 = 0x1.555555555543cp-3, C4 = 0x1.55555cf172b91p-5,
                 C5 = 0x1.1111167a4d017p-7;
    const uint64_t ux = dbits(x);
    uint32_t top = (uint32_t)(ux >> 52) & 0x7ff;
    if (top - 0x3c9u >= 0x408u - 0x3c9u) {     // |x| < 2^-54 or |x| >= 512
        if (top - 0x3c9u >= 0x80000000u) return 1.0 + x;
        if (top >= 0x409) {                    // |x| >= 1024, inf, NaN
            if (ux == 0xFFF0000000000000ull) return 0.0;
            if (top >= 0x7ff) return (ux << 12) ? quiet64(x) : x;
            return (ux >> 63) ? 0.0 : inf64();
        }
        top = 0;                               // large |x|: rescaled result
    }
    double kd = fmad(INV, x, SHIFT);
    const uint64_t ki = dbits(kd);
    kd -= SHIFT;
    const double r = fmad(kd, NL2LO, fmad(kd, NL2HI, x));
    const uint64_t idx = 2 * (ki & 127);
    const double tail = dfrom(ld(&EXP_TAB[idx]));
    const uint64_t sbits = ld(&EXP_TAB[idx + 1]) + (ki << 45);
    const double r2 = r * r;
    const double tmp = fmad(r2 * r2, fmad(r, C5, C4), fmad(r2, fmad(r, C3, C2), tail + r));
    if (top == 0) return exp64_special(tmp, sbits, ki);
    const double scale = dfrom(sbits);
    return fmad(scale, tmp, scale);
}

// ------------------------------------------------------------------ log64
// Near 1 (x in [1 - 2^-4, 1 + 0x1.09p-4]): log1p(x - 1) by a degree-12
// polynomial with the r^2/2 term split exactly. Elsewhere x = 2^k z, z in
// [0x1.6p-1, 0x1.6p0), log x = k ln2 + log c + log1p(z/c - 1) with (1/c,
// log c) from the table of 128 subintervals. (e_log.c)
LM_FN double log64(double x) {
    const double B0 = -0x1p-1, B1 = 0x1.5555555555577p-2, B2 = -0x1.ffffffffffdcbp-3, B3 = 0x1.999999995dd0cp-3,
                 B4 = -0x1.55555556745a7p-3, B5 = 0x1.24924a344de3p-3, B6 = -0x1.fffffa4423d65p-4,
                 B7 = 0x1.c7184282ad6cap-4, B8 = -0x1.999eb43b068ffp-4, B9 = 0x1.78182f7afd085p-4,
                 B10 = -0x1.5521375d145cdp-4;
    const double A0 = -0x1.0000000000001p-1, A1 = 0x1.555555551305bp-2, A2 = -0x1.fffffffeb459p-3,
                 A3 = 0x1.999b324f10111p-3, A4 = -0x1.55575e506c89fp-3;
    const double LN2HI = 0x1.62e42fefa3800p-1, LN2LO = 0x1.ef35793c76730p-45;
    uint64_t ix = dbits(x);
    const uint64_t LO = 0x3FEE000000000000ull;  // 1 - 2^-4
    const uint64_t HI = 0x3FF1090000000000ull;  // 1 + 0x1.09p-4
    if (ix - LO < HI - LO) {
        if (ix == 0x3FF0000000000000ull) return 0.0;
        const double r = x - 1.0, r2 = r * r, r3 = r * r2;
        const double p3 = fmad(r3, B10, fmad(r2, B9, fmad(r, B8, B7)));
        const double p2 = fmad(r3, p3, fmad(r2, B6, fmad(r, B5, B4)));
        const double p1 = fmad(r3, p2, fmad(r2, B3, fmad(r, B2, B1)));
        const double w = r * 0x1p27;
        const double rhi = (r + w) - w, rlo = r - rhi;
        const double w2 = (rhi * rhi) * B0;       // exact: rhi has 26 bits
        const double hi = r + w2;
        double lo = (r - hi) + w2;
        lo = fmad(B0 * rlo, rhi + r, lo);
        return fmad(r3, p1, lo) + hi;
    }
    const uint32_t top = (uint32_t)(ix >> 48);
    if (top - 0x0010u >= 0x7ff0u - 0x0010u) {  // subnormal, 0, negative, inf, NaN
        if ((ix << 1) == 0) return -inf64();
        if (ix == 0x7FF0000000000000ull) return x;
        if ((top & 0x8000u) || (top & 0x7ff0u) == 0x7ff0u)
            return ((ix << 1) > 0xFFE0000000000000ull) ? quiet64(x) : dnan64();
        ix = dbits(x * 0x1p52) - (52ull << 52);
    }
    const uint64_t d = ix - 0x3FE6000000000000ull;
    const int i = (int)((d >> 45) & 127);
    const double kd = (double)((int64_t)d >> 52);
    const double invc = ld(&LOG_TAB[2 * i]), logc = ld(&LOG_TAB[2 * i + 1]);
    const double z = dfrom(ix - (d & (0xfffull << 52)));
    const double r = fmad(z, invc, -1.0);
    const double w = fmad(kd, LN2HI, logc);
    const double hi = w + r;
    const double lo = fmad(kd, LN2LO, (w - hi) + r);
    const double r2 = r * r;
    const double q = fmad(r2, fmad(r, A4, A3), fmad(r, A2, A1));
    return fmad(r * r2, q, fmad(r2, A0, lo)) + hi;
}

// ------------------------------------------------------------------ sin64
// (s_sin.c) Constants: pi/2 = HP0 + HP1; pi/2 = MP1 + MP2 + PP3 + PP4 with
// MP1, MP2, PP3 short enough that n * each is exact for n < 2^26.
#define LM_BIG 0x1.8p45                        // table index shifter (1/128 steps)
#define LM_HP0 0x1.921fb54442d18p0
#define LM_HP1 0x1.1a62633145c07p-54
#define LM_MP1 0x1.921fb58000000p0
#define LM_MP2 -0x1.dde973c000000p-27
#define LM_PP3 -0x1.cb3b398000000p-55
#define LM_PP4 -0x1.d747f23e32ed7p-83

// sin(a + da) for small a: Taylor series to a^11 plus (1 - a^2/2) da
LM_FN double sin64_taylor(double xx, double a, double da) {
    const double S1 = -0x1.5555555555555p-3, S2 = 0x1.1111111110ecep-7, S3 = -0x1.a01a019db08b8p-13,
                 S4 = 0x1.71de27b9a7ed9p-19, S5 = -0x1.addffc2fcdf59p-26;
    const double p = fmad(fmad(fmad(fmad(S5, xx, S4), xx, S3), xx, S2), xx, S1);
    const double t = fmad(fmad(p, a, -(0.5 * da)), xx, da);
    return a + t;
}
#define LM_SN3 -1.66666666666664880952546298448555E-01
#define LM_SN5 8.33333214285722277379541354343671E-03
#define LM_CS2 4.99999999999999999999950396842453E-01
#define LM_CS4 -4.16666666666664434524222570944589E-02
#define LM_CS6 1.38888874007937613028114285595617E-03

// sin or cos of a + da (|a| < 0.86) from the table of i/128, evaluated
// without a branch on which: both of glibc's correction formulas are
// computed and one is selected (a warp whose lanes need different ones runs
// one body). With n even: sin(a + da), as s_sin.c's do_sin (Taylor series
// below |a| = 0.126; else sin(X_i) cos(d) + cos(X_i) sin(d), X_i = i/128
// nearest |a|). With n odd: cos(a + da), as do_cos (cos(X_i) cos(d) -
// sin(X_i) sin(d)). n & 2 negates the result.
LM_FN double sin64_quadrant(double a, double da, int n) {
    const bool cosq = (n & 1) != 0;
    const double dxs = (cosq ? (a < 0) : (a <= 0)) ? -da : da;
    const double ax = fabs(a);
    const double u = LM_BIG + ax;
    const double t = ax - (u - LM_BIG);
    const double x = cosq ? t + dxs : t;
    const double xx = x * x;
    const double ps = fmad(xx, LM_SN5, LM_SN3);
    const double pc = xx * fmad(xx, fmad(xx, LM_CS6, LM_CS4), LM_CS2);
    const double s = cosq ? fmad(x * xx, ps, x) : x + fmad(x * xx, ps, dxs);
    const double c = cosq ? pc : fmad(x, dxs, pc);
    const int k = (int)(uint32_t)dbits(u) << 2;
    const double sn = ld(&SINCOS_TAB[k]), ssn = ld(&SINCOS_TAB[k + 1]);
    const double cs = ld(&SINCOS_TAB[k + 2]), ccs = ld(&SINCOS_TAB[k + 3]);
    double r;
    if (cosq) {
        r = cs + fmad(-sn, s, fmad(-cs, c, fmad(-s, ssn, ccs)));
    } else if (ax < 0.126) {
        r = sin64_taylor(a * a, a, da);
    } else {
        r = copysign(sn + fmad(cs, s, fmad(-sn, c, fmad(s, ccs, ssn))), a);
    }
    return (n & 2) ? -r : r;
}
// |x| >= 105414350: x 2/pi = sum + b + bb from 24-bit chunks of 2/pi, each
// half of a 26-bit split of x multiplied exactly; (b + bb) pi/2 = a + aa.
// (branred.c, compiled without fused multiply-adds)
LM_SLOW int sin64_reduce_large(double x, double* a, double* aa) {
    const double SPLIT = 134217729.0, BIG = 0x1.8p52, BIG1 = 0x1.8p54;
    const double MP2B = -0x1.dde9740000000p-27;   // branred's own second part of pi/2
    x *= 0x1p-600;
    const double t0 = x * SPLIT;
    const double x1 = t0 - (t0 - x);
    const double x2 = x - x1;
    double sums[2], bs[2], bbs[2];
    for (int part = 0; part < 2; part++) {
        const double xp = part == 0 ? x1 : x2;
        double r[6], sum = 0.0, s, t, b, bb;
        int k = (int)((dbits(xp) >> 52) & 2047);
        k = (k - 450) / 24;
        if (k < 0) k = 0;
        double g = dfrom(dbits(0x1p576) - ((uint64_t)(k * 24) << 52));
        for (int i = 0; i < 6; i++) {
            r[i] = (xp * ld(&TWO_OVER_PI_24[k + i])) * g;
            g *= 0x1p-24;
        }
        for (int i = 0; i < 3; i++) {
            s = (r[i] + BIG) - BIG;
            sum += s;
            r[i] -= s;
        }
        t = 0.0;
        for (int i = 0; i < 6; i++) t += r[5 - i];
        bb = (((((r[0] - t) + r[1]) + r[2]) + r[3]) + r[4]) + r[5];
        s = (t + BIG) - BIG;
        sum += s;
        t -= s;
        b = t + bb;
        bb = (t - b) + bb;
        s = (sum + BIG1) - BIG1;
        sum -= s;
        sums[part] = sum; bs[part] = b; bbs[part] = bb;
    }
    double sum = sums[0] + sums[1];
    double b = bs[0] + bs[1];
    double bb = (fabs(bs[0]) > fabs(bs[1])) ? (bs[0] - b) + bs[1] : (bs[1] - b) + bs[0];
    if (b > 0.5) { b -= 1.0; sum += 1.0; }
    else if (b < -0.5) { b += 1.0; sum -= 1.0; }
    double s = b + (bb + bbs[0] + bbs[1]);
    double t = ((b - s) + bb) + (bbs[0] + bbs[1]);
    const double sp = s * SPLIT;
    const double t1 = sp - (sp - s), t2 = s - t1;
    b = s * LM_HP0;
    bb = (((t1 * LM_MP1 - b) + t1 * MP2B) + t2 * LM_MP1) + ((t2 * MP2B + s * LM_HP1) + t * LM_HP0);
    s = b + bb;
    t = (b - s) + bb;
    *a = s;
    *aa = t;
    return ((int)sum) & 3;
}
LM_SLOW double sin64_large(double x) {
    double a, da;
    const int n = sin64_reduce_large(x, &a, &da);
    return sin64_quadrant(a, da, n);
}
LM_FN double sin64(double x) {
    const uint32_t k = (uint32_t)(dbits(x) >> 32) & 0x7fffffffu;
    if (k < 0x3e500000u) return x;                       // |x| < 2^-26
    if (k >= 0x419921fbu) {                              // |x| >= 105414350, inf, NaN
        if (k < 0x7ff00000u) return sin64_large(x);
        return ((dbits(x) << 12) != 0) ? quiet64(x) : dnan64();
    }
    double a, da;
    int n;
    if (k < 0x3feb6000u) {                               // |x| < 0.855469: sin(x)
        a = x; da = 0.0; n = 0;
    } else if (k < 0x400368fdu) {                        // |x| < 2.426265: +-cos(pi/2 - |x|)
        a = LM_HP0 - fabs(x); da = LM_HP1; n = x < 0 ? 3 : 1;
    } else {                                             // Cody-Waite: x - n pi/2 in four parts
        const double t = fmad(x, 0x1.45f306dc9c883p-1, 0x1.8p52);   // x 2/pi + shifter
        const double xn = t - 0x1.8p52;
        const double y = fmad(-xn, LM_MP2, fmad(-xn, LM_MP1, x));
        n = (int)(dbits(t) & 3);
        const double t2 = fmad(-xn, LM_PP3, y);
        da = fmad(-xn, LM_PP3, y - t2);
        a = fmad(-xn, LM_PP4, t2);
        da += fmad(-xn, LM_PP4, t2 - a);
    }
    return sin64_quadrant(a, da, n);
}

// cos: 1 below 2^-27; do_cos below 0.855469; do_sin of pi/2 - |x| as a
// normalised double-double below 2.426265; quadrant n + 1 of the Cody-Waite
// or the large reduction above (s_sin.c's __cos).
LM_SLOW double cos64_large(double x) {
    double a, da;
    const int n = sin64_reduce_large(x, &a, &da);
    return sin64_quadrant(a, da, n + 1);
}
LM_FN double cos64(double x) {
    const uint32_t k = (uint32_t)(dbits(x) >> 32) & 0x7fffffffu;
    if (k < 0x3e400000u) return 1.0;                      // |x| < 2^-27
    if (k >= 0x419921fbu) {                              // |x| >= 105414350, inf, NaN
        if (k < 0x7ff00000u) return cos64_large(x);
        return ((dbits(x) << 12) != 0) ? quiet64(x) : dnan64();
    }
    double a, da;
    int n;
    if (k < 0x3feb6000u) {                               // |x| < 0.855469: cos(x)
        a = x; da = 0.0; n = 1;
    } else if (k < 0x400368fdu) {                        // |x| < 2.426265: sin(pi/2 - |x|)
        const double y = LM_HP0 - fabs(x);
        a = y + LM_HP1;
        da = (y - a) + LM_HP1;
        n = 0;
    } else {                                             // Cody-Waite: x - n pi/2 in four parts
        const double t = fmad(x, 0x1.45f306dc9c883p-1, 0x1.8p52);   // x 2/pi + shifter
        const double xn = t - 0x1.8p52;
        const double y = fmad(-xn, LM_MP2, fmad(-xn, LM_MP1, x));
        n = (int)(dbits(t) & 3) + 1;
        const double t2 = fmad(-xn, LM_PP3, y);
        da = fmad(-xn, LM_PP3, y - t2);
        a = fmad(-xn, LM_PP4, t2);
        da += fmad(-xn, LM_PP4, t2 - a);
    }
    return sin64_quadrant(a, da, n);
}

}  // namespace lm
}  // namespace ionp
