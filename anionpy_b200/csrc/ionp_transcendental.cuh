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

// ---------------------------------------------------------------------------
// float64 exp / log: a table-driven first pass accurate to about 2^-67
// (relative for exp, absolute for log), then Ziv's rounding test: if the
// first-pass value y_hi + y_lo, moved by its error bound either way, rounds to
// the same double, that double is the correctly rounded result; otherwise
// (about one argument in 2^11) the double-double evaluation decides. Every
// product that must be exact is a fused multiply-add (__fma_rn); everything
// else rounds as written (the library is built with -fmad=false).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void quick_two_sum(double a, double b, double* s, double* e) {  // |a| >= |b|
    *s = a + b;
    *e = b - (*s - a);
}
__device__ __forceinline__ void full_two_sum(double a, double b, double* s, double* e) {
    *s = a + b;
    const double bb = *s - a;
    *e = (a - (*s - bb)) + (b - bb);
}

// Tang's method with 64 table entries: x = k ln2/64 + r, |r| <= ln2/128,
// e^x = 2^(k >> 6) * 2^((k & 63)/64) * (1 + r + q), q = r^2/2 + ... + r^7/5040
// (the next term is below 2^-75). Error of y_hi + y_lo below 2^-66 relative.
__device__ __forceinline__ double exp_first(double x, bool* ok) {
    constexpr double INV = 1.0 / LN2_64_1;
    const double k = rint(x * INV);
    const int ki = (int)k;
    const int j = ki & 63, m = ki >> 6;
    const double p1 = k * LN2_64_1;
    const double p1e = __fma_rn(k, LN2_64_1, -p1);   // exact product error
    const double s = x - p1;                          // exact (Sterbenz)
    const double t = __fma_rn(k, LN2_64_2, p1e);
    double rh, rl;
    full_two_sum(s, -t, &rh, &rl);
    rl = rl - k * LN2_64_3;
    double q = __fma_rn(rh, 1.0 / 5040.0, 1.0 / 720.0);
    q = __fma_rn(q, rh, 1.0 / 120.0);
    q = __fma_rn(q, rh, 1.0 / 24.0);
    q = __fma_rn(q, rh, 1.0 / 6.0);
    q = __fma_rn(q, rh, 0.5);
    q = q * (rh * rh);
    const double tr = __fma_rn(rh, rl, rl) + q;      // e^(rh+rl) - 1 - rh
    const double th = __ldg(&EXP2_64_TAB[2 * j]), tl = __ldg(&EXP2_64_TAB[2 * j + 1]);
    const double ph = th * rh;
    const double pl = __fma_rn(th, rh, -ph);
    double sh, sl;
    quick_two_sum(th, ph, &sh, &sl);
    const double tail = __fma_rn(th, tr, __fma_rn(tl, rh, tl) + (pl + sl));
    double yh, yl;
    quick_two_sum(sh, tail, &yh, &yl);
    const double eb = yh * 0x1p-65;
    const double a = yh + (yl + eb), b = yh + (yl - eb);
    *ok = a == b;
    // 2^m, m in [-1021, 1022] on the first-pass range
    return a * __longlong_as_double((long long)(1023 + m) << 52);
}

// log x = e ln2 - log(inv_j) + log1p(r), r = y inv_j - 1 as an exact
// double-double (y = the mantissa in [1, 2), inv_j a 9-bit reciprocal,
// |r| <= 2^-7.6), log1p(r) = r + q, q to r^9/9. Near 1 (|x - 1| < 2^-7) log1p(x - 1) directly, with
// r^2/2 split exactly. Absolute error of y_hi + y_lo below 2^-66 (table
// path) or |r| 2^-66 (near 1).
__device__ __forceinline__ double log_first(double x, bool* ok) {
    double yh, yl, eb;
    const double d1 = x - 1.0;
    if (fabs(d1) < 0x1p-7) {
        const double r = d1;                          // exact (Sterbenz)
        const double hh = r * r;
        const double hl = __fma_rn(r, r, -hh);
        double q = __fma_rn(r, -1.0 / 10.0, 1.0 / 9.0);
        q = __fma_rn(q, r, -1.0 / 8.0);
        q = __fma_rn(q, r, 1.0 / 7.0);
        q = __fma_rn(q, r, -1.0 / 6.0);
        q = __fma_rn(q, r, 1.0 / 5.0);
        q = __fma_rn(q, r, -1.0 / 4.0);
        q = __fma_rn(q, r, 1.0 / 3.0);
        q = q * (hh * r);                             // r^3/3 - ... + r^10/10 (sign per term)
        double s, se;
        quick_two_sum(r, -0.5 * hh, &s, &se);
        const double tail = se + (q - 0.5 * hl);
        quick_two_sum(s, tail, &yh, &yl);
        eb = fabs(r) * 0x1p-65;
    } else {
        uint64_t bits = (uint64_t)__double_as_longlong(x);
        int e = 0;
        if (bits < (1ull << 52)) {                   // subnormal: scale into the normal range
            bits = (uint64_t)__double_as_longlong(x * 0x1p54);
            e = -54;
        }
        e += (int)(bits >> 52) - 1023;
        const double y = __longlong_as_double((long long)((bits & 0xFFFFFFFFFFFFFull) | 0x3FF0000000000000ull));
        const int j = (int)((bits >> 45) & 127);
        const double inv = __ldg(&LOG_INV_TAB[j]);
        const double lh = __ldg(&LOG_TAB[2 * j]), ll = __ldg(&LOG_TAB[2 * j + 1]);
        // r = y inv - 1 as rh + rl: the product split exactly, ph - 1 exact
        // (Sterbenz); r needs up to 54 bits, so one rounding would not do
        const double ph = y * inv;
        const double pl = __fma_rn(y, inv, -ph);
        double r, rl;
        quick_two_sum(ph - 1.0, pl, &r, &rl);
        double q = __fma_rn(r, 1.0 / 9.0, -1.0 / 8.0);
        q = __fma_rn(q, r, 1.0 / 7.0);
        q = __fma_rn(q, r, -1.0 / 6.0);
        q = __fma_rn(q, r, 1.0 / 5.0);
        q = __fma_rn(q, r, -1.0 / 4.0);
        q = __fma_rn(q, r, 1.0 / 3.0);
        q = __fma_rn(q, r, -0.5);
        q = q * (r * r);                              // log1p(r) - r
        q = q + (rl - r * rl);                        // + log1p(r + rl) - log1p(r), first order
        const double E = (double)e;
        const double ah = E * LN2_1;
        const double al = __fma_rn(E, LN2_1, -ah) + E * LN2_2;
        double s1, e1, s2, e2;
        full_two_sum(ah, lh, &s1, &e1);
        full_two_sum(s1, r, &s2, &e2);
        const double tail = ((e1 + e2) + (al + ll)) + q;
        quick_two_sum(s2, tail, &yh, &yl);
        eb = 0x1p-65 + fabs(yh) * 0x1p-90;
    }
    const double a = yh + (yl + eb), b = yh + (yl - eb);
    *ok = a == b;
    return a;
}

static __device__ __noinline__ double exp_slow(double x) {
    const dd::D2 r = dd::exp_dd(x);
    return r.hi + r.lo;  // the correctly rounded sum, also when hi is not
}
static __device__ __noinline__ double log_slow(double x) {
    const dd::D2 r = dd::log_dd(x);
    return r.hi + r.lo;  // the correctly rounded sum, also when hi is not
}

__device__ __forceinline__ double cr_exp(double x) {
    if (isnan_d(x)) return quiet_d(x);
    if (x > 709.8) return __longlong_as_double(0x7FF0000000000000ll);
    if (x < -745.2) return 0.0;
    if (x >= -708.0 && x <= 709.0) {  // normal results: the table-driven pass
        bool ok;
        const double r = exp_first(x, &ok);
        if (ok) return r;
    }
    return exp_slow(x);
}
__device__ __forceinline__ double cr_log(double x) {
    if (isnan_d(x)) return quiet_d(x);
    if (x < 0.0) return dnan_d();
    if (x == 0.0) return __longlong_as_double((long long)0xFFF0000000000000ull);
    if (isinf(x)) return x;
    bool ok;
    const double r = log_first(x, &ok);
    if (ok) return r;
    return log_slow(x);
}
// sin x for |x| <= 2^20: Cody-Waite reduction x = k pi/2 + r with pi/2 in
// three parts (r as a double-double, error below |k| 2^-104), then
// |r| = a + b with a = i/64 from a table of sin(a), cos(a) as double-double
// pairs and |b| <= 1/128:
//   sin(a + b) = S + C b + [S (cos b - 1) + C (sin b - b)]
//   cos(a + b) = C - S b + [C (cos b - 1) - S (sin b - b)]
// with the products C b, S b split exactly, the bracketed tails (below
// 2^-14 relative) in double and the first-order effect of b's low part on
// them kept. Error of y_hi + y_lo below about 2^-66 absolute, tested against
// 2^-64 (and 2^-62 relative when a = 0), plus the reduction error.
__device__ __forceinline__ double sin_first(double x, bool* ok) {
    constexpr double TWO_OVER_PI = 0.63661977236758134308;
    const double k = rint(x * TWO_OVER_PI);
    const int q = ((int)k) & 3;
    const double p1 = k * PI_2_1;
    const double p1e = __fma_rn(k, PI_2_1, -p1);
    const double s = x - p1;                          // exact (Sterbenz)
    const double t = __fma_rn(k, PI_2_2, p1e);
    double rh, rl;
    full_two_sum(s, -t, &rh, &rl);
    rl = rl - k * PI_2_3;
    const bool neg = rh < 0.0;
    if (neg) { rh = -rh; rl = -rl; }
    const int i = (int)rint(rh * 64.0);
    const double bh = rh - (double)i * 0.015625;      // exact
    const double bl = rl;
    const double b2 = bh * bh;
    double sbt = __fma_rn(b2, -1.0 / 5040.0, 1.0 / 120.0);
    sbt = __fma_rn(sbt, b2, -1.0 / 6.0);
    sbt = sbt * (b2 * bh);                            // sin b - b
    double cbm = __fma_rn(b2, 1.0 / 40320.0, -1.0 / 720.0);
    cbm = __fma_rn(cbm, b2, 1.0 / 24.0);
    cbm = __fma_rn(cbm, b2, -0.5);
    cbm = cbm * b2;                                   // cos b - 1
    const double sh = __ldg(&SINCOS_64_TAB[4 * i]), sl = __ldg(&SINCOS_64_TAB[4 * i + 1]);
    const double ch = __ldg(&SINCOS_64_TAB[4 * i + 2]), cl = __ldg(&SINCOS_64_TAB[4 * i + 3]);
    double s1, e1, tail;
    if ((q & 1) == 0) {   // sin r
        const double ph = ch * bh;
        const double pl = __fma_rn(ch, bh, -ph);
        full_two_sum(sh, ph, &s1, &e1);
        // ... - S b bl: the first-order effect of bl on S (cos b - 1)
        tail = (e1 + pl) + ((ch * bl + cl * bh) + sl) + ((sh * cbm + ch * sbt) - sh * (bh * bl));
    } else {              // cos r
        const double ph = sh * bh;
        const double pl = __fma_rn(sh, bh, -ph);
        full_two_sum(ch, -ph, &s1, &e1);
        tail = (e1 - pl) + (cl - (sh * bl + sl * bh)) + ((ch * cbm - sh * sbt) - ch * (bh * bl));
    }
    double yh, yl;
    quick_two_sum(s1, tail, &yh, &yl);
    const double eb = (i == 0 && (q & 1) == 0 ? fabs(yh) * 0x1p-62 : 0x1p-64) + fabs(k) * 0x1p-103 + 0x1p-104;
    const double a = yh + (yl + eb), b = yh + (yl - eb);
    *ok = a == b;
    // sin x = sin r, cos r, -sin r, -cos r for q = 0..3; sin(-r) = -sin r
    const bool flip = (q >= 2) != (neg && (q & 1) == 0);
    return flip ? -a : a;
}

static __device__ __noinline__ double sin_slow(double x) {
    const dd::D2 r = dd::sin_dd(x);
    return r.hi + r.lo;
}

__device__ __forceinline__ double cr_sin(double x) {
    if (isnan_d(x)) return quiet_d(x);
    if (isinf(x)) return dnan_d();
    if (x == 0.0) return x;
    const double ax = fabs(x);
    if (ax < 0x1p-26) return x;  // sin x = x (1 - x^2/6 ...) rounds to x
    if (ax <= 0x1p20) {
        bool ok;
        const double r = sin_first(x, &ok);
        if (ok) return r;
    }
    return sin_slow(x);
}

}  // namespace ionp
