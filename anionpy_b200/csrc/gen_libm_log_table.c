/* Selects the 128 (invc, logc) pairs of the float64 log reduction table
 * (ionp_libm.cuh, log64) and prints them, one "{invc, logc}," line each.
 *
 * The C library whose results the engine reproduces (glibc 2.39,
 * sysdeps/ieee754/dbl-64/e_log_data.c) publishes how its table was built:
 * for the i-th of 128 subintervals of [0x1.6p-1, 0x1.6p0) (split on the top
 * 7 mantissa bits of z - 0x1.6p-1), try the doubles invc within 2^29 ulps
 * of 1/center and keep one for which
 *   (1) logc = (double)log(1/invc) is a multiple of 2^-43, so that
 *       k*ln2hi + logc is exact, and
 *   (2) the rounding error of that logc is below 2^-66.
 * About 250 candidates per subinterval pass both tests; the source does not
 * state which of them it kept. This program enumerates them (logc on the
 * 2^-43 grid, invc = the double nearest exp(-logc), error from quad
 * precision) and keeps the candidate whose log, evaluated exactly as log64
 * evaluates it, agrees with the host C library's log() on 200,000 seeded
 * arguments from the subinterval (scaled by 2^e, e in [-20, 19], e != 0).
 * Exactly one candidate agrees in every subinterval; the program fails if
 * that ever stops being true.
 *
 * Build and run (x86-64 with FMA, glibc's FMA variant of log):
 *   gcc -O2 -fopenmp -ffp-contract=off gen_libm_log_table.c -lquadmath -lm
 */
#include <math.h>
#include <omp.h>
#include <quadmath.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static uint64_t bits_of(double d) { uint64_t u; memcpy(&u, &d, 8); return u; }
static double from_bits(uint64_t u) { double d; memcpy(&d, &u, 8); return d; }

/* polynomial of log64's table path: log1p(r) - r ~= r^2 (P0 + r P1 + ...) */
static const double P[5] = {-0x1.0000000000001p-1, 0x1.555555551305bp-2, -0x1.fffffffeb459p-3,
                            0x1.999b324f10111p-3, -0x1.55575e506c89fp-3};
static const double LN2_HI = 0x1.62e42fefa3800p-1, LN2_LO = 0x1.ef35793c76730p-45;
#define Z0 0x3fe6000000000000ULL
#define SAMPLES 200000

/* log64's table path for one candidate entry (same operations, same fused
 * multiply-adds, same order) */
static double table_path(double x, double invc, double logc) {
    uint64_t ix = bits_of(x), d = ix - Z0;
    double k = (double)((int64_t)d >> 52);
    double z = from_bits(ix - (d & (0xfffULL << 52)));
    double r = fma(z, invc, -1.0);
    double w = fma(k, LN2_HI, logc), hi = w + r;
    double lo = fma(k, LN2_LO, (w - hi) + r);
    double r2 = r * r;
    double q = fma(r2, fma(r, P[4], P[3]), fma(r, P[2], P[1]));
    return fma(r * r2, q, fma(r2, P[0], lo)) + hi;
}

static uint64_t next(uint64_t s[2]) {  /* xorshift128+ */
    uint64_t a = s[0];
    const uint64_t b = s[1];
    s[0] = b;
    a ^= a << 23;
    s[1] = a ^ b ^ (a >> 17) ^ (b >> 26);
    return s[1] + b;
}

int main(void) {
    const long long W = 1LL << 29;
    double invc_of[128], logc_of[128];
    int found[128];
    #pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < 128; i++) {
        double *xs = malloc(SAMPLES * sizeof(double)), *ys = malloc(SAMPLES * sizeof(double));
        uint64_t st[2] = {0x9E3779B97F4A7C15ULL * (uint64_t)(i + 7), 0xD1B54A32D192ED03ULL};
        for (int t = 0; t < SAMPLES; t++) {
            uint64_t u = next(st);
            uint64_t zb = Z0 + ((uint64_t)i << 45) + ((u >> 20) & ((1ULL << 45) - 1));
            int e = (int)((u >> 3) % 40) - 20;
            if (e == 0) e = 5;
            xs[t] = from_bits(zb) * ldexp(1.0, e);
            ys[t] = log(xs[t]);
        }
        double zlo = from_bits(Z0 + ((uint64_t)i << 45)), zhi = from_bits(Z0 + ((uint64_t)(i + 1) << 45));
        __float128 center = ((__float128)zlo + (__float128)zhi) / 2;
        double ic0 = (double)(1 / center);
        double icmin = from_bits(bits_of(ic0) - W), icmax = from_bits(bits_of(ic0) + W);
        long long m0 = (long long)ceilq(-logq((__float128)icmax) * 0x1p43Q);
        long long m1 = (long long)floorq(-logq((__float128)icmin) * 0x1p43Q);
        __float128 step = expq(-0x1p-43Q), e = 0;
        found[i] = 0;
        for (long long m = m0; m <= m1; m++) {
            e = ((m - m0) & 1023) == 0 ? expq(-(__float128)m * 0x1p-43Q) : e * step;
            double ic = (double)e;
            if (ic < icmin || ic > icmax) continue;
            __float128 err = ((__float128)ic - e) / e;   /* -log(ic) - m 2^-43, to first order */
            if (err < 0) err = -err;
            if (err >= 0x1p-66Q) continue;
            double lc = (double)((__float128)m * 0x1p-43Q);
            int agree = 1;
            for (int t = 0; t < SAMPLES && agree; t++)
                agree = bits_of(table_path(xs[t], ic, lc)) == bits_of(ys[t]);
            if (agree) { invc_of[i] = ic; logc_of[i] = lc; found[i]++; }
        }
        free(xs);
        free(ys);
    }
    for (int i = 0; i < 128; i++) {
        if (found[i] != 1) {
            fprintf(stderr, "subinterval %d: %d agreeing candidates\n", i, found[i]);
            return 1;
        }
    }
    for (int i = 0; i < 128; i++) printf("{%a, %a},\n", invc_of[i], logc_of[i]);
    return 0;
}
