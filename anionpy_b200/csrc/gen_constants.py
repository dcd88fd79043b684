"""Generates ionp_constants.h: mathematical constants for the correctly
rounded exp/log/sin kernels, computed here with mpmath at 2000-bit
precision (no library tables are copied):

* PI_2_1..3 / LN2_1..3: pi/2 and ln 2 split into three doubles whose sum is
  the constant to ~160 bits (each part is the round-to-nearest remainder);
* TWO_OVER_PI[]: the binary expansion of 2/pi in 32-bit words (bit 1 of the
  fraction is the MSB of word 0), enough for Payne-Hanek reduction of every
  finite double;
* EXP2_64_TAB[]: 2^(j/64), j = 0..63, as double-double pairs (hi, lo), and
  LN2_64_1/2/3: ln(2)/64 in three parts, for the table-driven float64 exp;
* LOG_INV_TAB[] / LOG_TAB[]: for y in [1 + j/128, 1 + (j+1)/128), a 9-bit
  reciprocal inv_j of the interval midpoint (inv_0 = 1 exactly) and
  -log(inv_j) as a double-double pair, for the table-driven float64 log
  (y * inv_j - 1 is exact as a double-double: one product split by a fused
  multiply-add);
* SINCOS_64_TAB[]: sin(i/64) and cos(i/64), i = 0..51, as double-double
  pairs (sin hi, sin lo, cos hi, cos lo), for the table-driven float64 sin.

Run: python anionpy_b200/csrc/gen_constants.py > anionpy_b200/csrc/ionp_constants.h
"""
import mpmath

mpmath.mp.prec = 2000


def split3(v):
    parts = []
    r = v
    for _ in range(3):
        d = float(r)
        parts.append(d)
        r = r - mpmath.mpf(d)
    return parts


def main():
    pi2 = split3(mpmath.pi / 2)
    ln2 = split3(mpmath.log(2))
    words = []
    frac = 2 / mpmath.pi  # < 1
    for _ in range(48):
        frac *= 2 ** 32
        w = int(mpmath.floor(frac))
        words.append(w)
        frac -= w
    print("// Generated by gen_constants.py (mpmath, 2000-bit precision). Do not edit.")
    print("#pragma once")
    print("#include <cstdint>")
    print("namespace ionp {")
    for name, parts in (("PI_2", pi2), ("LN2", ln2)):
        for i, p in enumerate(parts):
            print(f"constexpr double {name}_{i + 1} = {p.hex()};")
    print("// 2/pi = 0.w0 w1 w2 ... (32 bits per word)")
    print("__host__ __device__ constexpr uint32_t two_over_pi_word(int i) {")
    print("    constexpr uint32_t W[48] = {" + ", ".join(f"0x{w:08X}u" for w in words) + "};")
    print("    return (i >= 0 && i < 48) ? W[i] : 0u;")
    print("}")
    ln2_64 = split3(mpmath.log(2) / 64)
    for i, p in enumerate(ln2_64):
        print(f"constexpr double LN2_64_{i + 1} = {p.hex()};")
    print("// 2^(j/64): hi, lo")
    tab = []
    for j in range(64):
        v = mpmath.power(2, mpmath.mpf(j) / 64)
        hi = float(v)
        lo = float(v - mpmath.mpf(hi))
        tab += [hi, lo]
    print("__device__ static const double EXP2_64_TAB[128] = {" + ", ".join(t.hex() for t in tab) + "};")
    invs, logs = [], []
    for j in range(128):
        if j == 0:
            k = 512
        else:
            mid = 1 + (mpmath.mpf(j) + mpmath.mpf(0.5)) / 128
            k = int(mpmath.nint(512 / mid))
        inv = mpmath.mpf(k) / 512
        invs.append(float(inv))
        lv = -mpmath.log(inv)
        hi = float(lv)
        lo = float(lv - mpmath.mpf(hi))
        logs += [hi, lo]
    print("// 9-bit reciprocals of the log table intervals, and -log of each (hi, lo)")
    print("__device__ static const double LOG_INV_TAB[128] = {" + ", ".join(t.hex() for t in invs) + "};")
    print("__device__ static const double LOG_TAB[256] = {" + ", ".join(t.hex() for t in logs) + "};")
    sc = []
    for i in range(52):
        a = mpmath.mpf(i) / 64
        for v in (mpmath.sin(a), mpmath.cos(a)):
            hi = float(v)
            sc += [hi, float(v - mpmath.mpf(hi))]
    print("// sin(i/64) hi, lo, cos(i/64) hi, lo")
    print("__device__ static const double SINCOS_64_TAB[208] = {" + ", ".join(t.hex() for t in sc) + "};")
    print("}  // namespace ionp")


if __name__ == "__main__":
    main()
