"""Generates ionp_constants.h: mathematical constants for the correctly
rounded exp/log/sin kernels, computed here with mpmath at 2000-bit
precision (no library tables are copied):

* PI_2_1..3 / LN2_1..3: pi/2 and ln 2 split into three doubles whose sum is
  the constant to ~160 bits (each part is the round-to-nearest remainder);
* TWO_OVER_PI[]: the binary expansion of 2/pi in 32-bit words (bit 1 of the
  fraction is the MSB of word 0), enough for Payne-Hanek reduction of every
  finite double.

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
    print("}  // namespace ionp")


if __name__ == "__main__":
    main()
