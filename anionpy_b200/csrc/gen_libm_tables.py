"""Generates ionp_libm_tables.h, the tables of the exp/log/sin restatements
in ionp_libm.cuh.

The engine reproduces the host C library's results bit for bit (glibc 2.39
on x86-64, which the reference reaches through Rust's f32::exp/ln/sin and
f64::exp/ln/sin: ionp-core/src/ufunc.rs:4237-4367). Its tables are
mathematical functions of the index, computed here with mpmath (300 bits,
2400 for the digits of 2/pi) and rounded to nearest:

* EXPF_TAB[32]  2^(i/32) as double bits minus i << 47 (the exponent part
  that the caller adds back), for exp32;
* EXP_TAB[256]  for i < 128: the bits of t_i = 2^(i/128)/H_i - 1 and of
  H_i = (double)2^(i/128) minus i << 45, for exp64;
* LOGF_TAB[32]  (invc, logc) for 16 subintervals, for log32: invc is the
  published reduction constant (its choice is a search the source does not
  restate), logc = (double)log(1/invc) is computed here;
* LOG_TAB[256]  (invc, logc) for 128 subintervals, for log64, read from
  gen_libm_log_table.c (the published selection rule, see there);
* SINCOS_TAB[440]  sin(i/128) and cos(i/128), i < 110, each as a rounded
  double plus the rounded remainder, for sin64;
* TWO_OVER_PI_24[75]  2/pi in 24-bit chunks (2/pi = sum c_j 2^(-24(j+1))),
  for sin64's reduction of |x| >= 105414350;
* TWO_OVER_PI_W[24]  32-bit windows of 2/pi's bits ending at byte j, for
  sin32's reduction of |x| >= 120.

Run from this directory:
  python gen_libm_tables.py > ionp_libm_tables.h
(needs gcc with libquadmath and an x86-64 glibc with FMA for the log table).
"""
import os
import struct
import subprocess
import tempfile

import mpmath

mpmath.mp.prec = 300
HERE = os.path.dirname(os.path.abspath(__file__))

# log32's published reduction constants 1/c (16 subintervals of
# [0x1.66p-1, 0x1.66p0)); glibc sysdeps/ieee754/flt-32/e_logf_data.c
LOGF_INVC = [
    "0x1.661ec79f8f3bep+0", "0x1.571ed4aaf883dp+0", "0x1.49539f0f010bp+0", "0x1.3c995b0b80385p+0",
    "0x1.30d190c8864a5p+0", "0x1.25e227b0b8eap+0", "0x1.1bb4a4a1a343fp+0", "0x1.12358f08ae5bap+0",
    "0x1.0953f419900a7p+0", "0x1p+0", "0x1.e608cfd9a47acp-1", "0x1.ca4b31f026aap-1",
    "0x1.b2036576afce6p-1", "0x1.9c2d163a1aa2dp-1", "0x1.886e6037841edp-1", "0x1.767dcf5534862p-1",
]


def bits(d: float) -> int:
    return struct.unpack("<Q", struct.pack("<d", d))[0]


def log_table():
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "gen_log")
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-ffp-contract=off",
                               os.path.join(HERE, "gen_libm_log_table.c"), "-o", exe, "-lquadmath", "-lm"])
        out = subprocess.check_output([exe], text=True)
    rows = []
    for line in out.split("\n"):
        line = line.strip().strip(",").strip("{}")
        if line:
            a, b = (s.strip() for s in line.split(","))
            rows.append((float.fromhex(a), float.fromhex(b)))
    assert len(rows) == 128
    return rows


def emit(name, ctype, vals, fmt, per_line=4):
    print(f"LM_TAB {ctype} {name}[{len(vals)}] = {{")
    for i in range(0, len(vals), per_line):
        print("    " + ", ".join(fmt(v) for v in vals[i:i + per_line]) + ",")
    print("};")


def main():
    u64 = lambda v: f"0x{v:016x}ull"
    dbl = lambda v: v.hex()
    u32 = lambda v: f"0x{v:08x}u"

    expf = []
    for i in range(32):
        h = float(mpmath.power(2, mpmath.mpf(i) / 32))
        expf.append((bits(h) - (i << 47)) & (2 ** 64 - 1))
    exp = []
    for i in range(128):
        v = mpmath.power(2, mpmath.mpf(i) / 128)
        h = float(v)
        t = float(v / mpmath.mpf(h) - 1)
        exp += [bits(t), (bits(h) - (i << 45)) & (2 ** 64 - 1)]
    logf = []
    for s in LOGF_INVC:
        ic = float.fromhex(s)
        logf += [ic, float(-mpmath.log(mpmath.mpf(ic)))]
    logt = [v for row in log_table() for v in row]
    sincos = []
    for i in range(110):
        a = mpmath.mpf(i) / 128
        for f in (mpmath.sin, mpmath.cos):
            v = f(a)
            hi = float(v)
            sincos += [hi, float(v - mpmath.mpf(hi))]
    mpmath.mp.prec = 2400   # 75 chunks of 24 bits of 2/pi need ~1800 bits
    frac = 2 / mpmath.pi
    chunks = []
    for _ in range(75):
        frac *= 2 ** 24
        c = int(mpmath.floor(frac))
        chunks.append(float(c))
        frac -= c
    byts = []
    frac = 2 / mpmath.pi
    for _ in range(24):
        frac *= 256
        c = int(mpmath.floor(frac))
        byts.append(c)
        frac -= c
    wins = []
    for j in range(24):
        w = 0
        for b in byts[max(0, j - 3):j + 1]:
            w = (w << 8) | b
        wins.append(w)

    print("// Generated by gen_libm_tables.py. Do not edit.")
    print("// Tables of the exp/log/sin restatements in ionp_libm.cuh.")
    print("#pragma once")
    emit("EXPF_TAB", "unsigned long long", expf, u64)
    emit("EXP_TAB", "unsigned long long", exp, u64)
    emit("LOGF_TAB", "double", logf, dbl)
    emit("LOG_TAB", "double", logt, dbl)
    emit("SINCOS_TAB", "double", sincos, dbl)
    emit("TWO_OVER_PI_24", "double", chunks, lambda v: f"{int(v)}.0", per_line=8)
    emit("TWO_OVER_PI_W", "unsigned int", wins, u32, per_line=8)


if __name__ == "__main__":
    main()
