"""CPU check of the arithmetic behind the GPU division fast paths (`quot_fast`,
`floor_divide_fast`, `fmod_fast` and `udiv64_trunc` in
anionpy_b200/csrc/ionp_scalar.cuh), with exact rational arithmetic as the
judge of every claim.

The hardware reciprocal approximation is modelled by every float32 value
within 1 ulp of the exact reciprocal (its documented bound), so each pair is
checked for all the reciprocals the hardware may return. For every pair the
fast path accepts:
  * t = trunc(p) is the truncated quotient q or q + 1 in magnitude;
  * m = x - t*y is a representable value (one fused multiply-add is exact);
  * t - [m != 0 and sign(m) != sign(y)] is the exact floor of x / y;
  * m, with y added back (x's sign) when m has the sign opposite to x's, is
    the exact fmod of x and y.
Pairs: quotients a rounding away from integers at every scale up to the
fast path's limit (2^19 float32, 2^36 float64), divisors over the whole
accepted range 2^-125 ... 2^125, subnormal dividends."""
import math
from fractions import Fraction

import numpy as np

F32_MAX_Q = 2.0 ** 19
F64_MAX_Q = 2.0 ** 36


def rn32(fr):
    """a Fraction rounded to the nearest value with 24 significant bits (ties
    to even), as a float32: float32 rounding in the normal range (the
    subnormal dividends' products lie far below 1, where the fast path's
    outcome does not depend on their last bits)"""
    return np.float32(_rn_bits(fr, 24))


def rn64(fr):
    return _rn_bits(fr, 53)


def _rn_bits(fr, bits):
    """nearest binary float with `bits` significant bits (normal range,
    ties to even), as a Python float (exact for bits <= 53)"""
    if fr == 0:
        return 0.0
    s = -1 if fr < 0 else 1
    a = abs(fr)
    e = a.numerator.bit_length() - a.denominator.bit_length()
    if Fraction(2) ** e > a:
        e -= 1
    # a in [2^e, 2^(e+1)); scale the significand to an integer of `bits` bits
    sc = Fraction(2) ** (bits - 1 - e)
    v = a * sc
    n = v.numerator // v.denominator
    rem = v - n
    if rem > Fraction(1, 2) or (rem == Fraction(1, 2) and n % 2 == 1):
        n += 1
    return s * float(Fraction(n) / sc)


def rcp32_candidates(yf):
    """every float32 within 1 ulp of 1/yf (yf a float32, normal reciprocal)"""
    exact = 1 / Fraction(float(yf))
    r = rn32(exact)
    out = []
    for c in (np.nextafter(r, np.float32(-np.inf)), r, np.nextafter(r, np.float32(np.inf))):
        ulp = Fraction(float(np.spacing(np.float32(abs(c)))))
        if abs(Fraction(float(c)) - exact) <= ulp:
            out.append(c)
    return out


def check_pair(x, y, t, m_exact):
    """the four claims for one accepted pair (x, y, t as Fractions)"""
    q_exact = x / y
    q_trunc = Fraction(math.trunc(q_exact))
    assert abs(t) in (abs(q_trunc), abs(q_trunc) + 1), (x, y, t)
    # floor
    dec = m_exact != 0 and (m_exact < 0) != (y < 0)
    assert t - (1 if dec else 0) == math.floor(q_exact), (x, y, t)
    # fmod
    fm = m_exact
    if fm != 0 and (fm < 0) != (x < 0):
        fm = fm + (abs(y) if x > 0 else -abs(y))
    assert fm == x - q_trunc * y, (x, y, t)


def pairs(rng, n, qmax, emin, emax, dt):
    """seeded pairs: y over the accepted exponent range, quotients near
    integers of every scale up to qmax, both signs"""
    e = rng.integers(emin, emax + 1, n)
    y = rng.uniform(1.0, 2.0, n) * np.exp2(e.astype(np.float64)) * rng.choice([-1.0, 1.0], n)
    y = y.astype(dt)
    scale = np.exp2(rng.uniform(-3, math.log2(qmax), n))
    q = np.round(scale) + rng.choice([-1e-7, 0.0, 1e-7, 0.3, 0.5, 0.999], n) * (dt == np.float32) \
        + rng.choice([-1e-15, 0.0, 1e-15, 0.3, 0.5, 0.999], n) * (dt == np.float64)
    with np.errstate(over="ignore"):  # an infinite dividend is skipped by the caller
        x = (q * y.astype(np.float64) * rng.choice([-1.0, 1.0], n)).astype(dt)
    return x, y


def test_float32_fast_path_claims():
    rng = np.random.default_rng(20261204)
    x, y = pairs(rng, 6000, F32_MAX_Q, -125, 124, np.float32)
    # subnormal dividends over small divisors
    xs = (rng.uniform(-1, 1, 200) * 2.0 ** -128).astype(np.float32)
    ys = (rng.uniform(1, 2, 200) * np.exp2(rng.integers(-125, -100, 200).astype(np.float64))).astype(np.float32)
    x, y = np.concatenate([x, xs]), np.concatenate([y, ys])
    checked = 0
    for xf, yf in zip(x, y):
        if not (np.isfinite(xf) and 2.0 ** -125 <= abs(float(yf)) <= 2.0 ** 125):
            continue
        X, Y = Fraction(float(xf)), Fraction(float(yf))
        for rc in rcp32_candidates(yf):
            p = rn32(Fraction(float(rn32(X * Fraction(float(rc))))) * (1 + Fraction(1, 2 ** 20)))
            if not abs(float(p)) < F32_MAX_Q:
                continue
            t = Fraction(math.trunc(float(p)))
            m = X - t * Y
            assert Fraction(float(rn32(m))) == m, (xf, yf, t)  # one FMA is exact
            check_pair(X, Y, t, m)
            checked += 1
    assert checked >= 6000  # at least one modelled reciprocal per pair


def test_float64_fast_path_claims():
    rng = np.random.default_rng(20261205)
    x, y = pairs(rng, 4000, F64_MAX_Q, -125, 124, np.float64)
    checked = 0
    for xd, yd in zip(x, y):
        if not (np.isfinite(xd) and 2.0 ** -125 <= abs(float(yd)) <= 2.0 ** 125):
            continue
        X, Y = Fraction(float(xd)), Fraction(float(yd))
        yf = np.float32(yd)  # the float32 the reciprocal approximation sees
        for rc in rcp32_candidates(yf):
            r0 = Fraction(float(rc))
            e = Fraction(rn64(1 - Y * r0))           # fma(-y, r0, 1)
            r1 = Fraction(rn64(r0 + r0 * e))         # fma(r0, e, r0)
            p = rn64(Fraction(rn64(X * r1)) * (1 + Fraction(1, 2 ** 38)))
            if not abs(p) < F64_MAX_Q:
                continue
            t = Fraction(math.trunc(p))
            m = X - t * Y
            assert Fraction(rn64(m)) == m, (xd, yd, t)  # one FMA is exact
            check_pair(X, Y, t, m)
            checked += 1
    assert checked >= 4000  # at least one modelled reciprocal per pair


def _f32_rz(u):
    """a non-negative integer rounded toward zero to float32 (24 bits)"""
    if u < (1 << 24):
        return Fraction(u)
    sh = u.bit_length() - 24
    return Fraction((u >> sh) << sh)


def _f32_ru(u):
    """a positive integer rounded up to float32 (24 bits)"""
    if u < (1 << 24):
        return Fraction(u)
    sh = u.bit_length() - 24
    top = u >> sh
    if (top << sh) != u:
        top += 1
    return Fraction(top << sh)


def test_int64_quotient_estimate_claims():
    """`udiv64_trunc`: fq = rn(rn(rz(ux) * rcp(ru(uy))) * (1 - 2^-20)) stays
    below ux / uy, so q = trunc(fq) never overshoots (ux - q uy cannot wrap),
    and below 2^20 it is at most two below the true quotient, which the two
    remainder steps repair; for every float32 reciprocal within 1 ulp."""
    rng = np.random.default_rng(20261206)
    cases = []
    for _ in range(3000):
        kind = rng.integers(0, 4)
        uy = int(rng.integers(1, 1 << int(rng.integers(1, 63))))
        if kind == 0:    # near-multiples
            q = int(rng.integers(1, 1 << 20))
            ux = q * uy + int(rng.integers(-2, 3))
        elif kind == 1:  # quotients near the 2^20 limit
            ux = ((1 << 20) + int(rng.integers(-4, 4))) * uy + int(rng.integers(0, uy))
        elif kind == 2:  # powers of two
            uy = 1 << int(rng.integers(0, 40))
            ux = int(rng.integers(0, 1 << 62))
        else:            # random bits
            ux = int(rng.integers(0, 1 << 63))
        if 0 < ux < (1 << 64) and uy > 0 and ux >= uy:
            cases.append((ux, uy))
    checked = 0
    for ux, uy in cases:
        yr = float(_f32_ru(uy))
        for rc in rcp32_candidates(np.float32(yr)):
            fq = rn32(Fraction(float(rn32(_f32_rz(ux) * Fraction(float(rc))))) * (1 - Fraction(1, 2 ** 20)))
            if not float(fq) < 2.0 ** 20:
                continue
            q_est = math.trunc(float(fq))
            q = ux // uy
            assert q_est <= q, (ux, uy)          # ux - q_est uy does not wrap
            assert q - q_est <= 2, (ux, uy)      # two repairs suffice
            checked += 1
    assert checked >= 1000


def _fast_results(x, y, dt):
    """floor_divide / fmod / remainder of the fast path's formulas (the
    reciprocal taken correctly rounded, one of the values the hardware
    approximation may return), and the mask of pairs the fast path takes"""
    one = dt(1)
    if dt == np.float32:
        rc = one / y
        p = (x * rc) * np.float32(1 + 2.0 ** -20)
        lim, lo, hi = 2.0 ** 19, 2.0 ** -125, 2.0 ** 125
    else:
        rc = one / y
        p = (x * rc) * (1 + 2.0 ** -38)
        lim, lo, hi = 2.0 ** 36, 2.0 ** -125, 2.0 ** 125
    ok = np.isfinite(x) & (np.abs(y) >= lo) & (np.abs(y) <= hi) & (np.abs(p) < lim)
    t = np.trunc(np.where(ok, p, 0)).astype(dt)
    # m = x - t y is exact (test_*_fast_path_claims); computed exactly here
    m = np.array([float(Fraction(float(a)) - Fraction(float(b)) * Fraction(float(c)))
                  for a, b, c in zip(np.where(ok, x, 0), t, np.where(ok, y, 1))]).astype(dt)
    sx, sy, sm = np.signbit(x), np.signbit(y), np.signbit(m)
    f = np.where((m != 0) & (sm != sy), t - one, t)
    zero_xy = np.where(sx != sy, dt(-0.0), dt(0.0))
    fdiv = np.where(f == 0, zero_xy, f)
    v = np.where((m != 0) & (sm != sx), m + np.copysign(y, x), m)
    fmod = np.where(v == 0, np.copysign(dt(0.0), x), v)
    rem = np.where(fmod == 0, np.copysign(dt(0.0), y),
                   np.where((fmod < 0) != (y < 0), fmod + y, fmod))
    return ok, {"floor_divide": fdiv, "fmod": fmod, "remainder": rem}


def test_fast_path_results_match_the_oracle():
    """The fast path's result formulas (zero signs included) against the
    oracle's floor_divide / fmod / remainder, bit for bit, on the pairs the
    fast path takes."""
    from oracle import oracle as O
    rng = np.random.default_rng(20261207)
    for dt, qmax in ((np.float32, F32_MAX_Q), (np.float64, F64_MAX_Q)):
        x, y = pairs(rng, 6000, qmax, -125, 124, dt)
        x[:300] = rng.choice([0.0, -0.0], 300).astype(dt)            # signed zero dividends
        x[300:600] = (y[300:600] * dt(0.25)) * rng.choice([-1, 1], 300).astype(dt)  # |x / y| < 1
        ok, got = _fast_results(x, y, dt)
        assert ok.sum() > 5000
        ib = np.uint32 if dt == np.float32 else np.uint64
        for op, r in got.items():
            want, _ = O.binary(op, x, y)
            bad = np.nonzero(ok & (r.view(ib) != np.asarray(want).view(ib)))[0]
            assert bad.size == 0, (op, np.dtype(dt).name, x[bad[:3]], y[bad[:3]], r[bad[:3]], want[bad[:3]])
