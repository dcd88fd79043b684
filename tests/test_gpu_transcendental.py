"""GPU exp / log / sin: bit-exact against correctly rounded references and
within the reference's tolerance of its own libm (glibc) results.

The reference's recorded ULP tolerances (tests/differential/
ufunc_registry.py: exp 0, log 0, sin 1 for float32 / 0 for float64) are
measured against NumPy on the reference's macOS host. On Linux the reference
calls glibc, whose float32 expf/logf/sinf are not always correctly rounded
(expf is off by up to ~0.5000001 ULP); these kernels are correctly rounded,
so they agree with glibc bit for bit wherever glibc is correctly rounded and
differ by exactly 1 ULP elsewhere."""
import mpmath
import numpy as np
import pytest

from oracle import oracle as O
from tests._util import assert_bits_equal, ulp_distance

ap = pytest.importorskip("anionpy_b200")
pytestmark = pytest.mark.gpu


def inputs(fn, dt, n, seed):
    rng = np.random.default_rng(seed)
    if fn == "exp":
        x = rng.uniform(-110, 95, n)
    elif fn == "log":
        x = np.concatenate([1e6 * (1 - rng.random(n // 2)), np.exp(rng.uniform(-740, 709, n - n // 2))])
    else:
        x = np.concatenate([rng.standard_normal(n // 2) * 10, rng.uniform(-1e6, 1e6, n // 4),
                            np.exp(rng.uniform(0, 700, n - n // 2 - n // 4)) * rng.choice([-1, 1], n - n // 2 - n // 4)])
    specials = [0.0, -0.0, 1.0, -1.0, np.inf, -np.inf, np.nan, -np.nan, 1e-45, 5e-324, 88.72283, -103.97, 709.78,
                -745.13, 1e22, 3.4e38, 2.0 ** 24, np.pi, np.pi / 2, 1e-10]
    with np.errstate(all="ignore"):
        return np.concatenate([np.array(specials), x]).astype(dt)


def cr_f32(fn, x):
    xl = x.astype(np.longdouble)
    with np.errstate(all="ignore"):
        return getattr(np, fn)(xl).astype(np.float32)


def cr_f64(fn, x):
    mpmath.mp.prec = 140
    out = np.empty_like(x)
    f = {"exp": mpmath.exp, "log": mpmath.log, "sin": mpmath.sin}[fn]
    for i, v in enumerate(x):
        # zeros too: mpmath has no signed zero (sin(-0.0) is -0.0)
        if np.isnan(v) or np.isinf(v) or v == 0 or (fn == "log" and v <= 0) or (fn == "exp" and abs(v) > 800):
            with np.errstate(all="ignore"):
                out[i] = getattr(np, fn)(v)
            continue
        out[i] = float(f(mpmath.mpf(float(v))))
    return out


@pytest.mark.parametrize("fn", ["exp", "log", "sin"])
def test_float32_correctly_rounded(fn):
    x = inputs(fn, np.float32, 1 << 20, 1)
    got = getattr(ap, fn)(ap.from_numpy(x)).get()
    want = cr_f32(fn, x)
    nan = np.isnan(want)
    assert np.isnan(got[nan]).all()
    assert_bits_equal(got[~nan], want[~nan], f"{fn} float32 vs correctly rounded")
    # against the oracle (glibc), including NaN bits
    ref, _ = O.unary(fn, x)
    d = ulp_distance(got, ref)
    assert d.max() <= 1, f"{fn}: max ulp vs glibc {d.max()}"
    # every disagreement with glibc is an argument where glibc itself is not
    # correctly rounded (glibc 2.39 on x86-64: expf ~0.06%, logf ~0.01%,
    # sinf ~1% of these inputs); wherever glibc is correctly rounded the
    # results are identical bit for bit
    glibc_cr = ulp_distance(ref, want) == 0
    assert not np.any(d[glibc_cr & ~nan]), f"{fn}: differs from glibc where glibc is correctly rounded"
    assert got[nan].tobytes() == ref[nan].tobytes(), "NaN payloads"


@pytest.mark.parametrize("fn", ["exp", "log", "sin"])
def test_float64_correctly_rounded(fn):
    x = inputs(fn, np.float64, 20000, 2)
    got = getattr(ap, fn)(ap.from_numpy(x)).get()
    want = cr_f64(fn, x)
    nan = np.isnan(want)
    assert_bits_equal(got[~nan], want[~nan], f"{fn} float64 vs correctly rounded")
    ref, _ = O.unary(fn, x)
    d = ulp_distance(got, ref)
    assert d.max() <= 1, f"{fn}: max ulp vs glibc {d.max()}"
    assert got[nan].tobytes() == ref[nan].tobytes(), "NaN payloads"


def stress64(fn, n, seed):
    """float64 arguments at the edges of the table-driven first pass: near
    the table's interval ends, around |x - 1| = 2^-7 for log, subnormals,
    powers of two, the ends of exp's normal range, tiny arguments, sin near
    multiples of pi/2 and around the reduction limit 2^20."""
    rng = np.random.default_rng(seed)
    if fn == "exp":
        k = rng.integers(-65000, 65000, n // 2)
        parts = [k * (np.log(2) / 64) + rng.uniform(-1e-9, 1e-9, n // 2),
                 rng.uniform(-708.5, -707.5, n // 8), rng.uniform(708.5, 709.9, n // 8),
                 rng.uniform(-1e-12, 1e-12, n // 8) * np.exp2(-rng.integers(0, 40, n // 8))]
    elif fn == "sin":
        k = rng.integers(-600000, 600000, n // 4)
        parts = [k * (np.pi / 2) + rng.uniform(-1e-6, 1e-6, n // 4),
                 rng.integers(0, 52, n // 4) / 64.0 + rng.uniform(-2 ** -7, 2 ** -7, n // 4),
                 rng.uniform(-2 ** 21, 2 ** 21, n // 8), rng.uniform(-1e-7, 1e-7, n // 8),
                 (1 - 2 * rng.integers(0, 2, n // 8)) * np.exp2(rng.uniform(-30, 20, n // 8))]
    else:
        parts = [1 + rng.uniform(-2 ** -6, 2 ** -6, n // 2), 1 + rng.uniform(-1e-12, 1e-12, n // 8),
                 np.exp2(rng.integers(-1074, 1024, n // 8).astype(np.float64)),
                 rng.uniform(0, 1, n // 8) * 2.0 ** -1030, 1 + np.arange(1, 129) / 128.0]
    return np.concatenate(parts).astype(np.float64)


@pytest.mark.parametrize("fn", ["exp", "log", "sin"])
def test_float64_first_pass_edges(fn):
    x = stress64(fn, 24000, 5)
    got = getattr(ap, fn)(ap.from_numpy(x)).get()
    want = cr_f64(fn, x)
    ok = np.isfinite(want)
    assert_bits_equal(got[ok], want[ok], f"{fn} float64 edges vs correctly rounded")


@pytest.mark.parametrize("fn", ["exp", "log", "sin"])
def test_float16_and_int_promotion(fn):
    rng = np.random.default_rng(3)
    x16 = (rng.standard_normal(4096) * 4).astype(np.float16)
    if fn == "log":
        x16 = np.abs(x16)
    got = getattr(ap, fn)(ap.from_numpy(x16)).get()
    ref, _ = O.unary(fn, x16)
    assert got.dtype == np.float16
    assert ulp_distance(got, ref).max() <= 1
    xi = rng.integers(1, 100, 1000).astype(np.int16)  # int16 -> float32 loop
    g2 = getattr(ap, fn)(ap.from_numpy(xi)).get()
    r2, _ = O.unary(fn, xi)
    assert g2.dtype == r2.dtype == np.float32
    assert ulp_distance(g2, r2).max() <= 1


def test_log_fpe():
    with ap.errstate(divide="raise"):
        with pytest.raises(FloatingPointError, match="divide by zero encountered in log"):
            ap.log(ap.from_numpy(np.array([0.0, 1.0])))
    with ap.errstate(invalid="raise"):
        with pytest.raises(FloatingPointError, match="invalid value encountered in log"):
            ap.log(ap.from_numpy(np.array([0.0, -1.0], np.float32)))


@pytest.mark.parametrize("fn", ["exp", "log", "sin"])
@pytest.mark.parametrize("dt", [np.float32, np.float64], ids=lambda d: np.dtype(d).name)
def test_strided_slices(fn, dt):
    """Step-2 and step-3 slices (the one-strided-run path) give the same
    bits as the contiguous kernel, and log's FPE categories still fire."""
    x = inputs(fn, dt, 30000 if dt == np.float64 else 1 << 18, 9)
    d = ap.from_numpy(x)
    full = getattr(ap, fn)(d).get()
    for step in (2, 3):
        got = getattr(ap, fn)(d[::step]).get()
        assert_bits_equal(got, full[::step], f"{fn} {np.dtype(dt).name} step {step}")
    if fn == "log":
        with ap.errstate(divide="raise"):
            with pytest.raises(FloatingPointError, match="divide by zero encountered in log"):
                ap.log(ap.from_numpy(np.array([1.0, 5.0, 0.0, 7.0], dt))[::2])
