"""GPU exp / log / sin / cos: identical bits to the oracle, the host C library
that the reference's f32::exp/ln/sin/cos and f64::exp/ln/sin/cos call on
Linux (ionp-core/src/ufunc.rs:4237-4367). The reference records 0 ULP for exp
and log and for float64 sin and cos (tests/differential/ufunc_registry.py);
float32 sin and cos are held to the same 0 ULP here. NaN results must match
bit for bit too."""
import numpy as np
import pytest

from oracle import oracle as O
from tests._util import assert_bits_equal

ap = pytest.importorskip("anionpy_b200")
pytestmark = pytest.mark.gpu

SPECIALS = [0.0, -0.0, 1.0, -1.0, np.inf, -np.inf, np.nan, -np.nan, 1e-45, 5e-324, 88.72283, -103.97, 709.78,
            -745.13, 1e22, 3.4e38, 2.0 ** 24, np.pi, np.pi / 2, 1e-10, 120.0, -120.0, 105414350.0, 1e300, -1e300]


def check(fn, x, what):
    got = getattr(ap, fn)(ap.from_numpy(x)).get()
    want, _ = O.unary(fn, x)
    assert_bits_equal(got, want, f"{fn} {what}")


def f32_patterns(stride, offset):
    """every stride-th float32 bit pattern: all signs, exponents, NaN payloads"""
    return np.arange(offset, 1 << 32, stride, dtype=np.uint64).astype(np.uint32).view(np.float32)


@pytest.mark.parametrize("fn", ["exp", "log", "sin", "cos"])
def test_float32_bit_patterns(fn):
    check(fn, f32_patterns(251, 17), "float32 every 251st bit pattern")


@pytest.mark.parametrize("fn", ["exp", "log", "sin", "cos"])
@pytest.mark.parametrize("dt", [np.float32, np.float64], ids=lambda d: np.dtype(d).name)
def test_benchmark_distributions(fn, dt):
    """the distributions of the 2^28-element sweep: exp on U[-100, 100], log
    on U(0, 1e6], sin (and cos) on 10 N(0, 1)"""
    rng = np.random.default_rng(11)
    n = 1 << 20
    x = {"exp": rng.uniform(-100, 100, n), "log": 1e6 * (1 - rng.random(n)),
         "sin": 10 * rng.standard_normal(n), "cos": 10 * rng.standard_normal(n)}[fn]
    with np.errstate(all="ignore"):
        x = np.concatenate([np.array(SPECIALS), x]).astype(dt)
    check(fn, x, f"{np.dtype(dt).name} sweep distribution")


def f64_classes(fn, n, seed):
    """float64 arguments reaching every path of the restated algorithms:
    any bit pattern, moderate exponents, exp's subnormal and overflow ends,
    log near 1 and subnormals, sin and cos in each reduction range, near
    multiples of pi/2 and beyond 105414350"""
    rng = np.random.default_rng(seed)
    u = rng.integers(0, 2 ** 63, n, dtype=np.int64).astype(np.uint64) * np.uint64(2) + rng.integers(0, 2, n).astype(np.uint64)
    parts = [u.view(np.float64)]
    mant = (u & np.uint64(0x800FFFFFFFFFFFFF))
    parts.append((mant | (np.uint64(900) + u % np.uint64(250)) << np.uint64(52)).view(np.float64))
    if fn == "exp":
        parts += [rng.uniform(-745.2, -708, n), rng.uniform(705, 709.8, n), rng.uniform(-1e-10, 1e-10, n),
                  rng.integers(-65000, 65000, n) * (np.log(2) / 128) + rng.uniform(-1e-12, 1e-12, n)]
    elif fn == "log":
        parts += [rng.uniform(0.9, 1.1, n), 1 + rng.uniform(-1e-12, 1e-12, n),
                  (u & np.uint64(0x000FFFFFFFFFFFFF)).view(np.float64), 1e6 * (1 - rng.random(n))]
    else:
        big = (mant | (np.uint64(1049) + u % np.uint64(975)) << np.uint64(52)).view(np.float64)
        parts += [rng.uniform(-0.13, 0.13, n), rng.uniform(-2.5, 2.5, n), rng.uniform(-1e8, 1e8, n), big,
                  rng.integers(-600000, 600000, n) * (np.pi / 2) + rng.uniform(-1e-6, 1e-6, n)]
    return np.concatenate([np.array(SPECIALS)] + parts)


@pytest.mark.parametrize("fn", ["exp", "log", "sin", "cos"])
def test_float64_all_paths(fn):
    check(fn, f64_classes(fn, 1 << 18, 5), "float64 path classes")


@pytest.mark.parametrize("fn", ["exp", "log", "sin", "cos"])
def test_float16_and_int_promotion(fn):
    rng = np.random.default_rng(3)
    x16 = np.arange(1 << 16, dtype=np.uint32).astype(np.uint16).view(np.float16)   # every float16
    check(fn, x16, "every float16")
    for dt in (np.int8, np.int16, np.int32, np.uint16, np.bool_):   # -> float16 / float32 / float64 loops
        if dt == np.bool_:
            xi = rng.integers(0, 2, 1000).astype(np.bool_)
        else:
            info = np.iinfo(dt)
            xi = rng.integers(info.min, info.max, 4000, endpoint=True).astype(dt)
        got = getattr(ap, fn)(ap.from_numpy(xi)).get()
        want, _ = O.unary(fn, xi)
        assert_bits_equal(got, want, f"{fn} {np.dtype(dt).name}")


def test_log_fpe():
    with ap.errstate(divide="raise"):
        with pytest.raises(FloatingPointError, match="divide by zero encountered in log"):
            ap.log(ap.from_numpy(np.array([0.0, 1.0])))
    with ap.errstate(invalid="raise"):
        with pytest.raises(FloatingPointError, match="invalid value encountered in log"):
            ap.log(ap.from_numpy(np.array([0.0, -1.0], np.float32)))


@pytest.mark.parametrize("fn", ["exp", "log", "sin", "cos"])
@pytest.mark.parametrize("dt", [np.float32, np.float64], ids=lambda d: np.dtype(d).name)
def test_strided_slices(fn, dt):
    """Step-2 and step-3 slices and a reversed view give the oracle's bits,
    and log's FPE categories still fire on a strided view."""
    rng = np.random.default_rng(9)
    with np.errstate(all="ignore"):
        x = np.concatenate([np.array(SPECIALS), 30 * rng.standard_normal(1 << 17)]).astype(dt)
    d = ap.from_numpy(x)
    for view, host in ((d[::2], x[::2]), (d[::3], x[::3]), (d[::-1], x[::-1])):
        got = getattr(ap, fn)(view).get()
        want, _ = O.unary(fn, np.ascontiguousarray(host))
        assert_bits_equal(got, want, f"{fn} {np.dtype(dt).name} strided")
    if fn == "log":
        with ap.errstate(divide="raise"):
            with pytest.raises(FloatingPointError, match="divide by zero encountered in log"):
                ap.log(ap.from_numpy(np.array([1.0, 5.0, 0.0, 7.0], dt))[::2])
