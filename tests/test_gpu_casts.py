"""GPU parity of dtype conversion against the oracle: every one of the 12 x 12
(source, destination) pairs of the reference's Buffer::cast_to
(ionp-core/src/buffer.rs:64-330), including numpy's float -> narrow-int rule
(saturate to int32 first, then keep the low bits: 200.0 -> int8 is -56,
-1.5 -> uint8 is 255, inf -> int8 is -1), on contiguous and transposed
sources; and ndarray.astype's detect_cast_overflow report (fpe.rs:398)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests._util import ALL, assert_bits_equal, values

ap = pytest.importorskip("anionpy_b200")
pytestmark = pytest.mark.gpu

EDGES = [200.0, 130.0, -129.0, -1.5, 1.5, -0.5, 0.5, 255.5, 256.0, -256.0, 65535.5, 65536.0, -32769.0,
         2.0 ** 31, -(2.0 ** 31) - 1.0, 2.0 ** 32, 2.0 ** 63, -(2.0 ** 63), 2.0 ** 64, 1e10, -1e10, 1e300, -1e300,
         np.inf, -np.inf, np.nan, -0.0, 0.0, 65504.0, 70000.0, 1e-8, 3.4e38]


def source(dt, rng):
    body = values(dt, 2053, rng)
    if np.dtype(dt).kind == "f":
        with np.errstate(all="ignore"):
            edges = np.array(EDGES, np.float64).astype(dt)
        body = np.concatenate([edges, body])
    return body


@pytest.mark.parametrize("src", ALL, ids=lambda d: np.dtype(d).name)
def test_cast_all_pairs(src):
    rng = np.random.default_rng(51)
    host = source(src, rng)
    dev = ap.from_numpy(host)
    side = 17
    grid = values(src, side * 31, rng).reshape(31, side)
    dgrid = ap.from_numpy(grid)
    for dst in ALL:
        want = O.cast(host, dst)
        with ap.errstate(all="ignore"):
            got = dev.astype(dst)
        assert_bits_equal(got.get(), want, f"{np.dtype(src).name} -> {np.dtype(dst).name}")
        assert_bits_equal(dev._cast_to(dst).get(), want, f"{np.dtype(src).name} -> {np.dtype(dst).name} (cast_to)")
        wt = O.cast(np.ascontiguousarray(grid.T), dst)
        with ap.errstate(all="ignore"):
            gt = dgrid.T.astype(dst)
        assert_bits_equal(gt.get(), wt, f"{np.dtype(src).name} -> {np.dtype(dst).name} transposed source")


def test_astype_overflow_report():
    def raises(host, dst):
        with ap.errstate(invalid="raise"):
            try:
                ap.from_numpy(host).astype(dst)
            except FloatingPointError as e:
                assert "invalid value encountered in cast" in str(e)
                return True
        return False

    assert raises(np.array([1.0, 1e300]), np.int32)
    assert raises(np.array([1.0, np.nan]), np.int64)
    assert raises(np.array([np.inf], np.float32), np.uint8)
    assert raises(np.array([-1.0]), np.uint16)
    assert raises(np.array([np.inf], np.float16), np.int16)
    assert raises(np.array([2.0 ** 65]), np.uint64)
    assert not raises(np.array([2.0 ** 64]), np.uint64)       # u64::MAX as f64 rounds up to 2^64
    assert not raises(np.array([1.0, 2.0, -3.5]), np.int8)
    assert not raises(np.array([2.0 ** 63]), np.int64)        # i64::MAX as f64 is 2^63 itself
    assert not raises(np.array([np.nan, 1e300]), np.bool_)    # only integer destinations
    assert not raises(np.array([np.nan]), np.float32)         # float destinations never flag
    assert not raises(np.array([2 ** 40]), np.int8)           # integer narrowing wraps silently
    # the report comes from the whole array, any layout
    big = np.ones((64, 65))
    big[63, 64] = np.nan
    with ap.errstate(invalid="raise"):
        with pytest.raises(FloatingPointError, match="invalid value encountered in cast"):
            ap.from_numpy(big).T.astype(np.int32)


def test_astype_casting_rule():
    d = ap.from_numpy(np.array([1.5, 2.5]))
    with pytest.raises(TypeError, match="according to the rule 'safe'"):
        d.astype(np.int32, casting="safe")
    assert d.astype(np.float32, casting="same_kind").dtype == np.float32
