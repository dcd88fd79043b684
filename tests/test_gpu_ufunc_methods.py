"""GPU parity of the remaining ufunc methods against the oracle:
accumulate (and cumsum / cumprod), reduceat and outer
(ionp-core/src/ufunc.rs:7847-8483, 8212), on every dtype, C and transposed
layouts, every axis, and the long single fibers the split scan takes."""
import numpy as np
import pytest

from oracle import oracle as O
from tests._util import ALL, array, assert_bits_equal, values

ap = pytest.importorskip("anionpy_b200")
pytestmark = pytest.mark.gpu

ACC_OPS = ["add", "multiply", "maximum", "minimum", "subtract", "logical_and", "logical_or", "bitwise_xor",
           "floor_divide", "divide", "less"]


def legal(op, dt):
    try:
        O.reduce_compute_dtype(op, dt)
        return True
    except O.OracleError:
        return False


@pytest.mark.parametrize("op", ACC_OPS)
@pytest.mark.parametrize("dt", ALL, ids=lambda d: np.dtype(d).name)
def test_accumulate_axes_and_layouts(op, dt):
    if not legal(op, dt):
        with pytest.raises((TypeError, ValueError)):
            getattr(ap, op).accumulate(ap.from_numpy(values(dt, 8, np.random.default_rng(0))))
        return
    rng = np.random.default_rng(61)
    host = array(dt, (5, 6, 7), rng, zeros=0.05)
    if np.dtype(dt).kind == "f":
        host = (host / 4).astype(dt)
    dev = ap.from_numpy(host)
    for view, h in ((dev, host), (dev.transpose(2, 0, 1), host.transpose(2, 0, 1))):
        for axis in range(3):
            with np.errstate(all="ignore"):
                want = O.accumulate(op, h, axis)
            got = getattr(ap, op).accumulate(view, axis=axis)
            assert_bits_equal(got.get(), want, f"{op}.accumulate {np.dtype(dt).name} axis={axis}")


@pytest.mark.parametrize("op", ["add", "multiply", "maximum", "minimum", "bitwise_or", "logical_xor"])
@pytest.mark.parametrize("dt", [np.int8, np.int32, np.int64, np.uint64, np.float32, np.float64, np.float16, np.bool_],
                         ids=lambda d: np.dtype(d).name)
def test_accumulate_long_fibers(op, dt):
    """few long fibers: order-free folds take the three-pass split scan, the
    others one thread per fiber; both equal the sequential fold"""
    if not legal(op, dt):
        return
    rng = np.random.default_rng(62)
    for shape, axis in (((30011,), 0), ((3, 12007), 1), ((9001, 2), 0)):
        host = array(dt, shape, rng)
        if np.dtype(dt).kind == "f":
            host = np.where(rng.random(host.shape) < 0.5, host, -host).astype(dt)
        with np.errstate(all="ignore"):
            want = O.accumulate(op, host, axis)
        got = getattr(ap, op).accumulate(ap.from_numpy(host), axis=axis)
        assert_bits_equal(got.get(), want, f"{op}.accumulate {np.dtype(dt).name} {shape}")


@pytest.mark.parametrize("dt", [np.int8, np.bool_, np.int32, np.float32, np.float64, np.uint16], ids=lambda d: np.dtype(d).name)
def test_cumsum_cumprod(dt):
    rng = np.random.default_rng(63)
    host = array(dt, (4, 9), rng)
    dev = ap.from_numpy(host)
    for fn, op in (("cumsum", "add"), ("cumprod", "multiply")):
        with np.errstate(all="ignore"):
            want = O.accumulate(op, host.reshape(-1), 0)
        assert_bits_equal(getattr(ap, fn)(dev).get(), want, f"{fn} axis=None")
        for axis in (0, 1, -1):
            with np.errstate(all="ignore"):
                w = O.accumulate(op, host, axis % 2)
            assert_bits_equal(getattr(ap, fn)(dev, axis=axis).get(), w, f"{fn} axis={axis}")
            assert_bits_equal(getattr(dev, fn)(axis=axis).get(), w, f"ndarray.{fn} axis={axis}")
        # dtype= casts the input first and the result last
        with np.errstate(all="ignore"):
            w8 = O.cast(O.accumulate(op, O.cast(host, np.int8), 1), np.int8)
        assert_bits_equal(getattr(ap, fn)(dev, axis=1, dtype=np.int8).get(), w8, f"{fn} dtype=int8")
    # a 0-d input accumulates to shape (1,)
    assert ap.cumsum(ap.from_numpy(np.array(3.5))).shape == (1,)


@pytest.mark.parametrize("op", ["add", "multiply", "maximum", "subtract", "logical_or", "bitwise_and"])
@pytest.mark.parametrize("dt", [np.int16, np.int64, np.float32, np.float64, np.bool_], ids=lambda d: np.dtype(d).name)
def test_reduceat(op, dt):
    if not legal(op, dt):
        return
    rng = np.random.default_rng(64)
    host = array(dt, (8, 40), rng)
    dev = ap.from_numpy(host)
    for axis, idx in ((1, [0, 4, 4, 10, 3, 39]), (0, [0, 2, 7]), (1, [5]), (0, [7, 0, 3]), (1, [])):
        with np.errstate(all="ignore"):
            want = O.reduceat(op, host, idx, axis)
        got = getattr(ap, op).reduceat(dev, idx, axis=axis)
        assert_bits_equal(got.get(), want, f"{op}.reduceat {np.dtype(dt).name} axis={axis} {idx}")
    # a long segment over a transposed view
    big = array(dt, (3, 5000), rng)
    with np.errstate(all="ignore"):
        want = O.reduceat(op, np.ascontiguousarray(big.T), [0, 1, 2500], 0)
    got = getattr(ap, op).reduceat(ap.from_numpy(big).T, [0, 1, 2500], axis=0)
    assert_bits_equal(got.get(), want, f"{op}.reduceat transposed")
    with pytest.raises(IndexError, match="out-of-bounds"):
        getattr(ap, op).reduceat(dev, [0, 40], axis=1)


@pytest.mark.parametrize("op", ["add", "multiply", "maximum", "floor_divide", "less", "logical_and", "subtract"])
def test_outer(op):
    rng = np.random.default_rng(65)
    for da, db in ((np.float64, np.float32), (np.int32, np.int64), (np.int8, np.uint8), (np.bool_, np.bool_)):
        a = array(da, (3, 4), rng, zeros=0.1)
        b = array(db, (5,), rng, zeros=0.1)
        try:
            with np.errstate(all="ignore"):
                want = O.outer(op, a, b)
        except O.OracleError:
            with pytest.raises((TypeError, ValueError)):
                getattr(ap, op).outer(ap.from_numpy(a), ap.from_numpy(b))
            continue
        got = getattr(ap, op).outer(ap.from_numpy(a), ap.from_numpy(b))
        assert_bits_equal(got.get(), want, f"{op}.outer {np.dtype(da).name} x {np.dtype(db).name}")


def test_method_errors():
    d0 = ap.from_numpy(np.array(1.0))
    with pytest.raises(TypeError, match="cannot accumulate on a scalar"):
        ap.add.accumulate(d0)
    with pytest.raises(TypeError, match="cannot reduceat on a scalar"):
        ap.add.reduceat(d0, [0])
    with pytest.raises(ap.AxisError):
        ap.add.accumulate(ap.from_numpy(np.ones((2, 3))), axis=2)
    with pytest.raises(TypeError):
        ap.less.accumulate(ap.from_numpy(np.ones(4)))
