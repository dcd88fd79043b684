"""GPU parity of ufunc.at against the oracle (at_binary,
ionp-core/src/ufunc.rs:9577; at_math_binary, 9932; at_unary, 9301;
at_math_unary, 9805): every binary op over (target, values) dtype pairs that
keep the target's dtype, promote it (the whole-target round trip) or go
through bool, with repeated and negative indices, full / row / scalar
values, C, transposed and sliced targets; the unary ops; 0-d targets; values
that share memory with the target; and the reference's error cases."""
import numpy as np
import pytest

from oracle import oracle as O
from tests._util import ALL, array, assert_bits_equal

ap = pytest.importorskip("anionpy_b200")
pytestmark = pytest.mark.gpu

BIN_OPS = list(O.BINARY_AT_OPS)
UN_OPS = ["negative", "absolute", "invert", "logical_not", "sqrt", "exp", "log", "sin", "cos"]
IDX = [0, 3, -1, 0, 2, 3, 3, 5]


def oracle_at(op, host, idx, vals=None):
    """(result, exception class or None) of the oracle on a copy of host."""
    t = host.copy()
    try:
        with np.errstate(all="ignore"):
            O.at(op, t, idx, vals)
        return t, None
    except O.OracleError as e:
        return None, {"broadcast": ValueError}.get(e.status, TypeError)
    except (TypeError, ValueError, IndexError) as e:
        return None, type(e)


def dev_at(op, dev, idx, vals=None):
    uf = getattr(ap, op)
    with ap.errstate(all="ignore"):
        if vals is None:
            uf.at(dev, idx)
        else:
            uf.at(dev, idx, vals if isinstance(vals, ap.ndarray) else ap.from_numpy(np.asarray(vals)))


def check(op, host, dev_view, idx, vals, what):
    want, err = oracle_at(op, host, idx, vals)
    if err is not None:
        with pytest.raises(err):
            dev_at(op, dev_view, idx, vals)
        return
    dev_at(op, dev_view, idx, vals)
    assert_bits_equal(dev_view.get(), want, what)


@pytest.mark.parametrize("op", BIN_OPS)
@pytest.mark.parametrize("tdt", ALL, ids=lambda d: np.dtype(d).name)
def test_binary_at(op, tdt):
    rng = np.random.default_rng(71)
    for vdt in (tdt, np.int8, np.float64, np.bool_, np.uint32):
        host = array(tdt, (6, 5), rng)
        if np.dtype(tdt).kind == "f":
            host = (host / 4).astype(tdt)
        full = array(vdt, (len(IDX), 5), rng)
        row = array(vdt, (5,), rng)
        scal = array(vdt, (), rng)
        for name, vals in (("full", full), ("row", row), ("scalar", scal)):
            what = f"{op}.at {np.dtype(tdt).name} <- {np.dtype(vdt).name} {name}"
            check(op, host, ap.from_numpy(host), IDX, vals, what)
    # transposed and sliced targets: the update lands through the view
    host = array(tdt, (7, 6), rng)
    vals = array(tdt, (len(IDX), 7), rng)
    base = ap.from_numpy(np.ascontiguousarray(host))
    check(op, np.ascontiguousarray(host.T), base.T, IDX, vals, f"{op}.at transposed")
    big = array(tdt, (12, 9), rng)
    dbig = ap.from_numpy(big)
    check(op, big[::2, 1::3].copy(), dbig[::2, 1::3], IDX, array(tdt, (3,), rng), f"{op}.at sliced")


@pytest.mark.parametrize("op", UN_OPS)
@pytest.mark.parametrize("tdt", ALL, ids=lambda d: np.dtype(d).name)
def test_unary_at(op, tdt):
    rng = np.random.default_rng(73)
    host = array(tdt, (6, 4), rng)
    if np.dtype(tdt).kind == "f":
        host = (host / 8).astype(tdt)
    check(op, host, ap.from_numpy(host), IDX, None, f"{op}.at {np.dtype(tdt).name}")
    h1 = array(tdt, (9,), rng)
    check(op, h1, ap.from_numpy(h1), [1, 1, 1, -2, 4], None, f"{op}.at 1-d {np.dtype(tdt).name}")


def test_zero_d_and_empty():
    t = np.array(2.5)
    check("multiply", t, ap.from_numpy(t), [], np.array(3.0), "0-d multiply.at")
    check("sin", t, ap.from_numpy(t), [], None, "0-d sin.at")
    with pytest.raises(IndexError, match="too many indices for array: array is 0-dimensional, but 1 were indexed"):
        ap.add.at(ap.from_numpy(np.array(1.0)), [0], 1.0)
    # no index: nothing changes, except the promoted round trip, which the
    # reference makes for every element all the same
    big = np.array([2 ** 62 + 1, 3], np.int64)
    check("add", big, ap.from_numpy(big), [], np.array(0.5), "empty indices, promoting op")
    e = np.zeros((0, 3), np.float32)
    ap.add.at(ap.from_numpy(e), [], np.zeros((0, 3), np.float32))


def test_values_sharing_the_target():
    host = np.arange(10, dtype=np.int64)
    dev = ap.from_numpy(host)
    ap.add.at(dev, [1, 2, 3, 4], dev[0:4])
    want = host.copy()
    O.at("add", want, [1, 2, 3, 4], host[0:4].copy())
    assert_bits_equal(dev.get(), want, "values read before the update")


def test_large_repeated_indices():
    rng = np.random.default_rng(79)
    host = rng.standard_normal((1000, 33)).astype(np.float32)
    idx = rng.integers(-1000, 1000, 20000)
    vals = rng.standard_normal((20000, 33)).astype(np.float32)
    dev = ap.from_numpy(host)
    ap.add.at(dev, idx, ap.from_numpy(vals))
    want = host.copy()
    rows = np.where(idx < 0, idx + 1000, idx)
    for i, r in enumerate(rows):       # float32 adds, in index order
        want[r] = (want[r] + vals[i]).astype(np.float32)
    assert_bits_equal(dev.get(), want, "20000 repeated float32 updates")


def test_errors():
    d = ap.from_numpy(np.zeros((4, 3)))
    with pytest.raises(IndexError, match="index 4 is out of bounds for axis 0 with size 4"):
        ap.add.at(d, [1, 4], 1.0)
    with pytest.raises(IndexError, match="index -5 is out of bounds for axis 0 with size 4"):
        ap.add.at(d, [-5], 1.0)
    with pytest.raises(ValueError, match="array is not broadcastable to correct shape"):
        ap.add.at(d, [0, 1], ap.from_numpy(np.zeros((3, 3))))
    with pytest.raises(TypeError):
        ap.bitwise_and.at(d, [0], 1.0)
    with pytest.raises(TypeError):
        ap.subtract.at(ap.from_numpy(np.zeros(3, np.bool_)), [0], True)
    with pytest.raises(TypeError):
        ap.negative.at(ap.from_numpy(np.zeros(3, np.bool_)), [0])
    with pytest.raises(TypeError, match="first operand must be array"):
        ap.add.at(np.zeros(3), [0], 1.0)
    with pytest.raises(TypeError, match="indices must be an int, a sequence of ints, or an integer numpy array"):
        ap.add.at(d, [0.5], 1.0)
    with pytest.raises(TypeError, match="unary ufunc .at\\(\\) takes no third argument"):
        ap.exp.at(d, [0], 1.0)
    with pytest.raises(TypeError, match="binary ufunc .at\\(\\) requires a values argument"):
        ap.add.at(d, [0])
    # an int index alone is one index
    ap.add.at(d, 2, 5.0)
    assert d.get()[2].tolist() == [5.0, 5.0, 5.0]
