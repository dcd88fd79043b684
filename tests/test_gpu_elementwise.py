"""GPU parity of the element-wise ufunc path (ufunc __call__) against the
oracle: every binary/unary op the engine implements, every legal dtype,
broadcast / transposed / strided / reversed layouts, out=/where=/dtype=/
casting=, and the FPE category raised through errstate."""
import numpy as np
import pytest

from oracle import oracle as O
from tests._util import ALL, FLOATS, INTS, array, assert_bits_equal, values

ap = pytest.importorskip("anionpy_b200")
pytestmark = pytest.mark.gpu

FPE_BIT = {1: "divide", 2: "over", 4: "under", 8: "invalid"}
BIN = list(ap.BINARY_OPS)
EXACT_UNARY = ["negative", "absolute", "invert", "logical_not", "sqrt"]


def run(fn):
    """Call fn under errstate(all='call') and return (result, FPE category)."""
    seen = []
    with ap.errstate(all="call", call=lambda phrase, bit: seen.append(bit)):
        r = fn()
    return r, (FPE_BIT[seen[0]] if seen else None)


def to_host(r):
    return r.get() if isinstance(r, ap.ndarray) else np.asarray(r)


def oracle_or_error(fn):
    try:
        return fn(), None
    except O.OracleError as e:
        return None, e.status


def check_binary(op, a, b):
    want, werr = oracle_or_error(lambda: O.binary(op, a, b))
    if werr is not None:
        with pytest.raises((TypeError, ValueError)):
            getattr(ap, op)(ap.from_numpy(a) if isinstance(a, np.ndarray) else a,
                            ap.from_numpy(b) if isinstance(b, np.ndarray) else b)
        return
    got, cat = run(lambda: getattr(ap, op)(ap.from_numpy(a), ap.from_numpy(b)))
    assert_bits_equal(to_host(got), want[0], f"{op} {a.dtype}{a.shape} x {b.dtype}{b.shape}")
    assert cat == want[1], f"{op} {a.dtype} x {b.dtype}: fpe {cat} != {want[1]}"


@pytest.mark.parametrize("op", BIN)
@pytest.mark.parametrize("dt", ALL, ids=lambda d: np.dtype(d).name)
def test_binary_same_dtype_contiguous(op, dt):
    rng = np.random.default_rng(hash((op, np.dtype(dt).name)) % 2**32)
    z = 0.01 if op in ("floor_divide", "remainder", "fmod", "divide") else 0.0
    n = 4099
    a = values(dt, n, rng)
    b = values(dt, n, rng, zeros=z)
    if op in ("left_shift", "right_shift") and np.dtype(dt).kind in "iu":
        b = (rng.integers(-3, np.dtype(dt).itemsize * 8 + 3, n)).astype(dt)
    check_binary(op, a, b)


MIXED = [(np.int8, np.float32), (np.uint8, np.int8), (np.int32, np.float32), (np.bool_, np.float16),
         (np.uint64, np.int64), (np.int16, np.uint16), (np.float16, np.float64), (np.int64, np.float64),
         (np.bool_, np.int32), (np.uint32, np.float16)]


@pytest.mark.parametrize("op", ["add", "subtract", "multiply", "divide", "maximum", "floor_divide", "remainder",
                                "less", "equal", "logical_and", "bitwise_and", "minimum"])
@pytest.mark.parametrize("pair", MIXED, ids=lambda p: f"{np.dtype(p[0]).name}-{np.dtype(p[1]).name}")
def test_binary_mixed_dtypes(op, pair):
    rng = np.random.default_rng(7)
    a = values(pair[0], 1031, rng)
    b = values(pair[1], 1031, rng, zeros=0.01)
    check_binary(op, a, b)


SHAPES = [((1024, 1024), (1, 1024)), ((3, 1, 5), (4, 1)), ((7, 1), (1, 9)), ((), (5,)), ((6,), ()),
          ((2, 3, 4, 5), (3, 1, 5)), ((0, 5), (5,)), ((3, 0, 2), (1, 2)), ((1,), (1,)), ((2, 1, 3, 1, 2, 1), (4, 1, 1, 2, 1))]


@pytest.mark.parametrize("op", ["add", "multiply", "floor_divide", "divide", "remainder", "maximum", "less"])
@pytest.mark.parametrize("dt", [np.float64, np.float32, np.int32, np.int64, np.float16], ids=lambda d: np.dtype(d).name)
@pytest.mark.parametrize("shapes", SHAPES, ids=str)
def test_binary_broadcast(op, dt, shapes):
    rng = np.random.default_rng(11)
    a = array(dt, shapes[0], rng)
    b = array(dt, shapes[1], rng, zeros=0.05)
    check_binary(op, a, b)


def _views(base):
    yield "T", base.T
    yield "step2", base[::2]
    yield "rev", base[::-1]
    yield "F", np.asfortranarray(base)
    yield "step2inner", base[:, ::2]
    yield "offset", base[1:, 3:]


@pytest.mark.parametrize("op", ["add", "multiply", "maximum", "floor_divide", "subtract", "bitwise_and"])
@pytest.mark.parametrize("dt", [np.float32, np.float64, np.int32, np.int64], ids=lambda d: np.dtype(d).name)
def test_binary_layouts_and_order_k(op, dt):
    rng = np.random.default_rng(3)
    base = array(dt, (64, 96), rng)
    other = array(dt, (64, 96), rng, zeros=0.02)
    for name, v in _views(base):
        w = np.ascontiguousarray(other[: v.shape[0], : v.shape[1]]) if v.ndim == 2 else other
        if w.shape != v.shape:
            w = array(dt, v.shape, rng, zeros=0.02)
        want, werr = oracle_or_error(lambda: O.binary(op, v, w))
        if werr is not None:
            continue
        dv = ap.from_numpy(np.ascontiguousarray(base))
        # rebuild the same view on the device
        dview = {"T": dv.T, "step2": dv[::2], "rev": dv[::-1], "step2inner": dv[:, ::2], "offset": dv[1:, 3:]}.get(name)
        if name == "F":
            dview = ap.from_numpy(v)
        got, cat = run(lambda: getattr(ap, op)(dview, ap.from_numpy(w)))
        assert_bits_equal(got.get(), want[0], f"{op} {name}")
        assert cat == want[1]
        want_st = O.order_k_strides(want[0].shape, [v, w])
        assert list(got.elem_strides) == list(want_st), f"{op} {name}: strides {got.elem_strides} != {want_st}"


@pytest.mark.parametrize("dt", [np.float32, np.float64, np.int8, np.float16, np.int64], ids=lambda d: np.dtype(d).name)
@pytest.mark.parametrize("shape", [(45, 77), (33, 1000), (257, 40)])
def test_transposed_against_c_order_tiles(dt, shape):
    """A transposed view against a C-ordered operand (the shared-memory tile
    path), ragged tile edges, both output layouts via out=."""
    rng = np.random.default_rng(8)
    base = array(dt, shape[::-1], rng)
    w = array(dt, shape, rng)
    v = base.T
    for op in ("add", "maximum", "multiply"):
        want = O.binary(op, v, w)[0]
        db = ap.from_numpy(base)
        got = getattr(ap, op)(db.T, ap.from_numpy(w))
        assert_bits_equal(got.get(), want, f"{op} {shape}")
        for order in ("C", "F"):
            host_out = np.zeros(shape, want.dtype, order=order)
            dout = ap.from_numpy(host_out)
            getattr(ap, op)(db.T, ap.from_numpy(w), out=dout)
            assert_bits_equal(dout.get(), want, f"{op} {shape} out={order}")


@pytest.mark.parametrize("op", ["negative", "absolute", "invert", "logical_not", "sqrt"])
@pytest.mark.parametrize("dt", ALL, ids=lambda d: np.dtype(d).name)
def test_unary_exact(op, dt):
    rng = np.random.default_rng(5)
    a = values(dt, 4099, rng)
    want, werr = oracle_or_error(lambda: O.unary(op, a))
    if werr is not None:
        with pytest.raises((TypeError, ValueError)):
            getattr(ap, op)(ap.from_numpy(a))
        return
    got, cat = run(lambda: getattr(ap, op)(ap.from_numpy(a)))
    assert_bits_equal(got.get(), want[0], f"{op} {np.dtype(dt).name}")
    assert cat == want[1]
    # strided input
    v = a[::3]
    want2 = O.unary(op, v)[0]
    got2 = getattr(ap, op)(ap.from_numpy(a)[::3])
    assert_bits_equal(got2.get(), want2, f"{op} strided")


def test_out_where_casting():
    rng = np.random.default_rng(9)
    a = values(np.float64, 500, rng)
    b = values(np.float64, 500, rng)
    want = O.binary("add", a, b)[0]
    # out= of another dtype (same_kind float64 -> float32)
    out = ap.empty((500,), np.float32)
    r = ap.add(ap.from_numpy(a), ap.from_numpy(b), out=out)
    assert r is out
    assert_bits_equal(out.get(), O.cast(want, np.float32), "out= cast")
    # where= keeps the old values where False
    init = values(np.float64, 500, rng)
    out2 = ap.from_numpy(init)
    mask = rng.random(500) < 0.5
    ap.add(ap.from_numpy(a), ap.from_numpy(b), out=out2, where=ap.from_numpy(mask))
    exp = np.where(mask, want, init)
    assert_bits_equal(out2.get(), exp, "where=")
    # casting check on out=
    with pytest.raises(TypeError):
        ap.add(ap.from_numpy(a), ap.from_numpy(b), out=ap.empty((500,), np.int32))
    # dtype= precast
    ai = values(np.int32, 300, rng)
    bi = values(np.int32, 300, rng)
    got = ap.add(ap.from_numpy(ai), ap.from_numpy(bi), dtype=np.float64)
    assert_bits_equal(got.get(), O.binary("add", ai.astype(np.float64), bi.astype(np.float64))[0], "dtype=")


def test_in_place_aliasing():
    rng = np.random.default_rng(13)
    a = values(np.float32, 1000, rng)
    da = ap.from_numpy(a)
    ap.multiply(da, da, out=da)
    assert_bits_equal(da.get(), O.binary("multiply", a, a)[0], "in place")
    # overlapping shifted views go through a temporary
    b = values(np.float64, 1001, rng)
    db = ap.from_numpy(b)
    ap.add(db[:-1], db[1:], out=db[1:])
    exp = b.copy()
    exp[1:] = O.binary("add", b[:-1], b[1:])[0]
    assert_bits_equal(db.get(), exp, "overlap")


def test_errors_match_reference():
    with pytest.raises(ValueError, match="could not be broadcast"):
        ap.add(ap.from_numpy(np.ones(3)), ap.from_numpy(np.ones(4)))
    with pytest.raises(TypeError, match="boolean subtract"):
        ap.subtract(ap.from_numpy(np.ones(3, bool)), ap.from_numpy(np.ones(3, bool)))
    with pytest.raises(TypeError, match="bitwise_and"):
        ap.bitwise_and(ap.from_numpy(np.ones(3)), ap.from_numpy(np.ones(3)))
    with pytest.raises(TypeError, match="boolean negative"):
        ap.negative(ap.from_numpy(np.ones(3, bool)))


@pytest.mark.parametrize("mode", ["raise", "warn"])
def test_errstate_modes(mode):
    a = ap.from_numpy(np.array([1, 2, 3], np.int32))
    b = ap.from_numpy(np.array([1, 0, 3], np.int32))
    if mode == "raise":
        with ap.errstate(divide="raise"):
            with pytest.raises(FloatingPointError, match="divide by zero encountered in floor_divide"):
                ap.floor_divide(a, b)
    else:
        with pytest.warns(RuntimeWarning, match="divide by zero encountered in remainder"):
            ap.remainder(a, b)
    # float remainder by zero is silent (detect_remainder, fpe.rs:240)
    with ap.errstate(all="raise"):
        ap.remainder(ap.from_numpy(np.array([1.0])), ap.from_numpy(np.array([0.0])))


def test_scalar_operands_and_0d():
    r = ap.add(ap.from_numpy(np.arange(5, dtype=np.int8)), 3)
    assert r.dtype == np.int8
    s = ap.add(ap.from_numpy(np.array(2.5)), ap.from_numpy(np.array(1.0)))
    assert isinstance(s, np.float64) and s == 3.5


@pytest.mark.parametrize("op", ["floor_divide", "remainder", "fmod"])
@pytest.mark.parametrize("dt", [np.float32, np.float64], ids=lambda d: np.dtype(d).name)
def test_float_division_quotient_edges(op, dt):
    """floor_divide, remainder and fmod at the edges of their fast paths:
    quotients just below and above 2^19 / 2^20 / 2^23 (float32) and 2^36 /
    2^49 / 2^52 (float64), the limits of the approximate quotient and of the
    one-division paths; quotients a rounding away from an integer, exact
    multiples, divisors near 2^+-125 (the approximate quotient's range),
    zeros of both signs and huge quotients, against the oracle bit for
    bit."""
    rng = np.random.default_rng(77)
    f32 = dt == np.float32
    lims = [2.0 ** 19, 2.0 ** 20, 2.0 ** 23] if f32 else [2.0 ** 36, 2.0 ** 49, 2.0 ** 52]
    eps = 2.0 ** -23 if f32 else 2.0 ** -52
    n, g = 48000, 6
    m = n // g
    y = rng.standard_normal(n) * np.exp2(rng.integers(-20, 20, n))
    q = np.concatenate([rng.integers(1, 64, m).astype(np.float64)]
                       + [rng.integers(lim // 2, lim * 2, m).astype(np.float64) for lim in lims]
                       + [rng.integers(1, 1 << 16, n - 4 * m).astype(np.float64)])
    # divisors at the approximate quotient's range limits, small quotients
    edge = slice(n - m, n)
    y[edge] = rng.choice([-1.0, 1.0], m) * rng.uniform(1.0, 2.0, m) * np.exp2(
        rng.choice([-127, -126, -125, -124, 123, 124, 125], m).astype(np.float64))
    q[edge] = rng.integers(1, 4, m)
    x = q * y * (1 + rng.choice([-1.0, 0.0, 1.0], n) * eps) * rng.choice([-1.0, 1.0], n)
    x[-100:] = rng.choice([0.0, -0.0], 100)
    with np.errstate(over="ignore"):
        xs, ys = x.astype(dt), y.astype(dt)
    got = getattr(ap, op)(ap.from_numpy(xs), ap.from_numpy(ys)).get()
    want, _ = O.binary(op, xs, ys)
    assert_bits_equal(got, want, f"{op} {np.dtype(dt).name} quotient edges")


@pytest.mark.parametrize("dt", [np.float32, np.int32, np.uint32, np.float64, np.int64], ids=lambda d: np.dtype(d).name)
@pytest.mark.parametrize("shape", [(64, 64), (128, 192), (320, 64)])
def test_transposed_whole_vector_tiles(dt, shape):
    """Whole 64 x 64 (4-byte) or 32 x 32 (8-byte) tiles with 16-byte aligned
    rows: the vector tile kernel, both output layouts, FPE categories; a view
    whose rows start off a 16-byte boundary takes the scalar tile kernel and
    must give the same bits."""
    rng = np.random.default_rng(21)
    base = array(dt, shape[::-1], rng, zeros=0.02)
    w = array(dt, shape, rng, zeros=0.02)
    ops = ["add", "maximum", "multiply", "subtract", "floor_divide", "remainder"]
    if np.dtype(dt).kind in "iu":
        ops.append("bitwise_and")
    db, dw = ap.from_numpy(base), ap.from_numpy(w)
    for op in ops:
        want, wcat = O.binary(op, base.T, w)
        got, cat = run(lambda: getattr(ap, op)(db.T, dw))
        assert_bits_equal(got.get(), want, f"{op} {shape}")
        assert cat == wcat, f"{op} {shape}: FPE {cat} != {wcat}"
        for order in ("C", "F"):
            dout = ap.from_numpy(np.zeros(shape, want.dtype, order=order))
            getattr(ap, op)(db.T, dw, out=dout)
            assert_bits_equal(dout.get(), want, f"{op} {shape} out={order}")
    # rows starting one element past a 16-byte boundary
    big = array(dt, (shape[1] + 1, shape[0] + 1), rng)
    v = big[1:, 1:]
    want = O.binary("add", v.T, w)[0]
    got = ap.add(ap.from_numpy(big)[1:, 1:].T, dw)
    assert_bits_equal(got.get(), want, f"misaligned {shape}")


@pytest.mark.parametrize("dt", [np.int64, np.uint64], ids=lambda d: np.dtype(d).name)
def test_int64_division_quotient_ranges(dt):
    """floor_divide / remainder on 64-bit integers: full-range operands (small
    quotients), quotients around the 2^20 limit of the estimate path, huge
    quotients (the exact division), the extremes and zero divisors, each
    contiguous and through a step-2 slice."""
    rng = np.random.default_rng(33)
    info = np.iinfo(dt)
    n = 1 << 16
    y = rng.integers(1, 1 << 40, n, dtype=np.int64).astype(dt)
    q = rng.integers((1 << 20) - 4, (1 << 20) + 4, n).astype(dt)
    with np.errstate(all="ignore"):
        near = (q * y + rng.integers(0, 1 << 30, n).astype(dt) % y).astype(dt)
    parts_x = [rng.integers(info.min, info.max, n, dtype=dt, endpoint=True), near,
               rng.integers(info.min, info.max, n, dtype=dt, endpoint=True)]
    parts_y = [rng.integers(info.min, info.max, n, dtype=dt, endpoint=True), y,
               rng.integers(1, 1000, n).astype(dt)]
    ext = np.array([info.min, info.max, 0, 1, 2, info.max - 1, info.min + 1] + ([-1, -2] if dt == np.int64 else [3, 7]), dt)
    ex_x, ex_y = np.meshgrid(ext, ext)
    x = np.concatenate(parts_x + [ex_x.ravel()])
    yy = np.concatenate(parts_y + [ex_y.ravel()])
    if dt == np.int64:
        x[: n // 2] = -np.abs(x[: n // 2] // 2)
        yy[n: n + n // 2] = -yy[n: n + n // 2]
        x[2 * n + n // 3: 2 * n + n // 2] *= -1
    for op in ("floor_divide", "remainder"):
        want, wcat = O.binary(op, x, yy)
        got, cat = run(lambda: getattr(ap, op)(ap.from_numpy(x), ap.from_numpy(yy)))
        assert_bits_equal(got.get(), want, f"{op} contiguous")
        assert cat == wcat
        x2, y2 = np.repeat(x, 2), np.repeat(yy, 2)
        got2 = getattr(ap, op)(ap.from_numpy(x2)[::2], ap.from_numpy(y2)[::2])
        assert_bits_equal(got2.get(), want, f"{op} step-2")
