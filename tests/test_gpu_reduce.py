"""GPU parity of ufunc.reduce and argmin/argmax against the oracle:
pairwise-exact float add (wide runs, narrow axes, multi-run layouts, split
trees), f16 widening rules, sequential/associative folds, keepdims/initial/
where/dtype/out=, output layout, and the reference's error cases."""
import numpy as np
import pytest

from oracle import oracle as O
from tests._util import ALL, FLOATS, array, assert_bits_equal, values

ap = pytest.importorskip("anionpy_b200")
pytestmark = pytest.mark.gpu

RED_OPS = ["add", "multiply", "maximum", "minimum", "subtract", "divide", "floor_divide", "logical_and",
           "logical_or", "logical_xor", "bitwise_and", "bitwise_or", "bitwise_xor", "equal", "less"]


def to_host(r):
    return r.get() if isinstance(r, ap.ndarray) else np.asarray(r)


def check_reduce(op, a_np, dev, axis=0, **kw):
    try:
        want = O.reduce(op, a_np, axis=axis, **kw)
        werr = None
    except O.OracleError as e:
        want, werr = None, e.status
    if werr is not None:
        with pytest.raises((TypeError, ValueError)):
            getattr(ap, op).reduce(dev, axis=axis, **kw)
        return
    dkw = dict(kw)
    if "where" in dkw and isinstance(dkw["where"], np.ndarray):
        dkw["where"] = ap.from_numpy(dkw["where"])
    got = getattr(ap, op).reduce(dev, axis=axis, **dkw)
    assert_bits_equal(to_host(got), np.asarray(want), f"{op}.reduce {a_np.dtype}{a_np.shape} axis={axis} {kw}")
    if isinstance(got, ap.ndarray):
        axes = O.normalize_reduce_axes(axis, a_np.ndim)
        want_st = O.reduce_layout_strides(list(a_np.shape), O.elem_strides(a_np), axes, kw.get("keepdims", False))
        assert list(got.elem_strides) == list(want_st), f"{op} strides {got.elem_strides} != {want_st}"


@pytest.mark.parametrize("op", RED_OPS)
@pytest.mark.parametrize("dt", ALL, ids=lambda d: np.dtype(d).name)
def test_reduce_ops_dtypes(op, dt):
    rng = np.random.default_rng(21)
    a = array(dt, (37, 53), rng)
    d = ap.from_numpy(a)
    for axis in (0, 1, -1, None, (0, 1)):
        check_reduce(op, a, d, axis=axis)


PW_LENGTHS = [1, 2, 4, 7, 8, 9, 16, 31, 32, 64, 127, 128, 129, 136, 255, 256, 257, 1000, 1024, 4095, 4096, 5003,
              65536, 65537, 100003, 262147]


@pytest.mark.parametrize("dt", [np.float32, np.float64, np.float16], ids=lambda d: np.dtype(d).name)
@pytest.mark.parametrize("n", PW_LENGTHS)
def test_pairwise_lengths(dt, n):
    rng = np.random.default_rng(n)
    a = (rng.standard_normal(n) * 100).astype(dt)
    check_reduce("add", a, ap.from_numpy(a), axis=0)
    check_reduce("add", a, ap.from_numpy(a), axis=None, initial=2.5)


@pytest.mark.parametrize("shape,axis", [((8, 32768), -1), ((64, 1000), 1), ((1024, 1024), 1), ((3, 5, 16), -1),
                                        ((2, 3, 4, 5), (2, 3)), ((4, 5, 6), (0, 2)), ((6, 7, 8), None), ((16, 3, 5), 0),
                                        ((5, 4096), None), ((1, 7), 0), ((7, 1), 1)])
@pytest.mark.parametrize("dt", [np.float32, np.float64, np.float16], ids=lambda d: np.dtype(d).name)
@pytest.mark.parametrize("layout", ["C", "F", "T", "step"])
def test_float_add_layouts(shape, axis, dt, layout):
    rng = np.random.default_rng(31)
    base = array(dt, shape, rng)
    if layout == "F":
        a = np.asfortranarray(base)
        d = ap.from_numpy(a)
    elif layout == "T":
        a = base.T
        d = ap.from_numpy(base).T
        axis = tuple(base.ndim - 1 - x for x in (axis if isinstance(axis, tuple) else (axis,))) if axis is not None else None
        if isinstance(axis, tuple) and len(axis) == 1:
            axis = axis[0]
    elif layout == "step":
        big = array(dt, shape[:-1] + (shape[-1] * 2,), rng)
        a = big[..., ::2]
        d = ap.from_numpy(big)[..., ::2]
    else:
        a, d = base, ap.from_numpy(base)
    for kw in ({}, {"keepdims": True}, {"initial": 0.0, "keepdims": True}):
        check_reduce("add", a, d, axis=axis, **kw)
    check_reduce("multiply", a, d, axis=axis)
    check_reduce("maximum", a, d, axis=axis)


@pytest.mark.parametrize("dt", [np.float32, np.float64, np.float16, np.int32, np.int64, np.uint8, np.bool_],
                         ids=lambda d: np.dtype(d).name)
def test_where_initial_dtype(dt):
    rng = np.random.default_rng(41)
    a = array(dt, (23, 41), rng)
    d = ap.from_numpy(a)
    mask = rng.random((23, 41)) < 0.6
    for axis in (0, 1, None):
        check_reduce("add", a, d, axis=axis, where=mask)
        check_reduce("maximum", a, d, axis=axis, where=mask, initial=-5)
        check_reduce("add", a, d, axis=axis, initial=3)
        check_reduce("add", a, d, axis=axis, dtype=np.float64)
    check_reduce("add", a, d, axis=1, where=mask[0])  # broadcast mask
    # a mask without identity or initial is an error
    with pytest.raises(ValueError, match="identity"):
        ap.maximum.reduce(d, axis=0, where=ap.from_numpy(mask))


def test_empty_and_errors():
    e = np.zeros((0, 5), np.float64)
    de = ap.from_numpy(e)
    assert_bits_equal(ap.add.reduce(de, axis=0).get(), O.reduce("add", e, axis=0), "empty add")
    with pytest.raises(ValueError, match="zero-size array to reduction operation maximum"):
        ap.maximum.reduce(de, axis=0)
    with pytest.raises(ValueError, match="not reorderable"):
        ap.subtract.reduce(ap.from_numpy(np.ones((2, 3))), axis=None)
    with pytest.raises(TypeError):
        ap.less.reduce(ap.from_numpy(np.ones(3)))
    with pytest.raises(ap.AxisError):
        ap.add.reduce(ap.from_numpy(np.ones(3)), axis=2)


def test_out_param():
    rng = np.random.default_rng(2)
    a = array(np.float32, (40, 30), rng)
    out = ap.empty((30,), np.float64)
    r = ap.add.reduce(ap.from_numpy(a), axis=0, out=out)
    assert r is out
    assert_bits_equal(out.get(), O.reduce("add", a, axis=0).astype(np.float64), "out=")


# ---------------------------------------------------------------- argext
@pytest.mark.parametrize("which", ["argmax", "argmin"])
@pytest.mark.parametrize("dt", ALL, ids=lambda d: np.dtype(d).name)
def test_argext(which, dt):
    rng = np.random.default_rng(51)
    a = array(dt, (33, 70), rng)
    if np.dtype(dt).kind in "iub":
        a = (a % 5).astype(dt) if dt != np.bool_ else a  # many ties
    d = ap.from_numpy(a)
    for axis in (None, 0, 1, -1):
        for kd in (False, True):
            want = O.argext(which, a, axis=axis, keepdims=kd)
            got = getattr(ap, which)(d, axis=axis, keepdims=kd)
            assert_bits_equal(to_host(got), np.asarray(want), f"{which} axis={axis} keepdims={kd}")
    # transposed and strided views
    for v, dv in ((a.T, d.T), (a[:, ::3], d[:, ::3]), (a[::-1], d[::-1])):
        for axis in (None, 0, 1):
            assert_bits_equal(to_host(getattr(ap, which)(dv, axis=axis)), np.asarray(O.argext(which, v, axis=axis)),
                              f"{which} view axis={axis}")


@pytest.mark.parametrize("n", [1, 5, 64, 4097, 100000, 1 << 20])
def test_argext_long(n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal(n).astype(np.float32)
    if n > 10:
        a[n // 3] = np.nan
        a[2 * n // 3] = np.nan
    assert ap.argmax(ap.from_numpy(a)) == O.argext("argmax", a)
    b = rng.integers(0, 3, (4, n)).astype(np.int64)
    assert_bits_equal(ap.argmin(ap.from_numpy(b), axis=1).get(), O.argext("argmin", b, axis=1), "argmin rows")


def test_argext_errors():
    with pytest.raises(ValueError, match="empty sequence"):
        ap.argmax(ap.from_numpy(np.zeros(0)))
    with pytest.raises(ap.AxisError):
        ap.argmin(ap.from_numpy(np.zeros((2, 2))), axis=2)


WIDE = [((3, 2048), -1), ((2, 4096), 1), ((5, 5000), -1), ((2, 2049), 1), ((3, 65536), -1), ((2, 65544), 1),
        ((1, 300007), -1), ((2, 200000), -1), ((1 << 21,), 0), ((4, 8, 4096), (1, 2)), ((16, 8192), None)]


def _nan_payloads(a, rng, frac):
    """Scatter NaNs with distinct payloads and signs, so only the first NaN in
    fold order is the right answer."""
    flat = a.reshape(-1)
    pos = np.nonzero(rng.random(flat.size) < frac)[0]
    if flat.dtype == np.float32:
        pay = (0x7FC00000 | rng.integers(1, 1 << 22, pos.size)) | (rng.integers(0, 2, pos.size) << 31)
        flat.view(np.uint32)[pos] = pay.astype(np.uint32)
    else:
        pay = (0x7FF8000000000000 | rng.integers(1, 1 << 51, pos.size, dtype=np.int64)).astype(np.uint64)
        pay |= rng.integers(0, 2, pos.size).astype(np.uint64) << np.uint64(63)
        flat.view(np.uint64)[pos] = pay
    return a


@pytest.mark.parametrize("shape,axis", WIDE, ids=str)
@pytest.mark.parametrize("dt", [np.float32, np.float64], ids=lambda d: np.dtype(d).name)
def test_wide_rows_float(shape, axis, dt):
    """Contiguous runs of >= 2048 elements (the staged pairwise kernel and the
    order-free max/min kernel), aligned and unaligned row starts, split runs."""
    rng = np.random.default_rng(sum(shape))
    a = (rng.standard_normal(shape) * 50).astype(dt)
    a.reshape(-1)[rng.random(a.size) < 0.01] = 0.0
    a.reshape(-1)[rng.random(a.size) < 0.01] = -0.0
    d = ap.from_numpy(a)
    check_reduce("add", a, d, axis=axis)
    check_reduce("add", a, d, axis=axis, initial=1.25, keepdims=True)
    for op in ("maximum", "minimum"):
        check_reduce(op, a, d, axis=axis)
    nan = _nan_payloads(a.copy(), rng, 2e-4)
    dn = ap.from_numpy(nan)
    for op in ("maximum", "minimum", "add"):
        check_reduce(op, nan, dn, axis=axis)
    # a view whose start is 4 bytes past an aligned address
    flat = (rng.standard_normal(a.size + 1) * 3).astype(dt)
    check_reduce("add", flat[1:], ap.from_numpy(flat)[1:], axis=0)
    check_reduce("maximum", flat[1:], ap.from_numpy(flat)[1:], axis=0)


@pytest.mark.parametrize("shape,axis", WIDE, ids=str)
@pytest.mark.parametrize("dt", [np.int32, np.int64, np.uint32, np.uint64], ids=lambda d: np.dtype(d).name)
def test_wide_rows_int(shape, axis, dt):
    rng = np.random.default_rng(7 + sum(shape))
    a = array(dt, shape, rng)
    d = ap.from_numpy(a)
    for op in ("add", "multiply", "maximum", "minimum", "bitwise_and", "bitwise_or", "bitwise_xor"):
        check_reduce(op, a, d, axis=axis)
    check_reduce("add", a, d, axis=axis, initial=5, keepdims=True)


NARROW = [((40000, 16), np.float64), ((38000, 2), np.float64), ((38000, 6), np.float64), ((40000, 10), np.float64),
          ((38000, 32), np.float64), ((40000, 4), np.float32), ((40000, 12), np.float32), ((40000, 64), np.float32),
          ((4, 10000, 16), np.float64), ((40000, 16), np.int64), ((40000, 8), np.int32), ((40000, 20), np.uint32)]


@pytest.mark.parametrize("shape,dt", NARROW, ids=str)
def test_narrow_rows(shape, dt):
    """Many short C-contiguous rows reduced over the last axis (the staged
    thread-per-row kernel): leaf rule for float add, in-order folds else."""
    rng = np.random.default_rng(shape[-1])
    if np.dtype(dt).kind == "f":
        a = (rng.standard_normal(shape) * 20).astype(dt)
        a.reshape(-1)[rng.random(a.size) < 0.01] = -0.0
        ops = ("add", "maximum", "minimum")
    else:
        a = array(dt, shape, rng)
        ops = ("add", "multiply", "maximum", "minimum", "bitwise_xor")
    d = ap.from_numpy(a)
    for op in ops:
        check_reduce(op, a, d, axis=-1)
    check_reduce("add", a, d, axis=-1, keepdims=True, initial=3)
    if np.dtype(dt).kind == "f":
        nan = _nan_payloads(a.copy(), rng, 0.02)
        dn = ap.from_numpy(nan)
        for op in ("maximum", "minimum", "add"):
            check_reduce(op, nan, dn, axis=-1)


@pytest.mark.parametrize("shape", [(4096, 64), (2000, 300), (8192, 5), (1024, 4736)], ids=str)
@pytest.mark.parametrize("dt", [np.float32, np.float64, np.int32, np.int64, np.uint8, np.bool_], ids=lambda d: np.dtype(d).name)
def test_axis0_order_free_split(shape, dt):
    """Order-free folds over a long leading axis with few outputs: the axis
    is cut into parts folded in order on top."""
    rng = np.random.default_rng(shape[0] + shape[1])
    a = array(dt, shape, rng, specials=False)
    if np.dtype(dt).kind == "f":
        a = _nan_payloads(a, rng, 1e-3)
        a.reshape(-1)[rng.random(a.size) < 0.01] = -0.0
        ops = ("maximum", "minimum")
    elif dt == np.bool_:
        ops = ("logical_and", "logical_or", "logical_xor", "maximum")
    else:
        ops = ("add", "multiply", "maximum", "minimum", "bitwise_and", "bitwise_or", "bitwise_xor")
    d = ap.from_numpy(a)
    for op in ops:
        check_reduce(op, a, d, axis=0)
        check_reduce(op, a, d, axis=0, keepdims=True)
    if dt != np.bool_:
        check_reduce("maximum", a, d, axis=0, initial=a.reshape(-1)[5])


@pytest.mark.parametrize("which", ["argmax", "argmin"])
@pytest.mark.parametrize("shape,dt,axis", [((4096, 5000), np.float32, 0), ((2048, 4800), np.float64, 0),
                                           ((40000, 16), np.float64, 1), ((40000, 4), np.float32, -1),
                                           ((40000, 8), np.int16, 1), ((38000, 32), np.int64, 1),
                                           ((4, 10000, 16), np.float64, 2), ((1 << 21,), np.float32, 0),
                                           ((1 << 19,), np.int64, 0), ((64, 4096), np.float16, 1),
                                           ((1 << 18,), np.float16, 0), ((3, 70000), np.float32, 1)], ids=str)
def test_argext_split_and_narrow(which, shape, dt, axis):
    """Split column scans, the many-short-rows kernel and wide split scans,
    with ties and NaNs."""
    rng = np.random.default_rng(len(shape) + shape[-1])
    if np.dtype(dt).kind == "f":
        a = np.round(rng.standard_normal(shape) * 4).astype(dt)  # many ties, both signs
        if dt != np.float16:
            a = _nan_payloads(a, rng, 1e-4)
    else:
        a = rng.integers(-3, 4, shape).astype(dt)
    d = ap.from_numpy(a)
    for kd in (False, True):
        want = O.argext(which, a, axis=axis, keepdims=kd)
        got = getattr(ap, which)(d, axis=axis, keepdims=kd)
        assert_bits_equal(to_host(got), np.asarray(want), f"{which} {a.dtype}{shape} axis={axis} keepdims={kd}")


@pytest.mark.parametrize("shape", [(4096, 64), (512, 70000), (300, 1000)], ids=str)
@pytest.mark.parametrize("dt", [np.float32, np.float64], ids=lambda d: np.dtype(d).name)
def test_axis0_float_add_nan_payloads(shape, dt):
    """Sequential column sums with NaNs of distinct payloads, signaling NaNs
    (quieted by the first add) and infinities of both signs (inf - inf makes
    the default NaN): the plain-add fast path must fall back exactly."""
    rng = np.random.default_rng(shape[1])
    a = (rng.standard_normal(shape) * 10).astype(dt)
    a = _nan_payloads(a, rng, 2e-4)
    ib = np.uint32 if dt == np.float32 else np.uint64
    snan = np.array([0x7FA00001 if dt == np.float32 else 0x7FF4000000000001], ib).view(dt)[0]
    a[0, ::7] = snan
    a[shape[0] // 2, 3::11] = snan
    a[5, 1::13] = np.inf
    a[9, 1::13] = -np.inf
    d = ap.from_numpy(a)
    check_reduce("add", a, d, axis=0)
    check_reduce("add", a, d, axis=0, initial=0.5)
    check_reduce("add", a, d, axis=0, keepdims=True)


@pytest.mark.parametrize("case", [((300, 4740), np.float32, None), ((257, 40000), np.float32, None),
                                  ((260, 5000), np.float64, None), ((256, 20000), np.float64, None),
                                  ((300, 6000), np.float32, (16, 4816)), ((300, 6000), np.float32, (1, 4801)),
                                  ((290, 9000), np.int32, None), ((270, 5000), np.int64, None)], ids=str)
def test_axis0_many_columns(case):
    """Column folds over thousands of columns: a ragged last warp of
    columns, row counts that are not a multiple of any batch, columns past
    the 8 x 148 warps of one wave, a column slice whose rows are longer than
    the kept extent and an unaligned one; each op in row order, with NaN
    payloads, signaling NaNs, infinities and signed zeros for the floats
    (float max/min fold NaN-free batches through integer order keys)."""
    shape, dt, cols = case
    rng = np.random.default_rng(shape[0] * 7 + shape[1])
    if np.dtype(dt).kind == "f":
        a = (rng.standard_normal(shape) * 3).astype(dt)
        a = _nan_payloads(a, rng, 2e-4)
        ib = np.uint32 if dt == np.float32 else np.uint64
        a[0, ::17] = np.array([0x7FA00001 if dt == np.float32 else 0x7FF4000000000001], ib).view(dt)[0]
        a[7, 2::19] = np.inf
        a[11, 2::19] = -np.inf
        a.reshape(-1)[rng.random(a.size) < 0.01] = -0.0
        ops = ("add", "maximum", "minimum", "multiply", "subtract")
    else:
        a = rng.integers(-1000, 1000, shape).astype(dt)
        ops = ("add", "multiply", "maximum", "bitwise_xor", "subtract")
    base = ap.from_numpy(a)
    if cols is not None:
        a = a[:, cols[0]:cols[1]]
        d = base[:, cols[0]:cols[1]]
    else:
        d = base
    for op in ops:
        check_reduce(op, a, d, axis=0)
    check_reduce("add", a, d, axis=0, initial=a.dtype.type(2))
    check_reduce("maximum", a, d, axis=0, keepdims=True)


@pytest.mark.parametrize("shape,axis", [((64, 4096), 1), ((9, 32768), -1), ((3, 1 << 20), 1), ((1 << 22,), None),
                                        ((2, 16, 8192), (1, 2)), ((5, 65536), None)])
def test_float32_power_of_two_runs(shape, axis):
    """float32 add.reduce over power-of-two runs (the bulk-copy window
    kernel): NaN payloads of both signs, +inf / -inf pairs whose sum is the
    x86 default NaN, leaves with several NaN chains, split runs."""
    rng = np.random.default_rng(71)
    a = rng.standard_normal(shape, dtype=np.float32)
    flat = a.reshape(-1)
    n = flat.size
    pos = rng.permutation(n)
    k = max(n // 1000, 4)
    flat[pos[:k]] = np.array([0x7FC01234, 0xFFC05678, 0x7F800001, 0xFFA00000], np.uint32).view(np.float32)[np.arange(k) % 4]
    flat[pos[k:2 * k]] = np.inf
    flat[pos[2 * k:3 * k]] = -np.inf
    flat[pos[3 * k:4 * k]] = -0.0
    want = np.asarray(O.reduce("add", a, axis=axis))
    got = ap.add.reduce(ap.from_numpy(a), axis=axis)
    assert_bits_equal(np.asarray(got.get() if isinstance(got, ap.ndarray) else got).reshape(want.shape), want,
                      f"float32 add.reduce {shape} axis={axis}")
    # clean data: no NaN anywhere, the plain-add fast path alone
    b = rng.standard_normal(shape, dtype=np.float32)
    want = np.asarray(O.reduce("add", b, axis=axis, keepdims=True))
    got = ap.add.reduce(ap.from_numpy(b), axis=axis, keepdims=True)
    assert_bits_equal(got.get(), want, f"float32 add.reduce clean {shape}")
    # a view whose rows start off a 16-byte boundary takes another kernel
    if len(shape) == 2 and axis in (1, -1):
        c = rng.standard_normal((shape[0], shape[1] + 1), dtype=np.float32)
        v = c[:, 1:]
        want = np.asarray(O.reduce("add", v, axis=1))
        got = ap.add.reduce(ap.from_numpy(c)[:, 1:], axis=1)
        assert_bits_equal(got.get(), want, f"float32 add.reduce misaligned {shape}")


def test_float32_window_nan_rules():
    """Hand-placed NaN patterns for the float32 window kernel's shortcuts: a
    chain whose inf - inf comes before its first NaN element (default NaN),
    a NaN in a chain's first element, a NaN after an infinity, a chain with
    an inf - inf and no NaN element, several NaN payloads in one row (the
    leftmost must win), and a NaN early in a row followed by other NaNs in
    later windows (the rest of the unit is skipped)."""
    f = lambda u: np.array([u], np.uint32).view(np.float32)[0]
    rows, w = 12, 1 << 15
    a = np.random.default_rng(5).standard_normal((rows, w), dtype=np.float32)
    def at(r, leaf, chain, i):            # element i of chain `chain` of leaf `leaf`
        return r, 128 * leaf + chain + 8 * i
    # row 0: inf, -inf then a NaN in the same chain -> the default NaN wins
    a[at(0, 3, 2, 1)] = np.inf; a[at(0, 3, 2, 4)] = -np.inf; a[at(0, 3, 2, 9)] = f(0x7FC0AAAA)
    # row 1: NaN in element 0 of a chain, another NaN later in it
    a[at(1, 0, 5, 0)] = f(0x7FC01111); a[at(1, 0, 5, 7)] = f(0xFFC02222)
    # row 2: infinity then a NaN (no inf - inf): the NaN, quieted
    a[at(2, 7, 0, 2)] = np.inf; a[at(2, 7, 0, 3)] = f(0x7F800005)
    # row 3: inf - inf and no NaN element in the chain
    a[at(3, 31, 7, 14)] = np.inf; a[at(3, 31, 7, 15)] = -np.inf
    # row 4: NaNs of different payloads in different leaves and windows
    a[at(4, 40, 1, 3)] = f(0xFFC03333); a[at(4, 2, 6, 12)] = f(0x7FC04444); a[4, 20000] = f(0x7FC05555)
    # row 5: a NaN in the first window, other NaNs in every later window
    a[5, 100] = f(0x7FC06666)
    for k in range(1, 8):
        a[5, 4096 * k + 7] = f(0xFFC07777 + k)
    # row 6: +inf in one window, -inf in a later one: default NaN at a node
    a[6, 10] = np.inf; a[6, 30000] = -np.inf
    # row 7: several NaN chains in one leaf, the later ones with other payloads
    a[at(7, 5, 1, 8)] = f(0x7FC08888); a[at(7, 5, 2, 0)] = f(0x7FC09999); a[at(7, 5, 6, 3)] = f(0xFF800123)
    # row 8: a NaN in the last window only
    a[8, w - 3] = f(0x7FC0ABCD)
    for axis in (1, None):
        want = np.asarray(O.reduce("add", a, axis=axis))
        got = ap.add.reduce(ap.from_numpy(a), axis=axis)
        assert_bits_equal(np.asarray(got.get() if isinstance(got, ap.ndarray) else got).reshape(want.shape), want,
                          f"window NaN rules axis={axis}")
