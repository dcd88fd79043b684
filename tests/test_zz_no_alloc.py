"""GPU test of ionp_reduce_noalloc, the reduction entry point that allocates no
device memory.

Some callers cannot let the library call cudaMalloc: a process that reserves
its device memory once at start-up, a host runtime that owns every device
byte and passes in only its own buffers, or a latency-critical loop that
cannot take an allocation's implicit synchronisation. For them
ionp_reduce_noalloc keeps its scratch (the partial results of long runs) in a
fixed array inside the library. This test calls it through the C ABI and
checks, on two calls in a row and over a sequence of different calls, that
its results equal ionp_reduce's bit for bit (the tolerance every reduction
test here uses), that it leaves the caching allocator untouched, and that it
rejects what it cannot do with a clear error.

The file is named so that pytest collects it last."""
import ctypes

import numpy as np
import pytest

from anionpy_b200 import _lib
from oracle import oracle as O
from tests._util import assert_bits_equal

ap = pytest.importorskip("anionpy_b200")
pytestmark = pytest.mark.gpu

NOALLOC_LIMIT = 1 << 20  # IONP_NOALLOC_SCRATCH_BYTES in include/ionp_cuda.h
OPS = {"add": 0, "multiply": 2, "maximum": 4, "minimum": 5, "bitwise_and": 15}


def _bind():
    L = _lib.lib()
    P = ctypes.POINTER(_lib.IonpArr)
    L.ionp_reduce_noalloc.argtypes = [ctypes.c_int32, P, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32,
                                      ctypes.c_int32, ctypes.c_void_p, P, ctypes.c_void_p]
    L.ionp_reduce_noalloc.restype = ctypes.c_int32
    return L


def _axes(axis, nd):
    axes = list(range(nd)) if axis is None else sorted(a % nd for a in np.atleast_1d(axis))
    return (ctypes.c_int32 * max(len(axes), 1))(*axes), len(axes)


def _out_for(a, axes, keepdims, dtype):
    shp = [1 if i in axes else s for i, s in enumerate(a.shape)] if keepdims else \
        [s for i, s in enumerate(a.shape) if i not in axes]
    return ap.empty(tuple(shp), dtype)


def _stats():
    s = (ctypes.c_uint64 * 4)()
    _lib.check(_lib.lib().ionp_alloc_stats(s))
    return list(s)


def noalloc(op, a, axis, keepdims, initial, out_dtype):
    """ionp_reduce_noalloc into a fresh output of out_dtype; (status, out)."""
    L = _bind()
    cax, nax = _axes(axis, a.ndim)
    out = _out_for(a, list(cax)[:nax], keepdims, out_dtype)
    init_buf = None if initial is None else np.array([initial], dtype=out_dtype)
    da, do = a._desc(), out._desc()
    st = L.ionp_reduce_noalloc(OPS[op], ctypes.byref(da), cax, nax, int(keepdims),
                               None if init_buf is None else init_buf.ctypes.data, ctypes.byref(do), None)
    return st, out


def run_both(op, a, axis, keepdims=False, initial=None):
    """(ionp_reduce result, ionp_reduce_noalloc result), both as numpy."""
    L = _bind()
    kw = {"axis": axis, "keepdims": keepdims}
    if initial is not None:
        kw["initial"] = initial
    want = getattr(ap, op).reduce(a, **kw)
    want = want.get() if isinstance(want, ap.ndarray) else np.asarray(want)
    cax, nax = _axes(axis, a.ndim)
    axes_list = list(cax)[:nax]
    out = _out_for(a, axes_list, keepdims, want.dtype)
    init_buf = None
    if initial is not None:
        init_buf = np.array([initial], dtype=want.dtype)
    da, do = a._desc(), out._desc()
    before = _stats()
    st = L.ionp_reduce_noalloc(OPS[op], ctypes.byref(da), cax, nax, int(keepdims),
                               None if init_buf is None else init_buf.ctypes.data, ctypes.byref(do), None)
    _lib.check(st)
    _lib.check(L.ionp_stream_synchronize(None))
    after = _stats()
    assert after == before, f"the no-alloc call touched the caching allocator: {before} -> {after}"
    return want, out.get().reshape(want.shape)


CASES = [
    # (op, dtype, shape, axis, keepdims, initial): long runs split into
    # per-CTA segments, so their partials go through the static scratch
    ("add", np.float32, ((1 << 22) + 37,), 0, False, None),
    ("add", np.float64, (6, 300001), 1, False, None),
    ("add", np.float64, (3, 5, 100003), (1, 2), True, 0.0),
    ("add", np.float16, (4, 70001), -1, False, None),
    ("add", np.int32, (3, 1 << 20), 1, False, None),
    ("maximum", np.float32, (5, 400000), 1, False, None),
    ("minimum", np.float64, (1 << 21,), None, True, None),
    ("bitwise_and", np.uint16, (2, 300000), 1, False, None),
    ("multiply", np.int64, (7, 90001), 1, False, None),
    # short runs: no split, the static scratch is not needed
    ("add", np.float64, (512, 129), 1, False, 1.5),
    ("add", np.float32, (64, 3), 1, True, None),
]


def _data(dt, shape, seed):
    rng = np.random.default_rng(seed)
    n = int(np.prod(shape))
    if np.dtype(dt).kind == "f":
        x = rng.standard_normal(n).astype(dt)
        x[rng.random(n) < 1e-4] = np.nan
    elif np.dtype(dt).kind == "u":
        x = rng.integers(0, np.iinfo(dt).max, n, dtype=dt, endpoint=True)
    else:
        x = rng.integers(-1000, 1000, n).astype(dt)
    return x.reshape(shape)


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{np.dtype(c[1]).name}-{c[2]}-{c[3]}")
def test_noalloc_matches_reduce_twice(case):
    op, dt, shape, axis, keepdims, initial = case
    a = ap.from_numpy(_data(dt, shape, 5))
    for call in range(2):
        want, got = run_both(op, a, axis, keepdims, initial)
        assert_bits_equal(got, want, f"{op} {np.dtype(dt).name}{shape} axis={axis} call {call + 1}")


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{np.dtype(c[1]).name}-{c[2]}-{c[3]}")
def test_noalloc_matches_oracle(case):
    """The same cases against the oracle (the CPU restatement of the
    reference's reduce_axis), bit for bit."""
    op, dt, shape, axis, keepdims, initial = case
    host = _data(dt, shape, 5)
    kw = {"axis": axis, "keepdims": keepdims}
    if initial is not None:
        kw["initial"] = initial
    want = np.asarray(O.reduce(op, host, **kw))
    st, out = noalloc(op, ap.from_numpy(host), axis, keepdims, initial, want.dtype)
    _lib.check(st)
    assert_bits_equal(out.get().reshape(want.shape), want, f"{op} {np.dtype(dt).name}{shape} vs oracle")


def test_noalloc_widening_and_zero_d():
    """int8 and bool add.reduce widen to int64 on load; a 0-d input reduces
    to itself plus the seed. Each against ionp_reduce and the oracle."""
    rng = np.random.default_rng(8)
    for host in (rng.integers(-128, 128, (3, 200001)).astype(np.int8), rng.integers(0, 2, (2, 150001)).astype(np.bool_)):
        a = ap.from_numpy(host)
        want, got = run_both("add", a, 1)
        assert_bits_equal(got, want, f"add {host.dtype} vs ionp_reduce")
        assert_bits_equal(got, np.asarray(O.reduce("add", host, axis=1)), f"add {host.dtype} vs oracle")
    for v in (np.array(2.5), np.array(-7, np.int32)):
        want = np.asarray(O.reduce("add", v, axis=None))
        st, out = noalloc("add", ap.from_numpy(v), None, False, None, want.dtype)
        _lib.check(st)
        assert_bits_equal(out.get().reshape(want.shape), want, f"0-d {v.dtype}")


def test_noalloc_long_zero_stride_run():
    """A zero-stride view with a 2^32-element run (no memory behind it) splits
    into 2^16 segments: the top pass folds 2^16 partials per output, far more
    than shared memory holds at once. Pairwise sums of a constant power-of-two
    multiple are exact, so the result is known in closed form."""
    for dt, v in ((np.float64, 1.5), (np.float32, 1.0)):
        base = ap.from_numpy(np.array([v], dt))
        view = ap.ndarray(base._buf, (1 << 32,), dt, strides=(0,), offset=0)
        want, got = run_both("add", view, 0)
        assert_bits_equal(got, want, f"{np.dtype(dt).name} 2^32 zero-stride run vs ionp_reduce")
        assert float(got) == v * 2.0 ** 32, (float(got), v * 2.0 ** 32)


def test_noalloc_sequence_of_different_calls():
    """Each call overwrites the shared scratch; a later call with other sizes
    must not see the earlier call's partials."""
    for k, (op, dt, shape, axis, keepdims, initial) in enumerate(CASES[:6] + CASES[:3]):
        a = ap.from_numpy(_data(dt, shape, 100 + k))
        want, got = run_both(op, a, axis, keepdims, initial)
        assert_bits_equal(got, want, f"sequence call {k}: {op} {np.dtype(dt).name}{shape}")


def test_noalloc_rejects_oversized_and_unsupported():
    L = _bind()
    # 65537 outputs, each a run of 65537 int64 elements (an overlapping
    # sliding-window view of a 131073-element buffer): the runs split in two,
    # so the partials need 131074 x 8 bytes, over the 1 MiB limit. Rejected
    # before any launch.
    base = ap.from_numpy(np.arange(131073, dtype=np.int64))
    win = ap.ndarray(base._buf, (65537, 65537), np.int64, strides=(1, 1), offset=0)
    out = ap.empty((65537,), np.int64)
    cax, nax = _axes(1, 2)
    da, do = win._desc(), out._desc()
    st = L.ionp_reduce_noalloc(OPS["add"], ctypes.byref(da), cax, nax, 0, None, ctypes.byref(do), None)
    assert st == _lib.ERR_VALUE
    msg = _lib.last_error()
    assert "exceed" in msg and str(NOALLOC_LIMIT) in msg, msg
    # a narrow float add (axis 0 of a C-order array) folds in the column
    # kernel: not this entry point's job
    a = ap.from_numpy(np.ones((300, 400), np.float32))
    out = ap.empty((400,), np.float32)
    cax, nax = _axes(0, 2)
    da, do = a._desc(), out._desc()
    st = L.ionp_reduce_noalloc(OPS["add"], ctypes.byref(da), cax, nax, 0, None, ctypes.byref(do), None)
    assert st == _lib.ERR_UNSUPPORTED
    assert "use ionp_reduce" in _lib.last_error()
