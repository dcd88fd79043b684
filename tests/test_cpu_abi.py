"""CPU checks of the C ABI: the library loads, exports every symbol that
include/ionp_cuda.h declares, and its host-side rules (dtype promotion, loop
dtypes, casting, order='K' and reduction layouts) agree with the oracle and
with NumPy. No kernel is launched."""
import ctypes
import itertools
import os
import re

import numpy as np
import pytest

from anionpy_b200 import _lib
from oracle import oracle as O
from tests._util import ALL

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "ionp_cuda.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ionp_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_header_symbol():
    L = _lib.load_library()
    syms = header_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def _q(fn, *args):
    r = ctypes.c_int32(-1)
    st = fn(*args, ctypes.byref(r))
    return st, r.value


def test_promotion_matches_numpy_and_oracle():
    L = _lib.load_library()
    for a, b in itertools.product(ALL, ALL):
        st, r = _q(L.ionp_promote, _lib.code_of(a), _lib.code_of(b))
        assert st == 0
        assert _lib.DTYPES[r] == np.promote_types(a, b), (a, b)
        assert r == O.lib().oracle_promote(_lib.code_of(a), _lib.code_of(b))


@pytest.mark.parametrize("op", list(O.OPS))
def test_loop_dtypes_match_oracle(op):
    L = _lib.load_library()
    code = O.OPS[op]
    for a, b in itertools.product(ALL, ALL):
        if code >= 64:
            if b is not ALL[0]:
                continue
            st, r = _q(L.ionp_unary_out_dtype, code, _lib.code_of(a))
            want = O.lib().oracle_unary_out_dtype(code, _lib.code_of(a))
        else:
            st, r = _q(L.ionp_binary_out_dtype, code, _lib.code_of(a), _lib.code_of(b))
            want = O.lib().oracle_binary_out_dtype(code, _lib.code_of(a), _lib.code_of(b))
        if want < 0:
            assert st != 0, (op, a, b)
        else:
            assert st == 0 and r == want, (op, a, b, r, want)


def test_reduce_compute_dtype_matches_oracle():
    L = _lib.load_library()
    for op, code in O.OPS.items():
        if code >= 32:
            continue
        for a in ALL:
            st, r = _q(L.ionp_reduce_compute_dtype, code, _lib.code_of(a))
            want = O.lib().oracle_reduce_compute_dtype(code, _lib.code_of(a))
            if want < 0:
                assert st != 0, (op, a)
            else:
                assert st == 0 and r == want, (op, a)


def test_can_cast_matches_numpy():
    L = _lib.load_library()
    for rule in ("no", "equiv", "safe", "same_kind", "unsafe"):
        for a, b in itertools.product(ALL, ALL):
            st, r = _q(L.ionp_can_cast, _lib.code_of(a), _lib.code_of(b), _lib.CAST_RULES[rule])
            assert st == 0
            assert bool(r) == np.can_cast(a, b, rule), (a, b, rule)


def _desc(a: np.ndarray):
    d = _lib.IonpArr()
    d.dtype = _lib.code_of(a.dtype)
    d.ndim = a.ndim
    for i in range(a.ndim):
        d.shape[i] = a.shape[i]
        d.strides[i] = a.strides[i] // a.itemsize
    d.offset = 0
    d.data = 1
    return d


CASES = [
    [np.zeros((4, 5)), np.zeros((4, 5))],
    [np.zeros((4, 5)).T, np.zeros((5, 4))],
    [np.zeros((4, 5)).T, np.zeros((4, 5)).T],
    [np.zeros((2, 3, 4)).transpose(1, 2, 0), np.zeros((3, 4, 2))],
    [np.zeros((6, 8))[::2, ::-1], np.zeros((8,))],
    [np.zeros((3, 1, 5)), np.zeros((4, 1))],
    [np.asfortranarray(np.zeros((3, 4, 5))), np.zeros((5,))],
]


@pytest.mark.parametrize("ops", CASES)
def test_order_k_strides_match_oracle(ops):
    L = _lib.load_library()
    shape = np.broadcast_shapes(*[o.shape for o in ops])
    descs = [_desc(o) for o in ops]
    arr = (ctypes.POINTER(_lib.IonpArr) * len(descs))(*[ctypes.pointer(d) for d in descs])
    nd = len(shape)
    sh = (ctypes.c_int64 * max(nd, 1))(*shape)
    st = (ctypes.c_int64 * max(nd, 1))()
    assert L.ionp_order_k_strides(len(ops), arr, nd, sh, st) == 0
    assert list(st)[:nd] == O.order_k_strides(shape, ops)


@pytest.mark.parametrize("a", [np.zeros((4, 5, 6)), np.zeros((4, 5, 6)).transpose(2, 0, 1), np.zeros((7, 3))[::2],
                               np.asfortranarray(np.zeros((3, 4)))])
@pytest.mark.parametrize("keepdims", [False, True])
def test_reduce_layout_matches_oracle(a, keepdims):
    L = _lib.load_library()
    for axes in itertools.chain.from_iterable(itertools.combinations(range(a.ndim), k) for k in range(a.ndim + 1)):
        ax = (ctypes.c_int32 * max(len(axes), 1))(*axes)
        nd = ctypes.c_int32()
        sh = (ctypes.c_int64 * 32)()
        st = (ctypes.c_int64 * 32)()
        assert L.ionp_reduce_layout(ctypes.byref(_desc(a)), ax, len(axes), int(keepdims), ctypes.byref(nd), sh, st) == 0
        want = O.reduce_layout_strides(list(a.shape), O.elem_strides(a), list(axes), keepdims)
        assert list(st)[: nd.value] == want, (axes, keepdims)


def test_cast_scalar_matches_oracle():
    L = _lib.load_library()
    rng = np.random.default_rng(0)
    vals = [np.nan, -np.inf, 1e10, -1e10, 3.7, -3.7, 255.5, 65504.0, 70000.0, 1e-8, 2.0 ** 63, -2.0 ** 63]
    for sd in ALL:
        for dd in ALL:
            for v in vals + list(rng.standard_normal(4) * 1000):
                with np.errstate(all="ignore"):
                    src = np.array(v).astype(sd).reshape(())
                out = np.zeros(1, np.uint64)
                assert L.ionp_cast_scalar(src.ctypes.data, _lib.code_of(sd), out.ctypes.data, _lib.code_of(dd)) == 0
                got = out.view(np.uint8)[: np.dtype(dd).itemsize].view(dd)[0]
                want = O.cast(src, dd).reshape(())[()]
                assert np.array(got).tobytes() == np.array(want, dd).tobytes(), (sd, dd, v)


def _arr(dtype=10, shape=(4,), strides=None, data=0x1000, ndim=None):
    a = _lib.IonpArr()
    a.dtype = dtype
    a.ndim = len(shape) if ndim is None else ndim
    for i, s in enumerate(shape[:32]):
        a.shape[i] = s
    st = strides or [1] * len(shape)
    for i, s in enumerate(st[:32]):
        a.strides[i] = s
    a.offset = 0
    a.data = data
    return a


BAD = {
    "ndim > 32": (dict(ndim=33), _lib.ERR_INVALID, "ndim out of range"),
    "negative ndim": (dict(ndim=-1), _lib.ERR_INVALID, "ndim out of range"),
    "negative extent": (dict(shape=(4, -2)), _lib.ERR_INVALID, "negative extent"),
    "NULL data": (dict(data=None), _lib.ERR_INVALID, "NULL data"),
    "too many elements": (dict(shape=(1 << 40, 1 << 40)), _lib.ERR_INVALID, "2^62"),
    "complex dtype": (dict(dtype=12), _lib.ERR_UNSUPPORTED, "not supported"),
}


@pytest.mark.parametrize("case", list(BAD))
def test_malformed_descriptors_rejected_before_launch(case):
    """Every compute entry point validates its descriptors on the host and
    returns IONP_ERR_INVALID / IONP_ERR_UNSUPPORTED with a message, with no
    CUDA call (this runs without a GPU)."""
    L = _lib.load_library()
    kw, want, msg = BAD[case]
    bad, good = _arr(**kw), _arr()
    P = ctypes.byref
    calls = {
        "ionp_binary": lambda: L.ionp_binary(0, P(bad), P(good), P(good), None, None, None),
        "ionp_binary (out)": lambda: L.ionp_binary(0, P(good), P(good), P(bad), None, None, None),
        "ionp_unary": lambda: L.ionp_unary(81, P(bad), P(good), None, None, None),
        "ionp_cast": lambda: L.ionp_cast(P(bad), P(good), None),
        "ionp_astype": lambda: L.ionp_astype(P(bad), P(good), None, None),
        "ionp_reduce": lambda: L.ionp_reduce(0, P(bad), (ctypes.c_int32 * 1)(0), 1, 0, -1, None, None, P(good), None),
        "ionp_argext": lambda: L.ionp_argext(1, P(bad), -1, 0, P(good), None),
        "ionp_accumulate": lambda: L.ionp_accumulate(0, P(bad), 0, P(good), None),
        "ionp_reduceat": lambda: L.ionp_reduceat(0, P(bad), 0, (ctypes.c_int64 * 1)(0), 1, P(good), None),
    }
    for name, fn in calls.items():
        st = fn()
        assert st == want, f"{name}: status {st}, want {want}"
        assert msg in _lib.last_error(), f"{name}: {_lib.last_error()!r}"


def test_null_descriptor_and_bad_indices():
    L = _lib.load_library()
    good = _arr()
    assert L.ionp_binary(0, None, ctypes.byref(good), ctypes.byref(good), None, None, None) == _lib.ERR_INVALID
    assert "is NULL" in _lib.last_error()
    assert L.ionp_reduceat(0, ctypes.byref(good), 0, None, 3, ctypes.byref(good), None) == _lib.ERR_INVALID
    assert L.ionp_reduceat(0, ctypes.byref(good), 0, None, -1, ctypes.byref(good), None) == _lib.ERR_INVALID
