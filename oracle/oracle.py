"""TEST INFRASTRUCTURE ONLY -- the parity oracle's Python face.

ctypes wrapper over ``liboracle.so`` (``ionp_oracle.cpp``, a CPU restatement
of anionpy's ufunc engine). Only ``tests/``, ``__graft_entry__.smoke()`` and
the ``cpu_baseline`` leg of ``bench.py`` may import this module, and only to
check or time the reference behaviour; the product never calls it.

Besides the numeric calls it restates, in plain Python, the reference's
metadata rules that decide result layout (these touch shapes and strides
only):

* ``multi_sorted_stride_perm`` / ``apply_ufunc_order`` -- order='K' output
  layout of a ufunc call (ionp-core/src/array.rs:1153-1222,
  ionp-py/src/lib.rs:1290-1330);
* ``reduce_output_layout`` / ``relayout_for_reduction`` -- layout of a
  reduction result (ionp-core/src/array.rs:845-930);
* ``normalize_reduce_axes`` (ionp-core/src/ufunc.rs:7551-7632).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

# dtype codes in the order of ionp-core/src/dtype.rs:14
NP_DTYPES = [np.bool_, np.int8, np.int16, np.int32, np.int64, np.uint8, np.uint16,
             np.uint32, np.uint64, np.float16, np.float32, np.float64]
CODE = {np.dtype(t): i for i, t in enumerate(NP_DTYPES)}

OPS = {
    "add": 0, "subtract": 1, "multiply": 2, "divide": 3, "maximum": 4, "minimum": 5,
    "greater": 6, "greater_equal": 7, "less": 8, "less_equal": 9, "equal": 10, "not_equal": 11,
    "logical_and": 12, "logical_or": 13, "logical_xor": 14,
    "bitwise_and": 15, "bitwise_or": 16, "bitwise_xor": 17,
    "floor_divide": 18, "left_shift": 19, "right_shift": 20,
    "remainder": 32, "fmod": 33,
    "negative": 64, "absolute": 65, "invert": 66, "logical_not": 67,
    "sqrt": 80, "exp": 81, "log": 82, "sin": 83, "cos": 84,
}
FPE_NAMES = {0: None, 1: "divide", 2: "over", 4: "under", 8: "invalid"}
STATUS = {1: "broadcast", 2: "type", 3: "value", 4: "no_loop", 5: "axis", 9: "unsupported"}


class OrArr(ctypes.Structure):
    _fields_ = [("dtype", ctypes.c_int32), ("ndim", ctypes.c_int32),
                ("shape", ctypes.c_int64 * 32), ("strides", ctypes.c_int64 * 32),
                ("offset", ctypes.c_int64), ("data", ctypes.c_void_p)]


class OracleError(Exception):
    def __init__(self, status):
        super().__init__(STATUS.get(status, status))
        self.status = STATUS.get(status, status)


def build():
    """Compile liboracle.so from ionp_oracle.cpp (idempotent)."""
    src = os.path.join(_HERE, "ionp_oracle.cpp")
    if (not os.path.exists(_LIB_PATH)) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.POINTER(OrArr)
        L.oracle_binary.argtypes = [ctypes.c_int, P, P, P, ctypes.POINTER(ctypes.c_int)]
        L.oracle_unary.argtypes = [ctypes.c_int, P, P, ctypes.POINTER(ctypes.c_int)]
        L.oracle_reduce.argtypes = [ctypes.c_int, P, ctypes.c_int, ctypes.POINTER(ctypes.c_int32),
                                    ctypes.c_int, P, P, P]
        L.oracle_argext.argtypes = [ctypes.c_int, P, ctypes.c_int, P]
        L.oracle_cast.argtypes = [P, P]
        L.oracle_pairwise_f64.argtypes = [ctypes.c_void_p, ctypes.c_int64]
        L.oracle_pairwise_f64.restype = ctypes.c_double
        _lib = L
    return _lib


def _desc(a: np.ndarray) -> OrArr:
    d = OrArr()
    d.dtype = CODE[a.dtype]
    d.ndim = a.ndim
    for i in range(a.ndim):
        d.shape[i] = a.shape[i]
        st = a.strides[i]
        assert st % a.itemsize == 0
        d.strides[i] = st // a.itemsize
    d.offset = 0
    d.data = a.ctypes.data if a.size else (np.zeros(1, a.dtype).ctypes.data)
    return d


def np_dtype(code: int):
    return np.dtype(NP_DTYPES[code])


def binary_out_dtype(op: str, da, db):
    r = lib().oracle_binary_out_dtype(OPS[op], CODE[np.dtype(da)], CODE[np.dtype(db)])
    if r < 0:
        raise OracleError(-r)
    return np_dtype(r)


def unary_out_dtype(op: str, da):
    r = lib().oracle_unary_out_dtype(OPS[op], CODE[np.dtype(da)])
    if r < 0:
        raise OracleError(-r)
    return np_dtype(r)


def reduce_compute_dtype(op: str, da):
    r = lib().oracle_reduce_compute_dtype(OPS[op], CODE[np.dtype(da)])
    if r < 0:
        raise OracleError(-r)
    return np_dtype(r)


def binary(op: str, a: np.ndarray, b: np.ndarray):
    """(C-order result, fpe category name or None) of ufunc `op`(a, b)."""
    a = np.asarray(a)
    b = np.asarray(b)
    od = binary_out_dtype(op, a.dtype, b.dtype)
    try:
        shape = np.broadcast_shapes(a.shape, b.shape)
    except ValueError:
        raise OracleError(1) from None
    out = np.empty(shape, od)
    fpe = ctypes.c_int(0)
    st = lib().oracle_binary(OPS[op], _desc(a), _desc(b), _desc(out), ctypes.byref(fpe))
    if st:
        raise OracleError(st)
    return out, FPE_NAMES[fpe.value]


def unary(op: str, a: np.ndarray):
    a = np.asarray(a)
    od = unary_out_dtype(op, a.dtype)
    out = np.empty(a.shape, od)
    fpe = ctypes.c_int(0)
    st = lib().oracle_unary(OPS[op], _desc(a), _desc(out), ctypes.byref(fpe))
    if st:
        raise OracleError(st)
    return out, FPE_NAMES[fpe.value]


def cast(a: np.ndarray, dtype) -> np.ndarray:
    out = np.empty(a.shape, dtype)
    lib().oracle_cast(_desc(np.asarray(a)), _desc(out))
    return out


def normalize_reduce_axes(axis, ndim):
    """normalize_reduce_axes (ionp-core/src/ufunc.rs:7551-7632)."""
    if axis is None:
        return list(range(ndim))
    raw = list(axis) if isinstance(axis, (tuple, list)) else [axis]
    out = []
    for ax in raw:
        norm = ax + max(ndim, 1) if ax < 0 else ax
        if ndim == 0:
            if norm != 0:
                raise OracleError(5)
        elif norm < 0 or norm >= ndim:
            raise OracleError(5)
        out.append(max(norm, 0))
    if len(set(out)) != len(out):
        raise OracleError(3)
    return [] if ndim == 0 else sorted(out)


def reduce(op: str, a: np.ndarray, axis=0, dtype=None, keepdims=False, initial=None, where=None):
    """ufunc.reduce values (C-order over kept axes, keepdims re-inserted)."""
    a = np.asarray(a)
    axes = normalize_reduce_axes(axis, a.ndim)
    cd = np.dtype(dtype) if dtype is not None else reduce_compute_dtype(op, a.dtype)
    keep = [a.shape[i] for i in range(a.ndim) if i not in axes]
    out = np.empty(max(int(np.prod(keep)), 1) if not keep else keep, cd)
    if not keep:
        out = np.empty((1,), cd)
    ax = (ctypes.c_int32 * max(len(axes), 1))(*axes)
    ini = _desc(np.asarray(initial)) if initial is not None else None
    msk = None
    if where is not None:
        w = np.asarray(where)
        msk = _desc(w)
    st = lib().oracle_reduce(OPS[op], _desc(a), len(axes), ax, CODE[cd],
                             ctypes.byref(ini) if ini is not None else None,
                             ctypes.byref(msk) if msk is not None else None, _desc(out))
    if st:
        raise OracleError(st)
    res = out.reshape(keep) if keep else out.reshape(())
    if keepdims:
        res = res.reshape([1 if i in axes else a.shape[i] for i in range(a.ndim)])
    return res


def argext(which: str, a: np.ndarray, axis=None, keepdims=False):
    """argmin/argmax (ionp-py/src/reductions.rs:1198-1300, ufunc.rs:8131)."""
    a = np.asarray(a)
    ndim = a.ndim
    if axis is None:
        t = np.ascontiguousarray(a).reshape(-1)
        ax = 0
    else:
        ax = axis + max(ndim, 1) if axis < 0 else axis
        if ax < 0 or ax >= max(ndim, 1):
            raise OracleError(5)
        t = a
    keep = [t.shape[i] for i in range(t.ndim) if i != ax]
    out = np.empty(keep if keep else (1,), np.int64)
    st = lib().oracle_argext(1 if which == "argmax" else 0, _desc(t), ax, _desc(out))
    if st:
        raise OracleError(st)
    res = out.reshape(keep) if keep else out.reshape(())
    if keepdims and t.ndim != 0:
        res = res.reshape([1 if i == ax else t.shape[i] for i in range(t.ndim)])
    if axis is None and keepdims and ndim != 1:
        res = res.reshape([1] * ndim)
    return res


def pairwise_sum_f64(x: np.ndarray) -> float:
    x = np.ascontiguousarray(x, np.float64)
    return lib().oracle_pairwise_f64(x.ctypes.data, x.size)


# ---------------------------------------------------------------------------
# Layout rules (metadata only)
# ---------------------------------------------------------------------------
def c_strides(shape):
    st, acc = [0] * len(shape), 1
    for i in range(len(shape) - 1, -1, -1):
        st[i] = acc
        acc *= max(shape[i], 1)
    return st


def elem_strides(a: np.ndarray):
    return [s // a.itemsize for s in a.strides]


def multi_sorted_stride_perm(ndim, operands):
    """ionp-core/src/array.rs:1153-1205 (operands: list of (shape, elem strides))."""
    perm = list(range(ndim))
    for i0 in range(1, ndim):
        ax_j0 = perm[i0]
        ipos = i0
        i1 = i0
        while i1 > 0:
            i1 -= 1
            ax_j1 = perm[i1]
            ambig, shouldswap = True, False
            for shape, strides in operands:
                off = ndim - len(shape)
                if ax_j0 < off or ax_j1 < off:
                    continue
                s0, s1 = shape[ax_j0 - off], shape[ax_j1 - off]
                if s0 == 1 or s1 == 1:
                    continue
                st0, st1 = abs(strides[ax_j0 - off]), abs(strides[ax_j1 - off])
                if st0 <= st1:
                    shouldswap = False
                elif ambig:
                    shouldswap = True
                ambig = False
            if not ambig:
                if shouldswap:
                    ipos = i1
                else:
                    break
        if ipos != i0:
            perm[ipos + 1:i0 + 1] = perm[ipos:i0]
        perm[ipos] = ax_j0
    return perm


def perm_strides(shape, perm):
    """relayout_by_perm strides (array.rs:799-817)."""
    pshape = [shape[a] for a in perm]
    pst = c_strides(pshape)
    st = [0] * len(shape)
    for i, a in enumerate(perm):
        st[a] = pst[i]
    if int(np.prod(shape)) == 0:
        st = [0] * len(shape)
    return st


def _is_contig(a: np.ndarray, f: bool):
    return a.flags["F_CONTIGUOUS"] if f else a.flags["C_CONTIGUOUS"]


def order_k_strides(out_shape, operands):
    """Element strides of an order='K' ufunc result (lib.rs:1290-1330)."""
    nd = len(out_shape)
    if all(_is_contig(o, False) for o in operands):
        perm = list(range(nd))
    elif all(_is_contig(o, True) for o in operands):
        perm = list(range(nd))[::-1]
    else:
        perm = multi_sorted_stride_perm(nd, [(o.shape, elem_strides(o)) for o in operands])
    return perm_strides(list(out_shape), perm)


def reduce_layout_strides(shape, strides, axes, keepdims):
    """Strides of a reduction result (array.rs:845-930)."""
    nd = len(shape)
    retained = [i for i in range(nd) if i not in axes]
    full = sorted(range(nd), key=lambda x: -abs(strides[x]))
    local = {ax: i for i, ax in enumerate(retained)}
    local_perm = [local[ax] for ax in full if ax in local]
    kshape = [shape[a] for a in retained]
    st = perm_strides(kshape, local_perm)
    if not keepdims:
        return st
    pretend = list(shape)
    for a in axes:
        pretend[a] = 1
    perm = sorted(range(nd), key=lambda x: -abs(strides[x]))
    pshape = [pretend[a] for a in perm]
    pst = c_strides(pshape)
    full_st = [0] * nd
    for i, a in enumerate(perm):
        full_st[a] = pst[i]
    if int(np.prod(pretend)) == 0:
        full_st = [0] * nd
    return full_st


def mean(a: np.ndarray, axis=None, dtype=None, keepdims=False, where=None):
    """numpy's mean as the reference composes it (ionp-py/src/reductions.rs:
    1515-1734): (values, warned_empty, fpe category of the internal divide).
    Sum with add.reduce (float16 results sum in float32, bool/int input in
    float64 unless dtype= says otherwise), divide in float64 for float16 and
    float32 sums, cast back once; where= divides by the mask's count."""
    a = np.asarray(a)
    axes = normalize_reduce_axes(axis, a.ndim)
    over = None if dtype is None else np.dtype(dtype)
    default = np.dtype(np.float64) if over is None and (a.dtype == np.bool_ or a.dtype.kind in "iu") else over
    effective = default if default is not None else a.dtype
    f16_widen = effective == np.float16
    sum_cd = np.dtype(np.float32) if f16_widen else default
    mask = None if where is None else np.broadcast_to(np.asarray(where), a.shape)
    s = np.asarray(reduce("add", a, axis=tuple(axes), dtype=sum_cd, keepdims=False,
                          where=None if mask is None else mask))
    out_dt = s.dtype
    div_dt = np.dtype(np.float64) if out_dt in (np.float16, np.float32) else out_dt
    if mask is not None:
        count = np.asarray(reduce("add", cast(np.ascontiguousarray(mask), np.int64), axis=tuple(axes), keepdims=False))
    else:
        n = 1
        for ax in axes:
            n *= a.shape[ax]
        count = np.array(n, np.int64)
    cnt = cast(np.asarray(count), div_dt)
    num = cast(s, div_dt) if div_dt != out_dt else s
    warned = bool(np.any(cnt == 0))
    raw, cat = binary("divide", num, cnt)
    res = raw
    if div_dt != out_dt:
        res = cast(res, out_dt)
    if f16_widen:
        res = cast(res, np.float16)
    elif res.dtype != effective:
        res = cast(res, effective)
    if keepdims:
        res = res.reshape([1 if i in axes else a.shape[i] for i in range(a.ndim)])
    return res, warned, cat


def accumulate(op: str, a: np.ndarray, axis: int = 0):
    """accumulate_axis (ionp-core/src/ufunc.rs:7967-8035, accumulate_axis_generic
    7898): every fiber along `axis` folded left to right in the reduce-family
    compute dtype, acc = x0, acc = op(acc, x_i) -- one oracle ufunc call per
    step over all fibers at once (C-ordered result)."""
    a = np.asarray(a)
    cd = reduce_compute_dtype(op, a.dtype)
    x = np.moveaxis(cast(np.ascontiguousarray(a), cd), axis, 0)
    out = np.empty(x.shape, cd)
    if x.shape[0] == 0:
        return np.moveaxis(out, 0, axis)
    acc = np.ascontiguousarray(x[0])
    out[0, ...] = acc
    for i in range(1, x.shape[0]):
        acc = binary(op, acc, np.ascontiguousarray(x[i]))[0].astype(cd, copy=False).reshape(x.shape[1:])
        out[i, ...] = acc
    return np.ascontiguousarray(np.moveaxis(out, 0, axis))


def reduceat(op: str, a: np.ndarray, indices, axis: int = 0):
    """reduceat_binary_axis (ionp-core/src/ufunc.rs:8450, reduceat_axis_generic
    8322): segment k folds x[idx_k .. idx_{k+1}) left to right (to the axis
    end for the last), or is x[idx_k] alone when idx_{k+1} <= idx_k."""
    a = np.asarray(a)
    idx = [int(i) for i in np.asarray(indices).reshape(-1)]
    n = a.shape[axis]
    for i in idx:
        if i < 0 or i >= n:
            raise IndexError(f"index {i} out-of-bounds in {op}.reduceat [0, {n})")
    cd = reduce_compute_dtype(op, a.dtype)
    x = np.moveaxis(cast(np.ascontiguousarray(a), cd), axis, 0)
    out = np.empty((len(idx),) + x.shape[1:], cd)
    for k, start in enumerate(idx):
        nxt = idx[k + 1] if k + 1 < len(idx) else n
        acc = np.ascontiguousarray(x[start])
        for j in range(start + 1, nxt):
            acc = binary(op, acc, np.ascontiguousarray(x[j]))[0].astype(cd, copy=False).reshape(x.shape[1:])
        out[k, ...] = acc
    return np.ascontiguousarray(np.moveaxis(out, 0, axis))


def outer(op: str, a: np.ndarray, b: np.ndarray):
    """outer_binary (ionp-core/src/ufunc.rs:8212): op over the cross product,
    shape a.shape + b.shape."""
    a = np.asarray(a)
    b = np.asarray(b)
    return binary(op, a.reshape(a.shape + (1,) * b.ndim), b)[0]


BINARY_AT_OPS = ("add", "subtract", "multiply", "divide", "maximum", "minimum", "greater", "greater_equal", "less",
                 "less_equal", "equal", "not_equal", "logical_and", "logical_or", "logical_xor", "bitwise_and",
                 "bitwise_or", "bitwise_xor", "floor_divide", "left_shift", "right_shift", "remainder", "fmod")
LOGICAL = ("logical_and", "logical_or", "logical_xor")
COMPARE = ("greater", "greater_equal", "less", "less_equal", "equal", "not_equal")


def at_rows(shape, indices):
    """normalize_at_indices (ionp-core/src/ufunc.rs:9250): negative indices
    count from the end of axis 0; a 0-d target takes no index and applies
    the op once."""
    idx = [int(i) for i in np.asarray(indices, dtype=np.int64).reshape(-1)]
    if len(shape) == 0:
        if idx:
            raise IndexError(f"too many indices for array: array is 0-dimensional, but {len(idx)} were indexed")
        return [None]
    n = shape[0]
    rows = []
    for i in idx:
        j = i + n if i < 0 else i
        if j < 0 or j >= n:
            raise IndexError(f"index {i} is out of bounds for axis 0 with size {n}")
        rows.append(j)
    return rows


def _cc(x):
    """C-contiguous copy that keeps 0-d arrays 0-d."""
    return np.array(x, order="C")


def _row(t, r):
    return t[...] if r is None else t[r, ...]


def at(op: str, target: np.ndarray, indices, values=None):
    """ufunc.at in place on the numpy array `target`: at_binary
    (ionp-core/src/ufunc.rs:9577-9733), at_math_binary (9932), at_unary
    (9301) and at_math_unary (9805), one oracle ufunc call per index:
    * binary: values are broadcast against (len(indices),) + row shape as a
      whole; logical ops compute in bool and store 0/1 of the target dtype;
      comparisons compute in the target dtype (values cast to it) and store
      0/1 of it; other ops compute in the target dtype, or, when the ufunc
      promotes (target, values) to another dtype, on a whole-target copy in
      that dtype cast back at the end;
    * unary: logical_not in bool, stored back as 0/1; negative / absolute /
      invert only where they keep the dtype (else TypeError "'.at' would
      change dtype ..."); sqrt / exp / log / sin / cos in their float loop dtype,
      cast back after every application."""
    dt = target.dtype
    if values is None:
        math = op in ("sqrt", "exp", "log", "sin", "cos")
        if math:
            unary_out_dtype(op, dt)          # checked before the indices
        rows = at_rows(target.shape, indices)
        if op == "logical_not":
            for r in rows:
                _row(target, r)[...] = cast(np.asarray(cast(_row(target, r), np.bool_) == 0), dt)
            return target
        if not math:
            od = unary_out_dtype(op, dt)
            if od != dt:
                raise TypeError(f"'.at' would change dtype from {dt} to {od}, which is not supported")
        for r in rows:
            _row(target, r)[...] = cast(unary(op, _cc(_row(target, r)))[0], dt)
        return target
    values = np.asarray(values)
    rows = at_rows(target.shape, indices)
    vshape = ((len(rows),) + target.shape[1:]) if target.ndim else ()
    if op in LOGICAL:
        cd = np.dtype(np.bool_)
    elif op in COMPARE:
        cd = dt
    else:
        cd = binary_out_dtype(op, dt, values.dtype)
        if cd != dt:
            try:
                np.broadcast_to(values, vshape)
            except ValueError:
                raise OracleError(1) from None
            tmp = cast(_cc(target), cd)
            at(op, tmp, indices, values)
            target[...] = cast(tmp, dt)
            return target
    try:
        v = np.broadcast_to(cast(_cc(values), cd), vshape)
    except ValueError:
        raise OracleError(1) from None
    for i, r in enumerate(rows):
        row = _cc(_row(target, r))
        lhs = cast(row, cd) if op in LOGICAL else row
        res = binary(op, lhs, _cc(v[i] if target.ndim else v))[0]
        _row(target, r)[...] = cast(np.asarray(res), dt)
    return target
