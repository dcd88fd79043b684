"""The array reduction family: sum, prod, min, max, amin, amax, any, all and
mean, as functions and as ndarray methods.

sum ... all are the reference's thin wrappers over ufunc.reduce
(ionp-py/src/reductions.rs:1035-1150 through do_reduce_axis, :902-948):
axis defaults to None (every axis), keepdims to False, `initial=None` and
`where=None` mean "not given". mean (reductions.rs:1515-1734) is composed,
as there, from an add reduction, dtype casts and a true divide:

* result dtype: float64 for bool and integer input, the input's own dtype
  otherwise, or `dtype=`;
* float16 results sum in float32; float16 and float32 sums are divided in
  float64 and rounded back once;
* the count is the product of the reduced extents, or the per-slice count
  of a where= mask;
* an empty slice warns "Mean of empty slice", and the 0/0 divide reports its
  FPE category under the name "scalar divide" for a 0-d quotient, "divide"
  otherwise;
* the result takes the reduction's own layout (relayout_for_reduction).
"""
from __future__ import annotations

import builtins
import ctypes
import operator
import warnings

import numpy as np

from . import _fpstate
from ._array import asarray, ndarray
from ._lib import check, lib
from ._ufunc import _NOVALUE, _normalize_axes, _scalar_result, add, logical_and, logical_or, maximum, minimum

__all__ = ["sum", "prod", "min", "max", "amin", "amax", "any", "all", "mean", "cumsum", "cumprod"]


def _keepdims(k):
    """opt_index_like (reductions.rs): None is False; otherwise an index-like"""
    if k is None:
        return False
    return bool(operator.index(k))


def _where(w):
    return True if w is None else w


def _initial(v):
    return _NOVALUE if v is None else v


def sum(a, axis=None, dtype=None, out=None, keepdims=None, initial=None, where=None):  # noqa: A001
    """add.reduce over `axis` (default: every axis)."""
    return add.reduce(a, axis=axis, dtype=dtype, out=out, keepdims=_keepdims(keepdims), initial=_initial(initial),
                      where=_where(where))


def prod(a, axis=None, dtype=None, out=None, keepdims=None, initial=None, where=None):
    """multiply.reduce over `axis` (default: every axis)."""
    from ._ufunc import multiply
    return multiply.reduce(a, axis=axis, dtype=dtype, out=out, keepdims=_keepdims(keepdims),
                           initial=_initial(initial), where=_where(where))


def all(a, axis=None, out=None, keepdims=None, where=None):  # noqa: A001
    """logical_and.reduce over `axis` (default: every axis)."""
    return logical_and.reduce(a, axis=axis, out=out, keepdims=_keepdims(keepdims), where=_where(where))


def any(a, axis=None, out=None, keepdims=None, where=None):  # noqa: A001
    """logical_or.reduce over `axis` (default: every axis)."""
    return logical_or.reduce(a, axis=axis, out=out, keepdims=_keepdims(keepdims), where=_where(where))


def min(a, axis=None, out=None, keepdims=None, initial=None, where=None):  # noqa: A001
    """minimum.reduce over `axis` (default: every axis)."""
    return minimum.reduce(a, axis=axis, out=out, keepdims=_keepdims(keepdims), initial=_initial(initial),
                          where=_where(where))


def max(a, axis=None, out=None, keepdims=None, initial=None, where=None):  # noqa: A001
    """maximum.reduce over `axis` (default: every axis)."""
    return maximum.reduce(a, axis=axis, out=out, keepdims=_keepdims(keepdims), initial=_initial(initial),
                          where=_where(where))


amin = min
amax = max


def _mean_axis_check(axis, ndim):
    """mean_family_axis_check (reductions.rs:624): mean's own axis errors."""
    if axis is None:
        return
    items = axis if isinstance(axis, tuple) else (axis,)
    for item in items:
        if isinstance(item, float):
            raise TypeError("integer argument expected, got float")
        if isinstance(item, (bool, np.bool_)) and not isinstance(item, bool):
            raise TypeError(f"'{type(item).__module__}.{type(item).__name__}' object cannot be interpreted as an integer")
        if isinstance(item, bool):
            raw = 1 if item else 0
            if raw >= ndim:
                from ._lib import AxisError
                raise AxisError(f"axis {raw} is out of bounds for array of dimension {ndim}")
            raise TypeError("an integer is required")


def mean(a, axis=None, dtype=None, out=None, keepdims=None, where=None):
    """numpy's mean as the reference composes it (reductions.rs:1515)."""
    kd = _keepdims(keepdims)
    arr = a if isinstance(a, ndarray) else asarray(a)
    _mean_axis_check(axis, arr.ndim)
    if arr.ndim == 0 and axis is not None and not (isinstance(axis, tuple) and len(axis) == 0):
        ax0 = axis[0] if isinstance(axis, tuple) else axis
        from ._lib import AxisError
        raise AxisError(f"axis {operator.index(ax0)} is out of bounds for array of dimension 0")
    axes = _normalize_axes(axis, arr.ndim)
    over = None if dtype is None else np.dtype(dtype)
    if over is None and (arr.dtype == np.bool_ or arr.dtype.kind in "iu"):
        default = np.dtype(np.float64)
    else:
        default = over
    effective = default if default is not None else arr.dtype
    f16_widen = effective == np.float16
    sum_cd = np.dtype(np.float32) if f16_widen else default
    mask = None if where is None or where is True else asarray(where)
    s = add._reduce_nd(arr, axis=tuple(axes), dtype=sum_cd, keepdims=False,
                       where=True if mask is None else mask)
    out_dt = s.dtype
    div_dt = np.dtype(np.float64) if out_dt in (np.float16, np.float32) else out_dt
    if mask is not None:
        count = add._reduce_nd(_broadcast_to(mask, arr.shape)._cast_to(np.int64), axis=tuple(axes), keepdims=False)
    else:
        n = 1
        for ax in axes:
            n *= arr.shape[ax]
        count = asarray(np.array(n, np.int64))
    cnt = count._cast_to(div_dt)
    num = s._cast_to(div_dt) if div_dt != out_dt else s
    ch = cnt.get()
    if np.any(ch == 0):
        warnings.warn("Mean of empty slice", RuntimeWarning, stacklevel=2)
    # true_divide with the reference's FPE report (detect_divide_family)
    L = lib()
    shape = num.shape
    raw = ndarray.empty(shape, div_dt)
    fpe = ctypes.c_uint32(0)
    check(L.ionp_binary(3, ctypes.byref(num._desc()), ctypes.byref(cnt._desc()), ctypes.byref(raw._desc()), None,
                        ctypes.byref(fpe), None))
    if fpe.value:
        cat = _fpstate.category_of("divide", fpe.value)
        if cat:
            _fpstate.signal(cat, "scalar divide" if num.ndim == 0 else "divide", stacklevel=2)
    res = raw
    if div_dt != out_dt:
        res = res._cast_to(out_dt)
    if f16_widen:
        res = res._cast_to(np.float16)
    elif res.dtype != effective:
        res = res._cast_to(effective)
    # relayout onto the reduction's own layout (relayout_for_reduction)
    ax = (ctypes.c_int32 * (len(axes) or 1))(*axes)
    ond = ctypes.c_int32()
    osh = (ctypes.c_int64 * 32)()
    ost = (ctypes.c_int64 * 32)()
    check(L.ionp_reduce_layout(ctypes.byref(arr._desc()), ax, len(axes), int(kd), ctypes.byref(ond), osh, ost))
    rshape = tuple(osh[i] for i in range(ond.value))
    final = ndarray.empty(rshape, res.dtype, [ost[i] for i in range(ond.value)])
    if final.size:
        src = ndarray(res._buf, rshape, res.dtype, _c_strides(rshape), res._off) if res.flags["C_CONTIGUOUS"] else \
            res.copy().reshape(rshape)
        check(L.ionp_cast(ctypes.byref(src._desc()), ctypes.byref(final._desc()), None))
    if out is not None:
        if isinstance(out, tuple):
            out = out[0]
        if not isinstance(out, ndarray):
            raise TypeError("return arrays must be of ArrayType")
        if out.shape != final.shape:
            raise ValueError(f"output parameter has the wrong shape {out.shape}, expected {final.shape}")
        if final.size:
            check(L.ionp_cast(ctypes.byref(final._desc()), ctypes.byref(out._desc()), None))
        return out
    if final.ndim == 0:
        return _scalar_result(final)
    return final


def _accumulate_axis(uf, a, axis, dtype, out):
    """do_accumulate_axis (ionp-py/src/reductions.rs:1382): dtype= casts the
    input first and the result last; axis=None (and any axis of a 0-d
    array) accumulates the C-order ravel."""
    arr = a if isinstance(a, ndarray) else asarray(a)
    over = None if dtype is None else np.dtype(dtype)
    if over is not None:
        arr = arr._cast_to(over)
    if axis is None:
        target, ax = arr.reshape(-1), 0
    else:
        if isinstance(axis, (bool, np.bool_)) or isinstance(axis, float):
            raise TypeError(f"'{type(axis).__name__}' object cannot be interpreted as an integer")
        raw = operator.index(axis)
        nd = arr.ndim
        eff = builtins.max(nd, 1)  # this module's own max is the reduction
        norm = raw + eff if raw < 0 else raw
        if norm < 0 or norm >= eff:
            from ._lib import AxisError
            raise AxisError(f"axis {raw} is out of bounds for array of dimension {eff}")
        target, ax = (arr.reshape(-1), 0) if nd == 0 else (arr, norm)
    res = uf.accumulate(target, axis=ax)
    if over is not None and res.dtype != over:
        res = res._cast_to(over)
    if out is not None:
        return uf._write_out(res, out)
    return res


def cumsum(a, axis=None, dtype=None, out=None):
    """add.accumulate along `axis` (default: the C-order ravel)."""
    return _accumulate_axis(add, a, axis, dtype, out)


def cumprod(a, axis=None, dtype=None, out=None):
    """multiply.accumulate along `axis` (default: the C-order ravel)."""
    from ._ufunc import multiply
    return _accumulate_axis(multiply, a, axis, dtype, out)


def _broadcast_to(m, shape):
    """A zero-stride view of m with the given shape (numpy broadcasting)."""
    nd = len(shape)
    if m.ndim > nd:
        raise ValueError(f"could not broadcast where= mask of shape {m.shape} to {tuple(shape)}")
    st = [0] * (nd - m.ndim) + list(m.elem_strides)
    sh = [1] * (nd - m.ndim) + list(m.shape)
    for i in range(nd):
        if sh[i] != shape[i]:
            if sh[i] != 1:
                raise ValueError(f"could not broadcast where= mask of shape {m.shape} to {tuple(shape)}")
            st[i] = 0
    return ndarray(m._buf, tuple(shape), m.dtype, st, m._off)


def _c_strides(shape):
    st, acc = [], 1
    for s in reversed(shape):
        st.append(acc)
        acc *= (s if s > 0 else 1)
    return list(reversed(st))
