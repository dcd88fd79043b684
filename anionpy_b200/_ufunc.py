"""The ufunc objects: ``__call__``, ``.reduce`` and ``argmin``/``argmax``.

Mirrors the reference's PyO3 ``Ufunc`` pyclass (ionp-py/src/lib.rs:8697-10238)
and ``do_argext`` (ionp-py/src/reductions.rs:1174-1300): same names, keyword
arguments, casting checks, output layout rules and error types. All compute
goes through the C ABI of libionp_cuda.so on the GPU.
"""
from __future__ import annotations

import ctypes
import operator

import numpy as np

from . import _fpstate
from ._array import asarray, from_numpy, ndarray
from ._lib import AxisError, CAST_RULES, DTYPES, IonpArr, UFuncTypeError, check, code_of, lib

_NOVALUE = object()

# op codes (include/ionp_cuda.h)
BINARY_OPS = {
    "add": 0, "subtract": 1, "multiply": 2, "divide": 3, "maximum": 4, "minimum": 5,
    "greater": 6, "greater_equal": 7, "less": 8, "less_equal": 9, "equal": 10, "not_equal": 11,
    "logical_and": 12, "logical_or": 13, "logical_xor": 14,
    "bitwise_and": 15, "bitwise_or": 16, "bitwise_xor": 17,
    "floor_divide": 18, "left_shift": 19, "right_shift": 20,
    "remainder": 32, "fmod": 33,
}
UNARY_OPS = {
    "negative": 64, "absolute": 65, "invert": 66, "logical_not": 67,
    "sqrt": 80, "exp": 81, "log": 82, "sin": 83, "cos": 84,
}
# ops that have a post-hoc FPE detector (lib.rs:9077-9138)
_FPE_KIND = {"divide": "divide", "floor_divide": "divide", "remainder": "remainder", "fmod": "remainder",
             "multiply": "multiply", "sqrt": "sqrt", "log": "log"}


def _weak_scalar(x, other_dtype):
    """NEP 50 weak Python scalars (scalar_against, lib.rs:8104-8236)."""
    if isinstance(x, (bool, np.bool_)):
        return np.asarray(x, np.bool_)
    if isinstance(x, (np.generic,)):
        return np.asarray(x)
    if isinstance(x, int):
        if other_dtype is not None and other_dtype.kind in "iuf":
            if other_dtype.kind in "iu":
                info = np.iinfo(other_dtype)
                if not info.min <= x <= info.max:
                    raise OverflowError(f"Python integer {x} out of bounds for {other_dtype}")
            return np.asarray(x, other_dtype)
        return np.asarray(x, np.int64)
    if isinstance(x, float):
        if other_dtype is not None and other_dtype.kind == "f":
            return np.asarray(x, other_dtype)
        return np.asarray(x, np.float64)
    raise TypeError(f"unsupported operand type {type(x).__name__}")


def _operands(args):
    """Operands as device arrays; bare Python scalars are weak (NEP 50)."""
    dts = [a.dtype for a in args if isinstance(a, (ndarray, np.ndarray))]
    ref = dts[0] if dts else None
    out = []
    for a in args:
        if isinstance(a, ndarray):
            out.append(a)
        elif isinstance(a, np.ndarray):
            out.append(from_numpy(a))
        elif isinstance(a, (list, tuple)):
            out.append(from_numpy(np.asarray(a)))
        else:
            out.append(from_numpy(_weak_scalar(a, ref)))
    return out


def _fmt_shape(s):
    return "(" + ",".join(str(d) for d in s) + ("," if len(s) == 1 else "") + ")"


def _broadcast(shapes):
    """broadcast_shapes with the reference's error text (shape.rs:54-72)."""
    nd = max((len(s) for s in shapes), default=0)
    out = [1] * nd
    for s in shapes:
        for i, d in enumerate(s):
            k = nd - len(s) + i
            if out[k] == 1:
                out[k] = d
            elif d != 1 and d != out[k]:
                raise ValueError("operands could not be broadcast together with shapes "
                                 + " ".join(_fmt_shape(x) for x in shapes) + " ")
    return tuple(out)


def _scalar_result(r: ndarray):
    """A 0-d result becomes a numpy scalar (numpy_scalar_from_0d, lib.rs:8518)."""
    return r.get().reshape(())[()]


def _check_casting(casting):
    if casting not in CAST_RULES:
        raise ValueError(f"casting must be one of 'no', 'equiv', 'safe', 'same_kind', or 'unsafe'")
    return CAST_RULES[casting]


def _can_cast(a, b, rule) -> bool:
    r = ctypes.c_int32()
    check(lib().ionp_can_cast(code_of(a), code_of(b), rule, ctypes.byref(r)))
    return bool(r.value)


def _dt(code: int):
    return DTYPES[code]


class ufunc:
    """One ufunc object (ionp-py/src/lib.rs:8697 `Ufunc`)."""

    def __init__(self, name: str, nin: int, op: int):
        self.__name__ = name
        self.nin = nin
        self.nout = 1
        self.nargs = nin + 1
        self._op = op
        self._fpe = _FPE_KIND.get(name)

    def __repr__(self):
        return f"<ufunc '{self.__name__}'>"

    # ---- dtype resolution -------------------------------------------------
    def _result_dtype(self, dts):
        r = ctypes.c_int32()
        if self.nin == 2:
            check(lib().ionp_binary_out_dtype(self._op, code_of(dts[0]), code_of(dts[1]), ctypes.byref(r)))
        else:
            check(lib().ionp_unary_out_dtype(self._op, code_of(dts[0]), ctypes.byref(r)))
        return _dt(r.value)

    # ---- __call__ ----------------------------------------------------------
    def __call__(self, *args, out=_NOVALUE, where=True, dtype=None, casting="same_kind", order="K", subok=True, **kw):
        if kw:
            raise TypeError(f"{self.__name__}() got an unexpected keyword argument '{next(iter(kw))}'")
        if len(args) > self.nin:
            if len(args) > self.nargs:
                raise TypeError(f"{self.__name__}() takes from {self.nin} to {self.nargs} positional arguments but {len(args)} were given")
            if out is not _NOVALUE:
                raise TypeError("cannot specify 'out' as both a positional and keyword argument")
            out = args[self.nin]
            args = args[:self.nin]
        if len(args) < self.nin:
            raise TypeError(f"{self.__name__}() takes from {self.nin} to {self.nargs} positional arguments but {len(args)} were given")
        if isinstance(out, tuple):
            if len(out) != 1:
                raise ValueError("The 'out' tuple must have exactly one entry per ufunc output")
            out = out[0]
        if out is _NOVALUE:
            out = None
        rule = _check_casting(casting)
        if order not in ("K", "A", "C", "F", None):
            raise ValueError(f"order must be one of 'C', 'F', 'A', or 'K' (got '{order}')")
        ops = _operands(args)
        orig = list(ops)
        L = lib()
        # dtype= : precast the operands into the requested loop dtype
        if dtype is not None:
            dt = np.dtype(dtype)
            if self.nin == 2 and self._op in (6, 7, 8, 9, 10, 11, 12, 13, 14):
                if dt != np.bool_:
                    raise UFuncTypeError(f"No loop matching the specified signature and casting was found for ufunc {self.__name__}")
            else:
                cast = []
                for i, o in enumerate(ops):
                    if not _can_cast(o.dtype, dt, rule):
                        raise UFuncTypeError(f"Cannot cast ufunc '{self.__name__}' input {i} from {o.dtype!r} to {dt!r} with casting rule '{casting}'")
                    cast.append(o if o.dtype == dt else o._cast_to(dt))
                ops = cast
        elif rule <= 1:
            # casting='no'/'equiv' without dtype=: the loop dtype must equal the inputs
            rd = self._result_dtype([o.dtype for o in ops])
            loop = rd if self._op not in range(6, 15) else None
            if loop is not None and any(o.dtype != loop for o in ops):
                raise UFuncTypeError(f"Cannot cast ufunc '{self.__name__}' input from {ops[0].dtype!r} to {loop!r} with casting rule '{casting}'")
        rd = self._result_dtype([o.dtype for o in ops])
        shape = _broadcast([o.shape for o in ops]) if self.nin == 2 else ops[0].shape
        fpe = ctypes.c_uint32(0)
        want_fpe = self._fpe is not None
        if out is not None:
            if not isinstance(out, ndarray):
                raise TypeError("return arrays must be of ArrayType")
            _broadcast([o.shape for o in orig] + [out.shape])
            if tuple(_broadcast([shape, out.shape])) != out.shape:
                raise ValueError(f"non-broadcastable output operand with shape {out.shape} doesn't match the broadcast shape {shape}")
            if not _can_cast(rd, out.dtype, rule):
                raise UFuncTypeError(f"Cannot cast ufunc '{self.__name__}' output from {rd!r} to {out.dtype!r} with casting rule '{casting}'")
            mask = None
            if not (where is True):
                mask = asarray(where)
                if mask.dtype != np.bool_:
                    raise TypeError("where= mask must be boolean")
            res = out
        else:
            mask = None
            if order in ("K", None):
                descs = (ctypes.POINTER(IonpArr) * len(orig))(*[ctypes.pointer(o._desc()) for o in orig])
                nd = len(shape)
                sh = (ctypes.c_int64 * max(nd, 1))(*shape)
                st = (ctypes.c_int64 * max(nd, 1))()
                check(L.ionp_order_k_strides(len(orig), descs, nd, sh, st))
                strides = list(st)[:nd]
            elif order == "F" or (order == "A" and all(o.flags["F_CONTIGUOUS"] for o in orig)):
                strides, acc = [], 1
                for s in shape:
                    strides.append(acc)
                    acc *= max(s, 1)
            else:
                strides = None
            res = ndarray.empty(shape, rd, strides)
        wd = mask._desc() if mask is not None else None
        if self.nin == 2:
            st = L.ionp_binary(self._op, ctypes.byref(ops[0]._desc()), ctypes.byref(ops[1]._desc()), ctypes.byref(res._desc()),
                               ctypes.byref(wd) if wd is not None else None,
                               ctypes.byref(fpe) if want_fpe else None, None)
        else:
            st = L.ionp_unary(self._op, ctypes.byref(ops[0]._desc()), ctypes.byref(res._desc()),
                              ctypes.byref(wd) if wd is not None else None,
                              ctypes.byref(fpe) if want_fpe else None, None)
        check(st)
        if want_fpe and fpe.value:
            cat = _fpstate.category_of(self._fpe, fpe.value)
            if cat:
                _fpstate.signal(cat, self.__name__, stacklevel=3)
        if out is not None:
            return out
        if res.ndim == 0:
            return _scalar_result(res)
        return res

    # ---- reduce ------------------------------------------------------------
    def reduce(self, array, axis=0, dtype=None, out=None, keepdims=False, initial=_NOVALUE, where=True):
        res = self._reduce_nd(array, axis, dtype, out, keepdims, initial, where)
        if out is not None:
            return res
        if res.ndim == 0:
            return _scalar_result(res)
        return res

    def _reduce_nd(self, array, axis=0, dtype=None, out=None, keepdims=False, initial=_NOVALUE, where=True):
        """ufunc.reduce returning the device array (0-d included)."""
        if self.nin != 2:
            raise ValueError("reduce only supported for binary functions")
        a = array if isinstance(array, ndarray) else asarray(array)
        nd = a.ndim
        axes = _normalize_axes(axis, nd)
        L = lib()
        if dtype is not None:
            cd = np.dtype(dtype)
        else:
            r = ctypes.c_int32()
            check(L.ionp_reduce_compute_dtype(self._op, code_of(a.dtype), ctypes.byref(r)))
            cd = _dt(r.value)
        init_buf = None
        if initial is not _NOVALUE and initial is not None:
            iv = np.asarray(initial)
            if iv.dtype not in (np.dtype(t) for t in DTYPES):
                iv = iv.astype(np.float64)
            src = np.ascontiguousarray(iv.reshape(()))
            init_buf = np.zeros(1, np.uint64)
            check(L.ionp_cast_scalar(src.ctypes.data, code_of(src.dtype), init_buf.ctypes.data, code_of(cd)))
        mask = None
        if where is not True:
            mask = asarray(where)
        ax = (ctypes.c_int32 * max(len(axes), 1))(*axes)
        ond = ctypes.c_int32()
        osh = (ctypes.c_int64 * 32)()
        ost = (ctypes.c_int64 * 32)()
        check(L.ionp_reduce_layout(ctypes.byref(a._desc()), ax, len(axes), int(bool(keepdims)), ctypes.byref(ond), osh, ost))
        rshape = tuple(osh[i] for i in range(ond.value))
        if out is not None:
            if isinstance(out, tuple):
                out = out[0]
            if not isinstance(out, ndarray):
                raise TypeError("return arrays must be of ArrayType")
            if out.shape != rshape:
                raise ValueError(f"output parameter for reduction operation {self.__name__} has the wrong number of dimensions"
                                 if len(out.shape) != len(rshape) else
                                 f"output parameter for reduction operation {self.__name__} has a non-reduction dimension not equal to the input one.")
            if not _can_cast(cd, out.dtype, CAST_RULES["same_kind"]):
                raise UFuncTypeError(f"Cannot cast ufunc '{self.__name__}' output from {cd!r} to {out.dtype!r} with casting rule 'same_kind'")
            res = out
        else:
            res = ndarray.empty(rshape, cd, [ost[i] for i in range(ond.value)])
        md = mask._desc() if mask is not None else None
        check(L.ionp_reduce(self._op, ctypes.byref(a._desc()), ax, len(axes), int(bool(keepdims)),
                            code_of(cd) if dtype is not None else -1,
                            init_buf.ctypes.data if init_buf is not None else None,
                            ctypes.byref(md) if md is not None else None, ctypes.byref(res._desc()), None))
        return res


    # ---- accumulate / reduceat / outer ------------------------------------
    def _method_axis(self, a, axis, name):
        """normalize_ufunc_method_axis (ionp-py/src/lib.rs:121)."""
        nd = a.ndim
        eff = max(nd, 1)
        axis = operator.index(axis)
        norm = axis + eff if axis < 0 else axis
        if norm < 0 or norm >= eff:
            raise AxisError(f"axis {axis} is out of bounds for array of dimension {nd}")
        if nd == 0:
            raise TypeError(f"cannot {name} on a scalar")
        return norm

    def _write_out(self, res, out):
        """write_into_out_ufunc with casting='same_kind'."""
        if isinstance(out, tuple):
            out = out[0]
        if not isinstance(out, ndarray):
            raise TypeError("return arrays must be of ArrayType")
        if out.shape != res.shape:
            raise ValueError(f"non-broadcastable output operand with shape {out.shape} doesn't match the broadcast shape {res.shape}")
        if not _can_cast(res.dtype, out.dtype, CAST_RULES["same_kind"]):
            raise UFuncTypeError(f"Cannot cast ufunc '{self.__name__}' output from {res.dtype!r} to {out.dtype!r} with casting rule 'same_kind'")
        if res.size:
            check(lib().ionp_cast(ctypes.byref(res._desc()), ctypes.byref(out._desc()), None))
        return out

    def accumulate(self, array, axis=0, dtype=None, out=None):
        """accumulate_axis (ionp-core/src/ufunc.rs:7967): every fiber along
        `axis` folded in order; the result has the input's shape, its
        order='K' layout and the reduce-family compute dtype. `dtype=` is
        accepted and, like the reference, ignored."""
        if self.nin != 2:
            raise ValueError("accumulate only supported for binary functions")
        a = array if isinstance(array, ndarray) else asarray(array)
        ax = self._method_axis(a, axis, "accumulate")
        L = lib()
        r = ctypes.c_int32()
        check(L.ionp_reduce_compute_dtype(self._op, code_of(a.dtype), ctypes.byref(r)))
        cd = _dt(r.value)
        descs = (ctypes.POINTER(IonpArr) * 1)(ctypes.pointer(a._desc()))
        nd = a.ndim
        sh = (ctypes.c_int64 * max(nd, 1))(*a.shape)
        st = (ctypes.c_int64 * max(nd, 1))()
        check(L.ionp_order_k_strides(1, descs, nd, sh, st))
        res = ndarray.empty(a.shape, cd, list(st)[:nd])
        if res.size:
            check(L.ionp_accumulate(self._op, ctypes.byref(a._desc()), ax, ctypes.byref(res._desc()), None))
        if out is not None:
            return self._write_out(res, out)
        return res

    def reduceat(self, array, indices, axis=0, dtype=None, out=None):
        """reduceat_binary_axis (ionp-core/src/ufunc.rs:8450): segment k of
        every fiber along `axis` runs from indices[k] to indices[k+1] (the
        axis end for the last) and is folded in order, or is the single
        element indices[k] when the next index is not larger. C-ordered
        result in the reduce-family compute dtype; `dtype=` is ignored, as
        in the reference."""
        if self.nin != 2:
            raise ValueError("reduceat only supported for binary functions")
        a = array if isinstance(array, ndarray) else asarray(array)
        ax = self._method_axis(a, axis, "reduceat")
        idx = np.asarray(indices)
        if idx.dtype.kind not in "iu" and idx.size:
            raise TypeError("Cannot cast array data from dtype('float64') to dtype('int64') according to the rule 'safe'")
        idx = np.ascontiguousarray(idx.reshape(-1).astype(np.int64))
        L = lib()
        r = ctypes.c_int32()
        check(L.ionp_reduce_compute_dtype(self._op, code_of(a.dtype), ctypes.byref(r)))
        cd = _dt(r.value)
        shape = list(a.shape)
        shape[ax] = idx.size
        res = ndarray.empty(tuple(shape), cd)
        check(L.ionp_reduceat(self._op, ctypes.byref(a._desc()), ax,
                              idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), idx.size,
                              ctypes.byref(res._desc()), None))
        if out is not None:
            return self._write_out(res, out)
        return res

    def outer(self, A, B):
        """outer_binary (ionp-core/src/ufunc.rs:8212): op(A[i...], B[j...])
        over the full cross product, shape A.shape + B.shape, C order: the
        binary kernels on A viewed as A.shape + (1,) * B.ndim against B. Like
        the reference (ionp-py/src/lib.rs:10091), no FPE report."""
        if self.nin != 2:
            raise ValueError("outer product only supported for binary functions")
        a = A if isinstance(A, ndarray) else asarray(A)
        b = B if isinstance(B, ndarray) else asarray(B)
        av = ndarray(a._buf, tuple(a.shape) + (1,) * b.ndim, a.dtype, list(a.elem_strides) + [0] * b.ndim, a._off)
        shape = tuple(a.shape) + tuple(b.shape)
        rd = self._result_dtype([a.dtype, b.dtype])
        res = ndarray.empty(shape, rd)
        if res.size:
            check(lib().ionp_binary(self._op, ctypes.byref(av._desc()), ctypes.byref(b._desc()), ctypes.byref(res._desc()),
                                    None, None, None))
        return res


    def at(self, array, indices, b=None):
        """ufunc.at (ionp-py/src/lib.rs:10160): in place on `array`,
        array[indices[i], ...] = op(array[indices[i], ...], b[i, ...]) for i
        in order (repeated indices apply again), b broadcast against
        (len(indices),) + array.shape[1:]; unary ufuncs apply op once per
        occurrence. Computed in the array's dtype (promoting ufuncs: on a
        whole-array copy in the promoted dtype, cast back); no FPE report."""
        if not isinstance(array, ndarray):
            raise TypeError("first operand must be array")
        idx = _at_indices(indices)
        if self.nin == 1:
            if b is not None:
                raise TypeError("unary ufunc .at() takes no third argument")
            values = None
        else:
            if b is None:
                raise TypeError("binary ufunc .at() requires a values argument")
            values = b if isinstance(b, ndarray) else asarray(b)
        iv = np.ascontiguousarray(np.asarray(idx, dtype=np.int64).reshape(-1))
        check(lib().ionp_at(self._op, ctypes.byref(array._desc()), iv.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                            iv.size, None if values is None else ctypes.byref(values._desc()), None))
        return None


def _at_indices(obj):
    """extract_index_vec (ionp-py/src/lib.rs:8374): an int, or a sequence
    of ints (an integer array included)."""
    if isinstance(obj, ndarray):
        obj = obj.get()
    try:
        return [operator.index(obj)]
    except TypeError:
        pass
    if not isinstance(obj, (str, bytes)):
        try:
            return [operator.index(x) for x in obj]
        except TypeError:
            pass
    raise TypeError("indices must be an int, a sequence of ints, or an integer numpy array")


def _normalize_axes(axis, ndim):
    """normalize_reduce_axes (ionp-core/src/ufunc.rs:7551-7632)."""
    if axis is None:
        return list(range(ndim))
    raw = list(axis) if isinstance(axis, (tuple, list)) else [axis]
    out = []
    for a in raw:
        a = operator.index(a)
        norm = a + max(ndim, 1) if a < 0 else a
        if ndim == 0:
            if norm != 0:
                raise AxisError(f"axis {a} is out of bounds for array of dimension {ndim}")
        elif norm < 0 or norm >= ndim:
            raise AxisError(f"axis {a} is out of bounds for array of dimension {ndim}")
        out.append(max(norm, 0))
    if len(set(out)) != len(out):
        raise ValueError("duplicate value in 'axis'")
    return [] if ndim == 0 else sorted(out)


def _argext(is_max, a, axis=None, out=None, keepdims=False):
    """do_argext (ionp-py/src/reductions.rs:1198-1300)."""
    a = a if isinstance(a, ndarray) else asarray(a)
    nd = a.ndim
    keepdims = bool(keepdims)
    if axis is None:
        ax = -1
        shape = (1,) * nd if (keepdims and nd != 1) else ((1,) if keepdims else ())
    else:
        raw = operator.index(axis)
        ax = raw + max(nd, 1) if raw < 0 else raw
        if ax < 0 or ax >= max(nd, 1):
            raise AxisError(f"axis {raw} is out of bounds for array of dimension {max(nd, 1)}")
        shape = tuple((1 if i == ax else a.shape[i]) for i in range(nd) if keepdims or i != ax)
    res = ndarray.empty(shape, np.int64)
    check(lib().ionp_argext(int(is_max), ctypes.byref(a._desc()), ax if nd > 0 else 0, int(keepdims), ctypes.byref(res._desc()), None))
    if out is not None:
        if not isinstance(out, ndarray):
            raise TypeError("return arrays must be of ArrayType")
        check(lib().ionp_cast(ctypes.byref(res._desc()), ctypes.byref(out._desc()), None))
        return out
    if res.ndim == 0:
        return _scalar_result(res)
    return res


def argmax(a, axis=None, out=None, keepdims=False):
    return _argext(True, a, axis, out, keepdims)


def argmin(a, axis=None, out=None, keepdims=False):
    return _argext(False, a, axis, out, keepdims)


# ---- the ufunc objects (module registration, lib.rs:10266-10431) ----------
for _n, _c in BINARY_OPS.items():
    globals()[_n] = ufunc(_n, 2, _c)
for _n, _c in UNARY_OPS.items():
    globals()[_n] = ufunc(_n, 1, _c)
true_divide = globals()["divide"]
mod = globals()["remainder"]
abs = globals()["absolute"]
bitwise_not = globals()["invert"]
