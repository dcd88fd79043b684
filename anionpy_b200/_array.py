"""Device-resident ndarray: the B200 counterpart of NdArray
(ionp-core/src/array.rs:24 -- an `Arc<Buffer>` + shape + element strides +
offset). Storage comes from the engine's caching device allocator
(ionp_alloc), and views share their buffer exactly as NdArray views share
their `Arc<Buffer>`.
"""
from __future__ import annotations

import ctypes
import operator

import numpy as np

from . import _lib
from ._lib import IonpArr, check, code_of, lib


class DeviceBuffer:
    """One device allocation (freed back to the caching allocator)."""
    __slots__ = ("ptr", "nbytes", "__weakref__")

    def __init__(self, nbytes: int):
        p = ctypes.c_void_p()
        check(lib().ionp_alloc(ctypes.byref(p), max(int(nbytes), 1), None))
        self.ptr = p.value
        self.nbytes = int(nbytes)

    def __del__(self):
        try:
            if self.ptr:
                _lib.load_library().ionp_free(self.ptr, None)
        except Exception:
            pass
        self.ptr = None


def c_strides(shape):
    st, acc = [0] * len(shape), 1
    for i in range(len(shape) - 1, -1, -1):
        st[i] = acc
        acc *= max(int(shape[i]), 1)
    return st


class ndarray:
    """An N-d array in HBM with element strides, like the reference's NdArray."""
    __array_priority__ = 1000

    def __init__(self, buf: DeviceBuffer, shape, dtype, strides=None, offset: int = 0):
        self._buf = buf
        self._shape = tuple(int(s) for s in shape)
        self._dtype = np.dtype(dtype)
        self._st = tuple(int(s) for s in (strides if strides is not None else c_strides(self._shape)))
        self._off = int(offset)

    # ---- construction ----------------------------------------------------
    @classmethod
    def empty(cls, shape, dtype, strides=None):
        shape = tuple(int(s) for s in shape)
        dt = np.dtype(dtype)
        code_of(dt)
        n = int(np.prod(shape)) if shape else 1
        if strides is None:
            strides = c_strides(shape)
        # span of the layout (strides may be any permutation of C strides)
        span = 1
        for s, st in zip(shape, strides):
            if s == 0:
                span = 0
                break
            span += (s - 1) * abs(st)
        nbytes = max(span, n, 1) * dt.itemsize
        return cls(DeviceBuffer(nbytes), shape, dt, strides, 0)

    # ---- metadata -------------------------------------------------------
    @property
    def shape(self):
        return self._shape

    @property
    def dtype(self):
        return self._dtype

    @property
    def ndim(self):
        return len(self._shape)

    @property
    def size(self):
        return int(np.prod(self._shape)) if self._shape else 1

    @property
    def itemsize(self):
        return self._dtype.itemsize

    @property
    def nbytes(self):
        return self.size * self.itemsize

    @property
    def strides(self):
        """numpy-style byte strides."""
        return tuple(s * self.itemsize for s in self._st)

    @property
    def elem_strides(self):
        return self._st

    @property
    def offset(self):
        return self._off

    @property
    def data_ptr(self):
        return self._buf.ptr + self._off * self.itemsize

    def _contig(self, fortran: bool):
        if self.size == 0:
            return True
        expect = 1
        order = range(self.ndim) if fortran else range(self.ndim - 1, -1, -1)
        for i in order:
            if self._shape[i] == 1:
                continue
            if self._st[i] != expect:
                return False
            expect *= self._shape[i]
        return True

    @property
    def flags(self):
        return {"C_CONTIGUOUS": self._contig(False), "F_CONTIGUOUS": self._contig(True)}

    def _desc(self) -> IonpArr:
        d = IonpArr()
        d.dtype = code_of(self._dtype)
        d.ndim = self.ndim
        for i in range(self.ndim):
            d.shape[i] = self._shape[i]
            d.strides[i] = self._st[i]
        d.offset = self._off
        d.data = self._buf.ptr
        return d

    # ---- host transfer ---------------------------------------------------
    def get(self) -> np.ndarray:
        """Copy to a host numpy array (C order)."""
        src = self if self.flags["C_CONTIGUOUS"] else self.copy()
        out = np.empty(self._shape, self._dtype)
        if out.nbytes:
            L = lib()
            check(L.ionp_memcpy(out.ctypes.data, src.data_ptr, out.nbytes, 1, None))
            check(L.ionp_stream_synchronize(None))
        return out

    def __array__(self, dtype=None, copy=None):
        a = self.get()
        return a.astype(dtype) if dtype is not None else a

    def item(self):
        return self.get().item()

    def __repr__(self):
        return f"anionpy_b200.ndarray({self.get()!r}, device='cuda')"

    def __len__(self):
        if not self._shape:
            raise TypeError("len() of unsized object")
        return self._shape[0]

    def __bool__(self):
        if self.size != 1:
            raise ValueError("The truth value of an array with more than one element is ambiguous. Use a.any() or a.all()")
        return bool(self.get().reshape(()))

    def __float__(self):
        return float(self.get().reshape(()))

    def __int__(self):
        return int(self.get().reshape(()))

    # ---- views -----------------------------------------------------------
    def transpose(self, *axes):
        if not axes:
            axes = tuple(range(self.ndim))[::-1]
        elif len(axes) == 1 and isinstance(axes[0], (tuple, list)):
            axes = tuple(axes[0])
        axes = [a + self.ndim if a < 0 else a for a in axes]
        if sorted(axes) != list(range(self.ndim)):
            raise ValueError("axes don't match array")
        return ndarray(self._buf, [self._shape[a] for a in axes], self._dtype, [self._st[a] for a in axes], self._off)

    @property
    def T(self):
        return self.transpose()

    def __getitem__(self, key):
        if not isinstance(key, tuple):
            key = (key,)
        if any(k is Ellipsis for k in key):
            i = key.index(Ellipsis)
            fill = self.ndim - (len(key) - 1 - sum(1 for k in key if k is None))
            key = key[:i] + (slice(None),) * fill + key[i + 1:]
        shape, st, off, ax = [], [], self._off, 0
        for k in key:
            if k is None:
                shape.append(1)
                st.append(0)
                continue
            if ax >= self.ndim:
                raise IndexError("too many indices for array")
            n, s = self._shape[ax], self._st[ax]
            if isinstance(k, slice):
                start, stop, step = k.indices(n)
                cnt = len(range(start, stop, step))
                shape.append(cnt)
                st.append(s * step)
                off += start * s
            else:
                i = operator.index(k)
                if i < 0:
                    i += n
                if not 0 <= i < n:
                    raise IndexError(f"index {k} is out of bounds for axis {ax} with size {n}")
                off += i * s
            ax += 1
        for a in range(ax, self.ndim):
            shape.append(self._shape[a])
            st.append(self._st[a])
        return ndarray(self._buf, shape, self._dtype, st, off)

    def reshape(self, *shape):
        if len(shape) == 1 and isinstance(shape[0], (tuple, list)):
            shape = tuple(shape[0])
        shape = list(shape)
        if -1 in shape:
            known = int(np.prod([s for s in shape if s != -1])) or 1
            shape[shape.index(-1)] = self.size // known
        if int(np.prod(shape)) != self.size:
            raise ValueError(f"cannot reshape array of size {self.size} into shape {tuple(shape)}")
        src = self if self.flags["C_CONTIGUOUS"] else self.copy()
        return ndarray(src._buf, shape, self._dtype, c_strides(shape), src._off)

    def ravel(self):
        return self.reshape(-1)

    def copy(self, order="C"):
        out = ndarray.empty(self._shape, self._dtype)
        if self.size:
            check(lib().ionp_cast(ctypes.byref(self._desc()), ctypes.byref(out._desc()), None))
        return out

    def astype(self, dtype, order="K", casting="unsafe", subok=True, copy=True):
        """ndarray.astype (ionp-py/src/lib.rs:5960-6003): the casting= rule
        check, detect_cast_overflow (a float source cast to an integer
        dtype: NaN, infinity or out-of-range values report "invalid value
        encountered in cast" through errstate), then the cast."""
        from . import _fpstate
        from ._lib import CAST_RULES
        from ._ufunc import _can_cast
        dt = np.dtype(dtype)
        if casting not in CAST_RULES:
            raise ValueError("casting must be one of 'no', 'equiv', 'safe', 'same_kind', or 'unsafe'")
        if not _can_cast(self._dtype, dt, CAST_RULES[casting]):
            raise TypeError(f"Cannot cast array data from {self._dtype!r} to {dt!r} according to the rule '{casting}'")
        if dt == self._dtype and not copy:
            return self
        out = ndarray.empty(self._shape, dt)
        fpe = ctypes.c_uint32(0)
        check(lib().ionp_astype(ctypes.byref(self._desc()), ctypes.byref(out._desc()), ctypes.byref(fpe), None))
        if fpe.value & 8:
            _fpstate.signal("invalid", "cast", stacklevel=3)
        return out

    def _cast_to(self, dtype):
        """Buffer::cast_to (ionp-core/src/buffer.rs:210): a C-ordered copy in
        dtype, with no FPE check (the reference's internal casts)."""
        dt = np.dtype(dtype)
        out = ndarray.empty(self._shape, dt)
        if self.size:
            check(lib().ionp_cast(ctypes.byref(self._desc()), ctypes.byref(out._desc()), None))
        return out

    # ---- reductions (ndarray_attrs.rs:675-760: the same functions as
    # anionpy.sum etc., reached as methods) --------------------------------
    def sum(self, axis=None, dtype=None, out=None, keepdims=None, initial=None, where=None):
        from . import _reductions
        return _reductions.sum(self, axis, dtype, out, keepdims, initial, where)

    def prod(self, axis=None, dtype=None, out=None, keepdims=None, initial=None, where=None):
        from . import _reductions
        return _reductions.prod(self, axis, dtype, out, keepdims, initial, where)

    def min(self, axis=None, out=None, keepdims=None, initial=None, where=None):
        from . import _reductions
        return _reductions.min(self, axis, out, keepdims, initial, where)

    def max(self, axis=None, out=None, keepdims=None, initial=None, where=None):
        from . import _reductions
        return _reductions.max(self, axis, out, keepdims, initial, where)

    def all(self, axis=None, out=None, keepdims=None, where=None):
        from . import _reductions
        return _reductions.all(self, axis, out, keepdims, where)

    def any(self, axis=None, out=None, keepdims=None, where=None):
        from . import _reductions
        return _reductions.any(self, axis, out, keepdims, where)

    def mean(self, axis=None, dtype=None, out=None, keepdims=None, where=None):
        from . import _reductions
        return _reductions.mean(self, axis, dtype, out, keepdims, where)

    def cumsum(self, axis=None, dtype=None, out=None):
        from . import _reductions
        return _reductions.cumsum(self, axis, dtype, out)

    def cumprod(self, axis=None, dtype=None, out=None):
        from . import _reductions
        return _reductions.cumprod(self, axis, dtype, out)

    def argmax(self, axis=None, out=None, keepdims=False):
        from . import _ufunc
        return _ufunc.argmax(self, axis, out, keepdims)

    def argmin(self, axis=None, out=None, keepdims=False):
        from . import _ufunc
        return _ufunc.argmin(self, axis, out, keepdims)

    # ---- operators (thin wrappers over the ufuncs) -----------------------
    def _uf(name):
        def f(self, other):
            from . import _ufunc
            return getattr(_ufunc, name)(self, other)
        return f

    def _ruf(name):
        def f(self, other):
            from . import _ufunc
            return getattr(_ufunc, name)(other, self)
        return f

    __add__ = _uf("add")
    __radd__ = _ruf("add")
    __sub__ = _uf("subtract")
    __rsub__ = _ruf("subtract")
    __mul__ = _uf("multiply")
    __rmul__ = _ruf("multiply")
    __truediv__ = _uf("divide")
    __rtruediv__ = _ruf("divide")
    __floordiv__ = _uf("floor_divide")
    __rfloordiv__ = _ruf("floor_divide")
    __mod__ = _uf("remainder")
    __rmod__ = _ruf("remainder")
    __and__ = _uf("bitwise_and")
    __rand__ = _ruf("bitwise_and")
    __or__ = _uf("bitwise_or")
    __ror__ = _ruf("bitwise_or")
    __xor__ = _uf("bitwise_xor")
    __rxor__ = _ruf("bitwise_xor")
    __lshift__ = _uf("left_shift")
    __rshift__ = _uf("right_shift")
    __lt__ = _uf("less")
    __le__ = _uf("less_equal")
    __gt__ = _uf("greater")
    __ge__ = _uf("greater_equal")
    __eq__ = _uf("equal")
    __ne__ = _uf("not_equal")

    def __neg__(self):
        from . import _ufunc
        return _ufunc.negative(self)

    def __abs__(self):
        from . import _ufunc
        return _ufunc.absolute(self)

    def __invert__(self):
        from . import _ufunc
        return _ufunc.invert(self)

    __hash__ = None

    # reductions as methods (thin wrappers over ufunc.reduce / argext)
    def sum(self, axis=None, dtype=None, out=None, keepdims=False, initial=None, where=True):
        from . import _ufunc
        kw = {} if initial is None else {"initial": initial}
        return _ufunc.add.reduce(self, axis=axis, dtype=dtype, out=out, keepdims=keepdims, where=where, **kw)

    def max(self, axis=None, out=None, keepdims=False, initial=None, where=True):
        from . import _ufunc
        kw = {} if initial is None else {"initial": initial}
        return _ufunc.maximum.reduce(self, axis=axis, out=out, keepdims=keepdims, where=where, **kw)

    def min(self, axis=None, out=None, keepdims=False, initial=None, where=True):
        from . import _ufunc
        kw = {} if initial is None else {"initial": initial}
        return _ufunc.minimum.reduce(self, axis=axis, out=out, keepdims=keepdims, where=where, **kw)

    def argmax(self, axis=None, out=None, keepdims=False):
        from . import _ufunc
        return _ufunc.argmax(self, axis=axis, out=out, keepdims=keepdims)

    def argmin(self, axis=None, out=None, keepdims=False):
        from . import _ufunc
        return _ufunc.argmin(self, axis=axis, out=out, keepdims=keepdims)


def asarray(obj, dtype=None) -> ndarray:
    """Device array from a device array, numpy array or Python data."""
    if isinstance(obj, ndarray):
        return obj if dtype is None or np.dtype(dtype) == obj.dtype else obj.astype(dtype)
    host = np.asarray(obj, dtype=dtype)
    return from_numpy(host)


def from_numpy(host: np.ndarray, stream=None) -> ndarray:
    """Upload a host array, keeping its memory layout (strides) when it is a
    dense permutation of C order, else as a C-contiguous copy."""
    host = np.asarray(host)
    code_of(host.dtype)
    if host.flags["C_CONTIGUOUS"]:
        src, st = host, c_strides(host.shape)
    elif host.flags["F_CONTIGUOUS"] and host.size:
        src, st = host, [s // host.itemsize for s in host.strides]
    else:
        src = np.ascontiguousarray(host)
        st = c_strides(host.shape)
    out = ndarray.empty(host.shape, host.dtype, st)
    if src.nbytes:
        check(lib().ionp_memcpy(out.data_ptr, src.ctypes.data, src.nbytes, 0, stream))
        if stream is None:
            check(lib().ionp_stream_synchronize(None))
    return out


def array(obj, dtype=None) -> ndarray:
    return from_numpy(np.array(obj, dtype=dtype))


def empty(shape, dtype=np.float64) -> ndarray:
    if isinstance(shape, int):
        shape = (shape,)
    return ndarray.empty(shape, dtype)


def zeros(shape, dtype=np.float64) -> ndarray:
    return from_numpy(np.zeros(shape, dtype))


def ones(shape, dtype=np.float64) -> ndarray:
    return from_numpy(np.ones(shape, dtype))
