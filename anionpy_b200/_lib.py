"""ctypes binding of libionp_cuda.so (the C ABI in include/ionp_cuda.h).

The shared library is built in-tree by anionpy_b200/_build.py. There is no
fallback: if the library or a CUDA device is missing, using the engine raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libionp_cuda.so")
MAX_DIMS = 32

# dtype codes (ionp-core/src/dtype.rs:14 order)
NP_DTYPES = [np.bool_, np.int8, np.int16, np.int32, np.int64, np.uint8, np.uint16,
             np.uint32, np.uint64, np.float16, np.float32, np.float64]
CODE = {np.dtype(t): i for i, t in enumerate(NP_DTYPES)}
DTYPES = [np.dtype(t) for t in NP_DTYPES]

CAST_RULES = {"no": 0, "equiv": 1, "safe": 2, "same_kind": 3, "unsafe": 4}

# status codes
OK, ERR_BROADCAST, ERR_TYPE, ERR_VALUE, ERR_NO_LOOP, ERR_AXIS, ERR_CUDA, ERR_TIMEOUT, ERR_OOM, \
    ERR_UNSUPPORTED, ERR_INVALID, ERR_INDEX = range(12)

FPE_DIVIDE, FPE_OVER, FPE_UNDER, FPE_INVALID = 1, 2, 4, 8


class IonpArr(ctypes.Structure):
    _fields_ = [("dtype", ctypes.c_int32), ("ndim", ctypes.c_int32),
                ("shape", ctypes.c_int64 * MAX_DIMS), ("strides", ctypes.c_int64 * MAX_DIMS),
                ("offset", ctypes.c_int64), ("data", ctypes.c_void_p)]


class UFuncTypeError(TypeError):
    """numpy's ufunc type error (a TypeError subclass)."""


class AxisError(ValueError, IndexError):
    """numpy's AxisError (both a ValueError and an IndexError)."""


class IonpSchedule(ctypes.Structure):
    _fields_ = [("block_tile", ctypes.c_int32), ("vec_width", ctypes.c_int32),
                ("elems_per_thread", ctypes.c_int32), ("red_split", ctypes.c_int32)]


NUM_SCHEDULES = 48

_P = ctypes.POINTER(IonpArr)
_S = ctypes.POINTER(IonpSchedule)
_SIGS = {
    "ionp_promote": [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)],
    "ionp_binary_out_dtype": [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)],
    "ionp_unary_out_dtype": [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)],
    "ionp_reduce_compute_dtype": [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)],
    "ionp_can_cast": [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)],
    "ionp_cast_scalar": [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32],
    "ionp_order_k_strides": [ctypes.c_int32, ctypes.POINTER(_P), ctypes.c_int32, ctypes.POINTER(ctypes.c_int64),
                             ctypes.POINTER(ctypes.c_int64)],
    "ionp_reduce_layout": [_P, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32, ctypes.c_int32,
                           ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)],
    "ionp_binary": [ctypes.c_int32, _P, _P, _P, _P, ctypes.POINTER(ctypes.c_uint32), ctypes.c_void_p],
    "ionp_unary": [ctypes.c_int32, _P, _P, _P, ctypes.POINTER(ctypes.c_uint32), ctypes.c_void_p],
    "ionp_binary_nowait": [ctypes.c_int32, _P, _P, _P, _P, ctypes.c_void_p, ctypes.c_void_p],
    "ionp_unary_nowait": [ctypes.c_int32, _P, _P, _P, ctypes.c_void_p, ctypes.c_void_p],
    "ionp_cast": [_P, _P, ctypes.c_void_p],
    "ionp_astype": [_P, _P, ctypes.POINTER(ctypes.c_uint32), ctypes.c_void_p],
    "ionp_reduce": [ctypes.c_int32, _P, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                    ctypes.c_void_p, _P, _P, ctypes.c_void_p],
    "ionp_accumulate": [ctypes.c_int32, _P, ctypes.c_int32, _P, ctypes.c_void_p],
    "ionp_reduceat": [ctypes.c_int32, _P, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64), ctypes.c_int64, _P,
                      ctypes.c_void_p],
    "ionp_at": [ctypes.c_int32, _P, ctypes.POINTER(ctypes.c_int64), ctypes.c_int64, _P, ctypes.c_void_p],
    "ionp_argext": [ctypes.c_int32, _P, ctypes.c_int32, ctypes.c_int32, _P, ctypes.c_void_p],
    "ionp_alloc": [ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t, ctypes.c_void_p],
    "ionp_free": [ctypes.c_void_p, ctypes.c_void_p],
    "ionp_alloc_stats": [ctypes.POINTER(ctypes.c_uint64)],
    "ionp_alloc_trim": [],
    "ionp_last_error_message": [ctypes.c_char_p, ctypes.c_size_t],
    "ionp_memcpy": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int32, ctypes.c_void_p],
    "ionp_stream_create": [ctypes.POINTER(ctypes.c_void_p)],
    "ionp_stream_destroy": [ctypes.c_void_p],
    "ionp_stream_synchronize": [ctypes.c_void_p],
    "ionp_device_synchronize": [],
    "ionp_host_alloc": [ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t],
    "ionp_host_free": [ctypes.c_void_p],
    "ionp_event_create": [ctypes.POINTER(ctypes.c_void_p)],
    "ionp_event_destroy": [ctypes.c_void_p],
    "ionp_event_record": [ctypes.c_void_p, ctypes.c_void_p],
    "ionp_event_elapsed_ms": [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)],
    "ionp_set_device": [ctypes.c_int32],
    "ionp_reduce_noalloc": [ctypes.c_int32, _P, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32, ctypes.c_int32,
                            ctypes.c_void_p, _P, ctypes.c_void_p],
    "ionp_schedule_from_index": [ctypes.c_int32, _S],
    "ionp_batch_create": [ctypes.POINTER(ctypes.c_void_p)],
    "ionp_batch_destroy": [ctypes.c_void_p],
    "ionp_batch_add_binary": [ctypes.c_void_p, ctypes.c_int32, _P, _P, _P, _S, ctypes.POINTER(ctypes.c_int32)],
    "ionp_batch_add_reduce": [ctypes.c_void_p, ctypes.c_int32, _P, ctypes.c_int32, ctypes.c_int32, _P, _S,
                              ctypes.POINTER(ctypes.c_int32)],
    "ionp_batch_set_schedule": [ctypes.c_void_p, ctypes.c_int32, _S],
    "ionp_batch_finalize": [ctypes.c_void_p, ctypes.c_void_p],
    "ionp_batch_run": [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p],
    "ionp_batch_run_per_call": [ctypes.c_void_p, ctypes.c_void_p],
    "ionp_batch_fpe": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32), ctypes.c_void_p],
    "ionp_batch_info": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)],
    "ionp_batch_features": [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_float)],
    "ionp_mlp_create": [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_uint64],
    "ionp_mlp_destroy": [ctypes.c_void_p],
    "ionp_mlp_num_params": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)],
    "ionp_mlp_get": [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int64],
    "ionp_mlp_set_params": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64],
    "ionp_mlp_forward": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p],
    "ionp_mlp_gradients": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                           ctypes.POINTER(ctypes.c_float), ctypes.c_void_p],
    "ionp_mlp_train_step": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                            ctypes.c_float, ctypes.c_float, ctypes.POINTER(ctypes.c_float), ctypes.c_void_p],
    "ionp_batch_time_call": [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, _S, ctypes.c_int32,
                             ctypes.POINTER(ctypes.c_float), ctypes.c_void_p],
    "ionp_device_info": [ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32), ctypes.c_char_p, ctypes.c_size_t],
}

_lib = None
_lock = threading.Lock()


def load_library():
    """Load the in-tree shared library (raises if it was never built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with anionpy_b200._build.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int32
        L.ionp_launch_count.argtypes = []
        L.ionp_launch_count.restype = ctypes.c_uint64
        _lib = L
    return _lib


_device_checked = False


def lib():
    """The library, after checking once that a CUDA device is present."""
    global _device_checked
    L = load_library()
    if not _device_checked:
        n = ctypes.c_int32(0)
        L.ionp_device_info(ctypes.byref(n), None, None, 0)
        if n.value < 1:
            raise RuntimeError("anionpy_b200 needs a CUDA device; none is visible (there is no CPU fallback)")
        _device_checked = True
    return L


def last_error() -> str:
    buf = ctypes.create_string_buffer(2048)
    load_library().ionp_last_error_message(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int):
    """Raise the Python exception the reference raises for an IonpError."""
    if status == OK:
        return
    msg = last_error()
    if status in (ERR_BROADCAST, ERR_VALUE, ERR_INVALID):
        raise ValueError(msg)
    if status == ERR_TYPE:
        raise TypeError(msg)
    if status == ERR_NO_LOOP:
        raise UFuncTypeError(msg)
    if status == ERR_AXIS:
        raise AxisError(msg)
    if status == ERR_OOM:
        raise MemoryError(msg)
    if status == ERR_TIMEOUT:
        raise TimeoutError(msg)
    if status == ERR_UNSUPPORTED:
        raise TypeError(msg)
    if status == ERR_INDEX:
        raise IndexError(msg)
    raise RuntimeError(f"CUDA failure: {msg}")


def code_of(dtype) -> int:
    dt = np.dtype(dtype)
    if dt not in CODE:
        raise TypeError(f"dtype {dt} is not supported by the B200 ufunc engine")
    return CODE[dt]


def launch_count() -> int:
    return int(load_library().ionp_launch_count())
