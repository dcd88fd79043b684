"""anionpy_b200 -- anionpy's ufunc-engine hot path on NVIDIA B200.

Drop-in for the element-wise ufunc ``__call__`` (unary and binary, with
broadcasting and arbitrary strides), ``ufunc.reduce``, ``argmin``/``argmax``
and the reductions built on them (``sum``, ``prod``, ``min``, ``max``,
``any``, ``all``, ``mean``, also as array methods) of anionpy, computed by hand-written sm_100a CUDA kernels behind the
C ABI of ``libionp_cuda.so`` (include/ionp_cuda.h). Results are bit-exact with
anionpy's CPU path; errors and ``errstate`` behave the same way.
"""
from ._array import array, asarray, empty, from_numpy, ndarray, ones, zeros
from ._batch import Batch
from ._fpstate import errstate, geterr, geterrcall, seterr, seterrcall
from ._lib import AxisError, UFuncTypeError, launch_count
from ._ufunc import (BINARY_OPS, UNARY_OPS, absolute, add, argmax, argmin, bitwise_and, bitwise_not, bitwise_or,
                     bitwise_xor, cos, divide, equal, exp, floor_divide, fmod, greater, greater_equal, invert, left_shift,
                     less, less_equal, log, logical_and, logical_not, logical_or, logical_xor, maximum, minimum, mod,
                     multiply, negative, not_equal, remainder, right_shift, sin, sqrt, subtract, true_divide, ufunc)
from ._ufunc import abs  # noqa: A001
from ._reductions import all, amax, amin, any, cumprod, cumsum, max, mean, min, prod, sum  # noqa: A004

__all__ = [
    "ndarray", "array", "asarray", "empty", "zeros", "ones", "from_numpy",
    "errstate", "seterr", "geterr", "seterrcall", "geterrcall", "AxisError", "UFuncTypeError",
    "ufunc", "argmax", "argmin", "launch_count", "Batch",
    "sum", "prod", "min", "max", "amin", "amax", "any", "all", "mean", "cumsum", "cumprod",
] + list(BINARY_OPS) + list(UNARY_OPS) + ["true_divide", "mod", "abs", "bitwise_not"]
