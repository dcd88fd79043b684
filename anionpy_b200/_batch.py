"""Batched execution of many small ufunc calls (``ionp_batch_*`` in the C ABI).

A :class:`Batch` collects binary ufunc calls (add, subtract, multiply,
maximum, less, logical_and) and add/maximum reductions over one axis, then
runs all of them as ONE persistent kernel draining a device-side queue of
call descriptors, captured once in a CUDA graph and replayed. Every call
computes exactly what the same call through ``ufunc.__call__`` /
``ufunc.reduce`` computes; a call's schedule (see :func:`schedule`) changes
only how its work is tiled.

The reference runs each call on its own (ionp-py/src/lib.rs:9205 ``__call__``,
lib.rs:9959 ``reduce``); the batch has no counterpart there.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._array import ndarray
from ._lib import IonpSchedule, NUM_SCHEDULES, check, code_of, lib
from ._ufunc import BINARY_OPS

BATCH_BINARY = ("add", "subtract", "multiply", "maximum", "less", "logical_and")
BATCH_REDUCE = ("add", "maximum")

# schedule factors, in the index order of ionp_schedule_from_index
BLOCK_TILES = (128, 256, 512, 1024)
VEC_WIDTHS = (1, 2, 4)
ELEMS_PER_THREAD = (1, 4)
RED_SPLITS = (1, 2)
DEFAULT_SCHEDULE = (512, 1, 1, 1)  # the C library's default (ionp_batch.cu)


def schedule(idx: int) -> IonpSchedule:
    """Schedule number idx (0..47): block tile slowest, reduction split fastest."""
    s = IonpSchedule()
    check(lib().ionp_schedule_from_index(int(idx), ctypes.byref(s)))
    return s


def schedule_index(block_tile, vec_width, elems_per_thread, red_split) -> int:
    return (BLOCK_TILES.index(block_tile) * 12 + VEC_WIDTHS.index(vec_width) * 4 +
            ELEMS_PER_THREAD.index(elems_per_thread) * 2 + RED_SPLITS.index(red_split))


DEFAULT_INDEX = schedule_index(*DEFAULT_SCHEDULE)


def _sched(s):
    if s is None:
        return None
    if isinstance(s, IonpSchedule):
        return ctypes.byref(s)
    return ctypes.byref(schedule(int(s)))


class Batch:
    """A queue of calls run as one persistent kernel (optionally in a graph)."""

    def __init__(self):
        self._h = ctypes.c_void_p()
        check(lib().ionp_batch_create(ctypes.byref(self._h)))
        self._keep = []       # operands and outputs stay alive with the batch
        self.outputs = []
        self.kinds = []
        self._explicit = set()  # calls queued or set with a schedule of their own
        self._knobs_done = False

    def __del__(self):
        try:
            if self._h:
                lib().ionp_batch_destroy(self._h)
        except Exception:
            pass
        self._h = None

    def __len__(self):
        return len(self.outputs)

    # ---- building ---------------------------------------------------------
    def add_binary(self, name: str, a: ndarray, b: ndarray, out: ndarray | None = None, sched=None) -> int:
        """Queue ``name(a, b)``; returns the call id. The output (C order, the
        loop's result dtype) is allocated unless given."""
        L = lib()
        if out is None:
            r = ctypes.c_int32()
            check(L.ionp_binary_out_dtype(BINARY_OPS[name], code_of(a.dtype), code_of(b.dtype), ctypes.byref(r)))
            from ._lib import DTYPES
            shape = np.broadcast_shapes(a.shape, b.shape)
            out = ndarray.empty(shape, DTYPES[r.value])
        cid = ctypes.c_int32()
        da, db, do = a._desc(), b._desc(), out._desc()
        check(L.ionp_batch_add_binary(self._h, BINARY_OPS[name], ctypes.byref(da), ctypes.byref(db),
                                      ctypes.byref(do), _sched(sched), ctypes.byref(cid)))
        if sched is not None:
            self._explicit.add(cid.value)
        self._keep += [a, b]
        self.outputs.append(out)
        self.kinds.append(("binary", name))
        return cid.value

    def add_reduce(self, name: str, a: ndarray, axis: int, keepdims: bool = False, out: ndarray | None = None,
                   sched=None) -> int:
        """Queue ``name.reduce(a, axis)`` (C-contiguous a); returns the call id."""
        L = lib()
        axis = axis % a.ndim
        if out is None:
            r = ctypes.c_int32()
            check(L.ionp_reduce_compute_dtype(BINARY_OPS[name], code_of(a.dtype), ctypes.byref(r)))
            from ._lib import DTYPES
            shape = tuple(1 if i == axis else s for i, s in enumerate(a.shape)) if keepdims else \
                tuple(s for i, s in enumerate(a.shape) if i != axis)
            out = ndarray.empty(shape, DTYPES[r.value])
        cid = ctypes.c_int32()
        da, do = a._desc(), out._desc()
        check(L.ionp_batch_add_reduce(self._h, BINARY_OPS[name], ctypes.byref(da), int(axis), int(bool(keepdims)),
                                      ctypes.byref(do), _sched(sched), ctypes.byref(cid)))
        if sched is not None:
            self._explicit.add(cid.value)
        self._keep.append(a)
        self.outputs.append(out)
        self.kinds.append(("reduce", name))
        return cid.value

    def set_schedule(self, call: int, sched) -> None:
        s = sched if isinstance(sched, IonpSchedule) else schedule(int(sched))
        check(lib().ionp_batch_set_schedule(self._h, int(call), ctypes.byref(s)))
        self._explicit.add(int(call))

    def apply_knobs(self) -> dict:
        """Apply the run-time knobs (``_config.settings``) to the calls queued
        without a schedule of their own; done once, before the first run.
        Returns the settings used."""
        from ._config import settings
        cfg = settings()
        self._knobs_done = True
        free = [i for i in range(len(self)) if i not in self._explicit]
        if not free:
            return cfg
        L = lib()
        if cfg["batch_schedule"] is not None:
            picks = {i: cfg["batch_schedule"] for i in free}
        elif cfg["batch_picker"] == "stream":
            from .picker import StreamPicker
            all_picks = StreamPicker().pick(self)
            picks = {i: int(all_picks[i]) for i in free}
        elif cfg["batch_picker"] == "autotune":
            picks = {i: int(np.argmin(self.time_call(i, reps=3))) for i in free}
        else:
            return cfg
        for i, k in picks.items():
            s = schedule(k)
            check(L.ionp_batch_set_schedule(self._h, int(i), ctypes.byref(s)))
        return cfg

    def set_schedules(self, idxs) -> None:
        """Schedule idxs[i] for call i."""
        table = [schedule(k) for k in range(NUM_SCHEDULES)]
        f = lib().ionp_batch_set_schedule
        for i, k in enumerate(idxs):
            check(f(self._h, i, ctypes.byref(table[int(k)])))
            self._explicit.add(i)

    # ---- running ----------------------------------------------------------
    def finalize(self, stream=None) -> None:
        if not self._knobs_done:
            self.apply_knobs()
        check(lib().ionp_batch_finalize(self._h, stream))

    def run(self, graph: bool = True, stream=None) -> None:
        """All calls as one persistent kernel; graph=True replays a captured
        CUDA graph after the first run. The run-time knobs apply before the
        first run."""
        if not self._knobs_done:
            self.apply_knobs()
        check(lib().ionp_batch_run(self._h, int(bool(graph)), stream))

    def run_per_call(self, stream=None) -> None:
        """The same calls, one default-schedule launch per call (baseline)."""
        check(lib().ionp_batch_run_per_call(self._h, stream))

    def fpe(self, stream=None) -> np.ndarray:
        w = np.zeros(len(self), np.uint32)
        check(lib().ionp_batch_fpe(self._h, w.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), stream))
        return w

    def info(self) -> dict:
        v = (ctypes.c_int64 * 5)()
        check(lib().ionp_batch_info(self._h, v))
        return {"calls": v[0], "tiles": v[1], "grid": v[2], "smem": v[3], "bytes": v[4]}

    def time_call(self, call: int, scheds=None, reps: int = 5, stream=None) -> np.ndarray:
        """Device microseconds of call `call` run alone under each schedule
        (default: all 48)."""
        idx = list(range(NUM_SCHEDULES)) if scheds is None else [int(k) for k in scheds]
        arr = (IonpSchedule * len(idx))()
        for j, k in enumerate(idx):
            arr[j] = schedule(k)
        out = (ctypes.c_float * len(idx))()
        check(lib().ionp_batch_time_call(self._h, int(call), len(idx), arr, int(reps), out, stream))
        return np.frombuffer(out, np.float32).copy()
