"""Seeded synthetic workloads for the batched mixed stream and the schedule
picker.

``mixed_stream`` draws a stream of small ufunc calls: element counts
log-uniform in [10, 10^6], rank uniform in 1..4 with random size-1
(broadcast) axes on either operand, dtypes from {bool, int8, int16, int32,
int64, float16, float32, float64} combined by NumPy promotion; 70% binary
ufuncs from {add, multiply, subtract, maximum, less, logical_and}, 30%
add/maximum reductions over a random axis. A bool-bool subtract has no loop
(TypeError in the reference, ufunc.rs:1163-1167), so such draws are skipped
and counted.

The inputs of every call are their own device arrays, filled from per-dtype
pools of seeded random values (ints uniform over the dtype's range, floats
N(0,1) with 0.1% NaN, bools 0/1).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

DTYPES8 = ("bool", "int8", "int16", "int32", "int64", "float16", "float32", "float64")
BINARY6 = ("add", "multiply", "subtract", "maximum", "less", "logical_and")
REDUCE2 = ("add", "maximum")


@dataclass
class CallSpec:
    kind: str                      # "binary" | "reduce"
    op: str
    shapes: list                   # operand shapes
    dtypes: list                   # operand dtype names
    axis: int = 0                  # reduce only
    layouts: list = field(default_factory=list)  # per operand: "c", "T" (axes reversed), "s2" (step-2 inner axis)


def _shape(rng, n, rank):
    """rank extents whose product is close to n (log-uniform split)."""
    if rank == 1:
        return [n]
    w = rng.dirichlet(np.ones(rank))
    dims = [max(1, int(round(math.exp(x * math.log(n))))) for x in w]
    return dims


def mixed_stream(ncalls=10000, seed=7, n_min=10, n_max=10 ** 6):
    """(calls, skipped): `ncalls` valid CallSpecs and the count of skipped
    bool-subtract draws."""
    rng = np.random.default_rng(seed)
    calls, skipped = [], 0
    lo, hi = math.log(n_min), math.log(n_max)
    while len(calls) < ncalls:
        n = int(round(math.exp(rng.uniform(lo, hi))))
        rank = int(rng.integers(1, 5))
        shape = _shape(rng, n, rank)
        if rng.random() < 0.7:
            op = BINARY6[int(rng.integers(len(BINARY6)))]
            da = DTYPES8[int(rng.integers(8))]
            db = DTYPES8[int(rng.integers(8))]
            if op == "subtract" and np.promote_types(da, db) == np.bool_:
                skipped += 1
                continue
            sa = [d if rng.random() >= 0.25 else 1 for d in shape]
            sb = [d if rng.random() >= 0.25 else 1 for d in shape]
            calls.append(CallSpec("binary", op, [sa, sb], [da, db]))
        else:
            op = REDUCE2[int(rng.integers(2))]
            dt = DTYPES8[int(rng.integers(8))]
            axis = int(rng.integers(rank))
            calls.append(CallSpec("reduce", op, [shape], [dt], axis=axis))
    return calls, skipped


def picker_cases(ncases, seed, n_min=10, n_max=10 ** 6):
    """Cases of the schedule-picker study: drawn like the mixed stream, with
    binary operands also laid out as axis-reversed views (permuted) or step-2
    slices of the innermost axis (strided), 15% each, so that every stride
    class appears (contiguous / broadcast / permuted / strided)."""
    calls, _ = mixed_stream(ncases, seed=seed, n_min=n_min, n_max=n_max)
    rng = np.random.default_rng(seed + 1000)
    for c in calls:
        if c.kind == "binary":
            lay = []
            for _ in range(2):
                u = rng.random()
                lay.append("T" if u < 0.15 else ("s2" if u < 0.30 else "c"))
            c.layouts = lay
        else:
            c.layouts = ["c"]
    return calls


def pool_values(dt, n, rng):
    dt = np.dtype(dt)
    if dt == np.bool_:
        return rng.integers(0, 2, n).astype(np.bool_)
    if dt.kind in "iu":
        info = np.iinfo(dt)
        return rng.integers(info.min, info.max, n, dtype=dt, endpoint=True)
    x = rng.standard_normal(n).astype(dt)
    x[rng.random(n) < 0.001] = np.nan
    return x


class DevicePools:
    """One device pool of random values per dtype; operands are filled by
    device-to-device copies from random offsets of their dtype's pool."""

    def __init__(self, ap, pool_elems=1 << 24, seed=11):
        self.ap = ap
        self.rng = np.random.default_rng(seed)
        self.host = {}
        self.dev = {}
        self.n = pool_elems
        for d in DTYPES8:
            h = pool_values(d, pool_elems, self.rng)
            self.host[d] = h
            self.dev[d] = ap.from_numpy(h)

    def view(self, shape, dt, layout="c"):
        """A device array of the given logical shape laid out as `layout`
        ("c": C-contiguous, "T": the transpose of a C-contiguous array of the
        reversed shape, "s2": every other element of a C-contiguous array
        twice as long in the innermost axis); also its host copy."""
        shape = list(shape)
        if layout == "T" and len(shape) > 1:
            base, hb = self.array(shape[::-1], dt)
            return base.transpose(), hb.transpose()
        if layout == "s2" and len(shape) >= 1:
            wide = shape[:-1] + [2 * shape[-1]]
            base, hb = self.array(wide, dt)
            idx = (slice(None),) * (len(shape) - 1) + (slice(None, None, 2),)
            return base[idx], hb[idx]
        return self.array(shape, dt)

    def array(self, shape, dt):
        """A new C-contiguous device array of random values; also returns its
        host copy (a view of the pool)."""
        from . import _lib
        L = _lib.lib()
        n = int(np.prod(shape)) if len(shape) else 1
        if n > self.n:
            raise ValueError("operand larger than the value pool")
        off = int(self.rng.integers(0, self.n - n + 1))
        out = self.ap.empty(tuple(shape), dt)
        isz = np.dtype(dt).itemsize
        if n:
            _lib.check(L.ionp_memcpy(out.data_ptr, self.dev[dt].data_ptr + off * isz, n * isz, 2, None))
        return out, self.host[dt][off: off + n].reshape(shape)


def build_batch(ap, calls, pools, keep_host=False):
    """A Batch with every call queued (default schedules). Returns (batch,
    hosts) where hosts[i] are the call's host operand copies when keep_host."""
    from ._batch import Batch
    b = Batch()
    hosts = []
    for c in calls:
        if c.kind == "binary":
            (sa, sb), (da, db) = c.shapes, c.dtypes
            la, lb = c.layouts if c.layouts else ("c", "c")
            x, hx = pools.view(sa, da, la)
            y, hy = pools.view(sb, db, lb)
            b.add_binary(c.op, x, y)
            hosts.append((hx, hy) if keep_host else None)
        else:
            x, hx = pools.array(c.shapes[0], c.dtypes[0])
            b.add_reduce(c.op, x, c.axis)
            hosts.append((hx,) if keep_host else None)
    return b, hosts
