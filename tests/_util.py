"""Seeded test data and bit-exact comparison helpers."""
from __future__ import annotations

import numpy as np

SEED = 20260731  # the reference corpus seed (tests/differential/corpus.py:22)

ALL = [np.bool_, np.int8, np.int16, np.int32, np.int64, np.uint8, np.uint16, np.uint32, np.uint64,
       np.float16, np.float32, np.float64]
FLOATS = [np.float16, np.float32, np.float64]
INTS = [np.int8, np.int16, np.int32, np.int64, np.uint8, np.uint16, np.uint32, np.uint64]

_FSPECIAL = [np.nan, -np.nan, np.inf, -np.inf, 0.0, -0.0, 1.0, -1.0, 0.5, -2.5, 3.0, -3.0, 1e-30, -1e-30,
             5e-324, -5e-324, 1e-45, 6e-8, 1e300, -1e300, 65504.0, 3.4e38, 7.0, 2.0 ** 53, -(2.0 ** 54), 1.5]


def values(dt, n, rng, specials=True, zeros=0.0):
    """n values of dtype dt: specials first, then a seeded body."""
    dt = np.dtype(dt)
    if dt == np.bool_:
        return rng.integers(0, 2, n).astype(np.bool_)
    if dt.kind in "iu":
        info = np.iinfo(dt)
        body = rng.integers(info.min, info.max, n, dtype=dt, endpoint=True)
        if specials and n >= 8:
            ext = np.array([info.min, info.max, 0, 1, info.max - 1, info.min + 1] + ([-1] if dt.kind == "i" else [2]), dtype=dt)
            body[: len(ext)] = ext
        if zeros:
            body[rng.random(n) < zeros] = 0
        return body
    with np.errstate(all="ignore"):
        body = (rng.standard_normal(n) * 10).astype(dt)
        if specials:
            sp = np.array(_FSPECIAL, np.float64).astype(dt)
            k = min(len(sp), n)
            pos = rng.permutation(n)[: max(k, n // 20)]
            body[pos] = np.resize(sp, len(pos))
        if zeros:
            body[rng.random(n) < zeros] = 0
    return body


def array(dt, shape, rng, **kw):
    n = int(np.prod(shape)) if shape else 1
    return values(dt, n, rng, **kw).reshape(shape)


def bits(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a)
    if a.dtype == np.bool_:
        return a.view(np.uint8)
    return a.view({1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[a.itemsize])


def assert_bits_equal(got, want, what=""):
    got = np.asarray(got)
    want = np.asarray(want)
    assert got.dtype == want.dtype, f"{what}: dtype {got.dtype} != {want.dtype}"
    assert got.shape == want.shape, f"{what}: shape {got.shape} != {want.shape}"
    gb, wb = bits(got), bits(want)
    bad = np.nonzero(gb.reshape(-1) != wb.reshape(-1))[0]
    if len(bad):
        i = bad[0]
        raise AssertionError(f"{what}: {len(bad)} of {gb.size} elements differ; first at flat {i}: "
                             f"got {got.reshape(-1)[i]!r} ({gb.reshape(-1)[i]:#x}) want {want.reshape(-1)[i]!r} ({wb.reshape(-1)[i]:#x})")


def ulp_distance(got, want) -> np.ndarray:
    """Dawson ordered-integer distance; NaN vs non-NaN and +0 vs -0 count as
    infinite (the reference harness rule, tests/differential/harness.py:549)."""
    got = np.asarray(got)
    want = np.asarray(want)
    ib = {2: np.int16, 4: np.int32, 8: np.int64}[got.itemsize]
    g = got.view(ib).astype(np.int64)
    w = want.view(ib).astype(np.int64)
    big = np.iinfo(ib).min
    g = np.where(g < 0, big - g, g)
    w = np.where(w < 0, big - w, w)
    d = np.abs(g - w).astype(np.float64)
    gn, wn = np.isnan(got), np.isnan(want)
    d[gn & wn] = 0
    d[gn ^ wn] = np.inf
    z = (got == 0) & (want == 0) & (np.signbit(got) != np.signbit(want))
    d[z] = np.inf
    return d
