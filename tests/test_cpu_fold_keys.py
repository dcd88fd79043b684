"""CPU check of the order-key fold the column reductions use for float
maximum / minimum (`fkey` and `col_fold_batch` in
anionpy_b200/csrc/ionp_reduce.cuh): on NaN-free data the integer max / min
of the keys (a value's bits, with a negative value's magnitude bits
flipped) selects exactly the bits the sequential float_max / float_min fold
returns, the -0 / +0 ties included; checked against the oracle's reduce."""
import numpy as np
import pytest

from oracle import oracle as O


def keys(a):
    it = np.int32 if a.dtype == np.float32 else np.int64
    flip = it(0x7FFFFFFF) if it == np.int32 else it(0x7FFFFFFFFFFFFFFF)
    k = a.view(it)
    return np.where(k < 0, k ^ flip, k)


def unkey(k, dt):
    flip = k.dtype.type(0x7FFFFFFF) if dt == np.float32 else k.dtype.type(0x7FFFFFFFFFFFFFFF)
    return np.where(k < 0, k ^ flip, k).astype(k.dtype).view(dt)


@pytest.mark.parametrize("dt", [np.float32, np.float64], ids=lambda d: np.dtype(d).name)
@pytest.mark.parametrize("op", ["maximum", "minimum"])
def test_key_fold_matches_oracle(dt, op):
    rng = np.random.default_rng(7 + (op == "minimum"))
    a = np.round(rng.standard_normal((300, 257)) * 2).astype(dt)  # many ties
    a[rng.random(a.shape) < 0.3] = 0.0
    a[rng.random(a.shape) < 0.3] *= -1                            # -0 among the zeros
    a[:, :4] = rng.choice([0.0, -0.0], (300, 4)).astype(dt)      # columns of zeros only
    a[:, 20:40] = -np.abs(a[:, 20:40]) - dt(0.5)                  # all negative
    a[:, 40:60] = np.abs(a[:, 40:60]) + dt(0.5)                   # all positive
    a[:, 60:64] = np.where(rng.random((300, 4)) < 0.5, dt(-0.0), dt(-1.0))  # -0 the largest
    a[5, 10] = np.inf
    a[7, 11] = -np.inf
    ib = np.uint32 if dt == np.float32 else np.uint64
    k = keys(a)
    got = unkey(k.max(axis=0) if op == "maximum" else k.min(axis=0), dt)
    want = np.asarray(O.reduce(op, a, axis=0))
    assert np.array_equal(got.view(ib), want.view(ib))
    # a seed folds first, as the kernels' accumulator does
    for seed in (dt(0.0), dt(-0.0), dt(1.5)):
        ks = keys(np.array([seed], dt))[0]
        kk = np.maximum(k.max(axis=0), ks) if op == "maximum" else np.minimum(k.min(axis=0), ks)
        got = unkey(kk, dt)
        want = np.asarray(O.reduce(op, a, axis=0, initial=seed))
        assert np.array_equal(got.view(ib), want.view(ib)), seed
