"""GPU parity of the reduction family (sum, prod, min, max, amin, amax, any,
all, mean; functions and ndarray methods) against the oracle, over the call
forms the reference's own differential suite uses for them
(tests/differential/ndarray_attrs_cases.py `_reduce_forms`: no arguments,
axis=None, axis 0 / -1, keepdims, leading / all / non-adjacent axis tuples,
out-of-range and duplicate axes, where=True/False, dtype=float64,
initial=), on every dtype and on C, Fortran and transposed inputs."""
import warnings

import numpy as np
import pytest

from oracle import oracle as O
from tests._util import ALL, array, assert_bits_equal

ap = pytest.importorskip("anionpy_b200")
pytestmark = pytest.mark.gpu

FAMILY = {  # function -> (ufunc op, has dtype=, has initial=, initial value)
    "sum": ("add", True, True, 2), "prod": ("multiply", True, True, 2),
    "min": ("minimum", False, True, 1), "max": ("maximum", False, True, 1),
    "amin": ("minimum", False, True, 1), "amax": ("maximum", False, True, 1),
    "all": ("logical_and", False, False, None), "any": ("logical_or", False, False, None),
}


def forms(nd, has_dtype, has_initial, init):
    f = [("no_args", {}), ("axis_none_explicit", {"axis": None})]
    if nd >= 1:
        f += [("axis0", {"axis": 0}), ("axis_last", {"axis": -1}), ("keepdims_axis0", {"axis": 0, "keepdims": True}),
              ("where_true_explicit", {"axis": 0, "where": True})]
    if nd >= 2:
        f += [("axis_tuple_leading", {"axis": tuple(range(nd - 1))}), ("axis_tuple_all", {"axis": tuple(range(nd))})]
    if nd >= 3:
        f += [("axis_tuple_noncontig", {"axis": (0, nd - 1)})]
    if has_dtype and nd >= 1:
        f += [("dtype_kwarg_float64", {"axis": 0, "dtype": np.float64})]
    if has_initial and nd >= 1:
        f += [("initial_kwarg", {"axis": 0, "initial": init}), ("where_false_no_initial", {"axis": 0, "where": False}),
              ("where_false_with_initial", {"axis": 0, "where": False, "initial": init})]
    return f


def inputs(dt):
    rng = np.random.default_rng(41)
    base = array(dt, (4, 5, 6), rng)
    if np.dtype(dt).kind == "f":
        base = (base / 8).astype(dt)    # keep products finite and interesting
    yield "C", base
    yield "F", np.asfortranarray(base)
    yield "T", base.transpose(2, 0, 1)
    yield "1d", array(dt, (37,), rng)
    yield "0d", array(dt, (), rng)


def to_host(r):
    return r.get() if isinstance(r, ap.ndarray) else np.asarray(r)


def want_of(op, host, kw):
    kw = dict(kw)
    where = kw.pop("where", None)
    if where is True:
        where = None
    if where is False:
        where = np.zeros(host.shape, np.bool_)
    axis = kw.pop("axis", None)
    try:
        return np.asarray(O.reduce(op, host, axis=axis, where=where, **kw)), None
    except O.OracleError as e:
        return None, e.status


@pytest.mark.parametrize("fn", list(FAMILY))
@pytest.mark.parametrize("dt", ALL, ids=lambda d: np.dtype(d).name)
def test_family_forms(fn, dt):
    op, has_dtype, has_initial, init = FAMILY[fn]
    for lay, host in inputs(dt):
        dev = ap.from_numpy(host) if lay not in ("F", "T") else (
            ap.from_numpy(np.ascontiguousarray(host.T)).T if lay == "F" else
            ap.from_numpy(np.ascontiguousarray(host.transpose(1, 2, 0))).transpose(2, 0, 1))
        for name, kw in forms(host.ndim, has_dtype, has_initial, init):
            want, err = want_of(op, host, kw)
            with warnings.catch_warnings():
                warnings.simplefilter("ignore")
                if err is not None:
                    with pytest.raises((ValueError, TypeError)):
                        getattr(ap, fn)(dev, **kw)
                    continue
                got = getattr(ap, fn)(dev, **kw)
                meth = getattr(dev, fn)(**kw) if hasattr(dev, fn) else got
            what = f"{fn} {np.dtype(dt).name} {lay} {name}"
            assert_bits_equal(to_host(got).reshape(want.shape), want, what)
            assert_bits_equal(to_host(meth).reshape(want.shape), want, what + " (method)")
            if want.ndim == 0 and "keepdims" not in kw:
                assert not isinstance(got, ap.ndarray), f"{what}: a 0-d result is a scalar"
        # the error forms
        if host.ndim >= 1:
            with pytest.raises(ap.AxisError):
                getattr(ap, fn)(dev, axis=100)
            with pytest.raises(ap.AxisError):
                getattr(ap, fn)(dev, axis=-100)
            with pytest.raises(ValueError):
                getattr(ap, fn)(dev, axis=(0, 0))


MEAN_FORMS = [("no_args", {}), ("axis0", {"axis": 0}), ("axis_last", {"axis": -1}),
              ("keepdims_axis0", {"axis": 0, "keepdims": True}), ("axis_tuple", {"axis": (0, 2)}),
              ("dtype_f64", {"axis": 1, "dtype": np.float64}), ("dtype_f32", {"axis": 1, "dtype": np.float32})]


@pytest.mark.parametrize("dt", ALL, ids=lambda d: np.dtype(d).name)
def test_mean(dt):
    rng = np.random.default_rng(43)
    host = array(dt, (6, 7, 8), rng)
    if np.dtype(dt).kind == "f":
        host = np.where(np.isfinite(host), host, 0).astype(dt)
    for layout in ("C", "T"):
        h = host if layout == "C" else host.transpose(2, 1, 0)
        dev = ap.from_numpy(host) if layout == "C" else ap.from_numpy(host).transpose(2, 1, 0)
        for name, kw in MEAN_FORMS:
            want, warned, cat = O.mean(h, **kw)
            got = ap.mean(dev, **kw)
            what = f"mean {np.dtype(dt).name} {layout} {name}"
            assert_bits_equal(to_host(got).reshape(want.shape), want, what)
            assert_bits_equal(to_host(dev.mean(**kw)).reshape(want.shape), want, what + " (method)")
            if isinstance(got, ap.ndarray) and want.ndim:
                st = O.reduce_layout_strides(list(h.shape), [s // h.itemsize for s in h.strides],
                                             sorted((a % h.ndim) for a in np.atleast_1d(kw.get("axis", list(range(h.ndim))))),
                                             kw.get("keepdims", False))
                assert list(got.elem_strides) == list(st), f"{what}: strides {got.elem_strides} != {st}"
    # where= mask: divides by the mask's count per slice
    mask = rng.random((6, 7, 8)) < 0.6
    want, warned, cat = O.mean(host, axis=1, where=mask)
    got = ap.mean(ap.from_numpy(host), axis=1, where=ap.from_numpy(mask))
    assert_bits_equal(to_host(got), want, f"mean {np.dtype(dt).name} where=")


def test_mean_empty_slice_warns_and_reports_divide():
    a = np.zeros((0, 3))
    with pytest.warns(RuntimeWarning, match="Mean of empty slice"):
        with ap.errstate(invalid="warn"):
            with pytest.warns(RuntimeWarning, match="invalid value encountered in divide"):
                r = ap.mean(ap.from_numpy(a), axis=0)
    want, warned, cat = O.mean(a, axis=0)
    assert warned and cat == "invalid"
    assert_bits_equal(r.get(), want, "mean over an empty axis")
    with ap.errstate(invalid="raise"):
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            with pytest.raises(FloatingPointError, match="invalid value encountered in scalar divide"):
                ap.mean(ap.from_numpy(np.zeros((0,))))


def test_mean_axis_errors():
    d = ap.from_numpy(np.ones((3, 4)))
    with pytest.raises(TypeError, match="integer argument expected, got float"):
        ap.mean(d, axis=1.0)
    with pytest.raises(ap.AxisError):
        ap.mean(ap.from_numpy(np.array(1.0)), axis=0)
