"""CPU tests that pin the oracle (test infrastructure) before anything is
compared against it:

* the golden vectors of tests/golden/ (inputs from the reference's own
  differential corpus, outputs from NumPy for the items the reference
  declares bit-exact against NumPy) -- every case, byte for byte;
* the reference's reduce length sweep around the pairwise boundaries
  (tests/differential/ufunc_cases.py:156) against NumPy's add.reduce;
* the reference's inline Rust known-answer tests (ionp-core/src/ufunc.rs
  tests module);
* the FPE categories of ionp-core/src/fpe.rs on the reference's fperr cases;
* a planted mistake (a sequential sum in place of the pairwise tree) that
  the golden check must reject, like the reference's harness self-test.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _load():
    meta = json.load(open(os.path.join(GOLD, "corpus_numpy.json")))["cases"]
    arrs = np.load(os.path.join(GOLD, "corpus_numpy.npz"))
    return meta, arrs


def _run(c, A, reduce_impl=None):
    a = A[c["a"]]
    if c["kind"] == "binary":
        return O.binary(c["op"], a, A[c["b"]])[0]
    if c["kind"] == "unary":
        return O.unary(c["op"], a)[0]
    x = np.asfortranarray(a) if c.get("fortran") else a
    if c["kind"] == "reduce":
        return (reduce_impl or O.reduce)(c["op"], x, axis=c["axis"])
    return O.argext(c["op"], x, axis=c["axis"])


def test_golden_corpus_bit_exact():
    meta, A = _load()
    assert len(meta) > 4000
    bad = []
    for c in meta:
        try:
            r = np.asarray(_run(c, A))
            err = None
        except O.OracleError as e:
            r, err = None, e.status
        if "error" in c:
            if err is None:
                bad.append((c["label"], c["op"], "numpy raised", c["error"]))
            continue
        w = A[c["out"]]
        if err is not None or r.dtype != w.dtype or r.shape != w.shape or r.tobytes() != w.tobytes():
            bad.append((c["label"], c["op"], c["kind"], err))
    assert not bad, bad[:10]


@pytest.mark.parametrize("dt", [np.float16, np.float32, np.float64])
def test_pairwise_reduce_length_sweep(dt):
    rng = np.random.default_rng(20260731)
    for n in (2, 4, 7, 8, 9, 16, 32, 64, 127, 128, 129, 1000, 4097, 100003):
        x = (rng.standard_normal(n) * 10).astype(dt)
        got = O.reduce("add", x, axis=0)
        want = np.add.reduce(x)
        assert np.asarray(got).tobytes() == np.asarray(want).tobytes(), n


def test_c1_config_against_numpy():
    rng = np.random.default_rng(0)
    a = rng.uniform(-1, 1, (1024, 1024))
    b = rng.uniform(-1, 1, (1, 1024))
    assert O.binary("add", a, b)[0].tobytes() == np.add(a, b).tobytes()
    assert O.reduce("add", a, axis=1).tobytes() == np.add.reduce(a, axis=1).tobytes()
    assert O.reduce("maximum", a, axis=0).tobytes() == np.maximum.reduce(a, axis=0).tobytes()
    # narrow axis (axis 0 of C order) is sequential, not pairwise, in the reference
    assert O.reduce("add", a, axis=0).tobytes() == np.add.reduce(a, axis=0).tobytes()


def test_rust_known_answers():
    # add_same_shape / add_broadcasts_row_vector_over_matrix
    r, _ = O.binary("add", np.array([1.0, 2, 3]), np.array([10.0, 20, 30]))
    assert r.tolist() == [11, 22, 33]
    r, _ = O.binary("add", np.arange(6.0).reshape(2, 3), np.array([100.0, 200, 300]))
    assert r.tolist() == [[100, 201, 302], [103, 204, 305]]
    # add_promotes_dtype
    r, _ = O.binary("add", np.array([1, 2, 3], np.int32), np.array([0.5, 0.5, 0.5]))
    assert r.dtype == np.float64 and r.tolist() == [1.5, 2.5, 3.5]
    # multiply_bool_is_logical_and / add_bool_is_logical_or
    assert O.binary("multiply", np.array([1, 1, 0], bool), np.array([1, 0, 0], bool))[0].tolist() == [True, False, False]
    assert O.binary("add", np.array([1, 0, 0], bool), np.array([0, 0, 1], bool))[0].tolist() == [True, False, True]
    # broadcast_mismatch_is_an_error
    with pytest.raises(O.OracleError):
        O.binary("add", np.ones(3), np.ones(2))
    # add_on_transposed_view_matches_manual_layout
    r, _ = O.binary("add", np.arange(6.0).reshape(2, 3).T, np.array([1.0, 1.0]))
    assert r.reshape(-1).tolist() == [1, 4, 2, 5, 3, 6]
    # sqrt_special_values_match_numpy_exactly
    r, _ = O.unary("sqrt", np.array([-1.0, -0.0]))
    assert np.isnan(r[0]) and r[1] == 0 and np.signbit(r[1])
    # log_special_values_match_numpy_exactly
    r, _ = O.unary("log", np.array([0.0, -1.0, -0.0]))
    assert r[0] == -np.inf and np.isnan(r[1]) and r[2] == -np.inf
    # remainder_by_zero_int_is_zero_not_a_panic, MIN % -1 == 0, MIN // -1 wraps
    r, f = O.binary("remainder", np.array([5, -128], np.int8), np.array([0, -1], np.int8))
    assert r.tolist() == [0, 0] and f == "divide"
    r, _ = O.binary("floor_divide", np.array([-128], np.int8), np.array([-1], np.int8))
    assert r.tolist() == [-128]
    # fmod_and_remainder_float_sign_rules: remainder takes the divisor's sign
    r, f = O.binary("remainder", np.array([1.0, -1.0, 5.5]), np.array([-1.0, 1.0, -2.0]))
    assert np.signbit(r[0]) and not np.signbit(r[1]) and r[2] == -0.5 and f is None


def test_fpe_categories():
    z = np.array([0.0, 1.0])
    assert O.binary("divide", np.array([1.0, 2.0]), z)[1] == "divide"
    assert O.binary("divide", np.array([0.0, 2.0]), z)[1] == "invalid"
    assert O.binary("floor_divide", np.array([1, 2], np.int32), np.array([0, 1], np.int32))[1] == "divide"
    assert O.binary("floor_divide", np.array([0, 2], np.int32), np.array([0, 1], np.int32))[1] == "divide"  # int out: no invalid
    assert O.binary("remainder", np.array([1.0]), np.array([0.0]))[1] is None  # float %0 is silent
    assert O.binary("multiply", np.array([1e200]), np.array([1e200]))[1] == "over"
    assert O.binary("multiply", np.array([1e-200]), np.array([1e-200]))[1] == "under"
    assert O.binary("multiply", np.array([np.inf]), np.array([2.0]))[1] is None
    assert O.binary("add", np.array([1e308]), np.array([1e308]))[1] is None  # add overflow not flagged
    assert O.unary("sqrt", np.array([-1.0, 4.0]))[1] == "invalid"
    assert O.unary("log", np.array([0.0, 1.0]))[1] == "divide"
    assert O.unary("log", np.array([0.0, -1.0]))[1] == "invalid"
    assert O.unary("exp", np.array([1000.0]))[1] is None
    # the flat x[i % len] pairing of fpe.rs: (2,1) x (1,3) pairs a[i%2] with b[i%3]
    a = np.array([[0.0], [5.0]])
    b = np.array([[0.0, 1.0, 1.0]])
    assert O.binary("divide", a, b)[1] == "invalid"


def test_planted_mistake_is_caught():
    """A sequential left-to-right sum in place of the pairwise tree must
    disagree with the golden vectors (the check has teeth)."""
    meta, A = _load()

    def wrong_reduce(op, x, axis=0, **kw):
        if op == "add" and x.dtype.kind == "f" and x.size > 8:
            return np.asarray(np.cumsum(np.asarray(x, dtype=x.dtype), axis=axis, dtype=x.dtype)).take(-1, axis=axis if axis is not None else 0) \
                if axis is not None else np.cumsum(x.reshape(-1), dtype=x.dtype)[-1]
        return O.reduce(op, x, axis=axis, **kw)

    rng = np.random.default_rng(1)
    x = (rng.standard_normal(100003)).astype(np.float32)
    assert np.asarray(wrong_reduce("add", x)).tobytes() != np.add.reduce(x).tobytes()
    assert np.asarray(O.reduce("add", x)).tobytes() == np.add.reduce(x).tobytes()


def test_transcendentals_are_glibc_and_within_one_ulp_of_correct_rounding():
    """The oracle's exp/log/sin are glibc's (what Rust's f64::exp etc. call on
    Linux). Against a 64-bit-mantissa reference (x87 long double via
    np.longdouble) they are within 1 ULP in float64 and 1 ULP in float32."""
    import ctypes
    libm = ctypes.CDLL("libm.so.6")
    libm.exp.restype = ctypes.c_double
    libm.exp.argtypes = [ctypes.c_double]
    rng = np.random.default_rng(3)
    x = rng.uniform(-50, 50, 2000)
    got = O.unary("exp", x)[0]
    ref = np.array([libm.exp(float(v)) for v in x])
    assert got.tobytes() == ref.tobytes()
    ld = np.exp(x.astype(np.longdouble))
    err = np.abs((got.astype(np.longdouble) - ld) / np.spacing(got)).max()
    assert err <= 1.0


def test_oracle_mean_matches_numpy():
    """The oracle's mean (the reference's composition, reductions.rs:1515)
    equals NumPy's bit for bit on C-ordered inputs, which the reference
    declares; float16 sums in float32, float32 divides in float64."""
    rng = np.random.default_rng(1)
    for dt in (np.float16, np.float32, np.float64, np.int8, np.int32, np.int64, np.uint16, np.bool_):
        if np.dtype(dt).kind == "f":
            a = rng.standard_normal((6, 7, 8)).astype(dt)
        elif dt == np.bool_:
            a = rng.random((6, 7, 8)) < 0.5
        else:
            a = rng.integers(-100 if np.dtype(dt).kind == "i" else 0, 100, (6, 7, 8)).astype(dt)
        for kw in ({}, {"axis": 0}, {"axis": -1}, {"axis": (0, 2)}, {"axis": 1, "keepdims": True},
                   {"axis": 1, "dtype": np.float32}):
            got = O.mean(a, **kw)[0]
            want = np.asarray(np.mean(a, **kw))
            assert got.dtype == want.dtype and got.tobytes() == want.tobytes(), (np.dtype(dt).name, kw)
