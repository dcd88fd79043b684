"""Generates tests/golden/*.npz: golden vectors that pin the oracle.

Inputs come from the reference's own differential corpus
(Son0fSun/anionpy tests/differential/corpus.py: unary_corpus() and
binary_corpus(), seed 20260731), imported at generation time from a local
checkout of the reference, given as the first argument or in the
REFERENCE_ROOT environment variable. The
expected outputs are NumPy's, for the items the reference declares
bit-exact against NumPy (tests/differential/r.json and the coverage ledger:
add, subtract, multiply, divide, maximum, minimum, comparisons, logical and
bitwise ops, floor_divide, remainder, sum/add.reduce, maximum.reduce,
argmin/argmax). Transcendentals are not pinned to NumPy here: on x86 NumPy's
SIMD exp/log/sin differ from glibc, which is what the reference calls.

Run:  python tests/golden/make_golden.py <reference checkout>
(the produced .npz files are committed and used without it.)
"""
from __future__ import annotations

import json
import os
import sys
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = None

SUPPORTED = {np.dtype(t) for t in (np.bool_, np.int8, np.int16, np.int32, np.int64, np.uint8, np.uint16, np.uint32,
                                   np.uint64, np.float16, np.float32, np.float64)}
BINARY = ["add", "subtract", "multiply", "divide", "maximum", "minimum", "greater", "greater_equal", "less",
          "less_equal", "equal", "not_equal", "logical_and", "logical_or", "logical_xor", "bitwise_and",
          "bitwise_or", "bitwise_xor", "floor_divide", "remainder"]
UNARY = ["negative", "absolute", "invert", "logical_not", "sqrt"]
REDUCE = ["add", "maximum", "minimum", "multiply", "logical_and", "logical_or", "bitwise_xor"]


def main():
    global REF
    REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE_ROOT")
    if not REF or not os.path.isdir(os.path.join(REF, "tests", "differential")):
        sys.exit("usage: make_golden.py <reference checkout> (or set REFERENCE_ROOT)")
    sys.path.insert(0, os.path.join(REF, "tests", "differential"))
    import corpus  # the reference corpus builder (numpy only)

    arrays = {}
    meta = []

    def put(arr):
        k = f"x{len(arrays)}"
        arrays[k] = np.asarray(arr)
        return k

    def npres(fn):
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            with np.errstate(all="ignore"):
                try:
                    return fn(), None
                except Exception as e:  # numpy rejects: record the class
                    return None, type(e).__name__

    for p in corpus.binary_corpus():
        a, b = np.asarray(p.a), np.asarray(p.b)
        if a.dtype not in SUPPORTED or b.dtype not in SUPPORTED:
            continue
        for op in BINARY:
            r, err = npres(lambda: getattr(np, op)(a, b))
            entry = {"kind": "binary", "op": op, "label": p.label, "a": put(a), "b": put(b)}
            if err:
                entry["error"] = err
            else:
                entry["out"] = put(r)
            meta.append(entry)
    for c in corpus.unary_corpus():
        x = np.asarray(c.value)
        if x.dtype not in SUPPORTED:
            continue
        fortran = bool(x.ndim > 1 and x.flags["F_CONTIGUOUS"] and not x.flags["C_CONTIGUOUS"])
        xc = np.array(x, copy=True, order="C")
        for op in UNARY:
            r, err = npres(lambda: getattr(np, op)(x))
            entry = {"kind": "unary", "op": op, "label": c.label, "a": put(xc)}
            if err:
                entry["error"] = err
            else:
                entry["out"] = put(r)
            meta.append(entry)
        if x.ndim == 0 or not (x.flags["C_CONTIGUOUS"] or fortran):
            continue
        for op in REDUCE:
            for axis in (0, None, -1):
                r, err = npres(lambda: getattr(np, op).reduce(x, axis=axis))
                entry = {"kind": "reduce", "op": op, "label": c.label, "a": put(xc), "fortran": fortran,
                         "axis": axis}
                if err:
                    entry["error"] = err
                else:
                    entry["out"] = put(r)
                meta.append(entry)
        for which in ("argmax", "argmin"):
            for axis in (None, 0):
                r, err = npres(lambda: getattr(np, which)(x, axis=axis))
                entry = {"kind": "argext", "op": which, "label": c.label, "a": put(xc), "fortran": fortran, "axis": axis}
                if err:
                    entry["error"] = err
                else:
                    entry["out"] = put(r)
                meta.append(entry)
    np.savez_compressed(os.path.join(HERE, "corpus_numpy.npz"), **arrays)
    with open(os.path.join(HERE, "corpus_numpy.json"), "w") as f:
        json.dump({"numpy": np.__version__, "seed": corpus.SEED, "cases": meta}, f, indent=0)
    print(f"{len(meta)} cases, {len(arrays)} arrays")


if __name__ == "__main__":
    main()
