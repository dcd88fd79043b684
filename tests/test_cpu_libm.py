"""CPU check of the exp/log/sin/cos restatements the GPU kernels run
(anionpy_b200/csrc/ionp_libm.cuh), compiled for the host with the same
operations and fused multiply-adds, against the host C library (the
oracle's transcendentals): identical bits, NaNs included.

float32: every 61st bit pattern (about 70 million per function) by default;
IONP_LIBM_EXHAUSTIVE=1 checks all 2^32 patterns (about 35 s on 8 threads).
float64: 6 million seeded arguments per function over classes that reach
every path (subnormals, exp's overflow and underflow ends, log near 1, the
four reduction ranges of sin and cos); IONP_LIBM_F64=<n> sets the count."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "anionpy_b200", "csrc")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("libm") / "check_libm")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-pthread", "-I", CSRC,
                           os.path.join(HERE, "libm_check", "check_libm.cpp"), "-o", exe, "-lm"])
    return exe


def parse(out):
    rows = {}
    for line in out.strip().splitlines():
        name, n, d = line.split()
        rows[name] = (int(n.split("=")[1]), int(d.split("=")[1]))
    return rows


def test_float32_matches_c_library(checker):
    stride = "1" if os.environ.get("IONP_LIBM_EXHAUSTIVE") == "1" else "61"
    rows = parse(subprocess.check_output([checker, "f32", stride], text=True))
    assert set(rows) == {"exp32", "log32", "sin32", "cos32"}
    for name, (n, diff) in rows.items():
        assert n >= (1 << 32) // int(stride), name
        assert diff == 0, f"{name}: {diff} of {n} results differ from the C library"


def test_float64_matches_c_library(checker):
    count = os.environ.get("IONP_LIBM_F64", "6000000")
    rows = parse(subprocess.check_output([checker, "f64", count], text=True))
    assert set(rows) == {"exp64", "log64", "sin64", "cos64"}
    for name, (n, diff) in rows.items():
        assert n == int(count), name
        assert diff == 0, f"{name}: {diff} of {n} results differ from the C library"
