"""CPU check of the correctly rounded float32 exp/log/sin scheme of the GPU
kernels (ionp_transcendental.cuh / ionp_dd.cuh), compiled for the host and
compared on a sample of every float32 against (float)(long double libm).
The full sweep (stride 1, ~4.3e9 inputs per function) was run once with 0
differences; this test repeats it on a stride so the CPU suite stays fast."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "anionpy_b200", "csrc")


@pytest.fixture(scope="module")
def verifier(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cr") / "verify_f32")
    subprocess.check_call(["g++", "-O2", "-ffp-contract=off", "-std=c++17", "-pthread", "-I", CSRC,
                           os.path.join(HERE, "cr_check", "verify_f32.cpp"), "-o", exe, "-lm"])
    return exe


@pytest.mark.parametrize("which", [0, 1, 2], ids=["exp", "log", "sin"])
@pytest.mark.parametrize("slow", [0, 1], ids=["fast+slow", "slow-only"])
def test_float32_scheme_correctly_rounded(verifier, which, slow):
    out = subprocess.check_output([verifier, str(which), str(slow), "4099"], text=True)
    last = out.strip().splitlines()[-1]
    assert " diff=0 " in last + " ", out
    assert " n=0 " not in last
