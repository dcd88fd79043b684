"""Build step of the package: compiles libionp_cuda.so (sm_100a) in-tree."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")


def build(jobs: int | None = None, verbose: bool = False) -> str:
    """Run the csrc Makefile (nvcc, -gencode arch=compute_100a,code=sm_100a)."""
    jobs = jobs or max(os.cpu_count() or 4, 4)
    cmd = ["make", "-C", CSRC, f"-j{jobs}"]
    out = subprocess.run(cmd, capture_output=not verbose, text=True)
    if out.returncode != 0:
        raise RuntimeError("libionp_cuda.so build failed:\n" + (out.stdout or "")[-4000:] + (out.stderr or "")[-4000:])
    return os.path.join(HERE, "libionp_cuda.so")


if __name__ == "__main__":
    print(build(verbose=True))
