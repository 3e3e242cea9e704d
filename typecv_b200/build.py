"""Build libtba.so in-tree with nvcc for sm_100a (B200).

    python -m typecv_b200.build [--force]

The shared library lands next to this file (typecv_b200/libtba.so) so that it travels with the
source tree; nothing is installed elsewhere.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libtba.so")
SOURCES = ["tba_kernels.cu", "tba_batch.cu", "tba_adjoint.cu", "tba_observations.cu", "tba_checks.cu", "tba_api.cu",
           "tba_noalloc.cu"]
HEADERS = ["tba_math.cuh", "tba_engine.cuh", "tba_warp.cuh", "tba_batch.cuh", "tba_adjoint.cuh", "tba_observations.cuh",
           "tba_checks.cuh"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC", "-shared", "-Xptxas", "-v"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "tba.h"))
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    tmp = LIB + f".{os.getpid()}.tmp"
    cmd = [nvcc(), *NVCC_FLAGS, "-o", tmp, *[os.path.join(CSRC, f) for f in SOURCES]]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stderr[-4000:]}")
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
