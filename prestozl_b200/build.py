"""Build libjerk.so in-tree for sm_100a (nvcc, static cudart).

    python -m prestozl_b200.build
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = ["jerk_kernels.cu", "jerk_bank.cu", "jerk_realfft.cu", "jerk_polish.cu", "jerk_dedisp.cu", "jerk_plan.cpp", "jerk_server.cpp"]
HEADERS = ["jerk_fft.cuh", "jerk_kernels.cuh", "jerk_resp.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    target = os.path.join(LIBDIR, "libjerk.so")
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "jerk.h"))
    deps.append(os.path.abspath(__file__))
    if not force and not _stale(target, deps):
        return target
    cmd = [NVCC, "-O3", "-std=c++17", "--expt-relaxed-constexpr", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-shared",
           "-I" + os.path.join(ROOT, "include"), "-o", target]
    for f in SOURCES:
        p = os.path.join(CSRC, f)
        cmd += (["-x", "cu", p] if f.endswith(".cpp") else [p])
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return target


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
