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
    """Compile every source to an object in parallel, then link libjerk.so."""
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    target = os.path.join(LIBDIR, "libjerk.so")
    common = [os.path.join(CSRC, f) for f in HEADERS]
    common += [os.path.join(ROOT, "include", "jerk.h"), os.path.abspath(__file__)]
    flags = ["-O3", "-std=c++17", "--expt-relaxed-constexpr", *ARCH, "-lineinfo",
             "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include")]
    srcs = [os.path.join(CSRC, f) for f in SOURCES]
    if not force and not _stale(target, srcs + common):
        return target  # objects need not be present (a copy of the tree with the library)
    jobs = []
    objs = []
    for f in SOURCES:
        src = os.path.join(CSRC, f)
        obj = os.path.join(objdir, os.path.splitext(f)[0] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + common):
            cmd = [NVCC, *flags, "-c"] + (["-x", "cu", src] if f.endswith(".cpp") else [src])
            jobs.append(cmd + ["-o", obj])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)

    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1) or 1) as ex:
        for f in [ex.submit(run, c) for c in jobs]:
            f.result()
    run([NVCC, *ARCH, "-shared", "-o", target, *objs])
    return target


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
