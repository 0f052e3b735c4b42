"""Build recipe for libpeasoup_b200.so (sm_100a), in-tree.

    python -m peasoup_b200.build          # or peasoup_b200.build.build()

Steps: the CUDA and C++ sources are compiled with nvcc/g++ for sm_100a;
everything is linked against cuFFT into
peasoup_b200/libpeasoup_b200.so.  Objects go to peasoup_b200/_build/.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libpeasoup_b200.so")

CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Host code is compiled without floating-point contraction: the host float
# arithmetic (acceleration list, bin ranges) must round like the
# reference's host compiler.
HOST_FLAGS = "-fPIC,-O2,-ffp-contract=off,-fno-fast-math"
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", *ARCH, "-Xcompiler", HOST_FLAGS,
              f"-I{INCLUDE}", f"-I{CSRC}", f"-I{BUILD}"]

CU_SOURCES = ["psx_kernels.cu", "psx_fft.cu", "psx_fft4.cu", "psx_search.cu", "psx_tune.cu",
              "psx_dedisp.cu"]
CPP_SOURCES = ["psx_host.cpp", "psx_serve.cpp", "psx_output.cpp", "psx_sigproc.cpp"]


def _headers():
    """Every header of csrc/ (any change rebuilds every object)."""
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cuh", ".h")))


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    return r


def build(verbose: bool = False, force: bool = False) -> str:
    """Compile and link the library if any source is newer; returns its path."""
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in _headers()] + [os.path.join(INCLUDE, "peasoup_b200.h")]

    # 1. objects
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            jobs.append([NVCC, "-c", *NVCC_FLAGS, s, "-o", o])
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            jobs.append(["g++", "-c", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off",
                         "-fno-fast-math", f"-I{INCLUDE}", f"-I{CSRC}",
                         f"-I{os.path.join(CUDA, 'include')}", s, "-o", o])
    if jobs:
        with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for r in ex.map(_run, jobs):
                if verbose:
                    sys.stdout.write(r.stdout + r.stderr)

    # 2. link
    if force or jobs or _newer(LIB, objs):
        tmp = LIB + ".tmp"
        _run([NVCC, "-shared", *ARCH, *objs, "-lcufft", "-o", tmp])
        shutil.move(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
