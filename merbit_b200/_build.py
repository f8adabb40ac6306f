"""Builds the native libraries of merbit_b200 in-tree.

* ``libmerbit_b200.so``: every ``csrc/*.cu`` compiled for sm_100a with nvcc
  (``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``) and linked with
  the static CUDA runtime, so the library carries no dependency on the
  interpreter's libcudart.
* ``libmerbit_synth.so``: the OpenMP synthetic-matrix generators
  (``csrc/synth.cpp``).

Run ``python -m merbit_b200._build`` (``--force`` rebuilds everything).
Objects are only recompiled when a source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libmerbit_b200.so")
SYNTH = os.path.join(PKG, "libmerbit_synth.so")
EXAMPLE_SRC = os.path.join(PKG, "compat", "merbit_main.cpp")
EXAMPLE = os.path.join(PKG, "compat", "merbit_main")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                     "--expt-relaxed-constexpr", "-Xptxas", "-O3"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _hostcxx() -> str:
    # the system g++ carries libgomp; a CXX pointing elsewhere may not
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("g++ not found")


def _headers() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build(force: bool = False, verbose: bool = False) -> None:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    hdrs = _headers()
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    objs = []
    jobs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            jobs.append([nvcc] + NVCC_FLAGS + ["-c", s, "-o", o])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            for cmd, fut in zip(jobs, [ex.submit(_run, j) for j in jobs]):
                if verbose:
                    print(" ".join(cmd))
                fut.result()
    if force or jobs or _stale(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs)
    build_example(force)
    synth_src = os.path.join(CSRC, "synth.cpp")
    if force or _stale(SYNTH, [synth_src, os.path.join(ROOT, "include", "merbit_synth.h")]):
        _run([_hostcxx(), "-O3", "-fopenmp", "-fPIC", "-shared", "-std=c++17", "-o", SYNTH,
              synth_src])


def build_example(force: bool = False) -> None:
    """The C++ harness (merbit_b200/compat/merbit_main.cpp) against
    include/merbit_compat.hpp, libmerbit_b200.so and the CUDA runtime."""
    deps = [EXAMPLE_SRC, LIB, os.path.join(ROOT, "include", "merbit_compat.hpp"),
            os.path.join(ROOT, "include", "merbit.h")]
    if not (force or _stale(EXAMPLE, deps)):
        return
    _run([_hostcxx(), "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
          "-I", os.path.join(CUDA_HOME, "include"), EXAMPLE_SRC, "-o", EXAMPLE,
          "-L", PKG, "-lmerbit_b200", "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart",
          "-Wl,-rpath,$ORIGIN/..", "-Wl,-rpath," + os.path.join(CUDA_HOME, "lib64")])


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
    print(SYNTH)
