"""Builds the native libraries of merbit_b200 in-tree.

* ``libmerbit_b200.so``: every ``csrc/*.cu`` compiled for sm_100a with nvcc
  (``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``) and linked with
  the static CUDA runtime, so the library carries no dependency on the
  interpreter's libcudart.
* ``libmerbit_synth.so``: the OpenMP synthetic-matrix generators
  (``csrc/synth.cpp``).

Run ``python -m merbit_b200._build`` (``--force`` rebuilds everything).
An output is rebuilt only when the content digest of its inputs (sources,
headers, flags, compiler version) differs from the one recorded beside it
(``<output>.stamp``); file times play no part.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import hashlib
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


def _digest(files: list[str], extra: list[str]) -> str:
    """sha256 of the files' contents and the extra strings (flags, tools)."""
    h = hashlib.sha256()
    for f in files:
        h.update(f.encode())
        with open(f, "rb") as fh:
            h.update(fh.read())
    for e in extra:
        h.update(e.encode())
    return h.hexdigest()


def _stale(target: str, deps: list[str], extra: list[str]) -> bool:
    """True unless `target` exists and was built from exactly these inputs
    (its stamp file holds their content digest; file times are not used)."""
    stamp = target + ".stamp"
    if not (os.path.exists(target) and os.path.exists(stamp)):
        return True
    with open(stamp) as fh:
        return fh.read().strip() != _digest(deps, extra)


def _stamp(target: str, deps: list[str], extra: list[str]) -> None:
    with open(target + ".stamp", "w") as fh:
        fh.write(_digest(deps, extra) + "\n")


def _tool_version(tool: str) -> str:
    r = subprocess.run([tool, "--version"], capture_output=True, text=True)
    return r.stdout.strip()


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build(force: bool = False, verbose: bool = False) -> dict:
    """Compiles what changed and returns a report: the objects compiled, the
    libraries linked and whether each was up to date.  An output is rebuilt
    when the digest of its inputs (sources, headers, flags, compiler version)
    differs from the one recorded when it was built."""
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    nvcc_v = _tool_version(nvcc)
    hdrs = _headers()
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    objs = []
    jobs = []
    report = {"compiled": [], "linked": [], "up_to_date": []}
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        deps, extra = [s] + hdrs, NVCC_FLAGS + [nvcc_v]
        if force or _stale(o, deps, extra):
            jobs.append(([nvcc] + NVCC_FLAGS + ["-c", s, "-o", o], o, deps, extra))
        else:
            report["up_to_date"].append(os.path.basename(o))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            futs = [ex.submit(_run, j[0]) for j in jobs]
            for (cmd, o, deps, extra), fut in zip(jobs, futs):
                if verbose:
                    print(" ".join(cmd))
                fut.result()
                _stamp(o, deps, extra)
                report["compiled"].append(os.path.basename(o))
    lib_extra = ARCH + [nvcc_v]
    if force or jobs or _stale(LIB, objs, lib_extra):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs)
        _stamp(LIB, objs, lib_extra)
        report["linked"].append(os.path.basename(LIB))
    else:
        report["up_to_date"].append(os.path.basename(LIB))
    if build_example(force):
        report["linked"].append(os.path.basename(EXAMPLE))
    synth_src = os.path.join(CSRC, "synth.cpp")
    cxx = _hostcxx()
    synth_flags = ["-O3", "-fopenmp", "-fPIC", "-shared", "-std=c++17"]
    synth_deps = [synth_src, os.path.join(ROOT, "include", "merbit_synth.h")]
    synth_extra = synth_flags + [_tool_version(cxx)]
    if force or _stale(SYNTH, synth_deps, synth_extra):
        _run([cxx] + synth_flags + ["-o", SYNTH, synth_src])
        _stamp(SYNTH, synth_deps, synth_extra)
        report["linked"].append(os.path.basename(SYNTH))
    else:
        report["up_to_date"].append(os.path.basename(SYNTH))
    return report


def build_example(force: bool = False) -> bool:
    """The C++ harness (merbit_b200/compat/merbit_main.cpp) against
    include/merbit_compat.hpp, libmerbit_b200.so and the CUDA runtime.
    Returns whether it was linked."""
    deps = [EXAMPLE_SRC, LIB, os.path.join(ROOT, "include", "merbit_compat.hpp"),
            os.path.join(ROOT, "include", "merbit.h")]
    if not (force or _stale(EXAMPLE, deps, [])):
        return False
    _run([_hostcxx(), "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
          "-I", os.path.join(CUDA_HOME, "include"), EXAMPLE_SRC, "-o", EXAMPLE,
          "-L", PKG, "-lmerbit_b200", "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart",
          "-Wl,-rpath,$ORIGIN/..", "-Wl,-rpath," + os.path.join(CUDA_HOME, "lib64")])
    _stamp(EXAMPLE, deps, [])
    return True


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
    print(LIB)
    print(SYNTH)
