"""Seeded synthetic CSR workloads (numpy front end of libmerbit_synth.so).

These stand in for the Matrix Market graphs the reference harness loads by
id (src/main.cu:13, src/class.cu:60-141), which are not available: each
workload reproduces a shape, size and value distribution, from a fixed seed,
identically on every machine and for any thread count.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
SYNTH_PATH = os.path.join(PKG, "libmerbit_synth.so")

TAG_X = 0x58564543  # stream tag of x vectors
TAG_G = 0x47524144  # stream tag of upstream gradients

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(SYNTH_PATH):
            from . import _build

            _build.build()
        L = C.CDLL(SYNTH_PATH)
        i64, u64, d, p = C.c_int64, C.c_uint64, C.c_double, C.c_void_p
        L.merbit_synth_laplace2d.argtypes = [i64, i64, p, p, p]
        L.merbit_synth_stencil27_nnz.argtypes = [i64, i64, i64]
        L.merbit_synth_stencil27_nnz.restype = i64
        L.merbit_synth_stencil27.argtypes = [i64, i64, i64, u64, p, p, p]
        L.merbit_synth_zipf_rowptr.argtypes = [i64, i64, d, i64, d, u64, p]
        L.merbit_synth_zipf_rowptr.restype = i64
        L.merbit_synth_zipf_fill.argtypes = [i64, i64, u64, p, p, p]
        L.merbit_synth_rmat.argtypes = [i64, i64, d, d, d, u64, p, p, p]
        L.merbit_synth_rmat.restype = i64
        L.merbit_synth_uniform.argtypes = [u64, u64, i64, d, d, p]
        L.merbit_synth_normal.argtypes = [u64, u64, i64, p]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


@dataclass
class CSR:
    row_ptr: np.ndarray  # int32 [nrow+1]
    col: np.ndarray      # int32 [nnz]
    vals: np.ndarray     # float64 [nnz] (cast by the caller for other precisions)
    ncol: int
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def nrow(self) -> int:
        return len(self.row_ptr) - 1

    @property
    def nnz(self) -> int:
        return len(self.col)


def laplace2d(nx: int, ny: int) -> CSR:
    n = nx * ny
    nnz = 5 * n - 2 * nx - 2 * ny
    rp = np.empty(n + 1, np.int32)
    col = np.empty(nnz, np.int32)
    vals = np.empty(nnz, np.float64)
    if lib().merbit_synth_laplace2d(nx, ny, _p(rp), _p(col), _p(vals)) != 0:
        raise ValueError("laplace2d: bad size")
    return CSR(rp, col, vals, n, f"laplace2d_{nx}x{ny}")


def stencil27(nx: int, ny: int, nz: int, seed: int = 0) -> CSR:
    n = nx * ny * nz
    nnz = lib().merbit_synth_stencil27_nnz(nx, ny, nz)
    rp = np.empty(n + 1, np.int32)
    col = np.empty(nnz, np.int32)
    vals = np.empty(nnz, np.float64)
    if lib().merbit_synth_stencil27(nx, ny, nz, seed, _p(rp), _p(col), _p(vals)) != 0:
        raise ValueError("stencil27: bad size")
    return CSR(rp, col, vals, n, f"stencil27_{nx}x{ny}x{nz}")


def zipf(n: int, s: float = 1.8, cap: int = 200_000, empty_frac: float = 0.1,
         seed: int = 1, ncol: int | None = None) -> CSR:
    ncol = n if ncol is None else ncol
    rp = np.empty(n + 1, np.int32)
    nnz = lib().merbit_synth_zipf_rowptr(n, ncol, s, cap, empty_frac, seed, _p(rp))
    if nnz < 0:
        raise ValueError("zipf: bad parameters or nnz beyond int32")
    col = np.empty(nnz, np.int32)
    vals = np.empty(nnz, np.float64)
    if lib().merbit_synth_zipf_fill(n, ncol, seed, _p(rp), _p(col), _p(vals)) != 0:
        raise ValueError("zipf: fill failed")
    return CSR(rp, col, vals, ncol, f"zipf{s}_{n}")


def rmat(n: int, avg_degree: float, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int = 2) -> CSR:
    nedges = int(round(n * avg_degree))
    rp = np.empty(n + 1, np.int32)
    col = np.empty(max(nedges, 1), np.int32)
    vals = np.empty(max(nedges, 1), np.float64)
    nnz = lib().merbit_synth_rmat(n, nedges, a, b, c, seed, _p(rp), _p(col), _p(vals))
    if nnz < 0:
        raise ValueError("rmat: bad parameters")
    # views of the first nnz entries (the arrays were sized for every edge drawn)
    return CSR(rp, col[:nnz], vals[:nnz], n, f"rmat_{n}",
               {"edges_drawn": nedges, "avg_degree": avg_degree})


def uniform(seed: int, n: int, lo: float = -1.0, hi: float = 1.0, tag: int = TAG_X) -> np.ndarray:
    out = np.empty(n, np.float64)
    lib().merbit_synth_uniform(seed, tag, n, lo, hi, _p(out))
    return out


def normal(seed: int, n: int, tag: int = TAG_G) -> np.ndarray:
    out = np.empty(n, np.float64)
    lib().merbit_synth_normal(seed, tag, n, _p(out))
    return out


def to_bf16_bits(v: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even float64 -> bfloat16, returned as uint16 bits."""
    f = np.ascontiguousarray(v, dtype=np.float32).view(np.uint32)
    rounding = ((f >> 16) & 1) + 0x7FFF
    return ((f + rounding) >> 16).astype(np.uint16)


def bf16_bits_to_f64(b: np.ndarray) -> np.ndarray:
    return (b.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


# ---------------------------------------------------------------------------
# The named workloads (full sizes) and small instances of the same
# generators for parity tests.
# ---------------------------------------------------------------------------

def batch_rmat_specs(count: int = 128, seed: int = 2, nmin: int = 1000, nmax: int = 500_000,
                     dmin: float = 8.0, dmax: float = 64.0):
    """(n_i, avg_degree_i, seed_i) for the batched form: rows log-uniform in
    [nmin, nmax], average degree uniform in [dmin, dmax]."""
    u = uniform(seed, 2 * count, 0.0, 1.0, tag=0x42415443)
    specs = []
    for i in range(count):
        n = int(round(math.exp(math.log(nmin) + u[2 * i] * (math.log(nmax) - math.log(nmin)))))
        deg = dmin + u[2 * i + 1] * (dmax - dmin)
        specs.append((n, deg, seed * 1_000_003 + i))
    return specs


# Seed of the dense input vector x of each benchmark matrix (the Laplacian's
# x is drawn from seed 0, the power-law matrix's from seed 1, the
# differentiation form's X from seed 3); other workloads use seed 1.
X_SEEDS = {"laplace2d_256": 0, "zipf_2m": 1, "stencil27_160": 0, "zipf_1m_diff": 3}


def workload_x(name: str, n: int, k: int = 1) -> np.ndarray:
    """x ~ U[-1,1] of n entries (k > 1: an (n, k) row-major X) for `name`."""
    x = uniform(X_SEEDS.get(name, 1), n * k)
    return x if k == 1 else x.reshape(n, k)


def workload(name: str) -> CSR:
    if name == "laplace2d_256":
        return laplace2d(256, 256)
    if name == "zipf_2m":
        return zipf(2_000_000, 1.8, 200_000, 0.1, seed=1)
    if name == "stencil27_160":
        return stencil27(160, 160, 160, seed=0)
    if name == "zipf_1m_diff":
        return zipf(1_000_000, 1.8, 200_000, 0.1, seed=3)
    # small instances of the same generators
    if name == "laplace2d_small":
        return laplace2d(40, 33)
    if name == "zipf_small":
        return zipf(20_000, 1.8, 20_000, 0.1, seed=1)
    if name == "stencil27_small":
        return stencil27(14, 12, 10, seed=0)
    if name == "zipf_2k_diff":
        return zipf(2_000, 1.8, 2_000, 0.1, seed=3)
    raise KeyError(name)
