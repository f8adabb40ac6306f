"""ctypes front end of the CPU oracle and of the reference harness.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke``
and by ``bench.py``'s CPU-baseline leg (and its ``--impl reference`` arm),
never by the ``merbit_b200`` package.

* ``lib()`` -> oracle/_build/libmerbit_oracle.so (oracle/merbit_oracle.c):
  the C restatement of the reference's merge_search (include/utils.cuh:5-29),
  Tile_Kernel (include/tile.cuh:28-122) and an extended-precision SpMM/adjoint
  reference, plus the merge-path OpenMP FP64 SpMV used as the CPU baseline.
* ``ref()`` -> oracle/_ref/libmerbit_ref.so (oracle/ref_harness.cu): the
  reference's own merge_search / Tile_Kernel / merbit_kernel, compiled from
  the reference sources by oracle/Makefile.  ``None`` when not built.
* ``comp()`` -> oracle/_ref/libmerbit_competitors.so (oracle/competitors.cu):
  the libraries the reference compares against (cuSPARSE CSR_ALG2 / COO_ALG2,
  CUB DeviceSpmv, vendored CSR5 and HOLA), timed as src/spmv.cu calls them.
  ``None`` when not built.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libmerbit_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmerbit_ref.so")
COMP_SO = os.path.join(HERE, "_ref", "libmerbit_competitors.so")

F64, F32, BF16 = 0, 1, 2
_i64 = C.c_int64
_p = C.c_void_p

_lib = None
_ref = None
_ref_tried = False
_comp = None
_comp_tried = False


def build() -> None:
    """Run oracle/Makefile (oracle always; reference harness when the
    reference sources are present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.orc_merge_search.argtypes = [_p, _i64, _i64, _i64, C.POINTER(_i64), C.POINTER(_i64)]
        L.orc_merge_coords.argtypes = [_p, _i64, _i64, _i64, _i64, _p, _p]
        L.orc_tile_dims.argtypes = [_i64, _i64, C.c_int, C.POINTER(_i64), C.POINTER(_i64)]
        L.orc_tile_plan.argtypes = [_p, _i64, _i64, C.c_int, _p, _p, _p]
        L.orc_spmm.argtypes = [_i64, _p, _p, C.c_int, _p, C.c_int, _p, _i64, _i64, C.c_double,
                               _p, _p, _i64]
        L.orc_spmm_t.argtypes = [_i64, _i64, _p, _p, C.c_int, _p, C.c_int, _p, _i64, _i64, _p, _i64]
        L.orc_dval.argtypes = [_i64, _p, _p, C.c_int, _p, _i64, C.c_int, _p, _i64, _i64, _p]
        L.orc_spmv_omp_f64.argtypes = [_i64, _p, _p, _p, _p, _p, C.c_int]
        L.orc_spmv_omp_f64.restype = C.c_int
        L.orc_max_threads.restype = C.c_int
        L.orc_spmv_abs_omp_f64.argtypes = [_i64, _p, _p, _p, _p, _p, C.c_int]
        L.orc_spmv_abs_omp_f64.restype = C.c_int
        L.orc_spmm_omp_f32.argtypes = [_i64, _p, _p, _p, _p, _i64, _p, C.c_int]
        L.orc_spmm_omp_f32.restype = C.c_int
        _lib = L
    return _lib


def ref():
    """The reference harness, or None when oracle/_ref was not built."""
    global _ref, _ref_tried
    if not _ref_tried:
        _ref_tried = True
        if os.path.exists(REF_SO):
            R = C.CDLL(REF_SO)
            R.ref_merge_search.argtypes = [_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int),
                                           C.POINTER(C.c_int)]
            R.ref_tile_dims.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int),
                                        C.POINTER(C.c_int)]
            R.ref_tile_build.argtypes = [C.c_int, _p, C.c_int, C.c_int, _p, _p, _p]
            R.ref_merbit_spmv.argtypes = [C.c_int, _p, _p, C.c_int, C.c_int, _p, _p, _p,
                                          C.c_double, _p, _p, _p, _p]
            R.ref_merbit_time.argtypes = [C.c_int, _p, _p, C.c_int, C.c_int, _p, _p, _p, _p, _p,
                                          _p, C.c_int, _p]
            R.ref_merbit_time.restype = C.c_float
            R.ref_merbit_time_sigma.argtypes = [C.c_int, C.c_int, _p, _p, C.c_int, C.c_int, _p,
                                                _p, _p, _p, _p, _p, C.c_int, _p]
            R.ref_merbit_time_sigma.restype = C.c_float
            _ref = R
    return _ref


def comp():
    """The competitor-library harness, or None when oracle/_ref was not built.
    Every entry returns 0 or an error code; times are mean ms per call."""
    global _comp, _comp_tried
    if not _comp_tried:
        _comp_tried = True
        if os.path.exists(COMP_SO):
            L = C.CDLL(COMP_SO)
            f = C.POINTER(C.c_float)
            i = C.POINTER(C.c_int)
            L.comp_cusparse_time.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _p, _p, _p, _p,
                                             _p, _p, C.c_int, f]
            L.comp_cub_time.argtypes = [C.c_int, C.c_int, C.c_int, _p, _p, _p, _p, _p, C.c_int, f]
            L.comp_csr5_time.argtypes = [C.c_int, C.c_int, C.c_int, _p, _p, _p, _p, _p, C.c_int,
                                         f, f, i]
            L.comp_hola_time.argtypes = [C.c_int, C.c_int, C.c_int, _p, _p, _p, _p, _p, C.c_int,
                                         f, f]
            _comp = L
    return _comp


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_p)


def _code(a: np.ndarray) -> int:
    if a.dtype == np.float64:
        return F64
    if a.dtype == np.float32:
        return F32
    if a.dtype == np.uint16:
        return BF16
    raise TypeError(a.dtype)


def merge_search(row_ptr: np.ndarray, nnz: int, diag: int) -> tuple[int, int]:
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    cx, cy = _i64(), _i64()
    lib().orc_merge_search(_ptr(row_ptr), len(row_ptr) - 1, nnz, diag, C.byref(cx), C.byref(cy))
    return cx.value, cy.value


def merge_coords(row_ptr: np.ndarray, stride: int, count: int):
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    nrow = len(row_ptr) - 1
    nnz = int(row_ptr[-1])
    ox = np.empty(count, np.int32)
    oy = np.empty(count, np.int32)
    lib().orc_merge_coords(_ptr(row_ptr), nrow, nnz, stride, count, _ptr(ox), _ptr(oy))
    return ox, oy


def tile_dims(nrow: int, nnz: int, sigma: int) -> tuple[int, int]:
    t, l = _i64(), _i64()
    lib().orc_tile_dims(nrow, nnz, sigma, C.byref(t), C.byref(l))
    return t.value, l.value


def tile_plan(row_ptr: np.ndarray, sigma: int = 14):
    """(tile_x u32[T+1], tile_y u32[T+1], lane_desc u32|u64[lane_num])."""
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    nrow = len(row_ptr) - 1
    nnz = int(row_ptr[-1])
    T, Ln = tile_dims(nrow, nnz, sigma)
    tx = np.empty(T + 1, np.uint32)
    ty = np.empty(T + 1, np.uint32)
    desc = np.empty(max(Ln, 1), np.uint64)
    lib().orc_tile_plan(_ptr(row_ptr), nrow, nnz, sigma, _ptr(tx), _ptr(ty), _ptr(desc))
    desc = desc[:Ln]
    if sigma < 15:
        desc = desc.astype(np.uint32)
    return tx, ty, desc


def spmm(row_ptr, col, vals, x, k: int = 1, alpha: float = 1.0, with_abs: bool = True):
    """Extended-precision Y = alpha*A*X.  x is (ncol,) or (ncol, k) row-major.
    Returns (y, yabs) as float64 arrays of shape (nrow,) or (nrow, k)."""
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    vals = np.ascontiguousarray(vals)
    x = np.ascontiguousarray(x)
    nrow = len(row_ptr) - 1
    ldx = 1 if x.ndim == 1 else x.shape[1]
    y = np.empty((nrow, k), np.float64)
    ya = np.empty((nrow, k), np.float64) if with_abs else None
    lib().orc_spmm(nrow, _ptr(row_ptr), _ptr(col), _code(vals), _ptr(vals), _code(x), _ptr(x), k,
                   ldx, alpha, _ptr(y), _ptr(ya) if with_abs else None, k)
    if x.ndim == 1:
        y = y[:, 0]
        ya = ya[:, 0] if with_abs else None
    return y, ya


def spmm_t(row_ptr, col, vals, g, ncol: int):
    """Extended-precision dX = A^T G (G row-major (nrow, k))."""
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    vals = np.ascontiguousarray(vals)
    g = np.ascontiguousarray(g)
    nrow = len(row_ptr) - 1
    k = 1 if g.ndim == 1 else g.shape[1]
    dx = np.empty((ncol, k), np.float64)
    lib().orc_spmm_t(nrow, ncol, _ptr(row_ptr), _ptr(col), _code(vals), _ptr(vals), _code(g),
                     _ptr(g), k, k, _ptr(dx), k)
    return dx[:, 0] if g.ndim == 1 else dx


def dval(row_ptr, col, g, x):
    """Extended-precision dval[e] = G[row_e] . X[col_e]."""
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    g = np.ascontiguousarray(g)
    x = np.ascontiguousarray(x)
    nrow = len(row_ptr) - 1
    k = 1 if g.ndim == 1 else g.shape[1]
    out = np.empty(int(row_ptr[-1]), np.float64)
    lib().orc_dval(nrow, _ptr(row_ptr), _ptr(col), _code(g), _ptr(g), k, _code(x), _ptr(x), k, k,
                   _ptr(out))
    return out


def spmv_omp_f64(row_ptr, col, vals, x, y=None, nthreads: int = 0):
    """Merge-path OpenMP FP64 SpMV (the CPU baseline).  Returns (y, threads)."""
    nrow = len(row_ptr) - 1
    if y is None:
        y = np.empty(nrow, np.float64)
    n = lib().orc_spmv_omp_f64(nrow, _ptr(row_ptr), _ptr(col), _ptr(vals), _ptr(x), _ptr(y),
                               nthreads)
    return y, n


def spmv_abs_omp_f64(row_ptr, col, vals, x, nthreads: int = 0):
    """sum_j |a_ij| |x_j| per row in double (OpenMP): the denominator of the
    component-wise error for the full-size matrices."""
    nrow = len(row_ptr) - 1
    vals = np.ascontiguousarray(vals, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    y = np.empty(nrow, np.float64)
    lib().orc_spmv_abs_omp_f64(nrow, _ptr(row_ptr), _ptr(col), _ptr(vals), _ptr(x), _ptr(y),
                               nthreads)
    return y


def spmm_omp_f32(row_ptr, col, vals32, x32, k: int, y=None, nthreads: int = 0):
    """Row-parallel OpenMP float SpMM (batched-form CPU baseline)."""
    nrow = len(row_ptr) - 1
    if y is None:
        y = np.empty((nrow, k), np.float32)
    n = lib().orc_spmm_omp_f32(nrow, _ptr(row_ptr), _ptr(col), _ptr(vals32), _ptr(x32), k,
                               _ptr(y), nthreads)
    return y, n


def max_threads() -> int:
    return lib().orc_max_threads()


def ref_merge_search(row_ptr: np.ndarray, nnz: int, diag: int):
    R = ref()
    if R is None:
        return None
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    cx, cy = C.c_int(), C.c_int()
    R.ref_merge_search(_ptr(row_ptr), len(row_ptr) - 1, nnz, diag, C.byref(cx), C.byref(cy))
    return cx.value, cy.value


def rel_error(y, y_ref, y_abs, tiny: float = 1e-300):
    """Component-wise error |y - y_ref| / max(sum|a x|, tiny): (max, median)."""
    y = np.asarray(y, np.float64)
    e = np.abs(y - y_ref) / np.maximum(y_abs, tiny)
    if e.size == 0:
        return 0.0, 0.0
    return float(e.max()), float(np.median(e))
