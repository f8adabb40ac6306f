"""merbit_b200: merge-path tiled CSR SpMV/SpMM for NVIDIA B200 (sm_100a).

Python host side of the C ABI declared in ``include/merbit.h``.  PyTorch
supplies device memory and streams; every operation runs in the hand-written
CUDA kernels of ``libmerbit_b200.so`` (built in-tree by
``python -m merbit_b200._build``).  There is no CPU fallback: importing the
operations without the library raises.

Reference interfaces mirrored (paths relative to the MERBIT project root):

* ``merge_coords``  -> ``merge_search<SIGMA>``   include/utils.cuh:5-29
* ``tile_build``    -> ``TILE<BLOCK,SIGMA>``     include/tile.cuh:4-122
* ``Plan.spmv``     -> ``merbit_kernel`` via ``Fun_Merbit``
                       include/tile.cuh:476-615
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import torch

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libmerbit_b200.so")

F64, F32, BF16 = 0, 1, 2
PLAN_SKIP_VALIDATE = 0x1
PLAN_NO_TUNE = 0x2

_DT_OF = {torch.float64: F64, torch.float32: F32, torch.bfloat16: BF16}
_XY_OF = {F64: torch.float64, F32: torch.float32, BF16: torch.float32}

STATUS = {
    0: "MERBIT_OK",
    1: "MERBIT_ERR_INVALID",
    2: "MERBIT_ERR_MATRIX",
    3: "MERBIT_ERR_OVERFLOW",
    4: "MERBIT_ERR_CUDA",
    5: "MERBIT_ERR_TIMEOUT",
    6: "MERBIT_ERR_UNSUPPORTED",
}


class MerbitError(RuntimeError):
    def __init__(self, status: int, detail: str):
        self.status = status
        self.detail = detail
        super().__init__(f"{STATUS.get(status, status)}: {detail}")


class _PlanInfo(C.Structure):
    _fields_ = [
        ("nrow", C.c_int32), ("ncol", C.c_int32), ("nnz", C.c_int32), ("dtype", C.c_int32),
        ("block", C.c_int32), ("items_per_thread", C.c_int32), ("tile_items", C.c_int32),
        ("num_tiles", C.c_int32), ("vectorized", C.c_int32), ("kind", C.c_int32),
        ("l1_carveout", C.c_int32), ("gather_l2_only", C.c_int32),
        ("metadata_bytes", C.c_int64), ("algorithmic_bytes", C.c_double),
        ("max_row_len", C.c_int32),
    ]


_P = C.c_void_p
# name -> (restype, argtypes); the complete exported surface of include/merbit.h
SIGNATURES = {
    "merbit_merge_coords": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int64, C.c_int64, _P, _P, _P]),
    "merbit_tile_dims": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, _P, _P]),
    "merbit_tile_build": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, _P, _P, _P, _P]),
    "merbit_plan_create": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, _P, _P, _P, C.c_int,
                                     C.c_uint32, _P]),
    "merbit_plan_destroy": (C.c_int, [_P]),
    "merbit_plan_get_info": (C.c_int, [_P, _P]),
    "merbit_plan_set_values": (C.c_int, [_P, _P]),
    "merbit_plan_tune": (C.c_int, [_P, _P, _P, _P]),
    "merbit_spmv": (C.c_int, [_P, C.c_double, _P, C.c_double, _P, _P]),
    "merbit_num_configs": (C.c_int, [C.c_int]),
    "merbit_config_desc": (C.c_int, [C.c_int, C.c_int32, _P, _P, _P]),
    "merbit_plan_set_config": (C.c_int, [_P, C.c_int32, _P]),
    "merbit_plan_config_usable": (C.c_int, [_P, C.c_int32, _P, _P]),
    "merbit_plan_check": (C.c_int, [_P, _P]),
    "merbit_pagerank_step": (C.c_int, [_P, C.c_double, _P, _P, _P, _P, _P]),
    "merbit_plan_selftest_wait": (C.c_int, [_P, C.c_int32, C.c_int32, _P]),
    "merbit_release_cached_memory": (C.c_int, []),
    "merbit_coo_sort": (C.c_int, [C.c_int32, _P, _P, _P, C.c_int, _P]),
    "merbit_coo_to_csr": (C.c_int, [C.c_int32, _P, C.c_int32, _P, _P]),
    "merbit_outdegree_values": (C.c_int, [C.c_int32, C.c_int32, _P, _P, C.c_int, _P]),
    "merbit_plan_transpose": (C.c_int, [_P, _P, _P]),
    "merbit_plan_transpose_refresh": (C.c_int, [_P, _P, _P]),
    "merbit_dval": (C.c_int, [_P, C.c_int32, _P, C.c_int64, _P, C.c_int64, _P, _P]),
    "merbit_spmm": (C.c_int, [_P, C.c_int32, C.c_double, _P, C.c_int64, C.c_double, _P,
                              C.c_int64, _P]),
    "merbit_spmm_dval": (C.c_int, [_P, C.c_int32, _P, C.c_int64, _P, C.c_int64, _P, C.c_int64,
                                   _P, _P]),
    "merbit_batch_create": (C.c_int, [_P, C.c_int32, _P, C.c_int32, _P, _P, _P, _P, _P]),
    "merbit_batch_spmm": (C.c_int, [_P, C.c_double, C.c_double, _P]),
    "merbit_batch_tune": (C.c_int, [_P, _P]),
    "merbit_batch_get_info": (C.c_int, [_P, _P]),
    "merbit_batch_get_matrix_config": (C.c_int, [_P, C.c_int32, _P, _P, _P]),
    "merbit_batch_set_matrix_config": (C.c_int, [_P, C.c_int32, C.c_int32, _P]),
    "merbit_batch_set_matrix_tile": (C.c_int, [_P, C.c_int32, C.c_int32, _P]),
    "merbit_batch_set_kernel": (C.c_int, [_P, C.c_int32, C.c_int32, _P]),
    "merbit_batch_destroy": (C.c_int, [_P]),
    "merbit_spmv_noalloc": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, _P, _P, _P, C.c_int,
                                      C.c_double, _P, C.c_double, _P, _P]),
    "merbit_spmv_noalloc_check": (C.c_int, [_P]),
    "merbit_spmv_noalloc_selftest_wait": (C.c_int, [C.c_int32, C.c_int32, _P]),
    "merbit_status_string": (C.c_char_p, [C.c_int]),
    "merbit_last_cuda_error": (C.c_int, []),
    "merbit_last_error_detail": (C.c_char_p, []),
}

# measurement support (include/merbit_bench.h)
BENCH_SIGNATURES = {
    "merbit_bench_gather": (C.c_int, [_P, C.c_int32, _P, C.c_int64, _P, C.c_int32, _P]),
}

_lib = None


def lib() -> C.CDLL:
    """The native library, with argument types set.  Raises if it is not
    built: there is no fallback path."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing; build it with `python -m merbit_b200._build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in {**SIGNATURES, **BENCH_SIGNATURES}.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(status: int) -> None:
    if status != 0:
        detail = lib().merbit_last_error_detail().decode(errors="replace")
        raise MerbitError(status, detail)


def _stream_ptr(stream) -> _P:
    if stream is None:
        stream = torch.cuda.current_stream()
    return _P(stream.cuda_stream)


def _dptr(t: torch.Tensor | None) -> _P:
    return _P(t.data_ptr()) if t is not None else _P(0)


def _need_cuda(t: torch.Tensor, name: str, dtype=None) -> None:
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if dtype is not None and t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


def merge_coords(row_ptr: torch.Tensor, nnz: int, stride: int, count: int, stream=None):
    """Merge-path coordinates at diagonals i*stride (include/utils.cuh:5-29).
    Returns int32 tensors (coord_x, coord_y)."""
    _need_cuda(row_ptr, "row_ptr", torch.int32)
    cx = torch.empty(count, dtype=torch.int32, device=row_ptr.device)
    cy = torch.empty(count, dtype=torch.int32, device=row_ptr.device)
    _check(lib().merbit_merge_coords(_dptr(row_ptr), row_ptr.numel() - 1, nnz, stride, count,
                                     _dptr(cx), _dptr(cy), _stream_ptr(stream)))
    return cx, cy


def release_cached_memory(device=None) -> None:
    """Return the released blocks of the library's device memory pool
    (merbit_release_cached_memory); blocks of live plans stay."""
    with torch.cuda.device(device if device is not None else torch.cuda.current_device()):
        _check(lib().merbit_release_cached_memory())


def tile_dims(nrow: int, nnz: int, sigma: int) -> tuple[int, int]:
    t, l = C.c_int32(), C.c_int32()
    _check(lib().merbit_tile_dims(nrow, nnz, sigma, C.byref(t), C.byref(l)))
    return t.value, l.value


def tile_build(row_ptr: torch.Tensor, nnz: int, sigma: int = 14, stream=None):
    """The reference Merbit plan (TILE<BLOCK,SIGMA>, include/tile.cuh:4-122):
    (tile_x u32[T+1], tile_y u32[T+1], lane_desc u32|u64[lane_num]) as int32 /
    int64 tensors holding the same bits."""
    _need_cuda(row_ptr, "row_ptr", torch.int32)
    nrow = row_ptr.numel() - 1
    T, Ln = tile_dims(nrow, nnz, sigma)
    dev = row_ptr.device
    tx = torch.empty(T + 1, dtype=torch.int32, device=dev)
    ty = torch.empty(T + 1, dtype=torch.int32, device=dev)
    desc = torch.empty(max(Ln, 1), dtype=torch.int32 if sigma < 15 else torch.int64, device=dev)
    _check(lib().merbit_tile_build(_dptr(row_ptr), nrow, nnz, sigma, _dptr(tx), _dptr(ty),
                                   _dptr(desc), _stream_ptr(stream)))
    return tx, ty, desc[:Ln]


def coo_sort(major: torch.Tensor, minor: torch.Tensor, vals: torch.Tensor | None = None,
             stream=None) -> None:
    """Sorts COO triplets in place by (major, minor), stably -- GRAPH::sort
    (src/class.cu:143-177) with major = col_ind for sort(false)."""
    _need_cuda(major, "major", torch.int32)
    _need_cuda(minor, "minor", torch.int32)
    n = major.numel()
    if minor.numel() != n or (vals is not None and vals.numel() != n):
        raise ValueError("major, minor and vals must have the same length")
    if vals is not None:
        _need_cuda(vals, "vals")
        if vals.dtype not in _DT_OF:
            raise TypeError(f"unsupported value dtype {vals.dtype}")
    _check(lib().merbit_coo_sort(n, _dptr(major), _dptr(minor), _dptr(vals),
                                 _DT_OF[vals.dtype] if vals is not None else 0, _stream_ptr(stream)))


def coo_to_csr(sorted_rows: torch.Tensor, nrow: int, stream=None) -> torch.Tensor:
    """row_ptr[nrow+1] of a sorted row-index array (cusparseXcoo2csr as
    include/tile.cuh:574 calls it, zero-based)."""
    _need_cuda(sorted_rows, "sorted_rows", torch.int32)
    rp = torch.empty(nrow + 1, dtype=torch.int32, device=sorted_rows.device)
    _check(lib().merbit_coo_to_csr(sorted_rows.numel(), _dptr(sorted_rows), nrow, _dptr(rp),
                                   _stream_ptr(stream)))
    return rp


def outdegree_values(row_ind: torch.Tensor, nrow: int, dtype=torch.float64,
                     stream=None) -> torch.Tensor:
    """values[e] = 1 / (entries sharing row_ind[e]) -- the loader's PageRank
    weights (Fun_Values, src/class.cu:2-34)."""
    _need_cuda(row_ind, "row_ind", torch.int32)
    if dtype not in _DT_OF:
        raise TypeError(f"unsupported value dtype {dtype}")
    out = torch.empty(row_ind.numel(), dtype=dtype, device=row_ind.device)
    _check(lib().merbit_outdegree_values(row_ind.numel(), nrow, _dptr(row_ind), _dptr(out),
                                         _DT_OF[dtype], _stream_ptr(stream)))
    return out


@dataclass
class PlanInfo:
    nrow: int
    ncol: int
    nnz: int
    dtype: int
    block: int
    items_per_thread: int
    tile_items: int
    num_tiles: int
    vectorized: bool
    kind: int
    l1_carveout: int
    gather_l2_only: bool
    metadata_bytes: int
    algorithmic_bytes: float
    max_row_len: int


class Plan:
    """One CSR matrix prepared for repeated products (merbit_plan_create).

    row_ptr / col_idx: int32 CUDA tensors; vals: float64, float32 or bfloat16
    CUDA tensor.  x and y are float64 for float64 values and float32 otherwise.
    The plan references (does not copy) the tensors and keeps them alive.
    """

    def __init__(self, row_ptr: torch.Tensor, col_idx: torch.Tensor, vals: torch.Tensor,
                 ncol: int | None = None, validate: bool = True, stream=None):
        _need_cuda(row_ptr, "row_ptr", torch.int32)
        _need_cuda(col_idx, "col_idx", torch.int32)
        _need_cuda(vals, "vals")
        if vals.dtype not in _DT_OF:
            raise TypeError(f"unsupported value dtype {vals.dtype}")
        self.dtype = _DT_OF[vals.dtype]
        self.xy_dtype = _XY_OF[self.dtype]
        self.nrow = row_ptr.numel() - 1
        self.nnz = col_idx.numel()
        self.ncol = self.nrow if ncol is None else int(ncol)
        self.device = row_ptr.device
        self._keep = [row_ptr, col_idx, vals]
        self.row_ptr, self.col_idx, self.vals = row_ptr, col_idx, vals
        self._h = _P()
        flags = 0 if validate else PLAN_SKIP_VALIDATE
        with torch.cuda.device(self.device):
            _check(lib().merbit_plan_create(C.byref(self._h), self.nrow, self.ncol, self.nnz,
                                            _dptr(row_ptr), _dptr(col_idx), _dptr(vals),
                                            self.dtype, flags, _stream_ptr(stream)))

    def close(self) -> None:
        if self._h:
            lib().merbit_plan_destroy(self._h)
            self._h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> PlanInfo:
        i = _PlanInfo()
        _check(lib().merbit_plan_get_info(self._h, C.byref(i)))
        return PlanInfo(i.nrow, i.ncol, i.nnz, i.dtype, i.block, i.items_per_thread,
                        i.tile_items, i.num_tiles, bool(i.vectorized), i.kind, i.l1_carveout,
                        bool(i.gather_l2_only), i.metadata_bytes, i.algorithmic_bytes,
                        i.max_row_len)

    def set_values(self, vals: torch.Tensor) -> None:
        _need_cuda(vals, "vals", self.vals.dtype)
        if vals.numel() != self.nnz:
            raise ValueError("vals has the wrong length")
        _check(lib().merbit_plan_set_values(self._h, _dptr(vals)))
        self.vals = vals
        self._keep[2] = vals

    def _vec(self, t: torch.Tensor, n: int, name: str) -> None:
        _need_cuda(t, name, self.xy_dtype)
        if t.numel() != n:
            raise ValueError(f"{name} must have {n} elements, got {t.numel()}")

    def spmv(self, x: torch.Tensor, y: torch.Tensor | None = None, alpha: float = 1.0,
             beta: float = 0.0, stream=None) -> torch.Tensor:
        """y = alpha*A*x + beta*y (beta == 0 never reads y)."""
        self._vec(x, self.ncol, "x")
        if y is None:
            y = torch.empty(self.nrow, dtype=self.xy_dtype, device=self.device)
        else:
            self._vec(y, self.nrow, "y")
        _check(lib().merbit_spmv(self._h, float(alpha), _dptr(x), float(beta), _dptr(y),
                                 _stream_ptr(stream)))
        return y

    def pagerank_step(self, x: torch.Tensor, teleport: torch.Tensor, damp: float = 0.85,
                      y: torch.Tensor | None = None, residual: torch.Tensor | None = None,
                      stream=None) -> torch.Tensor:
        """y = damp*A*x + (1-damp)*teleport in one launch; when `residual` (a
        float64 CUDA tensor of one element) is given it receives
        sum|y - x| from the same launch."""
        self._vec(x, self.ncol, "x")
        self._vec(teleport, self.nrow, "teleport")
        if y is None:
            y = torch.empty(self.nrow, dtype=self.xy_dtype, device=self.device)
        else:
            self._vec(y, self.nrow, "y")
        if residual is not None and (not residual.is_cuda or residual.dtype != torch.float64
                                     or residual.numel() < 1):
            raise TypeError("residual must be a float64 CUDA tensor with one element")
        _check(lib().merbit_pagerank_step(self._h, float(damp), _dptr(x), _dptr(teleport),
                                          _dptr(y), _dptr(residual), _stream_ptr(stream)))
        return y

    def _mat(self, t: torch.Tensor, rows: int, name: str) -> int:
        if not t.is_cuda or t.dtype != self.xy_dtype:
            raise TypeError(f"{name} must be a CUDA {self.xy_dtype} tensor")
        if t.dim() != 2 or t.shape[0] != rows or (rows > 1 and t.stride(1) != 1):
            raise ValueError(f"{name} must be a row-major ({rows}, k) matrix")
        return t.stride(0) if rows > 1 else t.shape[1]

    def spmm(self, X: torch.Tensor, Y: torch.Tensor | None = None, alpha: float = 1.0,
             beta: float = 0.0, stream=None) -> torch.Tensor:
        """Y = alpha*A*X + beta*Y for row-major X (ncol, k) -> Y (nrow, k)."""
        ldx = self._mat(X, self.ncol, "X")
        k = X.shape[1]
        if Y is None:
            Y = torch.empty(self.nrow, k, dtype=self.xy_dtype, device=self.device)
        ldy = self._mat(Y, self.nrow, "Y")
        if Y.shape[1] != k:
            raise ValueError("X and Y must have the same number of columns")
        if k == 0:
            return Y
        _check(lib().merbit_spmm(self._h, k, float(alpha), _dptr(X), max(ldx, k), float(beta),
                                 _dptr(Y), max(ldy, k), _stream_ptr(stream)))
        return Y

    def tune(self, x: torch.Tensor | None = None, stream=None) -> PlanInfo:
        """Time every kernel configuration on this matrix and keep the fastest
        (cached per matrix signature for the process)."""
        if x is None:
            x = torch.ones(self.ncol, dtype=self.xy_dtype, device=self.device)
        y = torch.empty(self.nrow, dtype=self.xy_dtype, device=self.device)
        _check(lib().merbit_plan_tune(self._h, _dptr(x), _dptr(y), _stream_ptr(stream)))
        return self.info()

    def configs(self) -> list[tuple[int, int, int, int]]:
        """[(index, kind, block, items_per_thread)] of the kernel configurations
        this plan can run (kind 0 CTA tiles, 1 warp tiles -- needs 16-byte
        aligned arrays --, 3 row groups with items_per_thread lanes per row)."""
        out = []
        for i in range(lib().merbit_num_configs(self.dtype)):
            k, b, p, ok = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
            _check(lib().merbit_config_desc(self.dtype, i, C.byref(k), C.byref(b), C.byref(p)))
            _check(lib().merbit_plan_config_usable(self._h, i, C.byref(ok), _stream_ptr(None)))
            if ok.value:
                out.append((i, k.value, b.value, p.value))
        return out

    def set_config(self, idx: int, stream=None) -> None:
        _check(lib().merbit_plan_set_config(self._h, idx, _stream_ptr(stream)))

    def check(self, stream=None) -> None:
        """Raise MerbitError if a device-side wait of any launch ran out."""
        _check(lib().merbit_plan_check(self._h, _stream_ptr(stream)))

    def selftest_wait(self, which: int = 0, wait_us: int = 2000, stream=None) -> None:
        """Launch one bounded device wait (0: carry, 1: mbarrier) on a flag
        nothing sets; the next check() raises MERBIT_ERR_TIMEOUT."""
        _check(lib().merbit_plan_selftest_wait(self._h, which, wait_us, _stream_ptr(stream)))


class _BatchInfo(C.Structure):
    _fields_ = [("count", C.c_int32), ("k", C.c_int32), ("dtype", C.c_int32),
                ("tile_items", C.c_int32), ("vector_width", C.c_int32),
                ("total_tiles", C.c_int32), ("nnz", C.c_int64), ("algorithmic_bytes", C.c_double),
                ("kernel", C.c_int32), ("variant", C.c_int32)]


class Batch:
    """Many plans times k right-hand sides in one persistent launch
    (merbit_batch_create / merbit_batch_spmm).  Xs[i] (ncol_i, k) and
    Ys[i] (nrow_i, k) are bound at creation; refill them between runs."""

    def __init__(self, plans: list[Plan], Xs: list[torch.Tensor], Ys: list[torch.Tensor],
                 stream=None):
        if not (len(plans) == len(Xs) == len(Ys)) or not plans:
            raise ValueError("plans, Xs and Ys must have the same non-zero length")
        k = Xs[0].shape[1]
        self.plans, self.Xs, self.Ys, self.k = list(plans), list(Xs), list(Ys), k
        n = len(plans)
        hp = (_P * n)(*[p._h for p in plans])
        hx = (_P * n)(*[_dptr(x) for x in Xs])
        hy = (_P * n)(*[_dptr(y) for y in Ys])
        ldx = (C.c_int64 * n)(*[p._mat(x, p.ncol, "X") if x.shape[1] == k else -1
                                for p, x in zip(plans, Xs)])
        ldy = (C.c_int64 * n)(*[p._mat(y, p.nrow, "Y") if y.shape[1] == k else -1
                                for p, y in zip(plans, Ys)])
        ldx = (C.c_int64 * n)(*[max(v, k) if v >= 0 else -1 for v in ldx])
        ldy = (C.c_int64 * n)(*[max(v, k) if v >= 0 else -1 for v in ldy])
        self._h = _P()
        _check(lib().merbit_batch_create(C.byref(self._h), n, hp, k, hx, ldx, hy, ldy,
                                         _stream_ptr(stream)))

    def run(self, alpha: float = 1.0, beta: float = 0.0, stream=None) -> None:
        _check(lib().merbit_batch_spmm(self._h, float(alpha), float(beta), _stream_ptr(stream)))

    def tune(self, stream=None):
        _check(lib().merbit_batch_tune(self._h, _stream_ptr(stream)))
        return self.info()

    def info(self) -> dict:
        i = _BatchInfo()
        _check(lib().merbit_batch_get_info(self._h, C.byref(i)))
        return {f: getattr(i, f) for f, _ in _BatchInfo._fields_}

    def matrix_configs(self) -> list[tuple[int, int, int]]:
        """[(kernel, tile_items, items_per_thread)] of every matrix of the
        batch (merbit_batch_get_matrix_config)."""
        out = []
        for i in range(len(self.plans)):
            k, t, p = C.c_int32(), C.c_int32(), C.c_int32()
            _check(lib().merbit_batch_get_matrix_config(self._h, i, C.byref(k), C.byref(t),
                                                        C.byref(p)))
            out.append((k.value, t.value, p.value))
        return out

    def set_kernel(self, kernel: int, option: int, stream=None) -> None:
        """kernel 0: SpMM kernel with `option` merge items per tile (256,
        512 or an odd tile of k); kernel 1: warp-tile kernel (k = 1) in
        variant `option` (0-9)."""
        _check(lib().merbit_batch_set_kernel(self._h, kernel, option, _stream_ptr(stream)))

    def set_matrix_config(self, index: int, items_per_thread: int, stream=None) -> None:
        """Items per lane (7, 11, 15, 19 or 23, as the variant takes) of
        matrix `index` on the warp-tile kernel (k = 1, aligned arrays)."""
        _check(lib().merbit_batch_set_matrix_config(self._h, index, items_per_thread,
                                                    _stream_ptr(stream)))

    def set_matrix_tile(self, index: int, tile_items: int, stream=None) -> None:
        """Merge items per tile of matrix `index` on the SpMM kernel (k = 4,
        8, 16, 32 at vector width 4): the other tile of the batch's pair."""
        _check(lib().merbit_batch_set_matrix_tile(self._h, index, tile_items,
                                                  _stream_ptr(stream)))

    def close(self) -> None:
        if self._h:
            lib().merbit_batch_destroy(self._h)
            self._h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pagerank(plan: Plan, damp: float = 0.85, tol: float = 1e-10, maxiter: int = 100,
             perrnd: int = 1, teleport: torch.Tensor | None = None,
             x0: torch.Tensor | None = None):
    """Power iteration x <- damp*A*x + (1-damp)*teleport on a square plan,
    with the PARAMETER scaffold's knobs (include/class.cuh:119-146): at most
    `maxiter` rounds of `perrnd` fused steps each; the L1 residual of the
    last step of a round is read on the host once per round and iteration
    stops when it is <= tol.  teleport defaults to the uniform 1/n vector,
    x0 to teleport.  Returns (x, steps, residual per round)."""
    n = plan.nrow
    if plan.ncol != n:
        raise ValueError("pagerank needs a square plan")
    dt = plan.xy_dtype
    if teleport is None:
        teleport = torch.full((n,), 1.0 / max(n, 1), dtype=dt, device=plan.device)
    x = (teleport if x0 is None else x0).clone()
    y = torch.empty_like(x)
    res = torch.zeros(1, dtype=torch.float64, device=plan.device)
    history = []
    steps = 0
    for _ in range(maxiter):
        for _ in range(perrnd):
            plan.pagerank_step(x, teleport, damp, y=y, residual=res)
            x, y = y, x
            steps += 1
        r = float(res.item())
        history.append(r)
        if r <= tol:
            break
    return x, steps, history
