"""merbit_spmv_noalloc: the SpMV entry point that allocates no device memory.

It exists for callers that cannot allocate on the call path (code running
under CUDA stream capture, hosts whose device memory belongs to their own
pool allocator, loops that cannot take cudaMalloc's implicit sync).  Its
scratch is a fixed file-scope device array, so it is checked here against
the plan-based entry point (merbit_plan_create + merbit_spmv) on two calls in
a row, with the same component-wise tolerance as the other SpMV tests.

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import merbit_b200 as mb
from merbit_b200 import synth
from tests.helpers import to_cuda

TOL = {"f64": 1e-13, "f32": 1e-6, "bf16": 1e-6}
DT = {"f64": mb.F64, "f32": mb.F32, "bf16": mb.BF16}


def _abs_rowsum(A, x):
    """sum_j |a_ij x_j| per row, the denominator of the component-wise error."""
    rows = np.repeat(np.arange(A.nrow), np.diff(A.row_ptr))
    return np.bincount(rows, weights=np.abs(A.vals) * np.abs(x[A.col]), minlength=A.nrow)


def _call(A, rp, col, v, dtype, x, y, alpha=1.0, beta=0.0):
    s = torch.cuda.current_stream().cuda_stream
    return mb.lib().merbit_spmv_noalloc(A.nrow, A.ncol, A.nnz, C.c_void_p(rp.data_ptr()),
                                        C.c_void_p(col.data_ptr()), C.c_void_p(v.data_ptr()),
                                        DT[dtype], alpha, C.c_void_p(x.data_ptr()), beta,
                                        C.c_void_p(y.data_ptr()), C.c_void_p(s))


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32", "bf16"])
def test_noalloc_matches_plan_entry_point(dtype):
    A = synth.zipf(40_000, 1.8, 20_000, 0.1, seed=4)
    xt = torch.float64 if dtype == "f64" else torch.float32
    xh = synth.uniform(9, A.ncol).astype(np.float64 if dtype == "f64" else np.float32)
    rp, col, v = to_cuda(A, dtype)
    x = torch.from_numpy(xh).cuda()
    plan = mb.Plan(rp, col, v, ncol=A.ncol)
    y_ref = plan.spmv(x).cpu().numpy().astype(np.float64)
    stored = v.double().cpu().numpy() if dtype == "bf16" else A.vals
    Ab = synth.CSR(A.row_ptr, A.col, stored, A.ncol)
    denom = np.maximum(_abs_rowsum(Ab, xh.astype(np.float64)), 1e-300)
    for call in range(2):
        y = torch.full((A.nrow,), float("nan"), dtype=xt, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        assert _call(A, rp, col, v, dtype, x, y) == 0, mb.lib().merbit_last_error_detail()
        torch.cuda.synchronize()
        if call == 1:
            # after the first call's one-time set-up nothing is allocated
            # (free memory can only grow: the library's memory pool may hand
            # blocks of destroyed plans back to the device at a synchronization)
            assert torch.cuda.mem_get_info()[0] >= free_before
        err = np.abs(y.cpu().numpy().astype(np.float64) - y_ref) / denom
        assert np.isfinite(err).all()
        assert err.max() <= TOL[dtype], (call, err.max())


@pytest.mark.gpu
def test_noalloc_alpha_beta_two_calls():
    A = synth.workload("laplace2d_small")
    xh = synth.uniform(3, A.ncol)
    rp, col, v = to_cuda(A, "f64")
    x = torch.from_numpy(xh).cuda()
    y0 = torch.from_numpy(synth.uniform(5, A.nrow)).cuda()
    plan = mb.Plan(rp, col, v, ncol=A.ncol)
    y_ref = plan.spmv(x, y0.clone(), alpha=0.5, beta=-2.0).cpu().numpy()
    denom = np.maximum(0.5 * _abs_rowsum(A, xh) + 2.0 * np.abs(y0.cpu().numpy()), 1e-300)
    for _ in range(2):
        y = y0.clone()
        assert _call(A, rp, col, v, "f64", x, y, alpha=0.5, beta=-2.0) == 0
        torch.cuda.synchronize()
        assert (np.abs(y.cpu().numpy() - y_ref) / denom).max() <= TOL["f64"]


def test_noalloc_rejects_oversized_matrix():
    """Sizes beyond the fixed scratch are refused before any device work."""
    L = mb.lib()
    rc = L.merbit_spmv_noalloc(40_000_000, 40_000_000, 30_000_000, C.c_void_p(16),
                               C.c_void_p(16), C.c_void_p(16), mb.F64, 1.0, C.c_void_p(16), 0.0,
                               C.c_void_p(16), None)
    assert rc == 1
    assert b"scratch limit" in L.merbit_last_error_detail()
