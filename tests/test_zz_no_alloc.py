"""merbit_spmv_noalloc: the SpMV entry point that allocates no device memory.

It exists for callers that cannot allocate on the call path (hosts whose
device memory belongs to their own pool allocator, loops that cannot take
cudaMalloc's implicit sync).  Its scratch is a fixed file-scope device array,
so it is checked here against the plan-based entry point (merbit_plan_create
+ merbit_spmv) on two calls in a row, with the same component-wise tolerance
as the other SpMV tests: on a power-law matrix, rows spanning many tiles,
arrays that are not 16-byte aligned, the largest matrix the array admits,
and after a device-side wait of an earlier call ran out.

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import merbit_b200 as mb
from merbit_b200 import synth
from tests.helpers import csr_from_lengths, to_cuda

TOL = {"f64": 1e-13, "f32": 1e-6, "bf16": 1e-6}
DT = {"f64": mb.F64, "f32": mb.F32, "bf16": mb.BF16}


def _abs_rowsum(A, x):
    """sum_j |a_ij x_j| per row, the denominator of the component-wise error."""
    rows = np.repeat(np.arange(A.nrow), np.diff(A.row_ptr))
    return np.bincount(rows, weights=np.abs(A.vals) * np.abs(x[A.col]), minlength=A.nrow)


MAX_ITEMS = 32768 * 1792  # nrow + nnz the fixed scratch admits


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


def _check_against_plan(A, dtype, rp, col, v, calls=2):
    """Two no-alloc calls in a row against the plan entry point, each within
    the component-wise tolerance, and the device status clean after them."""
    xt = torch.float64 if dtype == "f64" else torch.float32
    xh = synth.uniform(11, A.ncol).astype(np.float64 if dtype == "f64" else np.float32)
    x = torch.from_numpy(xh).cuda()
    plan = mb.Plan(rp, col, v, ncol=A.ncol)
    y_ref = plan.spmv(x).cpu().numpy().astype(np.float64)
    plan.close()
    stored = v.double().cpu().numpy() if dtype != "f64" else A.vals
    Ab = synth.CSR(A.row_ptr, A.col, stored, A.ncol)
    denom = np.maximum(_abs_rowsum(Ab, xh.astype(np.float64)), 1e-300)
    for call in range(calls):
        y = torch.full((A.nrow,), float("nan"), dtype=xt, device="cuda")
        assert _call(A, rp, col, v, dtype, x, y) == 0, mb.lib().merbit_last_error_detail()
        torch.cuda.synchronize()
        err = np.abs(y.cpu().numpy().astype(np.float64) - y_ref) / denom
        assert np.isfinite(err).all()
        assert err.max() <= TOL[dtype], (call, err.max())
    assert mb.lib().merbit_spmv_noalloc_check(None) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("lengths", [[100_000], [0, 3, 2_000_000, 0, 5] + [7] * 1000],
                         ids=["one_row_56_tiles", "row_of_1117_tiles"])
def test_noalloc_rows_spanning_many_tiles(lengths):
    """Rows whose merge items cover many 1,792-item tiles finish through the
    look-back over the carry slots of the fixed array."""
    A = csr_from_lengths(lengths, ncol=2_500_000, seed=7)
    rp, col, v = to_cuda(A, "f64")
    _check_against_plan(A, "f64", rp, col, v)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_noalloc_on_arrays_off_16_byte_boundaries(dtype):
    """col_idx and vals as views one element past an aligned base: the
    call takes the non-vectorized loads."""
    A = synth.zipf(20_000, 1.8, 5_000, 0.1, seed=8)
    rp, col, v = to_cuda(A, dtype)
    col_off = torch.empty(A.nnz + 1, dtype=col.dtype, device="cuda")[1:]
    v_off = torch.empty(A.nnz + 1, dtype=v.dtype, device="cuda")[1:]
    col_off.copy_(col)
    v_off.copy_(v)
    assert col_off.data_ptr() % 16 != 0 and v_off.data_ptr() % 16 != 0
    _check_against_plan(A, dtype, rp, col_off, v_off)


@pytest.mark.gpu
def test_noalloc_at_the_size_limit():
    """nrow + nnz exactly at the limit of the fixed array works; one more
    merge item is refused before any device work."""
    nrow = 720_256
    nnz = MAX_ITEMS - nrow
    rng = np.random.default_rng(12)
    cuts = np.sort(rng.integers(0, nnz + 1, nrow - 1))
    rp = np.concatenate([[0], cuts, [nnz]]).astype(np.int32)
    col = rng.integers(0, nrow, nnz, dtype=np.int32)
    vals = rng.standard_normal(nnz)
    A = synth.CSR(rp, col, vals, nrow)
    d_rp, d_col, d_v = to_cuda(A, "f64")
    _check_against_plan(A, "f64", d_rp, d_col, d_v)
    y = torch.empty(nrow + 1, dtype=torch.float64, device="cuda")
    x = torch.zeros(nrow, dtype=torch.float64, device="cuda")
    rc = mb.lib().merbit_spmv_noalloc(nrow + 1, nrow, nnz, C.c_void_p(d_rp.data_ptr()),
                                      C.c_void_p(d_col.data_ptr()), C.c_void_p(d_v.data_ptr()),
                                      mb.F64, 1.0, C.c_void_p(x.data_ptr()), 0.0,
                                      C.c_void_p(y.data_ptr()), None)
    assert rc == 1 and b"scratch limit" in mb.lib().merbit_last_error_detail()


@pytest.mark.gpu
@pytest.mark.parametrize("which", [0, 1], ids=["carry_wait", "mbarrier_wait"])
def test_noalloc_timeout_is_reported_and_does_not_spoil_later_calls(which):
    """A wait that runs out (the self-test form: a flag nothing sets, a 2 ms
    limit) is reported once by merbit_spmv_noalloc_check, and the calls made
    after it still produce correct rows spanning many tiles."""
    L = mb.lib()
    A = csr_from_lengths([0, 300_000, 4, 0, 90_000] + [3] * 5000, ncol=400_000, seed=9)
    rp, col, v = to_cuda(A, "f64")
    assert L.merbit_spmv_noalloc_check(None) == 0
    assert L.merbit_spmv_noalloc_selftest_wait(which, 2000, None) == 0
    torch.cuda.synchronize()
    xh = synth.uniform(13, A.ncol)
    x = torch.from_numpy(xh).cuda()
    plan = mb.Plan(rp, col, v, ncol=A.ncol)
    y_ref = plan.spmv(x).cpu().numpy()
    denom = np.maximum(_abs_rowsum(A, xh), 1e-300)
    for _ in range(2):
        y = torch.full((A.nrow,), float("nan"), dtype=torch.float64, device="cuda")
        assert _call(A, rp, col, v, "f64", x, y) == 0
        torch.cuda.synchronize()
        assert (np.abs(y.cpu().numpy() - y_ref) / denom).max() <= TOL["f64"]
    assert L.merbit_spmv_noalloc_check(None) == 5  # MERBIT_ERR_TIMEOUT, from the self-test
    assert b"wait ran out" in L.merbit_last_error_detail()
    assert L.merbit_spmv_noalloc_check(None) == 0  # cleared by the read


def test_noalloc_limit_and_selftest_arguments_need_no_gpu():
    """One merge item past the limit is refused before any device work, as
    are bad self-test arguments."""
    L = mb.lib()
    rc = L.merbit_spmv_noalloc(1, 1, MAX_ITEMS, C.c_void_p(16), C.c_void_p(16), C.c_void_p(16),
                               mb.F64, 1.0, C.c_void_p(16), 0.0, C.c_void_p(16), None)
    assert rc == 1 and b"scratch limit" in L.merbit_last_error_detail()
    assert L.merbit_spmv_noalloc_selftest_wait(2, 100, None) == 1
    assert L.merbit_spmv_noalloc_selftest_wait(0, 0, None) == 1
