"""Differentiation form on the GPU: the adjoint kernels against the
extended-precision oracle, torch.autograd.gradcheck (FP64 finite
differences) and a dense-matmul reference gradient, on a 2,000-row
instance of the Zipf(1.8) generator."""
import numpy as np
import pytest
import torch

import merbit_b200 as mb
from merbit_b200 import synth
from merbit_b200.autograd import SparseMatrix
from oracle import oracle as O
from tests.helpers import csr_from_lengths, edge_cases, stored_values, to_cuda


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("k", [1, 4, 16])
def test_transpose_spmm_vs_oracle(dtype, k):
    A = synth.workload("zipf_small")
    G = synth.normal(3, A.nrow * k).reshape(A.nrow, k)
    G = G.astype(np.float64 if dtype == "f64" else np.float32)
    rp, col, v = to_cuda(A, dtype)
    plan = mb.Plan(rp, col, v)
    M = SparseMatrix(rp, col, v)
    dX = M.transpose_plan().spmm(torch.from_numpy(G).cuda()).cpu().numpy()
    ref = O.spmm_t(A.row_ptr, A.col, stored_values(A, dtype), G, A.ncol)
    # component-wise: |dX - ref| / sum |a g|
    absA = np.abs(stored_values(A, dtype).astype(np.float64))
    den = O.spmm_t(A.row_ptr, A.col, absA, np.abs(G.astype(np.float64)), A.ncol)
    tol = 1e-13 if dtype == "f64" else 1e-6
    assert (np.abs(dX - ref) / np.maximum(den, 1e-300)).max() <= tol
    del plan


@pytest.mark.gpu
@pytest.mark.parametrize("name,A", edge_cases()[:8], ids=[c[0] for c in edge_cases()[:8]])
def test_transpose_edge_cases(name, A):
    G = synth.normal(5, A.nrow * 2).reshape(A.nrow, 2)
    rp, col, v = to_cuda(A, "f64")
    M = SparseMatrix(rp, col, v, ncol=A.ncol)
    dX = M.transpose_plan().spmm(torch.from_numpy(G).cuda()).cpu().numpy()
    ref = O.spmm_t(A.row_ptr, A.col, A.vals, G, A.ncol)
    den = O.spmm_t(A.row_ptr, A.col, np.abs(A.vals), np.abs(G), A.ncol)
    assert (np.abs(dX - ref) / np.maximum(den, 1e-300)).max() <= 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_dval_vs_oracle(dtype):
    A = synth.workload("zipf_small")
    k = 16
    X = synth.uniform(4, A.ncol * k).reshape(A.ncol, k)
    G = synth.normal(6, A.nrow * k).reshape(A.nrow, k)
    nt = np.float64 if dtype == "f64" else np.float32
    X, G = X.astype(nt), G.astype(nt)
    rp, col, v = to_cuda(A, dtype)
    M = SparseMatrix(rp, col, v)
    d = M.dval(torch.from_numpy(G).cuda(), torch.from_numpy(X).cuda()).cpu().numpy()
    ref = O.dval(A.row_ptr, A.col, G, X)
    den = O.dval(A.row_ptr, A.col, np.abs(G), np.abs(X))
    tol = 1e-13 if dtype == "f64" else 1e-6
    assert (np.abs(d - ref) / np.maximum(den, 1e-300)).max() <= tol


def _diff_instance():
    A = synth.workload("zipf_2k_diff")  # 2,000 rows of the differentiation generator
    return A


@pytest.mark.gpu
def test_gradcheck_fp64_finite_differences_fast_mode():
    """gradcheck on the whole 2,000-row instance (14,006 nonzeros, rows up
    to 960 entries, i.e. spanning several merge-path tiles), with respect to
    the values and X together.  Fast mode compares v^T J u for random u, v
    against FP64 central differences, so every entry takes part."""
    A = _diff_instance()
    assert A.nrow == 2000 and np.diff(A.row_ptr).max() > 512
    rp, col, v = to_cuda(A, "f64")
    vals = v.clone().requires_grad_(True)
    M = SparseMatrix(rp, col, vals, ncol=A.ncol)
    X = torch.from_numpy(synth.uniform(2, A.ncol * 3).reshape(A.ncol, 3)).cuda()
    X.requires_grad_(True)
    assert torch.autograd.gradcheck(lambda w, x: M.matmul(x, vals=w), (vals, X), eps=1e-6,
                                    atol=1e-9, rtol=1e-7, fast_mode=True)


@pytest.mark.gpu
@pytest.mark.parametrize("wrt", ["vals", "X"])
def test_gradcheck_fp64_finite_differences_full_jacobian(wrt):
    """The full Jacobian of the 2,000-row instance against FP64 central
    differences, one input at a time: d Y / d vals (14,006 x 2,000, k = 1)
    and d Y / d X (k = 2).  Y is linear in vals and in X, so a central
    difference has no truncation error at any step; the step 1e-4 keeps its
    rounding error (about max|Y| * 2^-52 / step, max|Y| ~ 30 on rows of up
    to 960 entries) below the 1e-9 absolute tolerance."""
    A = _diff_instance()
    rp, col, v = to_cuda(A, "f64")
    k = 1 if wrt == "vals" else 2
    vals = v.clone().requires_grad_(wrt == "vals")
    M = SparseMatrix(rp, col, vals, ncol=A.ncol)
    X = torch.from_numpy(synth.uniform(2, A.ncol * k).reshape(A.ncol, k)).cuda()
    X.requires_grad_(wrt == "X")
    if wrt == "vals":
        fn, inputs = (lambda w: M.matmul(X, vals=w)), (vals,)
    else:
        fn, inputs = (lambda x: M.matmul(x, vals=vals)), (X,)
    assert torch.autograd.gradcheck(fn, inputs, eps=1e-4, atol=1e-9, rtol=1e-7)


@pytest.mark.gpu
@pytest.mark.parametrize("k", [1, 16])
def test_grad_matches_dense_matmul(k):
    A = _diff_instance()
    rp, col, v = to_cuda(A, "f64")
    vals = v.clone().requires_grad_(True)
    M = SparseMatrix(rp, col, vals, ncol=A.ncol)
    X = torch.from_numpy(synth.uniform(9, A.ncol * k).reshape(A.ncol, k)).cuda()
    X.requires_grad_(True)
    G = torch.from_numpy(synth.normal(10, A.nrow * k).reshape(A.nrow, k)).cuda()
    Xin = X[:, 0] if k == 1 else X
    Gin = G[:, 0] if k == 1 else G
    Y = M.matmul(Xin, vals=vals)
    Y.backward(Gin)
    # dense reference
    rows = torch.from_numpy(np.repeat(np.arange(A.nrow), np.diff(A.row_ptr))).cuda()
    cols = col.long()
    vd = v.clone().requires_grad_(True)
    Xd = X.detach().clone().requires_grad_(True)
    D = torch.zeros(A.nrow, A.ncol, dtype=torch.float64, device="cuda")
    D = D.index_put((rows, cols), vd)
    Yd = D @ (Xd[:, 0] if k == 1 else Xd)
    Yd.backward(Gin)
    assert torch.allclose(Y, Yd, rtol=1e-12, atol=1e-12)
    assert torch.allclose(vals.grad, vd.grad, rtol=1e-12, atol=1e-12)
    assert torch.allclose(X.grad, Xd.grad, rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
def test_backward_deterministic_and_refresh():
    A = _diff_instance()
    rp, col, v = to_cuda(A, "f32")
    M = SparseMatrix(rp, col, v)
    G = torch.from_numpy(synth.normal(1, A.nrow * 4).reshape(A.nrow, 4).astype(np.float32)).cuda()
    d1 = M.transpose_plan().spmm(G).clone()
    d2 = M.transpose_plan().spmm(G).clone()
    assert torch.equal(d1.view(torch.int32), d2.view(torch.int32))
    # values change in place: the transpose values follow
    with torch.no_grad():
        v.mul_(2.0)
    d3 = M.transpose_plan(v).spmm(G)
    assert torch.allclose(d3, 2 * d1, rtol=1e-6, atol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("k,ld", [(1, 1), (2, 3), (3, 3), (8, 12), (16, 17), (32, 32), (40, 44)])
def test_dval_strided_operands(dtype, k, ld):
    """dval with leading dimensions larger than k (vector widths 1, 2 and 4
    are chosen from the alignment) against the oracle."""
    A = synth.workload("zipf_2k_diff")
    nt = np.float64 if dtype == "f64" else np.float32
    tt = torch.float64 if dtype == "f64" else torch.float32
    Xw = torch.from_numpy(synth.uniform(7, A.ncol * ld).reshape(A.ncol, ld).astype(nt)).cuda()
    Gw = torch.from_numpy(synth.normal(8, A.nrow * ld).reshape(A.nrow, ld).astype(nt)).cuda()
    X, G = Xw[:, :k], Gw[:, :k]
    rp, col, v = to_cuda(A, dtype)
    M = SparseMatrix(rp, col, v)
    out = torch.empty(A.nnz, dtype=tt, device="cuda")
    from merbit_b200 import _check, _dptr, _stream_ptr, lib

    _check(lib().merbit_dval(M.plan._h, k, _dptr(G), ld, _dptr(X), ld, _dptr(out),
                             _stream_ptr(None)))
    Gh, Xh = G.cpu().numpy(), X.cpu().numpy()
    ref = O.dval(A.row_ptr, A.col, np.ascontiguousarray(Gh), np.ascontiguousarray(Xh))
    den = O.dval(A.row_ptr, A.col, np.abs(Gh).astype(np.float64), np.abs(Xh).astype(np.float64))
    tol = 1e-13 if dtype == "f64" else 1e-6
    assert (np.abs(out.cpu().numpy() - ref) / np.maximum(den, 1e-300)).max() <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("k", [1, 2, 4, 8, 16, 32])
def test_fused_backward_matches_oracle(dtype, k):
    """merbit_spmm_dval: dX = A^T G and dval from one launch, against the
    oracle, on the power-law instance (long rows span many tiles)."""
    A = synth.workload("zipf_small")
    nt = np.float64 if dtype == "f64" else np.float32
    X = synth.uniform(4, A.ncol * k).reshape(A.ncol, k).astype(nt)
    G = synth.normal(6, A.nrow * k).reshape(A.nrow, k).astype(nt)
    rp, col, v = to_cuda(A, dtype)
    M = SparseMatrix(rp, col, v)
    out = M.backward_fused(torch.from_numpy(G).cuda(), torch.from_numpy(X).cuda())
    assert out is not None
    dX, dv = (t.cpu().numpy() for t in out)
    tol = 1e-13 if dtype == "f64" else 1e-6
    vals = stored_values(A, dtype)
    ref = O.spmm_t(A.row_ptr, A.col, vals, G, A.ncol)
    den = O.spmm_t(A.row_ptr, A.col, np.abs(vals.astype(np.float64)), np.abs(G.astype(np.float64)),
                   A.ncol)
    assert (np.abs(dX - ref) / np.maximum(den, 1e-300)).max() <= tol
    refv = O.dval(A.row_ptr, A.col, G, X)
    denv = O.dval(A.row_ptr, A.col, np.abs(G.astype(np.float64)), np.abs(X.astype(np.float64)))
    assert (np.abs(dv - refv) / np.maximum(denv, 1e-300)).max() <= tol


@pytest.mark.gpu
def test_fused_backward_strided_x_and_fallbacks():
    A = _diff_instance()
    rp, col, v = to_cuda(A, "f32")
    M = SparseMatrix(rp, col, v)
    k = 16
    Xw = torch.from_numpy(synth.uniform(2, A.ncol * 18).reshape(A.ncol, 18).astype(np.float32)).cuda()
    X = Xw[:, 1:17]  # leading dimension 18, offset by one float: narrower vector loads
    G = torch.from_numpy(synth.normal(3, A.nrow * k).reshape(A.nrow, k).astype(np.float32)).cuda()
    from merbit_b200 import _check, _dptr, _stream_ptr, lib

    T = M.transpose_plan()
    dX = torch.empty(A.ncol, k, device="cuda")
    dv = torch.empty(A.nnz, device="cuda")
    _check(lib().merbit_spmm_dval(T._h, k, _dptr(G), k, _dptr(X), 18, _dptr(dX), k, _dptr(dv),
                                  _stream_ptr(None)))
    ref_dx = T.spmm(G)
    ref_dv = M.dval(G, X.contiguous())
    assert torch.allclose(dX, ref_dx, rtol=1e-5, atol=1e-6)
    assert torch.allclose(dv, ref_dv, rtol=1e-5, atol=1e-6)
    # k outside {1,2,4,...,32} and bf16 values are declined
    assert M.backward_fused(G[:, :3].contiguous(), X[:, :3].contiguous()) is None
    rpb, colb, vb = to_cuda(A, "bf16")
    Mb = SparseMatrix(rpb, colb, vb)
    assert Mb.backward_fused(G, X.contiguous()) is None
    # the plan of A itself is not a transpose plan
    assert lib().merbit_spmm_dval(M.plan._h, k, _dptr(G), k, _dptr(X), 18, _dptr(dX), k, _dptr(dv),
                                  _stream_ptr(None)) == 1
