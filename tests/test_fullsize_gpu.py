"""Parity at the full sizes of the five benchmark configurations.

Each matrix is built by its own seeded generator at its benchmark size and
run through the configuration the tuner picks (the one the bench times):

  * Laplacian 256x256, FP64: against the oracle and against the reference
    merbit_kernel<double,256,14> run on this GPU (oracle/_ref);
  * Zipf(1.8) 2M rows, FP64: against the reference merbit_kernel (the
    oracle comparison is in test_spmv_gpu.py); FP32 and BF16 values with x
    FP32: against the oracle on the stored inputs;
  * 27-point stencil 160^3 (4,096,000 rows, 109,215,352 nonzeros) with
    values stored FP64, FP32 and BF16 and x FP32: against the oracle on the
    stored inputs;
  * 128 R-MAT matrices in one graph-captured batched launch, FP32 values,
    k = 1, 4, 8 and 32 right-hand sides;
  * Zipf(1.8) 1M rows, FP32, k = 16: the forward product and the fused
    backward (dX = A^T G and dval = G[row] . X[col]).

Tolerances (component-wise, e_i = |y_i - y*_i| / sum_j |a_ij x_j|):
1e-13 for FP64 against the oracle, 1e-12 against the reference kernel
(which finishes CTA-boundary rows with float atomics), 1e-6 for the
FP32/BF16 precision, batched and differentiation forms.
"""
import functools

import numpy as np
import pytest
import torch

import merbit_b200 as mb
from merbit_b200 import synth
from merbit_b200.autograd import SparseMatrix
from oracle import oracle as O
from tests.helpers import stored_values, to_cuda

TOL = {"f64": 1e-13, "f32": 1e-6, "bf16": 1e-6}
TOL_REF_KERNEL = 1e-12


@functools.lru_cache(maxsize=1)
def _stencil():
    return synth.workload("stencil27_160")


@functools.lru_cache(maxsize=1)
def _rmat_batch():
    specs = synth.batch_rmat_specs(128, seed=2)
    return [synth.rmat(n, d, seed=sd) for n, d, sd in specs]


def _tuned_spmv(A, dtype, x):
    rp, col, v = to_cuda(A, dtype)
    plan = mb.Plan(rp, col, v, ncol=A.ncol)
    xd = torch.from_numpy(x).cuda()
    plan.tune(xd)
    y = plan.spmv(xd)
    torch.cuda.synchronize()
    plan.check()
    out = y.cpu().numpy().astype(np.float64)
    plan.close()
    return out


def _reference_kernel_y(A, x):
    """y of the reference merbit_kernel<double,256,14> with its own TILE plan."""
    R = O.ref()
    if R is None:
        pytest.skip("reference harness oracle/_ref not built")
    rp, col, v = to_cuda(A, "f64")
    T, Ln = mb.tile_dims(A.nrow, A.nnz, 14)
    tx = torch.zeros(T + 1, dtype=torch.int32, device="cuda")
    ty = torch.zeros(T + 1, dtype=torch.int32, device="cuda")
    desc = torch.zeros(max(Ln, 1), dtype=torch.int32, device="cuda")
    assert R.ref_tile_build(14, rp.data_ptr(), A.nrow, A.nnz, tx.data_ptr(), ty.data_ptr(),
                            desc.data_ptr()) == 0
    xd = torch.from_numpy(x).cuda()
    yr = torch.zeros(A.nrow, dtype=torch.float64, device="cuda")
    zr = torch.zeros(A.nrow, dtype=torch.float64, device="cuda")
    assert R.ref_merbit_spmv(0, col.data_ptr(), v.data_ptr(), A.nrow, A.nnz, tx.data_ptr(),
                             ty.data_ptr(), desc.data_ptr(), 1.0, xd.data_ptr(), yr.data_ptr(),
                             zr.data_ptr(), None) == 0
    torch.cuda.synchronize()
    return yr.cpu().numpy()


@pytest.mark.gpu
def test_laplace2d_256_f64_vs_oracle_and_reference_kernel():
    A = synth.workload("laplace2d_256")
    assert (A.nrow, A.nnz) == (65_536, 326_656)
    x = synth.workload_x("laplace2d_256", A.ncol)
    y = _tuned_spmv(A, "f64", x)
    yo, ya = O.spmm(A.row_ptr, A.col, A.vals, x)
    assert O.rel_error(y, yo, ya)[0] <= TOL["f64"]
    yr = _reference_kernel_y(A, x)
    assert O.rel_error(y, yr, ya)[0] <= TOL_REF_KERNEL
    # the stencil's values and x are exact in double: 4x - neighbours
    assert np.abs(y - yo).max() <= 1e-14


@pytest.mark.gpu
def test_zipf_2m_f64_vs_reference_kernel():
    A = synth.workload("zipf_2m")
    x = synth.workload_x("zipf_2m", A.ncol)
    y = _tuned_spmv(A, "f64", x)
    yr = _reference_kernel_y(A, x)
    _, ya = O.spmm(A.row_ptr, A.col, A.vals, x)
    assert O.rel_error(y, yr, ya)[0] <= TOL_REF_KERNEL


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f32", "bf16"])
def test_zipf_2m_precision_form_vs_oracle(dtype):
    """The precision form on the headline matrix (values stored FP32/BF16,
    x FP32): within 1e-6 of the FP64 oracle on the stored inputs."""
    A = synth.workload("zipf_2m")
    x = synth.workload_x("zipf_2m", A.ncol).astype(np.float32)
    y = _tuned_spmv(A, dtype, x)
    yo, ya = O.spmm(A.row_ptr, A.col, stored_values(A, dtype), x)
    emax, emed = O.rel_error(y, yo, ya)
    assert emax <= TOL[dtype], (emax, emed)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32", "bf16"])
def test_stencil27_160_vs_oracle(dtype):
    """The precision form on the 27-point stencil: values stored FP32/BF16,
    x FP32, compensated FP32 accumulation, within 1e-6 of the FP64 oracle on
    the stored inputs; plus the plain FP64 run at 1e-13."""
    A = _stencil()
    assert (A.nrow, A.nnz) == (4_096_000, 109_215_352)
    x = synth.workload_x("stencil27_160", A.ncol)
    x = x if dtype == "f64" else x.astype(np.float32)
    y = _tuned_spmv(A, dtype, x)
    yo, ya = O.spmm(A.row_ptr, A.col, stored_values(A, dtype), x)
    emax, emed = O.rel_error(y, yo, ya)
    assert emax <= TOL[dtype], (emax, emed)


@pytest.mark.gpu
@pytest.mark.parametrize("k", [1, 4, 8, 32])
def test_rmat_batch128_vs_oracle(k):
    """128 R-MAT matrices times k FP32 right-hand sides in one persistent
    launch, tuned, captured in a CUDA graph and replayed twice (the second
    replay must give the same bits)."""
    mats = _rmat_batch()
    assert len(mats) == 128
    plans, Xd, Yd = [], [], []
    for i, A in enumerate(mats):
        rp, col, v = to_cuda(A, "f32")
        plans.append(mb.Plan(rp, col, v, ncol=A.ncol))
        X = synth.uniform(100 + i, A.ncol * k).astype(np.float32).reshape(A.ncol, k)
        Xd.append(torch.from_numpy(X).cuda())
        Yd.append(torch.full((A.nrow, k), float("nan"), dtype=torch.float32, device="cuda"))
    batch = mb.Batch(plans, Xd, Yd)
    batch.tune()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        batch.run(stream=s)
    g.replay()
    torch.cuda.synchronize()
    first = [y.clone() for y in Yd]
    g.replay()
    torch.cuda.synchronize()
    for p in plans:
        p.check()
    worst = 0.0
    for i, A in enumerate(mats):
        assert torch.equal(first[i], Yd[i]), i
        X = Xd[i].cpu().numpy()
        yo, ya = O.spmm(A.row_ptr, A.col, A.vals.astype(np.float32), X, k=k)
        e = O.rel_error(Yd[i].cpu().numpy(), yo, ya)[0]
        worst = max(worst, e)
        assert e <= TOL["f32"], (i, A.nrow, A.nnz, e)
    del g
    batch.close()


@pytest.mark.gpu
def test_zipf_1m_diff_k16_forward_and_fused_backward():
    """The differentiation form at its benchmark size: Y = A X and, from one
    launch on the transpose plan, dX = A^T G and dval = G[row] . X[col]."""
    A = synth.workload("zipf_1m_diff")
    k = 16
    X = synth.workload_x("zipf_1m_diff", A.ncol, k).astype(np.float32)
    G = synth.normal(3, A.nrow * k).astype(np.float32).reshape(A.nrow, k)
    rp, col, v = to_cuda(A, "f32")
    M = SparseMatrix(rp, col, v, ncol=A.ncol)
    Xd, Gd = torch.from_numpy(X).cuda(), torch.from_numpy(G).cuda()
    Y = M.plan.spmm(Xd).cpu().numpy()
    fused = M.backward_fused(Gd, Xd)
    assert fused is not None, "the fused backward takes FP32 at k = 16"
    dX, dval = (t.cpu().numpy().astype(np.float64) for t in fused)
    torch.cuda.synchronize()
    M.plan.check()
    v32 = A.vals.astype(np.float32)
    yo, ya = O.spmm(A.row_ptr, A.col, v32, X, k=k)
    assert O.rel_error(Y, yo, ya)[0] <= TOL["f32"]
    absv = np.abs(v32.astype(np.float64))
    dxo = O.spmm_t(A.row_ptr, A.col, v32, G, A.ncol)
    dxa = O.spmm_t(A.row_ptr, A.col, absv, np.abs(G.astype(np.float64)), A.ncol)
    assert O.rel_error(dX, dxo, dxa)[0] <= TOL["f32"]
    dvo = O.dval(A.row_ptr, A.col, G, X)
    dva = O.dval(A.row_ptr, A.col, np.abs(G.astype(np.float64)), np.abs(X.astype(np.float64)))
    assert O.rel_error(dval, dvo, dva)[0] <= TOL["f32"]
