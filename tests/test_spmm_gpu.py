"""SpMM (k right-hand sides) and batched SpMM parity on the GPU.

Tolerances as for the SpMV (component-wise vs the extended-precision
oracle): 1e-13 for f64, 1e-6 for f32 / bf16 values with f32 X.
"""
import numpy as np
import pytest
import torch

import merbit_b200 as mb
from merbit_b200 import synth
from oracle import oracle as O
from tests.helpers import csr_from_lengths, edge_cases, stored_values, to_cuda

TOL = {"f64": 1e-13, "f32": 1e-6, "bf16": 1e-6}


def _X(ncol, k, dtype, seed=3):
    x = synth.uniform(seed, ncol * k).reshape(ncol, k)
    return x.astype(np.float64 if dtype == "f64" else np.float32)


def _check(A, dtype, Y, X, alpha=1.0):
    yo, ya = O.spmm(A.row_ptr, A.col, stored_values(A, dtype), X, k=X.shape[1], alpha=alpha)
    e = np.abs(Y.astype(np.float64) - yo) / np.maximum(ya, 1e-300)
    return float(e.max()) if e.size else 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32", "bf16"])
@pytest.mark.parametrize("k", [1, 2, 3, 4, 8, 16, 32, 40])
def test_spmm_vs_oracle(dtype, k):
    A = synth.workload("zipf_small")
    X = _X(A.ncol, k, dtype)
    rp, col, v = to_cuda(A, dtype)
    plan = mb.Plan(rp, col, v)
    Y = plan.spmm(torch.from_numpy(X).cuda())
    torch.cuda.synchronize()
    assert _check(A, dtype, Y.cpu().numpy(), X) <= TOL[dtype]


@pytest.mark.gpu
@pytest.mark.parametrize("k", [1, 4, 32])
@pytest.mark.parametrize("name,A", edge_cases(), ids=[c[0] for c in edge_cases()])
def test_spmm_edge_cases(name, A, k):
    X = _X(A.ncol, k, "f32")
    rp, col, v = to_cuda(A, "f32")
    plan = mb.Plan(rp, col, v, ncol=A.ncol)
    Y = plan.spmm(torch.from_numpy(X).cuda())
    torch.cuda.synchronize()
    assert _check(A, "f32", Y.cpu().numpy(), X) <= TOL["f32"]


@pytest.mark.gpu
def test_spmm_strided_and_alpha_beta():
    A = synth.workload("laplace2d_small")
    k, ld = 8, 13
    Xfull = _X(A.ncol, ld, "f64")
    Xd = torch.from_numpy(Xfull).cuda()[:, :k]
    Y0 = torch.from_numpy(_X(A.nrow, ld, "f64", seed=8)).cuda()
    Y = Y0.clone()
    rp, col, v = to_cuda(A, "f64")
    mb.Plan(rp, col, v).spmm(Xd, Y[:, :k], alpha=0.5, beta=-1.5)
    yo, ya = O.spmm(A.row_ptr, A.col, A.vals, np.ascontiguousarray(Xfull[:, :k]), k=k, alpha=0.5)
    ref = yo - 1.5 * Y0.cpu().numpy()[:, :k]
    got = Y.cpu().numpy()
    assert np.abs(got[:, :k] - ref).max() / np.abs(ref).max() < 1e-13
    assert np.array_equal(got[:, k:], Y0.cpu().numpy()[:, k:])  # untouched columns


@pytest.mark.gpu
@pytest.mark.parametrize("k", [1, 4, 8, 32])
def test_batch_vs_oracle_and_graph_replay(k):
    specs = synth.batch_rmat_specs(12, seed=2, nmin=200, nmax=20_000, dmin=4, dmax=40)
    mats = [synth.rmat(n, d, seed=s) for n, d, s in specs]
    mats.append(csr_from_lengths([0, 3000, 0, 2, 9000, 1], ncol=12000, seed=4))  # long rows
    plans, Xs, Ys, Xh = [], [], [], []
    for A in mats:
        rp, col, v = to_cuda(A, "f32")
        plans.append(mb.Plan(rp, col, v, ncol=A.ncol))
        X = _X(A.ncol, k, "f32", seed=len(Xs) + 1)
        Xh.append(X)
        Xs.append(torch.from_numpy(X).cuda())
        Ys.append(torch.full((A.nrow, k), float("nan"), dtype=torch.float32, device="cuda"))
    b = mb.Batch(plans, Xs, Ys)
    b.tune()
    b.run()
    torch.cuda.synchronize()
    for A, X, Y in zip(mats, Xh, Ys):
        assert _check(A, "f32", Y.cpu().numpy(), X) <= TOL["f32"]
    # capture one launch in a CUDA graph, refill the inputs, replay
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        b.run(stream=s)
    for rep in range(3):
        for i, A in enumerate(mats):
            Xh[i] = _X(A.ncol, k, "f32", seed=100 * rep + i)
            Xs[i].copy_(torch.from_numpy(Xh[i]))
            Ys[i].fill_(float("nan"))
        g.replay()
        torch.cuda.synchronize()
        for A, X, Y in zip(mats, Xh, Ys):
            assert _check(A, "f32", Y.cpu().numpy(), X) <= TOL["f32"]
    info = b.info()
    assert info["count"] == len(mats) and info["k"] == k


@pytest.mark.gpu
def test_spmm_deterministic():
    A = csr_from_lengths([0, 70_000, 5, 0, 90_000, 1] * 2, ncol=200_000, seed=9)
    X = torch.from_numpy(_X(A.ncol, 8, "f32")).cuda()
    rp, col, v = to_cuda(A, "f32")
    plan = mb.Plan(rp, col, v, ncol=A.ncol)
    ys = [plan.spmm(X).clone() for _ in range(10)]
    for y in ys[1:]:
        assert torch.equal(y.view(torch.int32), ys[0].view(torch.int32))


def _offset(t: torch.Tensor) -> torch.Tensor:
    """The same values at an address 4 (int32/f32) or 8 (f64) bytes past a
    16-byte boundary, as a caller's slice of a larger buffer would be."""
    buf = torch.empty(t.numel() + 1, dtype=t.dtype, device=t.device)
    out = buf[1:]
    out.copy_(t)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32", "bf16"])
def test_spmm_and_batch_on_offset_arrays(dtype):
    """row_ptr, col_idx and vals that do not start on a 16-byte boundary:
    the SpMM stages them with plain loads instead of bulk copies (which need
    16-byte aligned addresses), alone and inside a batch."""
    mats = [synth.workload("zipf_small"),
            csr_from_lengths([0, 3000, 0, 2, 9000, 1, 7, 0], ncol=12000, seed=4)]
    plans, keep = [], []
    for A in mats:
        rp, col, v = to_cuda(A, dtype)
        rp, col, v = _offset(rp), _offset(col), _offset(v)
        keep.append((rp, col, v))
        plans.append(mb.Plan(rp, col, v, ncol=A.ncol))
        assert not plans[-1].info().vectorized
    for k in (1, 3, 8):
        for A, plan in zip(mats, plans):
            X = _X(A.ncol, k, dtype)
            Y = plan.spmm(torch.from_numpy(X).cuda())
            torch.cuda.synchronize()
            assert _check(A, dtype, Y.cpu().numpy(), X) <= TOL[dtype], (k, A.name)
    Xh = [_X(A.ncol, 4, dtype, seed=20 + i) for i, A in enumerate(mats)]
    Xs = [torch.from_numpy(X).cuda() for X in Xh]
    Ys = [torch.full((A.nrow, 4), float("nan"), dtype=Xs[0].dtype, device="cuda") for A in mats]
    b = mb.Batch(plans, Xs, Ys)
    b.run()
    torch.cuda.synchronize()
    for A, X, Y in zip(mats, Xh, Ys):
        assert _check(A, dtype, Y.cpu().numpy(), X) <= TOL[dtype], A.name
    b.close()
