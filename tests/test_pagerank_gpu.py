"""Fused PageRank step: y = damp*A*x + (1-damp)*teleport and the L1
residual sum|y - x| from one SpMV launch (the iteration the reference's
PARAMETER scaffold describes, include/class.cuh:119-146, with RESULT::norm,
include/class.cuh:157).  Checked against the extended-precision oracle for
y, against a float64 sum over the stored y for the residual, and, for the
whole iteration, against a scipy power iteration on the same graph."""
import math

import numpy as np
import pytest
import torch

import merbit_b200 as mb
from merbit_b200 import synth
from oracle import oracle as O
from tests.helpers import csr_from_lengths, edge_cases, stored_values, to_cuda

TOL = {"f64": 1e-13, "f32": 1e-6, "bf16": 1e-6}
XT = {"f64": np.float64, "f32": np.float32, "bf16": np.float32}
DAMP = 0.85


def _step_ref(A, dtype, x, t):
    yo, ya = O.spmm(A.row_ptr, A.col, stored_values(A, dtype), x)
    tt = t.astype(np.float64)
    return DAMP * yo + (1 - DAMP) * tt, DAMP * ya + (1 - DAMP) * np.abs(tt)


def _check_step(A, dtype, plan, x, t):
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    res = torch.zeros(1, dtype=torch.float64, device="cuda")
    y = plan.pagerank_step(xd, td, DAMP, residual=res)
    torch.cuda.synchronize()
    plan.check()
    yh = y.cpu().numpy()
    ref, den = _step_ref(A, dtype, x, t)
    assert O.rel_error(yh, ref, den)[0] <= TOL[dtype]
    want = math.fsum(np.abs(yh.astype(np.float64) - x.astype(np.float64)))
    assert abs(res.item() - want) <= 1e-12 * max(want, 1e-300)
    return y, res.item()


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32", "bf16"])
@pytest.mark.parametrize("workload", ["zipf_small", "laplace2d_small"])
def test_pagerank_step_every_config(dtype, workload):
    A = synth.workload(workload)
    x = synth.uniform(1, A.ncol).astype(XT[dtype])
    t = synth.uniform(2, A.nrow).astype(XT[dtype])
    rp, col, v = to_cuda(A, dtype)
    plan = mb.Plan(rp, col, v)
    cfgs = plan.configs()
    assert {0, 1, 3} <= {k for _, k, _, _ in cfgs}
    for idx, _, _, _ in cfgs:
        plan.set_config(idx)
        _check_step(A, dtype, plan, x, t)


@pytest.mark.gpu
@pytest.mark.parametrize("name,A", [c for c in edge_cases() if c[1].nrow == c[1].ncol],
                         ids=[c[0] for c in edge_cases() if c[1].nrow == c[1].ncol])
def test_pagerank_step_edge_cases(name, A):
    x = synth.uniform(3, A.ncol)
    t = synth.uniform(4, A.nrow)
    rp, col, v = to_cuda(A, "f64")
    _check_step(A, "f64", mb.Plan(rp, col, v), x, t)


@pytest.mark.gpu
def test_pagerank_step_is_deterministic_and_plain_spmv_unchanged():
    A = synth.workload("zipf_small")
    rp, col, v = to_cuda(A, "f64")
    plan = mb.Plan(rp, col, v)
    x = torch.from_numpy(synth.uniform(5, A.ncol)).cuda()
    t = torch.from_numpy(synth.uniform(6, A.nrow)).cuda()
    res = torch.zeros(1, dtype=torch.float64, device="cuda")
    outs = []
    for _ in range(3):
        y = plan.pagerank_step(x, t, DAMP, residual=res)
        outs.append((y.clone(), res.clone()))
    for y, r in outs[1:]:
        assert torch.equal(y.view(torch.int64), outs[0][0].view(torch.int64))
        assert torch.equal(r.view(torch.int64), outs[0][1].view(torch.int64))
    # without a residual the step is y = damp*Ax + (1-damp)*t all the same
    y2 = plan.pagerank_step(x, t, DAMP)
    assert torch.equal(y2, outs[0][0])
    # and the plain product in between is untouched by the fused launches
    yo, ya = O.spmm(A.row_ptr, A.col, A.vals, x.cpu().numpy())
    assert O.rel_error(plan.spmv(x).cpu().numpy(), yo, ya)[0] <= TOL["f64"]
    plan.check()


def _transition(A):
    """A graph's column-stochastic transition matrix as CSR of A^T with
    values 1/outdeg (the loader's weights, src/class.cu:2-34)."""
    rows = np.repeat(np.arange(A.nrow), np.diff(A.row_ptr))
    outdeg = np.diff(A.row_ptr).astype(np.float64)
    order = np.lexsort((rows, A.col))
    r_t, c_t = A.col[order], rows[order]
    vals = 1.0 / outdeg[c_t]
    rp = np.zeros(A.ncol + 1, np.int64)
    np.add.at(rp, r_t + 1, 1)
    rp = np.cumsum(rp).astype(np.int32)
    return synth.CSR(rp, c_t.astype(np.int32), vals, A.nrow, "transition")


@pytest.mark.gpu
@pytest.mark.parametrize("perrnd", [1, 4])
def test_pagerank_converges_to_scipy_power_iteration(perrnd):
    import scipy.sparse as sp

    P = _transition(synth.workload("zipf_small"))
    n = P.nrow
    rp, col, v = to_cuda(P, "f64")
    plan = mb.Plan(rp, col, v)
    x, steps, hist = mb.pagerank(plan, damp=DAMP, tol=1e-12, maxiter=400, perrnd=perrnd)
    assert hist[-1] <= 1e-12 and steps % perrnd == 0
    M = sp.csr_matrix((P.vals, P.col, P.row_ptr), shape=(n, n))
    xr = np.full(n, 1.0 / n)
    for _ in range(steps):
        xr = DAMP * (M @ xr) + (1 - DAMP) / n
    assert np.abs(x.cpu().numpy() - xr).sum() <= 1e-12
    # residual history is that of the iterates
    assert all(h > 0 for h in hist[:-1])


@pytest.mark.gpu
def test_pagerank_step_argument_errors():
    A = csr_from_lengths([3] * 100, ncol=50)
    rp, col, v = to_cuda(A, "f64")
    plan = mb.Plan(rp, col, v, ncol=50)
    x = torch.ones(50, dtype=torch.float64, device="cuda")
    t = torch.ones(100, dtype=torch.float64, device="cuda")
    with pytest.raises(mb.MerbitError):  # not square
        plan.pagerank_step(x, t)
    B = csr_from_lengths([3] * 100, ncol=100)
    plan = mb.Plan(*to_cuda(B, "f64"))
    x = torch.ones(100, dtype=torch.float64, device="cuda")
    with pytest.raises(mb.MerbitError):  # y aliases x
        plan.pagerank_step(x, t, y=x)
    with pytest.raises(mb.MerbitError):
        plan.pagerank_step(x, t, damp=1.5)
