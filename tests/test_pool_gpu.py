"""Device memory of the library: every plan buffer comes from one stream-
ordered pool per device that keeps released blocks mapped (up to 64 MiB).
Building and destroying plans in a loop must neither leak nor hand a live
plan's blocks to a new one."""
from __future__ import annotations

import numpy as np
import pytest

import merbit_b200 as mb
from merbit_b200 import synth
from merbit_b200.autograd import SparseMatrix
from oracle import oracle as O
from tests.helpers import to_cuda

KEEP = 64 << 20  # blocks the pool may keep mapped after release


def _rel_err(y, y_ref, yabs):
    return np.abs(y - y_ref) / np.maximum(yabs, 1e-300)


@pytest.mark.gpu
def test_create_destroy_loop_does_not_leak():
    import torch

    A = synth.zipf(200_000, 1.8, 50_000, 0.1, seed=21)
    rp, col, v = to_cuda(A, "f64")
    x = torch.from_numpy(synth.uniform(1, A.ncol)).cuda()
    # warm: first plan, first pool blocks
    p = mb.Plan(rp, col, v, ncol=A.ncol)
    p.spmv(x)
    p.close()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for i in range(40):
        if i % 10 == 0:  # adjoint buffers (nnz-sized) through the pool too
            S = SparseMatrix(rp, col, v, ncol=A.ncol)
            S.transpose_plan().close()
            S.plan.close()
        p = mb.Plan(rp, col, v, ncol=A.ncol)
        y = p.spmv(x)
        p.close()
        del y
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free0 - free1 <= KEEP + (8 << 20), (free0, free1)
    # emptied, the pool holds nothing: every block of the 40 plans came back
    mb.release_cached_memory()
    free2 = torch.cuda.mem_get_info()[0]
    assert free2 >= free1
    assert free0 - free2 <= 4 << 20, (free0, free2)


@pytest.mark.gpu
def test_reused_blocks_do_not_disturb_live_plans():
    import torch

    mats = [synth.zipf(30_000 + 7_000 * i, 1.8, 10_000, 0.1, seed=30 + i) for i in range(3)]
    xs = [synth.uniform(40 + i, A.ncol) for i, A in enumerate(mats)]
    refs = [O.spmm(A.row_ptr, A.col, A.vals, x) for A, x in zip(mats, xs)]
    dev = [to_cuda(A, "f64") for A in mats]
    xd = [torch.from_numpy(x).cuda() for x in xs]
    a = mb.Plan(*dev[0], ncol=mats[0].ncol)
    b = mb.Plan(*dev[1], ncol=mats[1].ncol)
    ya = a.spmv(xd[0])
    a.close()  # its blocks go back to the pool
    c = mb.Plan(*dev[2], ncol=mats[2].ncol)  # may take them
    for _ in range(3):
        yb = b.spmv(xd[1])
        yc = c.spmv(xd[2])
    torch.cuda.synchronize()
    for y, (y_ref, yabs) in ((ya, refs[0]), (yb, refs[1]), (yc, refs[2])):
        assert _rel_err(y.cpu().numpy(), y_ref, yabs).max() <= 1e-12
    assert b.check() is None and c.check() is None
    b.close()
    c.close()


@pytest.mark.gpu
def test_first_allocating_call_under_capture_is_refused():
    """A call that must allocate (here the first SpMM at this k, which
    allocates its carry slots) fails under stream capture instead of giving
    the plan memory that the captured graph owns; outside capture it then
    works."""
    import torch

    A = synth.zipf(20_000, 1.8, 5_000, 0.1, seed=50)
    rp, col, v = to_cuda(A, "f64")
    plan = mb.Plan(rp, col, v, ncol=A.ncol)
    X = torch.from_numpy(synth.uniform(51, A.ncol * 4).reshape(A.ncol, 4)).cuda()
    Y = torch.empty(A.nrow, 4, dtype=torch.float64, device="cuda")
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    with pytest.raises(mb.MerbitError) as ei:
        with torch.cuda.graph(g, stream=s):
            plan.spmm(X, Y, stream=s)
    assert "captured" in ei.value.detail
    del g
    plan.spmm(X, Y)
    torch.cuda.synchronize()
    y_ref, yabs = O.spmm(A.row_ptr, A.col, A.vals, X.cpu().numpy(), k=4)
    assert _rel_err(Y.cpu().numpy(), y_ref, yabs).max() <= 1e-12
