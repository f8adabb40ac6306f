"""The batched k = 1 warp-tile kernel (merbit_batch_spmm with one right-hand
side): many uneven matrices in one persistent launch, each with its own
tile size (7, 11, 15, 19 or 23 items per lane).

Each matrix's y must be bitwise the y of the single-matrix warp-tile SpMV
with the same items per lane (same partition, same order of additions),
where that SpMV configuration admits the matrix (its row_ptr window caps
the rows a tile may end; the batch kernel has no cap); every matrix is also
checked against the oracle (component-wise, 1e-13 f64, 1e-6 f32/bf16)."""
import numpy as np
import pytest
import torch

import merbit_b200 as mb
from merbit_b200 import synth
from oracle import oracle as O
from tests.helpers import csr_from_lengths, edge_cases, stored_values, to_cuda

TOL = {"f64": 1e-13, "f32": 1e-6, "bf16": 1e-6}
XT = {"f64": torch.float64, "f32": torch.float32, "bf16": torch.float32}


def _mats():
    specs = synth.batch_rmat_specs(10, seed=2, nmin=300, nmax=30_000, dmin=2, dmax=48)
    mats = [synth.rmat(n, d, seed=s) for n, d, s in specs]
    mats += [A for name, A in edge_cases() if A.nrow > 0 and A.nnz > 0]
    mats.append(csr_from_lengths([0] * 2000 + [5] + [0] * 3000, ncol=100, seed=3))  # empty runs
    return mats


def _warp_config(plan, ipt):
    """Index of a warp-tile SpMV configuration with `ipt` items per lane that
    this plan can run, or None."""
    for idx, kind, block, p in plan.configs():
        if kind == 1 and p == ipt:
            return idx
    return None


def _build(mats, dtype, beta_y0=None):
    plans, Xs, Ys, xh = [], [], [], []
    for i, A in enumerate(mats):
        rp, col, v = to_cuda(A, dtype)
        plans.append(mb.Plan(rp, col, v, ncol=A.ncol))
        x = synth.uniform(50 + i, A.ncol).astype(np.float64 if dtype == "f64" else np.float32)
        xh.append(x)
        Xs.append(torch.from_numpy(x).cuda().reshape(A.ncol, 1))
        Ys.append(torch.full((A.nrow, 1), float("nan"), dtype=XT[dtype], device="cuda"))
    return plans, Xs, Ys, xh


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32", "bf16"])
@pytest.mark.parametrize("variant,ipt", [(0, 7), (0, 11), (1, 15), (2, "mixed"), (3, 19),
                                         (4, 23), (3, "mixed"), (5, "mixed"), (6, "mixed"),
                                         (7, 11), (8, "mixed"), (9, "mixed")])
def test_batch_k1_matches_single_matrix_warp_kernel(dtype, variant, ipt):
    mats = _mats()
    plans, Xs, Ys, xh = _build(mats, dtype)
    batch = mb.Batch(plans, Xs, Ys)
    batch.set_kernel(1, variant)
    takes = {3: (15, 19, 23), 4: (15, 19, 23)}.get(variant, (7, 11) if variant >= 6 else (7, 11, 15))
    ipts = [takes[i % len(takes)] if ipt == "mixed" else ipt for i in range(len(mats))]
    for i, p in enumerate(ipts):
        batch.set_matrix_config(i, p)
    assert batch.info()["kernel"] == 1 and batch.info()["variant"] == variant
    assert [c[2] for c in batch.matrix_configs()] == ipts
    assert [c[1] for c in batch.matrix_configs()] == [32 * p for p in ipts]
    batch.run()
    torch.cuda.synchronize()
    for p in plans:
        p.check()
    compared = 0
    for i, (A, plan) in enumerate(zip(mats, plans)):
        y = Ys[i][:, 0].cpu().numpy().astype(np.float64)
        yo, ya = O.spmm(A.row_ptr, A.col, stored_values(A, dtype), xh[i])
        assert O.rel_error(y, yo, ya)[0] <= TOL[dtype], (i, A.nrow, A.nnz)
        cfg = _warp_config(plan, ipts[i])
        if cfg is not None:
            plan.set_config(cfg)
            ys = plan.spmv(Xs[i][:, 0])
            torch.cuda.synchronize()
            assert torch.equal(ys, Ys[i][:, 0]), (i, A.nrow, A.nnz, ipts[i])
            compared += 1
    # the single-matrix table has warp tiles of 7, 11, 15 and 23 items per lane
    if set(ipts) <= {7, 11, 15, 23}:
        assert compared >= len(mats) // 2
    batch.close()


@pytest.mark.gpu
def test_batch_k1_graph_replay_alpha_beta_and_tuning():
    """Captured once, replayed with new x and beta != 0; then tuned (the
    per-class search) and still correct; the tuner's choices are reported
    per matrix and reused by a new batch of the same matrices."""
    mats = _mats()
    plans, Xs, Ys, xh = _build(mats, "f64")
    y0 = [torch.from_numpy(synth.uniform(90 + i, A.nrow)).cuda().reshape(A.nrow, 1)
          for i, A in enumerate(mats)]
    batch = mb.Batch(plans, Xs, Ys)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        batch.run(alpha=0.5, beta=-2.0, stream=s)
    for rep in range(3):
        for i, A in enumerate(mats):
            xh[i] = synth.uniform(200 + 10 * rep + i, A.ncol)
            Xs[i].copy_(torch.from_numpy(xh[i]).reshape(A.ncol, 1))
            Ys[i].copy_(y0[i])
        g.replay()
        torch.cuda.synchronize()
        for i, A in enumerate(mats):
            yo, ya = O.spmm(A.row_ptr, A.col, A.vals, xh[i], alpha=0.5)
            ref = yo - 2.0 * y0[i][:, 0].cpu().numpy()
            den = ya + 2.0 * np.abs(y0[i][:, 0].cpu().numpy())
            e = np.abs(Ys[i][:, 0].cpu().numpy() - ref) / np.maximum(den, 1e-300)
            assert e.max() <= TOL["f64"], (rep, i)
    del g
    info = batch.tune()
    cfgs = batch.matrix_configs()
    assert len(cfgs) == len(mats)
    if info["kernel"] == 1:
        assert all(c[2] in (7, 11, 15, 19, 23) and c[1] == 32 * c[2] for c in cfgs)
        # a new batch of the same matrices starts from the cached choices
        b2 = mb.Batch(plans, Xs, Ys)
        assert b2.info()["kernel"] == 1
        assert [c[2] for c in b2.matrix_configs()] == [c[2] for c in cfgs]
        b2.close()
    batch.run()
    torch.cuda.synchronize()
    for i, A in enumerate(mats):
        yo, ya = O.spmm(A.row_ptr, A.col, A.vals, xh[i])
        assert O.rel_error(Ys[i][:, 0].cpu().numpy(), yo, ya)[0] <= TOL["f64"], i
    batch.close()


def test_batch_matrix_config_arguments_need_no_gpu():
    L = mb.lib()
    assert L.merbit_batch_set_matrix_config(None, 0, 11, None) == 1
    assert L.merbit_batch_get_matrix_config(None, 0, None, None, None) == 1
    assert L.merbit_batch_set_kernel(None, 1, 0, None) == 1


@pytest.mark.gpu
def test_batch_kernel_selection_and_refusals():
    """Every SpMM tile size of each k, and the warp-tile variants at k = 1,
    give the oracle's answer; items per lane a variant does not take are
    refused, as is the warp-tile kernel at k > 1."""
    mats = _mats()[:6]
    for k in (1, 2, 4, 8, 16, 32):
        plans, Xs, Ys, xh = [], [], [], []
        for i, A in enumerate(mats):
            rp, col, v = to_cuda(A, "f32")
            plans.append(mb.Plan(rp, col, v, ncol=A.ncol))
            x = synth.uniform(70 + i, A.ncol * k).astype(np.float32).reshape(A.ncol, k)
            xh.append(x)
            Xs.append(torch.from_numpy(x).cuda())
            Ys.append(torch.empty(A.nrow, k, dtype=torch.float32, device="cuda"))
        batch = mb.Batch(plans, Xs, Ys)
        odd = {1: (288, 480), 2: (224, 352), 4: (288, 480), 8: (272, 496), 16: (264, 504),
               32: (260, 508)}[k]
        base = (256,) if k == 2 else (256, 512)
        choices = [(0, t) for t in base + odd] + ([(1, v) for v in range(10)] if k == 1 else [])
        for kern, opt in choices:
            batch.set_kernel(kern, opt)
            batch.run()
            torch.cuda.synchronize()
            for i, A in enumerate(mats):
                yo, ya = O.spmm(A.row_ptr, A.col, A.vals.astype(np.float32), xh[i], k=k)
                assert O.rel_error(Ys[i].cpu().numpy(), yo, ya)[0] <= TOL["f32"], (k, kern, opt, i)
        if k == 1:
            batch.set_kernel(1, 0)
            with pytest.raises(mb.MerbitError):
                batch.set_matrix_config(0, 23)
        else:
            with pytest.raises(mb.MerbitError):
                batch.set_kernel(1, 0)
        batch.close()


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [0, 6])
def test_batch_k1_with_empty_members(variant):
    """Members with no rows, with rows but no nonzeros, and with a single
    giant row sit between ordinary ones; warps cross them on the way."""
    mats = [csr_from_lengths([], ncol=5, seed=1),
            synth.rmat(2000, 10, seed=3),
            csr_from_lengths([0] * 700, ncol=50, seed=2),
            csr_from_lengths([], ncol=1, seed=1),
            csr_from_lengths([90_000], ncol=120_000, seed=4),
            synth.rmat(5000, 6, seed=6)]
    plans, Xs, Ys, xh = _build(mats, "f64")
    batch = mb.Batch(plans, Xs, Ys)
    batch.set_kernel(1, variant)
    for rep in range(2):
        batch.run()
        torch.cuda.synchronize()
        for i, A in enumerate(mats):
            if A.nrow == 0:
                continue
            y = Ys[i][:, 0].cpu().numpy()
            yo, ya = O.spmm(A.row_ptr, A.col, A.vals, xh[i])
            assert O.rel_error(y, yo, ya)[0] <= TOL["f64"], (rep, i)
            assert np.all(y[np.diff(A.row_ptr) == 0] == 0)
    batch.close()
