"""Seeded random CSR matrices through every kernel configuration, on the GPU.

The fixed edge cases (tests/helpers.py: edge_cases) pin the shapes the merge
path is known to find hard.  These cases draw the shapes instead: row counts
from 1 to 30,000, rectangular column counts, a mixture of empty, short,
medium and a few very long rows (so tiles end anywhere: inside giant rows,
on runs of empty rows, at row boundaries), duplicate and unsorted column
indices (CSR allows both; the product sums every stored entry), and every
fourth matrix on 4-byte-offset arrays, which rules out the 16-byte bulk and
vector loads.  Each matrix runs through every configuration the tuner could
pick, in every value type, and through the SpMM with a random k, against the
extended-precision oracle with the tolerances of the other parity tests.
"""
import math

import numpy as np
import pytest
import torch

import merbit_b200 as mb
from merbit_b200 import synth
from merbit_b200.autograd import SparseMatrix
from oracle import oracle as O
from tests.helpers import stored_values, to_cuda

TOL = {"f64": 1e-13, "f32": 1e-6, "bf16": 1e-6}
XT = {"f64": np.float64, "f32": np.float32, "bf16": np.float32}
SEEDS = range(16)


def random_csr(seed: int, square: bool = False) -> synth.CSR:
    rng = np.random.default_rng(1000 + seed)
    nrow = int(rng.integers(1, 30_001))
    ncol = int(rng.integers(1, 60_001))
    if square:
        ncol = nrow
    u = rng.random(nrow)
    L = np.zeros(nrow, np.int64)  # u >= 0.85: empty
    short = u < 0.55
    L[short] = rng.integers(1, 12, int(short.sum()))
    med = (u >= 0.55) & (u < 0.80)
    L[med] = rng.integers(12, 600, int(med.sum()))
    lng = (u >= 0.80) & (u < 0.85)
    L[lng] = rng.integers(600, 4_000, int(lng.sum()))
    # a few giant rows that span many tiles of every size
    for r in rng.choice(nrow, size=min(nrow, int(rng.integers(0, 4))), replace=False):
        L[r] = int(rng.integers(5_000, 60_000))
    # keep the oracle quick: at most ~1.5 M nonzeros
    tot = int(L.sum())
    if tot > 1_500_000:
        L = (L * (1_500_000 / tot)).astype(np.int64)
    rp = np.zeros(nrow + 1, np.int64)
    np.cumsum(L, out=rp[1:])
    nnz = int(rp[-1])
    col = rng.integers(0, ncol, nnz).astype(np.int32)  # duplicates allowed
    if seed % 2 == 0:  # sorted within rows on even seeds, as stored order otherwise
        rows = np.repeat(np.arange(nrow), L)
        col = col[np.lexsort((col, rows))]
    vals = rng.standard_normal(nnz)
    return synth.CSR(rp.astype(np.int32), col, vals, ncol, f"fuzz{seed}")


def _offset(t: torch.Tensor) -> torch.Tensor:
    """The same values at an address 4 bytes past a 16-byte boundary."""
    buf = torch.empty(t.numel() + 1, dtype=t.dtype, device=t.device)
    out = buf[1:]
    out.copy_(t)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("seed", SEEDS)
def test_random_csr_every_config_and_dtype(seed):
    A = random_csr(seed)
    unaligned = seed % 4 == 3
    x64 = synth.uniform(seed + 7, A.ncol)
    empty = np.diff(A.row_ptr) == 0
    for dtype in ("f64", "f32", "bf16"):
        x = x64.astype(XT[dtype])
        yo, ya = O.spmm(A.row_ptr, A.col, stored_values(A, dtype), x)
        rp, col, v = to_cuda(A, dtype)
        if unaligned and A.nnz > 0:
            col, v = _offset(col), _offset(v)
        plan = mb.Plan(rp, col, v, ncol=A.ncol)
        xd = torch.from_numpy(x).cuda()
        cfgs = plan.configs()
        if unaligned and A.nnz > 0:
            assert all(kind != 1 for _, kind, _, _ in cfgs)  # no bulk copies from these
        for idx, kind, block, ipt in cfgs:
            plan.set_config(idx)
            y = plan.spmv(xd).cpu().numpy()
            e = O.rel_error(y, yo, ya)[0]
            assert e <= TOL[dtype], (dtype, idx, kind, block, ipt, e)
            assert np.all(y[empty] == 0), (dtype, idx)
        plan.check()

        # SpMM with a random number of right-hand sides (tuned configuration)
        k = int(np.random.default_rng(seed).choice([1, 2, 3, 4, 8, 16, 32]))
        X = synth.uniform(seed + 11, A.ncol * k).reshape(A.ncol, k).astype(XT[dtype])
        plan.tune(xd)
        Y = plan.spmm(torch.from_numpy(X).cuda()).cpu().numpy()
        Yo, Ya = O.spmm(A.row_ptr, A.col, stored_values(A, dtype), X, k=k)
        Ye = np.abs(Y.astype(np.float64) - Yo) / np.maximum(Ya, 1e-300)
        assert (Ye.max() if Ye.size else 0.0) <= TOL[dtype], (dtype, k, float(Ye.max()))
        plan.check()
        plan.close()


@pytest.mark.gpu
@pytest.mark.parametrize("seed", SEEDS)
def test_random_partition_bit_exact(seed):
    """merge_search coordinates and the reference TILE plan, bit for bit."""
    A = random_csr(seed)
    rp = torch.from_numpy(A.row_ptr).cuda()
    total = A.nrow + A.nnz
    for stride in (14, 448, 480, 3072):
        count = min(total // stride + 2, 200_000)
        cx, cy = mb.merge_coords(rp, A.nnz, stride, count)
        ox, oy = O.merge_coords(A.row_ptr, stride, count)
        assert np.array_equal(cx.cpu().numpy(), ox), stride
        assert np.array_equal(cy.cpu().numpy(), oy), stride
    for sigma in (14, 20):
        tx, ty, desc = mb.tile_build(rp, A.nnz, sigma)
        ox, oy, od = O.tile_plan(A.row_ptr, sigma)
        assert np.array_equal(tx.cpu().numpy().view(np.uint32), ox)
        assert np.array_equal(ty.cpu().numpy().view(np.uint32), oy)
        d = desc.cpu().numpy()
        assert np.array_equal(d.view(np.uint32) if sigma < 15 else d.view(np.uint64), od)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(8))
def test_random_adjoints(seed):
    """dX = A^T G through the transpose plan, dval = G[row].X[col], and the
    fused backward, against the oracle (every fourth matrix on offset
    arrays)."""
    A = random_csr(seed)
    rng = np.random.default_rng(seed)
    k = int(rng.choice([1, 2, 4, 8, 16, 32]))
    for dtype in ("f64", "f32"):
        nt = XT[dtype]
        X = synth.uniform(seed + 4, A.ncol * k).reshape(A.ncol, k).astype(nt)
        G = synth.normal(seed + 6, A.nrow * k).reshape(A.nrow, k).astype(nt)
        rp, col, v = to_cuda(A, dtype)
        if seed % 4 == 3 and A.nnz > 0:
            col, v = _offset(col), _offset(v)
        M = SparseMatrix(rp, col, v, ncol=A.ncol)
        Gd, Xd = torch.from_numpy(G).cuda(), torch.from_numpy(X).cuda()
        vals = stored_values(A, dtype)
        absv = np.abs(vals.astype(np.float64))
        ref = O.spmm_t(A.row_ptr, A.col, vals, G, A.ncol)
        den = O.spmm_t(A.row_ptr, A.col, absv, np.abs(G.astype(np.float64)), A.ncol)
        refv = O.dval(A.row_ptr, A.col, G, X)
        denv = O.dval(A.row_ptr, A.col, np.abs(G.astype(np.float64)), np.abs(X.astype(np.float64)))
        tol = TOL[dtype]
        dX = M.transpose_plan().spmm(Gd).cpu().numpy()
        assert (np.abs(dX - ref) / np.maximum(den, 1e-300)).max(initial=0.0) <= tol, (dtype, k)
        dv = M.dval(Gd, Xd).cpu().numpy()
        assert (np.abs(dv - refv) / np.maximum(denv, 1e-300)).max(initial=0.0) <= tol, (dtype, k)
        out = M.backward_fused(Gd, Xd)
        if out is not None:
            fX, fv = (t.cpu().numpy() for t in out)
            assert (np.abs(fX - ref) / np.maximum(den, 1e-300)).max(initial=0.0) <= tol
            assert (np.abs(fv - refv) / np.maximum(denv, 1e-300)).max(initial=0.0) <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(4))
def test_random_batch(seed):
    """Five random matrices in one persistent batched launch (random k and
    value type, one of them on offset arrays), tuned, against the oracle."""
    rng = np.random.default_rng(50 + seed)
    k = int(rng.choice([1, 2, 4, 8, 16, 32]))
    dtype = ("f64", "f32", "bf16")[seed % 3]
    mats = [random_csr(100 + 5 * seed + j) for j in range(5)]
    plans, Xh, Xs, Ys = [], [], [], []
    for j, A in enumerate(mats):
        rp, col, v = to_cuda(A, dtype)
        if j == 2 and A.nnz > 0:
            rp, col, v = _offset(rp), _offset(col), _offset(v)
        plans.append(mb.Plan(rp, col, v, ncol=A.ncol))
        X = synth.uniform(200 + j, A.ncol * k).reshape(A.ncol, k).astype(XT[dtype])
        Xh.append(X)
        Xs.append(torch.from_numpy(X).cuda())
        Ys.append(torch.full((A.nrow, k), float("nan"), dtype=Xs[-1].dtype, device="cuda"))
    b = mb.Batch(plans, Xs, Ys)
    b.tune()
    b.run()
    torch.cuda.synchronize()
    for A, X, Y in zip(mats, Xh, Ys):
        Yo, Ya = O.spmm(A.row_ptr, A.col, stored_values(A, dtype), X, k=k)
        e = np.abs(Y.cpu().numpy().astype(np.float64) - Yo) / np.maximum(Ya, 1e-300)
        assert e.max(initial=0.0) <= TOL[dtype], (dtype, k, A.name)
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(4))
def test_random_pagerank_step(seed):
    """The fused PageRank step (damped SpMV + teleport + L1 residual) on
    random square matrices, every configuration."""
    A = random_csr(seed, square=True)
    dtype = ("f64", "f32", "bf16", "f64")[seed]
    x = synth.uniform(seed + 1, A.ncol).astype(XT[dtype])
    t = synth.uniform(seed + 2, A.nrow).astype(XT[dtype])
    yo, ya = O.spmm(A.row_ptr, A.col, stored_values(A, dtype), x)
    ref = 0.85 * yo + 0.15 * t.astype(np.float64)
    den = 0.85 * ya + 0.15 * np.abs(t.astype(np.float64))
    rp, col, v = to_cuda(A, dtype)
    plan = mb.Plan(rp, col, v)
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    for idx, kind, _, ipt in plan.configs():
        plan.set_config(idx)
        res = torch.zeros(1, dtype=torch.float64, device="cuda")
        y = plan.pagerank_step(xd, td, 0.85, residual=res).cpu().numpy()
        assert O.rel_error(y, ref, den)[0] <= TOL[dtype], (dtype, idx, kind, ipt)
        want = math.fsum(np.abs(y.astype(np.float64) - x.astype(np.float64)))
        assert abs(res.item() - want) <= 1e-12 * max(want, 1e-300), (dtype, idx)
    plan.check()


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(4))
def test_random_front_end_to_spmv(seed):
    """The harness front end end to end, as Fun_Merbit runs it: shuffled COO
    triplets (duplicates included) -> stable sort by row -> coo_to_csr ->
    plan -> SpMV, against the oracle on the same matrix built by numpy; and
    the loader's 1/outdegree weights against numpy."""
    A = random_csr(200 + seed)
    dtype = ("f64", "f32", "bf16", "f64")[seed]
    rng = np.random.default_rng(300 + seed)
    rows = np.repeat(np.arange(A.nrow, dtype=np.int32), np.diff(A.row_ptr))
    perm = rng.permutation(A.nnz)
    td = {"f64": torch.float64, "f32": torch.float32, "bf16": torch.bfloat16}[dtype]
    dr = torch.from_numpy(rows[perm]).cuda()
    # values stored as the oracle's stored_values rounds them
    _, dc, dv = to_cuda(synth.CSR(A.row_ptr, A.col[perm], A.vals[perm], A.ncol, "shuffled"), dtype)
    mb.coo_sort(dr, dc, dv)  # by (row, col), stable
    order = np.lexsort((A.col[perm], rows[perm]))
    assert np.array_equal(dr.cpu().numpy(), rows[perm][order])
    assert np.array_equal(dc.cpu().numpy(), A.col[perm][order])
    rp = mb.coo_to_csr(dr, A.nrow)
    assert np.array_equal(rp.cpu().numpy(), A.row_ptr)
    B = synth.CSR(A.row_ptr, A.col[perm][order], A.vals[perm][order], A.ncol, "sorted")
    x = synth.uniform(seed + 9, A.ncol).astype(XT[dtype])
    yo, ya = O.spmm(B.row_ptr, B.col, stored_values(B, dtype), x)
    plan = mb.Plan(rp, dc, dv, ncol=A.ncol)
    plan.tune(torch.from_numpy(x).cuda())
    y = plan.spmv(torch.from_numpy(x).cuda()).cpu().numpy()
    assert O.rel_error(y, yo, ya)[0] <= TOL[dtype]
    w = mb.outdegree_values(dr, A.nrow, td).to(torch.float64).cpu().numpy()
    ref = torch.from_numpy(1.0 / np.diff(A.row_ptr)[rows]).to(td).to(torch.float64).numpy()
    assert np.array_equal(w, ref)


def test_random_csr_generator_is_seeded_and_valid():
    """CPU: the generator is deterministic and yields a valid CSR with the
    mixture the GPU test relies on."""
    for seed in (0, 3, 5):
        A, B = random_csr(seed), random_csr(seed)
        assert np.array_equal(A.row_ptr, B.row_ptr) and np.array_equal(A.col, B.col)
        assert A.row_ptr[0] == 0 and A.row_ptr[-1] == A.nnz
        assert np.all(np.diff(A.row_ptr) >= 0)
        assert A.nnz == 0 or (A.col.min() >= 0 and A.col.max() < A.ncol)
    lens = np.concatenate([np.diff(random_csr(s).row_ptr) for s in range(4)])
    assert (lens == 0).any() and (lens >= 5_000).any() and (lens < 12).any()
