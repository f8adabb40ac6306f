"""Batches on the SpMM kernel whose matrices take different tile sizes
(merbit_batch_set_matrix_tile): one launch runs matrices with tiles of
either size of a pair (256/512, or the two odd tiles of k), at vector
width 4 and k = 4, 8, 16, 32.

Each matrix's Y must be bitwise the Y of the same matrix in a batch where
every matrix takes its tile size (same partition, same order of
additions), and within 1e-6 of the oracle (component-wise, FP32)."""
import numpy as np
import pytest
import torch

import merbit_b200 as mb
from merbit_b200 import synth
from oracle import oracle as O
from tests.helpers import csr_from_lengths, to_cuda

PAIRS = {4: [(256, 512), (288, 480)], 8: [(256, 512), (272, 496)],
         16: [(256, 512), (264, 504)], 32: [(256, 512), (260, 508)]}


def _mats():
    specs = synth.batch_rmat_specs(8, seed=5, nmin=300, nmax=20_000, dmin=2, dmax=40)
    mats = [synth.rmat(n, d, seed=s) for n, d, s in specs]
    mats.append(csr_from_lengths([], ncol=4, seed=1))                  # no rows
    mats.append(csr_from_lengths([0] * 900 + [3] + [0] * 400, ncol=60, seed=2))
    mats.append(csr_from_lengths([30_000], ncol=40_000, seed=3))        # one long row
    return mats


def _operands(mats, k):
    plans, Xs, Ys, xh = [], [], [], []
    for i, A in enumerate(mats):
        rp, col, v = to_cuda(A, "f32")
        plans.append(mb.Plan(rp, col, v, ncol=A.ncol))
        x = synth.uniform(300 + i, A.ncol * k).astype(np.float32).reshape(A.ncol, k)
        xh.append(x)
        Xs.append(torch.from_numpy(x).cuda())
        Ys.append(torch.full((A.nrow, k), float("nan"), dtype=torch.float32, device="cuda"))
    return plans, Xs, Ys, xh


@pytest.mark.gpu
@pytest.mark.parametrize("k", [4, 8, 16, 32])
def test_mixed_tile_batch_matches_uniform_batches_and_oracle(k):
    mats = _mats()
    plans, Xs, Ys, xh = _operands(mats, k)
    batch = mb.Batch(plans, Xs, Ys)
    for lo, hi in PAIRS[k]:
        # each tile size alone: the bits every matrix must reproduce
        uniform = {}
        for t in (lo, hi):
            batch.set_kernel(0, t)
            assert batch.info()["vector_width"] == 4
            batch.run()
            torch.cuda.synchronize()
            uniform[t] = [y.clone() for y in Ys]
        batch.set_kernel(0, lo)
        tiles = [hi if i % 3 == 1 else lo for i in range(len(mats))]
        for i, t in enumerate(tiles):
            if t != lo:
                batch.set_matrix_tile(i, t)
        assert [c[1] for c in batch.matrix_configs()] == tiles
        for y in Ys:
            y.fill_(float("nan"))
        batch.run()
        torch.cuda.synchronize()
        for p in plans:
            p.check()
        for i, A in enumerate(mats):
            assert torch.equal(Ys[i], uniform[tiles[i]][i]), (k, lo, hi, i)
            if A.nrow:
                yo, ya = O.spmm(A.row_ptr, A.col, A.vals.astype(np.float32), xh[i], k=k)
                assert O.rel_error(Ys[i].cpu().numpy(), yo, ya)[0] <= 1e-6, (k, lo, hi, i)
        # setting every matrix back to one size leaves a uniform batch
        for i, t in enumerate(tiles):
            if t != lo:
                batch.set_matrix_tile(i, lo)
        assert {c[1] for c in batch.matrix_configs()} == {lo}
    # a tile outside the batch's pair is refused
    batch.set_kernel(0, 256)
    with pytest.raises(mb.MerbitError):
        batch.set_matrix_tile(0, PAIRS[k][1][1])
    batch.close()


@pytest.mark.gpu
def test_tuned_batch_reports_its_tiles_and_stays_correct():
    """After the tuner's per-class choice the batch reports each matrix's
    tile (two sizes at most, a pair when they differ) and gives the
    oracle's answer."""
    mats = _mats()
    k = 8
    plans, Xs, Ys, xh = _operands(mats, k)
    batch = mb.Batch(plans, Xs, Ys)
    info = batch.tune()
    cfgs = batch.matrix_configs()
    tiles = sorted({c[1] for c in cfgs})
    assert info["kernel"] == 0 and len(tiles) <= 2
    if len(tiles) == 2:
        assert tuple(tiles) in PAIRS[k]
    batch.run()
    torch.cuda.synchronize()
    for i, A in enumerate(mats):
        if A.nrow:
            yo, ya = O.spmm(A.row_ptr, A.col, A.vals.astype(np.float32), xh[i], k=k)
            assert O.rel_error(Ys[i].cpu().numpy(), yo, ya)[0] <= 1e-6, i
    batch.close()


@pytest.mark.gpu
def test_matrix_tile_refused_on_warp_kernel_and_narrow_vectors():
    mats = _mats()[:4]
    plans, Xs, Ys, _ = _operands(mats, 1)
    batch = mb.Batch(plans, Xs, Ys)
    assert batch.info()["kernel"] == 1
    with pytest.raises(mb.MerbitError):
        batch.set_matrix_tile(0, 512)
    batch.close()
    plans, Xs, Ys, _ = _operands(mats, 2)  # vector width 2 at k = 2: no pairs
    batch = mb.Batch(plans, Xs, Ys)
    with pytest.raises(mb.MerbitError):
        batch.set_matrix_tile(0, 512)
    batch.close()


def test_matrix_tile_arguments_need_no_gpu():
    L = mb.lib()
    assert L.merbit_batch_set_matrix_tile(None, 0, 512, None) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("k,tile", [(2, 352), (4, 480), (8, 496), (16, 504), (32, 508)])
def test_untuned_batch_defaults(k, tile):
    """An untuned batch starts from the tile the tuner picks on the R-MAT
    batch (staged products at k = 2, the odd tile of k at vector width 4);
    with a leading dimension that rules out wide vectors it keeps 256."""
    mats = _mats()[:5]
    plans, Xs, Ys, xh = _operands(mats, k)
    batch = mb.Batch(plans, Xs, Ys)
    info = batch.info()
    assert info["kernel"] == 0 and info["tile_items"] == tile
    batch.run()
    torch.cuda.synchronize()
    for i, A in enumerate(mats):
        if A.nrow:
            yo, ya = O.spmm(A.row_ptr, A.col, A.vals.astype(np.float32), xh[i], k=k)
            assert O.rel_error(Ys[i].cpu().numpy(), yo, ya)[0] <= 1e-6, (k, i)
    batch.close()
    # X with a leading dimension of k + 1: scalar loads only
    Xw = [torch.zeros(A.ncol, k + 1, dtype=torch.float32, device="cuda") for A in mats]
    for X, x in zip(Xw, xh):
        X[:, :k] = torch.from_numpy(x).cuda()
    b2 = mb.Batch(plans, [X[:, :k] for X in Xw], Ys)
    assert b2.info()["tile_items"] == 256 and b2.info()["vector_width"] == 1
    b2.close()
