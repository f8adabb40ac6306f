"""Partition parity on the GPU: merge-path coordinates and the reference's
TILE plan format must match bit for bit -- against the C oracle
(oracle/merbit_oracle.c, pinned to the reference's own merge_search) and,
when oracle/_ref is built, against the reference Tile_Kernel itself."""
import numpy as np
import pytest
import torch

import merbit_b200 as mb
from oracle import oracle as O
from tests.helpers import edge_cases

CASES = edge_cases()


@pytest.mark.gpu
@pytest.mark.parametrize("name,A", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("stride", [1, 14, 448, 2048, 3072])
def test_merge_coords_bit_exact(name, A, stride):
    rp = torch.from_numpy(A.row_ptr).cuda()
    total = A.nrow + A.nnz
    count = min(total // stride + 2, 200_000)
    cx, cy = mb.merge_coords(rp, A.nnz, stride, count)
    ox, oy = O.merge_coords(A.row_ptr, stride, count)
    assert np.array_equal(cx.cpu().numpy(), ox)
    assert np.array_equal(cy.cpu().numpy(), oy)


@pytest.mark.gpu
@pytest.mark.parametrize("name,A", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("sigma", [7, 14, 20, 32])
def test_tile_plan_bit_exact(name, A, sigma):
    rp = torch.from_numpy(A.row_ptr).cuda()
    tx, ty, desc = mb.tile_build(rp, A.nnz, sigma)
    ox, oy, od = O.tile_plan(A.row_ptr, sigma)
    assert np.array_equal(tx.cpu().numpy().view(np.uint32), ox)
    assert np.array_equal(ty.cpu().numpy().view(np.uint32), oy)
    d = desc.cpu().numpy()
    d = d.view(np.uint32) if sigma < 15 else d.view(np.uint64)
    assert np.array_equal(d, od)


@pytest.mark.gpu
@pytest.mark.parametrize("name,A", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("sigma", [7, 14, 20, 32])
def test_tile_plan_matches_reference_kernel(name, A, sigma):
    R = O.ref()
    if R is None:
        pytest.skip("reference harness oracle/_ref not built")
    if A.nrow + A.nnz == 0:
        pytest.skip("reference launch needs at least one lane")
    rp = torch.from_numpy(A.row_ptr).cuda()
    T, Ln = mb.tile_dims(A.nrow, A.nnz, sigma)
    rtx = torch.zeros(T + 1, dtype=torch.int32, device="cuda")
    rty = torch.zeros(T + 1, dtype=torch.int32, device="cuda")
    rdesc = torch.zeros(max(Ln, 1), dtype=torch.int32 if sigma < 15 else torch.int64,
                        device="cuda")
    torch.cuda.synchronize()
    assert R.ref_tile_build(sigma, rp.data_ptr(), A.nrow, A.nnz, rtx.data_ptr(),
                            rty.data_ptr(), rdesc.data_ptr()) == 0
    tx, ty, desc = mb.tile_build(rp, A.nnz, sigma)
    assert torch.equal(tx, rtx)
    assert torch.equal(ty, rty)
    assert torch.equal(desc, rdesc[:Ln])
