"""Generates the golden fixtures that pin the CPU oracle to the reference.

All outputs come from the reference's OWN code, compiled from its sources
into oracle/_ref/libmerbit_ref.so by oracle/Makefile:

  --cpu   merge_coords.npz   reference merge_search (include/utils.cuh:5-29,
                             host-callable) at every diagonal of stride 1,
                             14 and 448 on small matrices
  --gpu   tile_plan.npz      reference Tile_Kernel<256,SIGMA> plan
                             (include/tile.cuh:28-104), SIGMA = 7, 14, 20, 32
          merbit_kernel_y.npz  reference merbit_kernel<V,256,14> y = A x
                             (include/tile.cuh:476-561), V = double and float

--gpu needs a CUDA device.  Usage:
  python tests/golden/make_golden.py --cpu [--out DIR]
  python tests/golden/make_golden.py --gpu [--out DIR]
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from merbit_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402


def cases():
    rng = np.random.default_rng(2024)

    def from_len(L, ncol, seed):
        L = np.asarray(L, np.int64)
        r = np.random.default_rng(seed)
        rp = np.concatenate([[0], np.cumsum(L)]).astype(np.int32)
        col = np.concatenate([np.sort(r.choice(ncol, int(l), replace=False)) for l in L]
                             + [np.zeros(0, np.int64)]).astype(np.int32)
        return synth.CSR(rp, col, r.standard_normal(int(rp[-1])), ncol)

    out = {
        "lap12x10": synth.laplace2d(12, 10),
        "st27_5x5x4": synth.stencil27(5, 5, 4, seed=0),
        "zipf3000": synth.zipf(3000, 1.8, 3000, 0.1, seed=1),
        "ragged500": from_len(rng.integers(0, 30, 500), 400, 1),
        "giant5000": from_len([0, 5000, 0, 0, 7, 0], 6000, 2),
        "empty300": from_len([0] * 300, 10, 3),
        "aligned": from_len([447] * 4 + [448] * 4 + [0] * 3 + [449] * 4, 1000, 4),
    }
    return out


def make_cpu(outdir):
    if O.ref() is None:
        raise SystemExit("oracle/_ref not built (make -C oracle)")
    data = {}
    for name, A in cases().items():
        total = A.nrow + A.nnz
        data[f"{name}_row_ptr"] = A.row_ptr
        for stride in (1, 14, 448):
            count = total // stride + 2
            xs = np.empty(count, np.int32)
            ys = np.empty(count, np.int32)
            for i in range(count):
                d = min(i * stride, total)
                xs[i], ys[i] = O.ref_merge_search(A.row_ptr, A.nnz, d)
            data[f"{name}_x_{stride}"] = xs
            data[f"{name}_y_{stride}"] = ys
    np.savez_compressed(os.path.join(outdir, "merge_coords.npz"), **data)


def make_gpu(outdir):
    import torch

    R = O.ref()
    if R is None:
        raise SystemExit("oracle/_ref not built (make -C oracle)")
    plans, ys = {}, {}
    for name, A in cases().items():
        rp = torch.from_numpy(A.row_ptr).cuda()
        plans[f"{name}__row_ptr"] = A.row_ptr
        for sigma in (7, 14, 20, 32):
            ln = (A.nrow + A.nnz + sigma - 1) // sigma
            tn = (ln + 31) // 32
            tx = torch.zeros(tn + 1, dtype=torch.int32, device="cuda")
            ty = torch.zeros(tn + 1, dtype=torch.int32, device="cuda")
            dd = torch.zeros(max(ln, 1), dtype=torch.int32 if sigma < 15 else torch.int64,
                             device="cuda")
            assert R.ref_tile_build(sigma, rp.data_ptr(), A.nrow, A.nnz, tx.data_ptr(),
                                    ty.data_ptr(), dd.data_ptr()) == 0
            plans[f"{name}__tx_{sigma}"] = tx.cpu().numpy().view(np.uint32)
            plans[f"{name}__ty_{sigma}"] = ty.cpu().numpy().view(np.uint32)
            d = dd.cpu().numpy()[:ln]
            plans[f"{name}__desc_{sigma}"] = d.view(np.uint32) if sigma < 15 else d.view(np.uint64)
        # reference kernel output
        ln = (A.nrow + A.nnz + 13) // 14
        tn = (ln + 31) // 32
        tx = torch.zeros(tn + 1, dtype=torch.int32, device="cuda")
        ty = torch.zeros(tn + 1, dtype=torch.int32, device="cuda")
        dd = torch.zeros(max(ln, 1), dtype=torch.int32, device="cuda")
        assert R.ref_tile_build(14, rp.data_ptr(), A.nrow, A.nnz, tx.data_ptr(), ty.data_ptr(),
                                dd.data_ptr()) == 0
        x = synth.uniform(5, A.ncol)
        col = torch.from_numpy(A.col).cuda()
        ys[f"{name}__row_ptr"] = A.row_ptr
        ys[f"{name}__col"] = A.col
        ys[f"{name}__v64"] = A.vals
        ys[f"{name}__x64"] = x
        for code, vt in ((0, torch.float64), (1, torch.float32)):
            v = torch.from_numpy(A.vals).cuda().to(vt)
            xd = torch.from_numpy(x).cuda().to(vt)
            y = torch.zeros(max(A.nrow, 1), dtype=vt, device="cuda")
            z = torch.zeros(max(A.nrow, 1), dtype=vt, device="cuda")
            assert R.ref_merbit_spmv(code, col.data_ptr(), v.data_ptr(), A.nrow, A.nnz,
                                     tx.data_ptr(), ty.data_ptr(), dd.data_ptr(), 1.0,
                                     xd.data_ptr(), y.data_ptr(), z.data_ptr(), None) == 0
            torch.cuda.synchronize()
            ys[f"{name}__y{64 if code == 0 else 32}"] = y.cpu().numpy()[:A.nrow]
    np.savez_compressed(os.path.join(outdir, "tile_plan.npz"), **plans)
    np.savez_compressed(os.path.join(outdir, "merbit_kernel_y.npz"), **ys)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--cpu", action="store_true")
    ap.add_argument("--gpu", action="store_true")
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    if a.cpu:
        make_cpu(a.out)
    if a.gpu:
        make_gpu(a.out)
