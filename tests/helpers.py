"""Shared test helpers: small matrices that exercise the merge-path corner
cases, and conversions between numpy CSR and CUDA tensors."""
from __future__ import annotations

import numpy as np

from merbit_b200 import synth


def csr_from_lengths(lengths, ncol=None, seed=0, dtype=np.float64):
    lengths = np.asarray(lengths, dtype=np.int64)
    nrow = len(lengths)
    ncol = ncol if ncol is not None else max(nrow, 1)
    rng = np.random.default_rng(seed)
    rp = np.zeros(nrow + 1, np.int64)
    np.cumsum(np.minimum(lengths, ncol), out=rp[1:])
    nnz = int(rp[-1])
    col = np.empty(nnz, np.int32)
    for r in range(nrow):
        L = rp[r + 1] - rp[r]
        if L:
            col[rp[r]:rp[r + 1]] = np.sort(rng.choice(ncol, size=L, replace=False))
    vals = rng.standard_normal(nnz).astype(dtype)
    return synth.CSR(rp.astype(np.int32), col, vals, ncol, "lengths")


def edge_cases():
    """(name, CSR) pairs covering the shapes the reference's merge path has
    to get right: empty matrix, no nonzeros, empty rows at tile edges, one
    row spanning many tiles, single row, dense-ish rows, ragged tails."""
    out = []
    out.append(("one_row_one_nnz", csr_from_lengths([1])))
    out.append(("all_empty_rows", csr_from_lengths([0] * 5000, ncol=10)))
    out.append(("single_giant_row", csr_from_lengths([100_000], ncol=200_000, seed=1)))
    out.append(("giant_rows_between_empties",
                csr_from_lengths([0, 0, 60_000, 0, 3, 0, 45_000, 0, 0, 1], ncol=100_000, seed=2)))
    rng = np.random.default_rng(3)
    out.append(("ragged", csr_from_lengths(rng.integers(0, 40, 7777), ncol=5000, seed=3)))
    out.append(("short_rows_many_empty",
                csr_from_lengths(rng.integers(0, 3, 30000) * (rng.random(30000) < 0.5),
                                 ncol=30000, seed=4)))
    # every row exactly fills a tile boundary for common tile sizes
    out.append(("row_len_2047", csr_from_lengths([2047] * 10, ncol=4096, seed=5)))
    out.append(("row_len_448", csr_from_lengths([447] * 20 + [448] * 20 + [449] * 20,
                                                ncol=1000, seed=6)))
    out.append(("laplace2d_small", synth.workload("laplace2d_small")))
    out.append(("stencil27_small", synth.workload("stencil27_small")))
    out.append(("zipf_small", synth.workload("zipf_small")))
    return out


def to_cuda(A, dtype="f64", device="cuda"):
    import torch

    rp = torch.from_numpy(A.row_ptr).to(device)
    col = torch.from_numpy(A.col).to(device)
    if dtype == "f64":
        v = torch.from_numpy(np.ascontiguousarray(A.vals, np.float64)).to(device)
    elif dtype == "f32":
        v = torch.from_numpy(np.ascontiguousarray(A.vals, np.float32)).to(device)
    elif dtype == "bf16":
        v = torch.from_numpy(synth.to_bf16_bits(A.vals).view(np.int16)).to(device).view(
            torch.bfloat16)
    else:
        raise ValueError(dtype)
    return rp, col, v


def stored_values(A, dtype):
    """The values exactly as the GPU stores them, as the oracle's input."""
    if dtype == "f64":
        return np.ascontiguousarray(A.vals, np.float64)
    if dtype == "f32":
        return np.ascontiguousarray(A.vals, np.float32)
    return synth.to_bf16_bits(A.vals)
