"""The tuner's signature cache (merbit_plan_tune -> merbit_plan_create).

A plan created after a tuning run of a matrix with the same signature
starts from the configuration that won there.  The signature buckets the
row count, the nonzero count, the density and the longest row, so a
row-group configuration tuned on a 27-point stencil (short, even rows) must
not reach a power-law matrix of the same size class, whose longest row
would serialize the row-group kernel."""
import math

import numpy as np
import pytest

from merbit_b200 import synth
from tests.helpers import to_cuda


def _bucket(v: float) -> int:
    """log2 bucket of the library's signature (floor(log2 v), 0 below 2)."""
    return 0 if v < 2.0 else int(math.floor(math.log2(v)))


def _size_class(A):
    return (_bucket(A.nrow), _bucket(A.nnz), _bucket(4.0 * A.nnz / A.nrow))


def _ms_per_spmv(plan, x, y, reps=20, trials=3):
    import torch

    s = torch.cuda.current_stream()
    best = float("inf")
    for _ in range(trials):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(reps):
            plan.spmv(x, y)
        e1.record(s)
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / reps)
    return best


def test_stencil_and_power_law_share_a_size_class():
    """CPU: the two matrices of the GPU test differ only in their longest row."""
    S = synth.stencil27(64, 64, 64, seed=0)
    Z = synth.zipf(64 * 64 * 64, 1.8, 100_000, 0.1, seed=21)
    assert _size_class(S) == _size_class(Z)
    assert np.diff(S.row_ptr).max() == 27
    assert np.diff(Z.row_ptr).max() > 1000


@pytest.mark.gpu
def test_row_group_choice_of_a_stencil_does_not_reach_a_power_law_matrix():
    import torch

    import merbit_b200 as mb

    S = synth.stencil27(64, 64, 64, seed=0)
    Z = synth.zipf(64 * 64 * 64, 1.8, 100_000, 0.1, seed=21)
    assert _size_class(S) == _size_class(Z)
    rs, cs, vs = to_cuda(S, "f64")
    xs = torch.from_numpy(synth.uniform(1, S.ncol)).cuda()
    ps = mb.Plan(rs, cs, vs, ncol=S.ncol)
    info_s = ps.tune(xs)
    assert info_s.max_row_len == 27
    assert info_s.kind == 3, "the tuner is expected to pick row groups on the stencil"
    # a second stencil plan of the same signature starts from the cached choice
    ps2 = mb.Plan(rs, cs, vs, ncol=S.ncol)
    assert ps2.info().kind == 3

    rz, cz, vz = to_cuda(Z, "f64")
    xz = torch.from_numpy(synth.uniform(2, Z.ncol)).cuda()
    yz = torch.empty(Z.nrow, dtype=torch.float64, device="cuda")
    pz = mb.Plan(rz, cz, vz, ncol=Z.ncol)  # untuned, same size class
    iz = pz.info()
    assert iz.max_row_len == int(np.diff(Z.row_ptr).max())
    assert iz.kind != 3, "a cached row-group choice reached a power-law matrix"
    t_untuned = _ms_per_spmv(pz, xz, yz)
    pz.tune(xz)
    t_tuned = _ms_per_spmv(pz, xz, yz)
    assert t_untuned <= 1.2 * t_tuned, (t_untuned, t_tuned)
    for p in (ps, ps2, pz):
        p.close()
