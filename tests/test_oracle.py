"""CPU: the oracle against the reference's own code and golden fixtures.

* orc_merge_search vs the reference's host merge_search (oracle/_ref, built
  from the reference sources) on every diagonal of many small matrices;
* orc_merge_search / orc_tile_plan / orc_spmm vs the committed fixtures in
  tests/golden/ (made by tests/golden/make_golden.py from the reference's
  merge_search, Tile_Kernel and merbit_kernel);
* the extended-precision SpMM and the OpenMP baseline against exact
  rational arithmetic on tiny cases.
"""
import os
from fractions import Fraction

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import csr_from_lengths, edge_cases

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _random_rowptr(rng, nrow):
    L = rng.integers(0, 8, size=nrow) * (rng.random(nrow) < 0.7)
    if nrow and rng.random() < 0.3:
        L[rng.integers(0, nrow)] = int(rng.integers(20, 300))
    return np.concatenate([[0], np.cumsum(L)]).astype(np.int32)


def test_merge_search_matches_reference_host_code():
    if O.ref() is None:
        pytest.skip("reference harness oracle/_ref not built")
    rng = np.random.default_rng(1)
    for _ in range(200):
        rp = _random_rowptr(rng, int(rng.integers(0, 50)))
        nnz = int(rp[-1])
        for d in range(len(rp) - 1 + nnz + 1):
            assert O.merge_search(rp, nnz, d) == O.ref_merge_search(rp, nnz, d)


def test_merge_search_tie_rule():
    # rows: [0,2), [2,2) empty, [2,5): at x == row end the row end goes first
    rp = np.array([0, 2, 2, 5], np.int32)
    path = [O.merge_search(rp, 5, d) for d in range(9)]
    assert path == [(0, 0), (1, 0), (2, 0), (2, 1), (2, 2), (3, 2), (4, 2), (5, 2), (5, 3)]


def _golden(name):
    p = os.path.join(GOLDEN, name)
    if not os.path.exists(p):
        pytest.skip(f"fixture {name} not generated")
    return np.load(p)


def test_merge_coords_vs_golden():
    g = _golden("merge_coords.npz")
    for key in sorted(k for k in g.files if k.endswith("_row_ptr")):
        case = key[: -len("_row_ptr")]
        rp = g[key]
        for stride in (1, 14, 448):
            ox, oy = O.merge_coords(rp, stride, len(g[f"{case}_x_{stride}"]))
            assert np.array_equal(ox, g[f"{case}_x_{stride}"]), case
            assert np.array_equal(oy, g[f"{case}_y_{stride}"]), case


def test_tile_plan_vs_golden():
    g = _golden("tile_plan.npz")
    cases = sorted({k.split("__")[0] for k in g.files})
    assert cases
    for case in cases:
        rp = g[f"{case}__row_ptr"]
        for sigma in (7, 14, 20, 32):
            if f"{case}__tx_{sigma}" not in g.files:
                continue
            tx, ty, desc = O.tile_plan(rp, sigma)
            assert np.array_equal(tx, g[f"{case}__tx_{sigma}"]), (case, sigma)
            assert np.array_equal(ty, g[f"{case}__ty_{sigma}"]), (case, sigma)
            assert np.array_equal(desc, g[f"{case}__desc_{sigma}"]), (case, sigma)


def test_spmm_vs_reference_kernel_golden():
    """The oracle's y agrees with the reference merbit_kernel's y (stored from
    a B200 run) within the reference kernel's own rounding."""
    g = _golden("merbit_kernel_y.npz")
    cases = sorted({k.split("__")[0] for k in g.files})
    assert cases
    for case in cases:
        rp, col, x = g[f"{case}__row_ptr"], g[f"{case}__col"], g[f"{case}__x64"]
        v64 = g[f"{case}__v64"]
        yo, ya = O.spmm(rp, col, v64, x)
        e = np.abs(g[f"{case}__y64"] - yo) / np.maximum(ya, 1e-300)
        assert e.max() <= 1e-12, case
        yo32, ya32 = O.spmm(rp, col, v64.astype(np.float32), x.astype(np.float32))
        e32 = np.abs(g[f"{case}__y32"].astype(np.float64) - yo32) / np.maximum(ya32, 1e-300)
        assert e32.max() <= 1e-5, case


def test_tile_plan_self_consistency():
    """Decoding the descriptors walks the same merge path as merge_search."""
    for name, A in edge_cases()[:6]:
        if A.nrow + A.nnz == 0:
            continue
        sigma = 14
        tx, ty, desc = O.tile_plan(A.row_ptr, sigma)
        T, Ln = O.tile_dims(A.nrow, A.nnz, sigma)
        assert tx[T] == A.nnz and ty[T] == A.nrow
        for gid in range(0, Ln, max(1, Ln // 300)):
            t = gid // 32
            wx, wy = int(tx[t]), int(ty[t]) & 0x7FFFFFFF
            d = int(desc[gid])
            dx, dy = d & 0x1FF, (d >> 9) & 0x1FF
            assert O.merge_search(A.row_ptr, A.nnz, gid * sigma) == (wx + dx, wy + dy)


def test_spmm_exact_small():
    rng = np.random.default_rng(4)
    A = csr_from_lengths(rng.integers(0, 6, 40), ncol=30, seed=4)
    x = rng.standard_normal(30)
    y, _ = O.spmm(A.row_ptr, A.col, A.vals, x)
    for r in range(A.nrow):
        ex = sum((Fraction(float(A.vals[e])) * Fraction(float(x[A.col[e]]))
                  for e in range(A.row_ptr[r], A.row_ptr[r + 1])), Fraction(0))
        assert y[r] == float(ex)


def test_spmm_multi_rhs_and_adjoint_consistent():
    rng = np.random.default_rng(5)
    A = csr_from_lengths(rng.integers(0, 9, 300), ncol=200, seed=5)
    X = rng.standard_normal((200, 3))
    G = rng.standard_normal((300, 3))
    Y, _ = O.spmm(A.row_ptr, A.col, A.vals, X, k=3)
    dX = O.spmm_t(A.row_ptr, A.col, A.vals, G, 200)
    dv = O.dval(A.row_ptr, A.col, G, X)
    # <G, A X> == <A^T G, X> == sum_e dval_e * a_e
    lhs = float((G * Y).sum())
    assert np.isclose(lhs, float((dX * X).sum()), rtol=1e-12)
    assert np.isclose(lhs, float((dv * A.vals).sum()), rtol=1e-12)


def test_omp_baseline_matches_oracle():
    for name, A in edge_cases():
        x = np.random.default_rng(0).uniform(-1, 1, A.ncol)
        y, nt = O.spmv_omp_f64(A.row_ptr, A.col, A.vals, x)
        yo, ya = O.spmm(A.row_ptr, A.col, A.vals, x)
        assert O.rel_error(y, yo, ya)[0] <= 1e-12, name
        assert nt >= 1


@pytest.mark.parametrize("nthreads", [1, 2, 3, 7, 64])
def test_omp_baseline_thread_counts(nthreads):
    A = csr_from_lengths([0, 5000, 1, 0, 2, 7000, 0], ncol=9000, seed=3)
    x = np.linspace(-1, 1, A.ncol)
    y, _ = O.spmv_omp_f64(A.row_ptr, A.col, A.vals, x, nthreads=nthreads)
    yo, ya = O.spmm(A.row_ptr, A.col, A.vals, x)
    assert O.rel_error(y, yo, ya)[0] <= 1e-12
