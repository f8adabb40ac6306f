"""CPU: the seeded generators give the documented shapes, sorted unique
columns, and the same bits on every call."""
import numpy as np

from merbit_b200 import synth


def _sorted_unique_rows(A):
    rp, c = A.row_ptr, A.col.astype(np.int64)
    for r in range(0, A.nrow, max(1, A.nrow // 2000)):
        seg = c[rp[r]:rp[r + 1]]
        assert np.all(np.diff(seg) > 0)
        if len(seg):
            assert seg[0] >= 0 and seg[-1] < A.ncol


def test_laplace2d_exact_shape():
    A = synth.laplace2d(256, 256)
    assert (A.nrow, A.nnz) == (65_536, 326_656)
    assert set(np.unique(A.vals)) == {-1.0, 4.0}
    _sorted_unique_rows(A)
    # row sums: 0 inside, positive on the boundary
    rs = np.add.reduceat(A.vals, A.row_ptr[:-1])
    assert rs.min() == 0.0 and rs.max() == 2.0


def test_stencil27_shape_and_dominance():
    A = synth.stencil27(9, 8, 7, seed=0)
    assert A.nnz == (3 * 9 - 2) * (3 * 8 - 2) * (3 * 7 - 2)
    _sorted_unique_rows(A)
    for r in range(A.nrow):
        s, e = A.row_ptr[r], A.row_ptr[r + 1]
        d = A.vals[s:e][A.col[s:e] == r][0]
        off = np.abs(A.vals[s:e]).sum() - abs(d)
        assert np.isclose(d, off + 1.0)


def test_stencil27_full_size_nnz():
    assert synth.lib().merbit_synth_stencil27_nnz(160, 160, 160) == 109_215_352


def test_zipf_properties_and_determinism():
    A = synth.zipf(50_000, 1.8, 20_000, 0.1, seed=1)
    B = synth.zipf(50_000, 1.8, 20_000, 0.1, seed=1)
    assert np.array_equal(A.row_ptr, B.row_ptr) and np.array_equal(A.col, B.col)
    assert np.array_equal(A.vals, B.vals)
    L = np.diff(A.row_ptr)
    assert 0.08 < (L == 0).mean() < 0.12
    assert L.max() <= 20_000
    # P(L = 1 | nonempty) for Zipf(1.8) capped at 2e4 is 1/H(1.8) ~ 0.57
    assert 0.52 < (L[L > 0] == 1).mean() < 0.62
    _sorted_unique_rows(A)
    C = synth.zipf(50_000, 1.8, 20_000, 0.1, seed=2)
    assert not np.array_equal(A.row_ptr, C.row_ptr)


def test_rmat_dedup_and_range():
    A = synth.rmat(3000, 20.0, seed=5)
    _sorted_unique_rows(A)
    assert 0 < A.nnz <= 3000 * 20
    B = synth.rmat(3000, 20.0, seed=5)
    assert np.array_equal(A.col, B.col)


def test_batch_specs_ranges():
    specs = synth.batch_rmat_specs(128, seed=2)
    assert len(specs) == 128
    assert all(1000 <= n <= 500_000 and 8 <= d <= 64 for n, d, _ in specs)


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.0078125, -3.14159, 0.0, 1e-30])
    bits = synth.to_bf16_bits(v)
    back = synth.bf16_bits_to_f64(bits)
    assert back[0] == 1.0 and back[1] == 1.0  # tie to even
    assert back[2] == 1.0078125
    assert abs(back[3] + 3.14159) < 0.02
