"""SpMV parity on the GPU, through the C ABI.

Tolerances (component-wise, e_i = |y_i - y*_i| / sum_j |a_ij x_j| against
the extended-precision oracle computed on the stored values):
  * f64 (plain form):            1e-13
  * f32 / bf16 (precision form): 1e-6   (the precision target)
and against the reference merbit_kernel (oracle/_ref, its own float atomics):
  * f64: 1e-12,  f32: 1e-5 (the reference accumulates in plain float)
"""
import numpy as np
import pytest
import torch

import merbit_b200 as mb
from merbit_b200 import synth
from oracle import oracle as O
from tests.helpers import csr_from_lengths, edge_cases, stored_values, to_cuda

CASES = edge_cases()
TOL = {"f64": 1e-13, "f32": 1e-6, "bf16": 1e-6}
XT = {"f64": torch.float64, "f32": torch.float32, "bf16": torch.float32}


def _x(A, dtype, seed=7):
    x = synth.uniform(seed, A.ncol)
    return x.astype(np.float64 if dtype == "f64" else np.float32)


def _run(A, dtype, x, alpha=1.0, beta=0.0, y0=None, tune=False):
    rp, col, v = to_cuda(A, dtype)
    plan = mb.Plan(rp, col, v, ncol=A.ncol)
    if tune:
        plan.tune()
    xd = torch.from_numpy(x).cuda()
    y = None if y0 is None else torch.from_numpy(y0).cuda()
    y = plan.spmv(xd, y, alpha=alpha, beta=beta)
    torch.cuda.synchronize()
    plan.check()
    return plan, y.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32", "bf16"])
@pytest.mark.parametrize("name,A", CASES, ids=[c[0] for c in CASES])
def test_spmv_vs_oracle(name, A, dtype):
    x = _x(A, dtype)
    _, y = _run(A, dtype, x)
    yo, ya = O.spmm(A.row_ptr, A.col, stored_values(A, dtype), x)
    emax, emed = O.rel_error(y, yo, ya)
    assert emax <= TOL[dtype], (emax, emed)
    # rows with no nonzeros are exactly zero
    empty = np.diff(A.row_ptr) == 0
    assert np.all(y[empty] == 0)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32", "bf16"])
@pytest.mark.parametrize("workload", ["zipf_small", "laplace2d_small", "stencil27_small"])
def test_spmv_every_config(dtype, workload):
    """Every tile configuration the tuner can pick gives the oracle's answer."""
    A = synth.workload(workload)
    x = _x(A, dtype)
    yo, ya = O.spmm(A.row_ptr, A.col, stored_values(A, dtype), x)
    rp, col, v = to_cuda(A, dtype)
    plan = mb.Plan(rp, col, v)
    xd = torch.from_numpy(x).cuda()
    cfgs = plan.configs()
    assert {0, 1, 3} <= {k for _, k, _, _ in cfgs}
    for idx, kind, block, ipt in cfgs:
        plan.set_config(idx)
        assert plan.info().tile_items == {0: block * ipt, 1: 32 * ipt, 3: 0}[kind]
        y = plan.spmv(xd)
        torch.cuda.synchronize()
        plan.check()
        assert O.rel_error(y.cpu().numpy(), yo, ya)[0] <= TOL[dtype], (idx, kind, block, ipt)
    plan.tune(xd)
    y = plan.spmv(xd)
    assert O.rel_error(y.cpu().numpy(), yo, ya)[0] <= TOL[dtype]


# The precision form's bound per row: products rounded to f32 (1 unit),
# blocks of 4 of them summed in f32 before each TwoSum (3 units), and y
# rounded to f32 on the store (1 unit): 5 units of sum |a x|.
F32_FORM_BOUND = 5 * 2.0 ** -24


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f32", "bf16"])
def test_precision_form_error_bound(dtype):
    """Positive values and x (no cancellation, so the bound is tight
    relative to |y|): every configuration stays within 5 units of sum |a x|
    per row, on single-row tiles (one row of 100,000 entries), the walk
    (rows of 37), a power-law matrix and the row groups (stencil)."""
    mats = [csr_from_lengths([100_000], ncol=150_000, seed=5),
            csr_from_lengths([37] * 3_000, ncol=20_000, seed=6),
            synth.workload("zipf_small"), synth.workload("stencil27_small")]
    for A in mats:
        A = synth.CSR(A.row_ptr, A.col, 0.5 + 0.5 * np.abs(np.tanh(A.vals)), A.ncol, A.name)
        x = (0.5 + 0.5 * synth.uniform(9, A.ncol, 0.0, 1.0)).astype(np.float32)
        yo, ya = O.spmm(A.row_ptr, A.col, stored_values(A, dtype), x)
        rp, col, v = to_cuda(A, dtype)
        plan = mb.Plan(rp, col, v, ncol=A.ncol)
        xd = torch.from_numpy(x).cuda()
        for idx, kind, block, ipt in plan.configs():
            plan.set_config(idx)
            y = plan.spmv(xd)
            torch.cuda.synchronize()
            emax = O.rel_error(y.cpu().numpy(), yo, ya)[0]
            assert emax <= F32_FORM_BOUND, (A.name, idx, kind, ipt, emax)
        plan.close()


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_alpha_beta(dtype):
    A = synth.workload("zipf_small")
    x = _x(A, dtype)
    y0 = synth.uniform(11, A.nrow).astype(x.dtype)
    _, y = _run(A, dtype, x, alpha=-2.5, beta=0.75, y0=y0)
    yo, ya = O.spmm(A.row_ptr, A.col, stored_values(A, dtype), x, alpha=-2.5)
    ref = yo + 0.75 * y0.astype(np.float64)
    err = np.abs(y - ref) / np.maximum(ya + 0.75 * np.abs(y0), 1e-300)
    assert err.max() <= TOL[dtype] * 4


@pytest.mark.gpu
def test_beta_zero_ignores_nan_in_y():
    A = synth.workload("laplace2d_small")
    x = _x(A, "f64")
    y0 = np.full(A.nrow, np.nan)
    _, y = _run(A, "f64", x, beta=0.0, y0=y0)
    assert np.isfinite(y).all()


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_deterministic_bitwise(dtype):
    """No float atomics: repeated launches give identical bits."""
    A = csr_from_lengths([0, 70_000, 5, 0, 90_000, 1] * 3, ncol=200_000, seed=9)
    x = _x(A, dtype)
    rp, col, v = to_cuda(A, dtype)
    plan = mb.Plan(rp, col, v, ncol=A.ncol)
    xd = torch.from_numpy(x).cuda()
    ys = [plan.spmv(xd).clone() for _ in range(20)]
    for y in ys[1:]:
        assert torch.equal(y.view(torch.int64 if dtype == "f64" else torch.int32),
                           ys[0].view(torch.int64 if dtype == "f64" else torch.int32))


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32", "bf16"])
def test_unaligned_pointers_scalar_path(dtype):
    """Views that start off a 16-byte boundary take the scalar-load kernel."""
    A = synth.workload("zipf_small")
    rp, col, v = to_cuda(A, dtype)
    col2 = torch.empty(col.numel() + 1, dtype=col.dtype, device="cuda")
    col2[1:] = col
    v2 = torch.empty(v.numel() + 1, dtype=v.dtype, device="cuda")
    v2[1:] = v
    plan = mb.Plan(rp, col2[1:], v2[1:])
    assert not plan.info().vectorized
    x = _x(A, dtype)
    y = plan.spmv(torch.from_numpy(x).cuda()).cpu().numpy()
    yo, ya = O.spmm(A.row_ptr, A.col, stored_values(A, dtype), x)
    assert O.rel_error(y, yo, ya)[0] <= TOL[dtype]


@pytest.mark.gpu
def test_rectangular():
    A = csr_from_lengths(np.arange(300) % 17, ncol=50_000, seed=12)
    x = _x(A, "f64")
    _, y = _run(A, "f64", x)
    yo, ya = O.spmm(A.row_ptr, A.col, A.vals, x)
    assert O.rel_error(y, yo, ya)[0] <= TOL["f64"]


@pytest.mark.gpu
def test_empty_matrix():
    rp = torch.zeros(1, dtype=torch.int32, device="cuda")
    col = torch.zeros(0, dtype=torch.int32, device="cuda")
    v = torch.zeros(0, dtype=torch.float64, device="cuda")
    plan = mb.Plan(rp, col, v, ncol=0)
    y = plan.spmv(torch.zeros(0, dtype=torch.float64, device="cuda"))
    assert y.numel() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("bad", ["rp0", "rpn", "decreasing", "col_high", "col_neg"])
def test_malformed_structure_rejected(bad):
    A = synth.workload("laplace2d_small")
    rp, col, v = A.row_ptr.copy(), A.col.copy(), A.vals
    if bad == "rp0":
        rp[0] = 1
    elif bad == "rpn":
        rp[-1] -= 1
    elif bad == "decreasing":
        rp[10] = rp[12] + 1
    elif bad == "col_high":
        col[100] = A.ncol
    else:
        col[5] = -1
    with pytest.raises(mb.MerbitError) as ei:
        mb.Plan(torch.from_numpy(rp).cuda(), torch.from_numpy(col).cuda(),
                torch.from_numpy(v).cuda(), ncol=A.ncol)
    assert ei.value.status == 2


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_vs_reference_merbit_kernel(dtype):
    """Same y as the reference merbit_kernel<V,256,14> run on this GPU."""
    R = O.ref()
    if R is None:
        pytest.skip("reference harness oracle/_ref not built")
    for name, A in edge_cases():
        if A.nrow == 0 or A.nrow + A.nnz < 1:
            continue
        x = _x(A, dtype)
        _, y = _run(A, dtype, x)
        rp, col, v = to_cuda(A, dtype)
        T, Ln = mb.tile_dims(A.nrow, A.nnz, 14)
        tx = torch.zeros(T + 1, dtype=torch.int32, device="cuda")
        ty = torch.zeros(T + 1, dtype=torch.int32, device="cuda")
        desc = torch.zeros(max(Ln, 1), dtype=torch.int32, device="cuda")
        assert R.ref_tile_build(14, rp.data_ptr(), A.nrow, A.nnz, tx.data_ptr(), ty.data_ptr(),
                                desc.data_ptr()) == 0
        xd = torch.from_numpy(x).cuda()
        yr = torch.zeros(A.nrow, dtype=XT[dtype], device="cuda")
        zr = torch.zeros(A.nrow, dtype=XT[dtype], device="cuda")
        assert R.ref_merbit_spmv(0 if dtype == "f64" else 1, col.data_ptr(), v.data_ptr(),
                                 A.nrow, A.nnz, tx.data_ptr(), ty.data_ptr(), desc.data_ptr(),
                                 1.0, xd.data_ptr(), yr.data_ptr(), zr.data_ptr(), None) == 0
        torch.cuda.synchronize()
        _, ya = O.spmm(A.row_ptr, A.col, stored_values(A, dtype), x)
        e = np.abs(y.astype(np.float64) - yr.cpu().numpy().astype(np.float64))
        e = e / np.maximum(ya, 1e-300)
        tol = 1e-12 if dtype == "f64" else 1e-5
        assert e.max() <= tol, (name, e.max())


@pytest.mark.gpu
def test_full_size_zipf_f64_vs_oracle():
    """The bench workload itself (Zipf(1.8), 2M rows), against the oracle."""
    A = synth.workload("zipf_2m")
    x = synth.uniform(1, A.ncol)
    _, y = _run(A, "f64", x, tune=True)
    yo, ya = O.spmm(A.row_ptr, A.col, A.vals, x)
    emax, emed = O.rel_error(y, yo, ya)
    assert emax <= TOL["f64"], (emax, emed)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_alternating_kernels_share_carry_slots(dtype):
    """Launches that alternate between kernel kinds and tile sizes on one
    plan (as the tuner does) must each see clean carry / swap slots."""
    A = synth.workload("zipf_small")
    x = _x(A, dtype)
    yo, ya = O.spmm(A.row_ptr, A.col, stored_values(A, dtype), x)
    rp, col, v = to_cuda(A, dtype)
    plan = mb.Plan(rp, col, v)
    xd = torch.from_numpy(x).cuda()
    cfgs = plan.configs()
    warp = [c[0] for c in cfgs if c[1] == 1]
    cta = [c[0] for c in cfgs if c[1] == 0]
    rows = [c[0] for c in cfgs if c[1] == 3]
    order = [warp[0], cta[0], warp[0], rows[0], warp[1], cta[1], cta[0], rows[-1], warp[0],
             warp[-1], cta[-1], rows[1], warp[0]]
    for idx in order * 2:
        plan.set_config(idx)
        y = plan.spmv(xd)
        torch.cuda.synchronize()
        assert O.rel_error(y.cpu().numpy(), yo, ya)[0] <= TOL[dtype], idx
    plan.check()


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("name,A", CASES, ids=[c[0] for c in CASES])
def test_row_groups_edge_cases(name, A, dtype):
    """Every row-group configuration (2-32 lanes per row, both gather hints)
    on the edge cases: empty rows, a 100k-entry row, ragged tails."""
    x = _x(A, dtype)
    yo, ya = O.spmm(A.row_ptr, A.col, stored_values(A, dtype), x)
    rp, col, v = to_cuda(A, dtype)
    plan = mb.Plan(rp, col, v, ncol=A.ncol)
    xd = torch.from_numpy(x).cuda()
    rows = [c for c in plan.configs() if c[1] == 3]
    assert len(rows) >= 5
    for idx, _, _, lpr in rows:
        plan.set_config(idx)
        y = plan.spmv(xd).cpu().numpy()
        assert O.rel_error(y, yo, ya)[0] <= TOL[dtype], (idx, lpr)
        assert np.all(y[np.diff(A.row_ptr) == 0] == 0)
    plan.check()


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("workload", ["zipf_small", "stencil27_small"])
def test_graph_replay_every_config(dtype, workload):
    """Every configuration captured in a CUDA graph and replayed: three SpMVs
    per graph (an odd count, so the launch epoch's parity differs from one
    replay to the next), four replays with new x each time, no host-side
    reset in between; every y against the oracle."""
    A = synth.workload(workload)
    rp, col, v = to_cuda(A, dtype)
    plan = mb.Plan(rp, col, v, ncol=A.ncol)
    nt = np.float64 if dtype == "f64" else np.float32
    xs = [torch.from_numpy(_x(A, dtype, seed=40 + j)).cuda() for j in range(3)]
    ys = [torch.empty(A.nrow, dtype=xs[0].dtype, device="cuda") for _ in range(3)]
    s = torch.cuda.Stream()
    for idx, kind, _, _ in plan.configs():
        plan.set_config(idx)
        plan.spmv(xs[0], ys[0])  # first launch outside capture (function attributes)
        torch.cuda.synchronize()
        s.wait_stream(torch.cuda.current_stream())
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            for j in range(3):
                plan.spmv(xs[j], ys[j], stream=s)
        for rep in range(4):
            xh = [synth.uniform(100 * rep + 10 * idx + j, A.ncol).astype(nt) for j in range(3)]
            for j in range(3):
                xs[j].copy_(torch.from_numpy(xh[j]))
                ys[j].fill_(float("nan"))
            g.replay()
            torch.cuda.synchronize()
            for j in range(3):
                yo, ya = O.spmm(A.row_ptr, A.col, stored_values(A, dtype), xh[j])
                e = O.rel_error(ys[j].cpu().numpy(), yo, ya)[0]
                assert e <= TOL[dtype], (idx, kind, rep, j, e)
        del g
        plan.check()


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32", "bf16"])
def test_warp_configs_with_equal_tiles_agree_bitwise(dtype):
    """Warp-tile configurations that differ only in carveout, gather hint,
    row_ptr window or walk (staged products or the register walk) share the
    partition and the order of every addition: their y are the same bits."""
    mats = [A for _, A in edge_cases()] + [synth.rmat(3000, 12, seed=5)]
    for A in mats:
        if A.nrow == 0:
            continue
        x = _x(A, dtype)
        rp, col, v = to_cuda(A, dtype)
        plan = mb.Plan(rp, col, v, ncol=A.ncol)
        xd = torch.from_numpy(x).cuda()
        by_ipt = {}
        for idx, kind, block, ipt in plan.configs():
            if kind == 1:
                by_ipt.setdefault(ipt, []).append(idx)
        for ipt, idxs in by_ipt.items():
            ys = []
            for idx in idxs:
                plan.set_config(idx)
                ys.append(plan.spmv(xd).clone())
            torch.cuda.synchronize()
            plan.check()
            for idx, y in zip(idxs[1:], ys[1:]):
                assert torch.equal(y, ys[0]), (A.name, ipt, idxs[0], idx)
        plan.close()
