"""The reference's C++ host API (include/merbit_compat.hpp): a harness in
the shape of src/main.cu builds against it and, on a GPU, loads Matrix
Market graphs the way the reference does (symmetric doubling, basezero,
1/outdegree values) and runs Fun_Merbit's 400 SpMVs."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "merbit_b200", "compat", "merbit_main")


def test_example_harness_builds():
    from merbit_b200 import _build

    _build.build()
    assert os.access(EXE, os.X_OK)


def test_compat_header_compiles_for_float(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text('#include "merbit_compat.hpp"\nstd::fstream FSTR;\n'
                   'void f(const ENV& e, const PARAMETER<float>& p) { Fun_Merbit<float,256,20>(e, p); }\n'
                   'int main() { return 0; }\n')
    r = subprocess.run(["/usr/bin/g++", "-std=c++17", "-fsyntax-only", "-I",
                        os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include", str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def _write_mtx(path, n, entries, symmetric=False, basezero=False):
    kind = "symmetric" if symmetric else "general"
    hdr = f"%%MatrixMarket matrix coordinate real {kind}" + (" basezero" if basezero else "")
    with open(path, "w") as f:
        f.write(hdr + "\n% a comment\n")
        f.write(f"{n} {n} {len(entries)}\n")
        for r, c in entries:
            f.write(f"{r} {c} 1.5\n")


def _expected(n, entries, symmetric, basezero):
    rows, cols = [], []
    for r, c in entries:
        r0, c0 = (r, c) if basezero else (r - 1, c - 1)
        rows.append(r0)
        cols.append(c0)
    if symmetric:
        rows, cols = rows + cols, cols + rows
    rows, cols = np.array(rows), np.array(cols)
    outdeg = np.bincount(rows, minlength=n).astype(np.float64)
    vals = 1.0 / outdeg[rows]
    y = np.zeros(n)
    np.add.at(y, cols, vals)  # CSR rows are col_ind, x = 1 (tile.cuh:571-601)
    return y


@pytest.mark.gpu
@pytest.mark.parametrize("symmetric,basezero", [(False, False), (True, False), (False, True)])
def test_fun_merbit_on_matrix_market(tmp_path, symmetric, basezero):
    rng = np.random.default_rng(11)
    n = 3000
    lo = 0 if basezero else 1
    entries = sorted({(int(r), int(c)) for r, c in rng.integers(lo, n + lo, size=(20000, 2))})
    mtx = tmp_path / "g.mtx"
    _write_mtx(mtx, n, entries, symmetric, basezero)
    cfg = tmp_path / "config.txt"
    cfg.write_text(f"1 /nonexistent 1 1 1\n7 {mtx} {n} {n} {len(entries)}\n")
    log = tmp_path / "log.txt"
    yout = tmp_path / "y.bin"
    r = subprocess.run([EXE, "7", str(cfg), str(log), "0", str(yout)], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "graph = 7, block = 256, sigma = 14" in r.stdout
    line = log.read_text().strip()
    assert re.fullmatch(r"7&MERBIT&14&[0-9.e+-]+&[0-9.e+-]+", line), line
    y = np.fromfile(yout, dtype=np.float64)
    ref = _expected(n, entries, symmetric, basezero)
    assert np.allclose(y, ref, rtol=1e-13, atol=1e-15)


@pytest.mark.gpu
def test_missing_graph_id_is_an_error(tmp_path):
    cfg = tmp_path / "config.txt"
    cfg.write_text("1 /nonexistent 1 1 1\n")
    r = subprocess.run([EXE, "5", str(cfg), str(tmp_path / "log.txt")], capture_output=True,
                       text=True, timeout=60)
    assert r.returncode == 1 and "graph id" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("n", [0, 1, 1000, 300_000])
def test_coo_sort_stable_against_numpy(n):
    import torch
    import merbit_b200 as mb

    rng = np.random.default_rng(n)
    major = rng.integers(0, 500, n).astype(np.int32)
    minor = rng.integers(0, 50, n).astype(np.int32)  # many duplicate (major, minor) pairs
    vals = np.arange(n, dtype=np.float64)
    dM, dm, dv = (torch.from_numpy(a).cuda() for a in (major, minor, vals))
    mb.coo_sort(dM, dm, dv)
    order = np.lexsort((minor, major))  # stable: ties keep input order
    assert np.array_equal(dM.cpu().numpy(), major[order])
    assert np.array_equal(dm.cpu().numpy(), minor[order])
    assert np.array_equal(dv.cpu().numpy(), vals[order])


@pytest.mark.gpu
@pytest.mark.parametrize("nrow,n", [(1, 0), (10, 1), (5000, 40000), (7, 100)])
def test_coo_to_csr_against_numpy(nrow, n):
    import torch
    import merbit_b200 as mb

    rng = np.random.default_rng(nrow + n)
    rows = np.sort(rng.integers(0, nrow, n)).astype(np.int32)
    rp = mb.coo_to_csr(torch.from_numpy(rows).cuda(), nrow).cpu().numpy()
    assert np.array_equal(rp, np.searchsorted(rows, np.arange(nrow + 1), side="left"))


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32", "bf16"])
def test_outdegree_values_against_numpy(dtype):
    import torch
    import merbit_b200 as mb

    td = {"f64": torch.float64, "f32": torch.float32, "bf16": torch.bfloat16}[dtype]
    rng = np.random.default_rng(3)
    nrow = 2000
    rows = rng.zipf(1.8, 50000).clip(1, nrow).astype(np.int32) - 1
    v = mb.outdegree_values(torch.from_numpy(rows).cuda(), nrow, td)
    ref = torch.from_numpy(1.0 / np.bincount(rows, minlength=nrow)[rows]).to(td)
    assert torch.equal(v.cpu(), ref)


@pytest.mark.gpu
def test_outdegree_values_rejects_out_of_range_rows():
    import torch
    import merbit_b200 as mb

    rows = torch.tensor([0, 1, 5, 2], dtype=torch.int32, device="cuda")
    with pytest.raises(mb.MerbitError):
        mb.outdegree_values(rows, 3)
