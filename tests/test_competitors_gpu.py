"""The reference's comparison libraries, run through oracle/competitors.cu
(cuSPARSE CSR_ALG2 / COO_ALG2, CUB DeviceSpmv, CSR5, HOLA; called as the
reference's src/spmv.cu calls them).  They are timing baselines, not part of
the product: these tests show that each harness entry computes the same
FP64 SpMV as the oracle, so that the times bench.py reports for them are
times of the right product."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from merbit_b200 import synth
from oracle import oracle as O
from tests.helpers import csr_from_lengths

SYMBOLS = ["comp_cusparse_time", "comp_cub_time", "comp_csr5_time", "comp_hola_time"]


def _matrices():
    rng = np.random.default_rng(11)
    return [
        ("zipf_small", synth.workload("zipf_small")),
        ("stencil27_small", synth.workload("stencil27_small")),
        ("laplace2d_small", synth.workload("laplace2d_small")),
        ("ragged_with_empty_rows", csr_from_lengths(rng.integers(0, 40, 20000), ncol=20000,
                                                    seed=12)),
    ]


def test_competitor_library_exports():
    L = O.comp()
    if L is None:
        pytest.skip("competitor harness oracle/_ref not built")
    for s in SYMBOLS:
        assert hasattr(L, s), s


@pytest.mark.gpu
@pytest.mark.parametrize("name,A", _matrices(), ids=lambda v: v if isinstance(v, str) else "")
def test_competitors_compute_the_same_spmv(name, A):
    import torch

    L = O.comp()
    if L is None:
        pytest.skip("competitor harness oracle/_ref not built")
    vals = np.ascontiguousarray(A.vals, np.float64)
    x = synth.uniform(0, A.ncol)
    y_ref, yabs = O.spmm(A.row_ptr, A.col, vals, x)
    rp = torch.from_numpy(A.row_ptr).cuda()
    col = torch.from_numpy(A.col).cuda()
    v = torch.from_numpy(vals).cuda()
    xd = torch.from_numpy(x).cuda()
    y = torch.zeros(A.nrow, dtype=torch.float64, device="cuda")
    ms, bms, sig = C.c_float(), C.c_float(), C.c_int()

    def check(label, rc):
        assert rc == 0, (label, rc)
        assert ms.value > 0, label
        e = np.abs(y.cpu().numpy() - y_ref) / np.maximum(yabs, 1e-300)
        assert e.max() <= 1e-12, (label, float(e.max()))
        y.zero_()

    check("cusparse_csr_alg2", L.comp_cusparse_time(0, A.nrow, A.ncol, A.nnz, rp.data_ptr(), None,
                                                    col.data_ptr(), v.data_ptr(), xd.data_ptr(),
                                                    y.data_ptr(), 3, C.byref(ms)))
    rows = torch.from_numpy(np.repeat(np.arange(A.nrow, dtype=np.int32),
                                      np.diff(A.row_ptr))).cuda()
    check("cusparse_coo_alg2", L.comp_cusparse_time(1, A.nrow, A.ncol, A.nnz, rp.data_ptr(),
                                                    rows.data_ptr(), col.data_ptr(), v.data_ptr(),
                                                    xd.data_ptr(), y.data_ptr(), 3, C.byref(ms)))
    check("cub_device_spmv", L.comp_cub_time(A.nrow, A.ncol, A.nnz, rp.data_ptr(),
                                             col.data_ptr(), v.data_ptr(), xd.data_ptr(),
                                             y.data_ptr(), 3, C.byref(ms)))
    col_w, v_w = col.clone(), v.clone()
    check("csr5", L.comp_csr5_time(A.nrow, A.ncol, A.nnz, rp.data_ptr(), col_w.data_ptr(),
                                   v_w.data_ptr(), xd.data_ptr(), y.data_ptr(), 3, C.byref(bms),
                                   C.byref(ms), C.byref(sig)))
    # destroy() transposes the CSR5 arrays back to CSR order
    assert torch.equal(col_w, col) and torch.equal(v_w, v)
    check("hola", L.comp_hola_time(A.nrow, A.ncol, A.nnz, rp.data_ptr(), col.data_ptr(),
                                   v.data_ptr(), xd.data_ptr(), y.data_ptr(), 3, C.byref(bms),
                                   C.byref(ms)))
