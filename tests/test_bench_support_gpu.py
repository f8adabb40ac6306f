"""The measurement probe of include/merbit_bench.h: merbit_bench_gather sums
x at every index (indices outside [0, nx) read x[0]), so the rate bench.py
reports is a rate of gathers that really happened."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import merbit_b200 as mb


@pytest.mark.gpu
@pytest.mark.parametrize("n", [8, 1 << 12, (1 << 20) + 8 * 37])
def test_gather_probe_sums_every_gathered_value(n):
    import torch

    rng = np.random.default_rng(n)
    nx = 5000
    idx = rng.integers(-10, nx + 10, n).astype(np.int32)
    x = rng.standard_normal(nx)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    xd = torch.from_numpy(x).cuda()
    idd = torch.from_numpy(idx).cuda()
    out = torch.zeros(sms * 2048, dtype=torch.float64, device="cuda")
    st = mb.lib().merbit_bench_gather(C.c_void_p(xd.data_ptr()), nx, C.c_void_p(idd.data_ptr()), n,
                                      C.c_void_p(out.data_ptr()), out.numel(), None)
    assert st == 0, mb.lib().merbit_last_error_detail()
    torch.cuda.synchronize()
    safe = np.where((idx >= 0) & (idx < nx), idx, 0)
    expect = x[safe].sum()
    got = float(out.sum())
    assert abs(got - expect) <= 1e-9 * np.abs(x[safe]).sum()
