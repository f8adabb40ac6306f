"""Failure detection without a GPU fault: every device-side spin of the
kernels (the cross-CTA carry wait, the mbarrier wait on staged copies) has a
time limit after which it records MERBIT_ERR_TIMEOUT and returns.  The
self-test entry point runs each wait on a flag nothing sets; the host reads
the status through merbit_plan_check and the context stays usable."""
import numpy as np
import pytest

from tests.helpers import csr_from_lengths, to_cuda


@pytest.mark.gpu
@pytest.mark.parametrize("which", [0, 1], ids=["carry_wait", "mbarrier_wait"])
def test_bounded_wait_reports_timeout_and_context_survives(which):
    import torch
    import merbit_b200 as mb

    A = csr_from_lengths(np.full(3000, 5), ncol=3000, seed=2)
    rp, col, v = to_cuda(A, "f64")
    plan = mb.Plan(rp, col, v)
    x = torch.ones(A.ncol, dtype=torch.float64, device="cuda")
    y0 = plan.spmv(x).clone()
    plan.check()
    plan.selftest_wait(which, wait_us=2000)
    with pytest.raises(mb.MerbitError) as ei:
        plan.check()
    assert ei.value.status == 5  # MERBIT_ERR_TIMEOUT
    plan.check()  # the status was cleared by the read
    # the context and the plan still work
    y1 = plan.spmv(x)
    plan.check()
    assert torch.equal(y0, y1)


def test_selftest_argument_checks_need_no_gpu():
    import merbit_b200 as mb

    L = mb.lib()
    assert L.merbit_plan_selftest_wait(None, 0, 100, None) == 1  # null plan: MERBIT_ERR_INVALID
