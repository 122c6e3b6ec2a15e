"""Failure detection on a B200, without faulting or hanging the GPU (ssblasSetFaultInjection):

  * a tensor-core GEMM launch whose first thread block skips one operand copy: the waits on that
    copy run out after a short limit, the kernel records the error in the device flag and exits
    (its other blocks finish normally, tensor memory is released), and the call returns
    SSBLAS_STATUS_INTERNAL_ERROR with the run info's device_error set; the next call on the same
    process is correct;
  * a workspace allocation that fails: SSBLAS_STATUS_ALLOC_FAILED, nothing launched, C untouched.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture
def S():
    import torch
    assert torch.cuda.is_available()
    import ssblasex_b200 as S
    S.set_math_mode(S.SSBLAS_MATH_PLAIN)
    yield S
    S.set_fault_injection(S.SSBLAS_FAULT_NONE)
    S.set_math_mode(S.SSBLAS_MATH_PLAIN)


def test_skipped_copy_is_reported_and_the_next_call_is_correct(S):
    from ssblasex_b200 import runner, workloads as W
    p = W.make_problem("i8", 1, 0, 256, 512, 512, 4, 1, 0, seed=81)
    dp = runner.DeviceProblem(p)
    assert S.set_fault_injection(S.SSBLAS_FAULT_SKIP_COPY) == 0
    st, _ = runner.call(p, mode="device_array", dp=dp)
    info = S.last_run_info()
    assert st == S.SSBLAS_STATUS_INTERNAL_ERROR
    assert info["path"] == "i8_tcgen05" and info["device_error"] != 0
    for _ in range(2):
        dp.reset_c()
        st, C = runner.call(p, mode="device_array", dp=dp)
        assert st == 0 and S.last_run_info()["device_error"] == 0
        np.testing.assert_array_equal(C, O.restated_gemm(p)[1])


def test_allocation_failure_leaves_c_untouched(S):
    import torch
    from ssblasex_b200 import runner, workloads as W
    p = W.make_problem("f64", 0, 1, 200, 180, 300, 3, 1.0, 0.5, seed=82, dist="expspread")
    dp = runner.DeviceProblem(p)
    before = dp.C.clone()
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
    assert S.set_fault_injection(S.SSBLAS_FAULT_ALLOC) == 0
    st, _ = runner.call(p, mode="device_array", dp=dp)
    assert st == S.SSBLAS_STATUS_ALLOC_FAILED
    assert torch.equal(dp.C, before)
    st, C = runner.call(p, mode="device_array", dp=dp)
    assert st == 0
    np.testing.assert_array_equal(C.view(np.uint64), O.ozaki_f64(p, 7)[1].view(np.uint64))
