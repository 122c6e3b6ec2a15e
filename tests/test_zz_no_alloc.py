"""ssblasGemmBatchedExNoAlloc on a B200, through the C ABI.

The allocation-free entry point serves callers that cannot let a library allocate device memory
(a pool allocator that owns all of the GPU's memory, or a loop where a synchronising cudaMalloc
is not allowed). Its scratch is one fixed device array shared by all calls, so the checks are:
two calls in a row -- of different shapes, so the second one runs over the first one's leftover
scratch -- each give exactly the result of the regular entry point in the same (Ozaki FP64)
mode, and a problem larger than the array is refused without touching C.

This file is collected last, so a run that stops at its first failure has already run every
other test; it also passes on its own in a fresh process.
"""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(S, p, dp):
    Ad, Bd, Cd = dp.device_arrays()
    al = np.array([p.alpha], np.float64)
    be = np.array([p.beta], np.float64)
    return S.lib().ssblasGemmBatchedExNoAlloc(p.transa, p.transb, p.m, p.n, p.k, al.ctypes.data, Ad.data_ptr(),
                                              S.SSBLAS_R_64F, p.lda, Bd.data_ptr(), S.SSBLAS_R_64F, p.ldb,
                                              be.ctypes.data, Cd.data_ptr(), S.SSBLAS_R_64F, p.ldc, p.batch, 0, 0)


def test_noalloc_matches_the_regular_entry_point_on_two_calls_in_a_row():
    import torch
    assert torch.cuda.is_available()
    import ssblasex_b200 as S
    from ssblasex_b200 import runner, workloads as W
    problems = [
        W.make_problem("f64", 0, 1, 300, 200, 500, 3, 0.75, -0.5, seed=31, dist="expspread"),
        W.make_problem("f64", 1, 0, 129, 260, 1030, 2, 1.0, 0.0, seed=32, dist="expspread"),
    ]
    S.set_ozaki_slices(0)
    try:
        for p in problems:
            # the regular entry point in the same mode (uses the library's allocated workspace)
            S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
            st, want = runner.call(p, mode="device_array")
            assert st == 0 and S.last_run_info()["path"] == "ozaki_tcgen05"
            # the allocation-free entry point on fresh device copies of the same inputs
            S.set_math_mode(S.SSBLAS_MATH_PLAIN)    # it does not depend on the math mode
            dp = runner.DeviceProblem(p)
            assert _noalloc(S, p, dp) == 0
            got = dp.C.cpu().numpy()
            # same algorithm and operation order: the results agree bit for bit
            np.testing.assert_array_equal(got.view(np.uint64), want.view(np.uint64))
    finally:
        S.set_math_mode(S.SSBLAS_MATH_PLAIN)


def test_noalloc_refuses_problems_beyond_its_scratch():
    import torch
    import ssblasex_b200 as S
    from ssblasex_b200 import runner, workloads as W
    # 7 slices * (1024 + 1024) * 1024 * 8 instances = 117 MB > the 64 MiB array
    p = W.make_problem("f64", 0, 0, 1024, 1024, 1024, 8, 1.0, 0.0, seed=1)
    dp = runner.DeviceProblem(p)
    before = dp.C.clone()
    assert _noalloc(S, p, dp) == S.SSBLAS_STATUS_INVALID_VALUE
    assert torch.equal(dp.C, before)
    # other type rows have no allocation-free variant
    al = np.array([1.0], np.float32)
    arr = torch.zeros(1, dtype=torch.int64, device="cuda")
    st = S.lib().ssblasGemmBatchedExNoAlloc(0, 0, 4, 4, 4, al.ctypes.data, arr.data_ptr(), S.SSBLAS_R_32F, 4,
                                            arr.data_ptr(), S.SSBLAS_R_32F, 4, al.ctypes.data, arr.data_ptr(),
                                            S.SSBLAS_R_32F, 4, 1, 0, 0)
    assert st == S.SSBLAS_STATUS_NOTIMPLEMENTED_ERROR


@pytest.mark.parametrize("slices,shape", [
    # few rows: both operands through the one-kernel slicer for long K
    (7, (128, 128, 4096, 4)),
    # one operand with enough rows for the two-kernel form (exponents, then digits per chunk);
    # (320 row blocks of 32 >= two per SM); 3 slices, so 3 * (10240 + 16) * 2064 bytes still fit
    (3, (10240, 16, 2064, 1)),
])
def test_noalloc_long_k_matches_the_regular_entry_point(slices, shape):
    """For 2048 < k <= 16384 the allocation-free entry point slices with its own kernels (the
    regular path uses the two-pass row-maximum / slab form, which needs workspace): the digits and
    therefore the results must still agree bit for bit."""
    import ssblasex_b200 as S
    from ssblasex_b200 import runner, workloads as W
    m, n, k, batch = shape
    p = W.make_problem("f64", 0, 1, m, n, k, batch, 1.0, 0.5, seed=k, dist="expspread")
    S.set_ozaki_slices(slices)
    try:
        S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
        st, want = runner.call(p, mode="device_array")
        assert st == 0 and S.last_run_info()["slices"] == slices
        S.set_math_mode(S.SSBLAS_MATH_PLAIN)
        for _ in range(2):
            dp = runner.DeviceProblem(p)
            assert _noalloc(S, p, dp) == 0
            info = S.last_run_info()
            assert info["path"] == "ozaki_tcgen05" and info["slices"] == slices
            np.testing.assert_array_equal(dp.C.cpu().numpy().view(np.uint64), want.view(np.uint64))
    finally:
        S.set_ozaki_slices(0)
        S.set_math_mode(S.SSBLAS_MATH_PLAIN)


def test_noalloc_refuses_k_beyond_one_exact_piece():
    import torch
    import ssblasex_b200 as S
    from ssblasex_b200 import runner, workloads as W
    p = W.make_problem("f64", 0, 1, 16, 16, 16385, 1, 1.0, 0.0, seed=2)
    dp = runner.DeviceProblem(p)
    before = dp.C.clone()
    assert _noalloc(S, p, dp) == S.SSBLAS_STATUS_INVALID_VALUE
    assert torch.equal(dp.C, before)
