"""The type and semantics extensions (ssblasSetExtensions) on a B200, through the C ABI. Each is
off by default; with it off the call behaves as the reference does (pinned by the golden status
cases and tests/test_abi_cpu.py).

  * SSBLAS_EXT_R16F: fp16 op(A), op(B), fp16 or fp32 C, fp32 accumulation on tcgen05 kind::f16
    (direct staging in every layout) and on the SIMT kernel (leading dimensions that cannot be
    staged directly): within FP32 accumulation error plus the one rounding of C to its type;
  * SSBLAS_EXT_R8U: unsigned int8 for either operand, bit-exact (int32 wrap-around);
  * SSBLAS_EXT_OP_C: op C gives exactly the op T result;
  * SSBLAS_EXT_K0_BETA: k = 0 scales C by beta (zeros for beta = 0, C not read);
  * SSBLAS_EXT_COMPUTE_TYPE: COMPUTE_32F on the fp32 row keeps FP32 arithmetic in the 3xBF16 mode.
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
    S.set_extensions(S.SSBLAS_EXT_NONE)
    S.set_math_mode(S.SSBLAS_MATH_PLAIN)


def int_exact(p, b):
    """alpha * op(A) op(B) + beta * C0 in wrapping int32, from exact int64 products."""
    want = (p.op_a(b).astype(np.int64) @ p.op_b(b).astype(np.int64) * int(p.alpha)
            + int(p.beta) * p.c_view(p.C, b).astype(np.int64))
    return ((want + 2 ** 31) % 2 ** 32 - 2 ** 31).astype(np.int32)


def f16_check(p, C):
    """FP32 accumulation of exact fp16 products, then one rounding to C's type."""
    for b in range(p.batch):
        a = p.op_a(b).astype(np.float64)
        bb = p.op_b(b).astype(np.float64)
        c0 = p.c_view(p.C, b).astype(np.float64)
        exact = p.alpha * (a @ bb) + p.beta * c0
        norm = abs(p.alpha) * (np.abs(a) @ np.abs(bb)) + abs(p.beta) * np.abs(c0)
        got = p.c_view(C, b).astype(np.float64)
        u_c = 2.0 ** -11 if p.C.dtype == np.float16 else 2.0 ** -24
        bound = 4 * p.k * 2.0 ** -24 * norm + u_c * np.abs(exact) + 2.0 ** -24
        assert np.all(np.abs(got - exact) <= bound), (p.name, b, float(np.max(np.abs(got - exact) / bound)))


@pytest.mark.parametrize("row", ["f16", "f16c32"])
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("aligned", [True, False])
def test_fp16_row(S, row, ta, tb, aligned):
    from ssblasex_b200 import runner, workloads as W
    m, n, k = 200, 136, 300
    al = (lambda x: -(-x // 8) * 8) if aligned else (lambda x: x + 1 if x % 8 == 0 else x)
    p = W.make_problem(row, ta, tb, m, n, k, 3, 0.75, -0.5, lda=al(m if ta == 0 else k),
                       ldb=al(k if tb == 0 else n), ldc=m + 2, seed=ta + 2 * tb + (0 if aligned else 10), name=row)
    assert runner.call(p, mode="device_array")[0] == S.SSBLAS_STATUS_INVALID_VALUE   # extension off
    S.set_extensions(S.SSBLAS_EXT_R16F)
    st, C = runner.call(p, mode="device_array")
    assert st == 0
    assert S.last_run_info()["path"] == ("f16_tcgen05" if aligned else "simt")
    f16_check(p, C)
    # the ld padding of C is untouched
    pad = C.reshape(p.batch, p.n, p.ldc)[:, :, p.m:]
    np.testing.assert_array_equal(pad, p.C.reshape(p.batch, p.n, p.ldc)[:, :, p.m:])


@pytest.mark.parametrize("row", ["u8", "u8s8", "s8u8"])
@pytest.mark.parametrize("ta,tb,aligned", [(1, 0, True), (0, 1, True), (0, 0, False), (1, 1, True)])
def test_unsigned_int8_rows(S, row, ta, tb, aligned):
    from ssblasex_b200 import runner, workloads as W
    m, n, k = 150, 270, 333
    al = (lambda x: -(-x // 16) * 16) if aligned else (lambda x: x)
    p = W.make_problem(row, ta, tb, m, n, k, 2, 3, -1, lda=al(m if ta == 0 else k), ldb=al(k if tb == 0 else n),
                       seed=11 + ta + 2 * tb)
    assert runner.call(p, mode="device_array")[0] == S.SSBLAS_STATUS_INVALID_VALUE   # extension off
    S.set_extensions(S.SSBLAS_EXT_R8U)
    st, C = runner.call(p, mode="device_array")
    assert st == 0 and S.last_run_info()["path"] == "i8_tcgen05"
    for b in range(p.batch):
        np.testing.assert_array_equal(p.c_view(C, b), int_exact(p, b))


@pytest.mark.parametrize("row", ["f32", "f64", "i8"])
def test_op_c_is_op_t(S, row):
    from ssblasex_b200 import runner, workloads as W
    p = W.make_problem(row, 1, 1, 70, 50, 90, 2, 1, 0, seed=5)
    S.set_extensions(S.SSBLAS_EXT_OP_C)
    st_t, C_t = runner.call(p, mode="device_array")
    st_c, C_c = runner.call(p, mode="device_array", transa=2, transb=2)
    assert st_t == st_c == 0
    np.testing.assert_array_equal(C_c, C_t)
    S.set_extensions(S.SSBLAS_EXT_NONE)
    assert runner.call(p, mode="device_array", transa=2)[0] == S.SSBLAS_STATUS_INVALID_VALUE


@pytest.mark.parametrize("row", ["f32", "f64", "i8", "f16"])
@pytest.mark.parametrize("beta", [0, 2])
@pytest.mark.parametrize("mode", ["device_array", "host_matrices"])
def test_k0_scales_c_by_beta(S, row, beta, mode):
    from ssblasex_b200 import runner, workloads as W
    p = W.make_problem(row, 0, 0, 33, 17, 5, 2, 3, beta, ldc=40, seed=9)
    S.set_extensions(S.SSBLAS_EXT_K0_BETA | S.SSBLAS_EXT_R16F)
    st, C = runner.call(p, mode=mode, k=0)
    assert st == 0
    for b in range(p.batch):
        want = (p.c_view(p.C, b).astype(np.float64) * beta).astype(p.C.dtype)
        np.testing.assert_array_equal(p.c_view(C, b), want)
    np.testing.assert_array_equal(C.reshape(2, 17, 40)[:, :, 33:], p.C.reshape(2, 17, 40)[:, :, 33:])
    assert runner.call(p, mode=mode, k=-1)[0] == S.SSBLAS_STATUS_INVALID_VALUE
    # without the extension: the reference's k = 0 convention (success, C untouched)
    S.set_extensions(S.SSBLAS_EXT_R16F)
    st, C = runner.call(p, mode=mode, k=0)
    assert st == 0
    np.testing.assert_array_equal(C, p.C)


def test_compute_type_32f_keeps_fp32_arithmetic(S):
    from ssblasex_b200 import workloads as W
    import ctypes as ct
    from ssblasex_b200 import runner
    p = W.make_problem("f32", 0, 0, 128, 128, 256, 2, 1.0, 0.0, seed=4)
    dp = runner.DeviceProblem(p)
    Ad, Bd, Cd = dp.device_arrays()
    al, be = np.array([1.0], np.float32), np.array([0.0], np.float32)

    def call(compute):
        return S.lib().ssblasGemmBatchedEx(0, 0, p.m, p.n, p.k, al.ctypes.data, Ad.data_ptr(), S.SSBLAS_R_32F, p.lda,
                                           Bd.data_ptr(), S.SSBLAS_R_32F, p.ldb, be.ctypes.data, Cd.data_ptr(),
                                           S.SSBLAS_R_32F, p.ldc, p.batch, compute, 0)
    S.set_math_mode(S.SSBLAS_MATH_FP32_BF16X3)
    assert call(S.SSBLAS_COMPUTE_32F) == 0 and S.last_run_info()["path"] == "bf16x3_tcgen05"   # ignored
    S.set_extensions(S.SSBLAS_EXT_COMPUTE_TYPE)
    assert call(S.SSBLAS_COMPUTE_32F) == 0 and S.last_run_info()["path"] == "simt"
    assert O.normalized_error(p, dp.C.cpu().numpy()) <= 4 * p.k * 2.0 ** -24
    assert call(S.SSBLAS_COMPUTE_DEFAULT_TYPE) == 0 and S.last_run_info()["path"] == "bf16x3_tcgen05"
    assert call(S.SSBLAS_COMPUTE_32I) == S.SSBLAS_STATUS_INVALID_VALUE
