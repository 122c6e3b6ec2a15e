"""Parity of the CUDA path with the reference, through the C ABI, on a B200.

  * golden vectors made by the reference itself: int8 bit-exact, fp within 4*k*u normalised by
    |alpha||op(A)||op(B)| + |beta||C|, under all three pointer conventions;
  * the reference's status conventions and its untouched-C cases;
  * seeded problems against the C restatement of the reference (oracle/) at sizes it finishes in
    seconds, and the named full-size workloads through size-independent checks.
"""
import numpy as np
import pytest

from golden_cases import fp_tolerance, load_cases, load_status_cases
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MODES = ["device_array", "host_array", "host_matrices"]


@pytest.fixture(scope="module")
def S():
    import torch
    assert torch.cuda.is_available()
    import ssblasex_b200 as S
    S.set_math_mode(S.SSBLAS_MATH_PLAIN)
    return S


def check(p, C, ref_C):
    if p.row == "i8":
        np.testing.assert_array_equal(C, ref_C, err_msg=p.name)
    else:
        tol = fp_tolerance(p)
        err = O.normalized_error(p, C)
        assert err <= tol, (p.name, err, tol)
        # entries outside the m x n part of each C keep their value
        if p.ldc > p.m:
            got = C.reshape(p.batch, p.n, p.ldc)[:, :, p.m:]
            np.testing.assert_array_equal(got, p.C.reshape(p.batch, p.n, p.ldc)[:, :, p.m:])


@pytest.mark.parametrize("mode", MODES)
def test_golden_vectors(S, golden, mode):
    from ssblasex_b200 import runner
    for p, ref_C, ref_st in load_cases(golden):
        st, C = runner.call(p, mode=mode)
        assert st == ref_st == 0, (p.name, st)
        check(p, C, ref_C)


@pytest.mark.parametrize("mode", MODES)
def test_status_cases_on_gpu(S, golden, mode):
    from ssblasex_b200 import runner
    for p, over, ref_C, ref_st in load_status_cases(golden):
        st, C = runner.call(p, mode=mode, **over)
        assert st == ref_st, (p.name, st, ref_st)
        np.testing.assert_array_equal(C, ref_C, err_msg=p.name)


def test_entry_point_64_matches(S, golden):
    from ssblasex_b200 import runner
    for p, ref_C, _ in list(load_cases(golden))[::7]:
        st, C = runner.call(p, mode="device_array", use_64=True)
        assert st == 0
        check(p, C, ref_C)


@pytest.mark.parametrize("row", ["f32", "f64", "i8"])
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_against_restated_oracle(S, row, ta, tb):
    """Medium shapes with ragged tails over every tile edge, ld > rows, beta != 0."""
    from ssblasex_b200 import runner, workloads as W
    al, be = (3, -2) if row == "i8" else (0.75, -1.5)
    p = W.make_problem(row, ta, tb, 203, 131, 700, 3, al, be, lda=None, seed=11 + 4 * ta + tb)
    st, C = runner.call(p, mode="device_array")
    assert st == 0
    st_o, C_o = O.restated_gemm(p)
    if row == "i8":
        np.testing.assert_array_equal(C, C_o)
    else:
        tol = fp_tolerance(p)
        assert O.normalized_error(p, C, rows=range(0, 203, 7)) <= tol
        assert O.normalized_error(p, C_o, rows=range(0, 203, 7)) <= tol


@pytest.mark.parametrize("row,mode", [("f32", 0), ("f64", 0), ("i8", 0), ("f64", 1), ("f32", 2)])
def test_host_matrices_pipelined(S, row, mode):
    """Host matrices (the reference's convention) in a batch large enough for the chunked,
    overlapped staging: the same result as with device pointers, and the callers' ld padding of
    C is untouched."""
    from ssblasex_b200 import runner, workloads as W
    S.set_math_mode(mode)
    try:
        al, be = (2, -1) if row == "i8" else (0.75, 0.5)
        p = W.make_problem(row, 1, 0, 100, 70, 130, 13, al, be, lda=136, ldb=136, ldc=104, seed=70 + mode,
                           dist="expspread" if row == "f64" else "uniform")
        st, C_host = runner.call(p, mode="host_matrices")
        assert st == 0
        st, C_dev = runner.call(p, mode="device_array")
        assert st == 0
        np.testing.assert_array_equal(C_host.view(np.uint8), C_dev.view(np.uint8))
        pad = C_host.reshape(p.batch, p.n, p.ldc)[:, :, p.m:]
        np.testing.assert_array_equal(pad, p.C.reshape(p.batch, p.n, p.ldc)[:, :, p.m:])
    finally:
        S.set_math_mode(0)


def test_beta_zero_never_reads_c(S):
    """C full of NaN with beta = 0 gives finite results (C is not read)."""
    from ssblasex_b200 import runner, workloads as W
    for row in ("f32", "f64"):
        p = W.make_problem(row, 0, 1, 70, 50, 40, 2, 1.0, 0.0, seed=5)
        p.C[:] = np.nan
        st, C = runner.call(p, mode="device_array")
        assert st == 0 and np.isfinite(p.c_view(C, 0)).all() and np.isfinite(p.c_view(C, 1)).all()


def test_int8_wraparound(S):
    from ssblasex_b200 import runner, workloads as W
    p = W.make_problem("i8", 1, 0, 96, 80, 1024, 2, 1 << 20, 1 << 14, seed=6)
    st, C = runner.call(p, mode="device_array")
    st_o, C_o = O.restated_gemm(p)
    assert st == 0
    np.testing.assert_array_equal(C, C_o)


# ------------------------------------------------------------- full-size named workloads ----
def test_fp32_batch64_128_full(S):
    from ssblasex_b200 import runner, workloads as W
    p = W.workload("fp32_batch64_128")
    st, C = runner.call(p, mode="device_array")
    assert st == 0
    st_o, C_o = O.restated_gemm(p)
    tol = fp_tolerance(p)
    assert O.normalized_error(p, C, instances=range(0, 64, 9), rows=range(0, 128, 5)) <= tol
    assert np.max(np.abs(C - C_o)) < 1e-3


def test_i8_batch512_512_full(S):
    """Bit-exact on every instance: integer checks with numpy int64 on all 512 instances."""
    from ssblasex_b200 import runner, workloads as W
    p = W.workload("i8_batch512_512")
    st, C = runner.call(p, mode="device_array")
    assert st == 0
    for b in range(p.batch):
        want = (p.op_a(b).astype(np.int64) @ p.op_b(b).astype(np.int64) * int(p.alpha)
                + int(p.beta) * p.c_view(p.C, b).astype(np.int64))
        want = ((want + 2 ** 31) % 2 ** 32 - 2 ** 31).astype(np.int32)
        np.testing.assert_array_equal(p.c_view(C, b), want, err_msg=f"instance {b}")


def test_f64_batch32_1024_plain_error(S):
    from ssblasex_b200 import runner, workloads as W
    p = W.workload("f64_batch32_1024")
    st, C = runner.call(p, mode="device_array")
    assert st == 0
    err = O.normalized_error(p, C, instances=[0, 17, 31], rows=range(0, 1024, 61))
    assert err <= fp_tolerance(p)


def test_fp32_batch4096_64_full(S):
    from ssblasex_b200 import runner, workloads as W
    p = W.workload("fp32_batch4096_64")
    st, C = runner.call(p, mode="device_array")
    assert st == 0
    tol = fp_tolerance(p)
    assert O.normalized_error(p, C, instances=range(0, 4096, 257)) <= tol


@pytest.fixture(scope="module")
def config_fixtures():
    import pathlib
    return np.load(pathlib.Path(__file__).resolve().parent / "golden" / "config_cases.npz")


@pytest.mark.parametrize("name,mode", [("fp32_batch64_128", 0), ("f64_batch32_1024", 0), ("f64_batch32_1024", 1),
                                       ("i8_batch512_512", 0), ("fp32_batch4096_64", 0), ("fp32_batch4096_64", 2)])
def test_reference_output_at_benchmark_shapes(S, config_fixtures, name, mode):
    """The CUDA path against the reference's own output at the benchmark configurations' shapes
    (tests/golden/config_cases.npz, made by running the reference): int8 bit-exact; plain fp and
    the Ozaki FP64 mode within 4*k*u normalised; 3xBF16 within its stated 2^-14."""
    from golden_cases import check_against_config_fixture, load_config_case
    from ssblasex_b200 import runner
    p, rows, ref_rows, ref_colsum = load_config_case(config_fixtures, name)
    S.set_math_mode(mode)
    try:
        st, C = runner.call(p, mode="device_array")
    finally:
        S.set_math_mode(S.SSBLAS_MATH_PLAIN)
    assert st == 0
    tol = 0.0 if p.row == "i8" else (2.0 ** -14 if mode == 2 else fp_tolerance(p))
    check_against_config_fixture(p, C, rows, ref_rows, ref_colsum, O.exact_f64, tol)
