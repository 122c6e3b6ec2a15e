"""The benchmark configurations at their full sizes on a B200, through the C ABI.

  * FP64 32 x 1024^3 NT (ld 1032, entries spread over 2^+-8): the Ozaki mode's error against the
    FP64-exact oracle is within 4 k u, within the stated a-priori bound, and no larger than the
    plain DMMA path's error on the same inputs (the equal-error condition of the speed target);
    the automatic slice count is 7.
  * FP32 4096 x 64^3 TT with 1% outliers (x 1e4): plain FFMA within 4 k u, 3xBF16 within its
    stated error against the FP64-exact value and within FP32 accumulation error of the exact
    value of its own three BF16 products.
  * The grouped workload of 10,000 uneven instances (half fp64 Ozaki, half fp32 3xBF16): a seeded
    sample of 500 instances against their CPU restatements (Ozaki bit for bit).
  * Rows whose entries span 2^+-30: the stated bound holds at the automatic slice count and at the
    counts other tolerances select.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

U64 = 2.0 ** -53
U32 = 2.0 ** -24


@pytest.fixture
def S():
    import torch
    assert torch.cuda.is_available()
    import ssblasex_b200 as S
    S.set_math_mode(S.SSBLAS_MATH_PLAIN)
    S.set_ozaki_slices(0)
    S.set_ozaki_tolerance(0)
    yield S
    S.set_math_mode(S.SSBLAS_MATH_PLAIN)
    S.set_ozaki_slices(0)
    S.set_ozaki_tolerance(0)


def test_ozaki_full_f64_batch32_1024_error_at_most_plain(S):
    from ssblasex_b200 import runner, workloads as W
    from bounds import check_ozaki
    p = W.workload("f64_batch32_1024")
    dp = runner.DeviceProblem(p)
    rows = np.arange(3, p.m, 127)                     # 9 rows of every instance, all 1024 columns
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
    st, C_oz = runner.call(p, mode="device_array", dp=dp)
    info = S.last_run_info()
    assert st == 0 and info["path"] == "ozaki_tcgen05" and info["slices"] == 7
    err_oz = O.normalized_error(p, C_oz, instances=range(p.batch), rows=rows)
    check_ozaki(p, C_oz, 7, range(p.batch), rows, O.exact_f64)
    S.set_math_mode(S.SSBLAS_MATH_PLAIN)
    dp.reset_c()
    st, C_pl = runner.call(p, mode="device_array", dp=dp)
    assert st == 0 and S.last_run_info()["path"] == "dmma"
    err_pl = O.normalized_error(p, C_pl, instances=range(p.batch), rows=rows)
    assert err_pl <= 4 * p.k * U64
    assert err_oz <= 4 * p.k * U64
    assert err_oz <= err_pl, (err_oz, err_pl)


def test_fp32_full_batch4096_64_both_modes(S):
    from ssblasex_b200 import runner, workloads as W
    p = W.workload("fp32_batch4096_64")
    dp = runner.DeviceProblem(p)
    sample = np.random.default_rng(11).choice(p.batch, 192, replace=False)
    st, C = runner.call(p, mode="device_array", dp=dp)
    assert st == 0
    assert O.normalized_error(p, C, instances=sample) <= 4 * p.k * U32
    S.set_math_mode(S.SSBLAS_MATH_FP32_BF16X3)
    dp.reset_c()
    st, C = runner.call(p, mode="device_array", dp=dp)
    assert st == 0 and S.last_run_info()["path"] == "bf16x3_tcgen05"
    for b in sample:
        emu = O.bf16x3_f32(p, b)
        ex, nrm = O.exact_f64(p, b)
        got = p.c_view(C, b).astype(np.float64)
        assert np.max(np.abs(got - emu) / nrm) <= 4 * p.k * U32, b
        assert np.max(np.abs(got - ex) / nrm) <= 2.0 ** -14, b


def test_grouped_full_10000_sampled(S):
    from ssblasex_b200 import runner, workloads as W
    probs = W.grouped_problems(count=10000)
    gd = runner.GroupedDevice(probs)
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI | S.SSBLAS_MATH_FP32_BF16X3)
    rng = np.random.default_rng(2024)
    sample = np.concatenate([rng.choice(5000, 250, replace=False), 5000 + rng.choice(5000, 250, replace=False)])
    for rep in range(2):                              # planned call, then the replayed graph
        gd.reset_c()
        assert gd.call(device_arrays=True) == 0
        assert S.last_run_info()["path"] == "grouped"
        res = gd.results()
        for i in sample:
            p, C = probs[i], res[i]
            if p.row == "f64":
                want = O.ozaki_f64(p, 7)[1]
                np.testing.assert_array_equal(C.view(np.uint64), want.view(np.uint64), err_msg=p.name)
            else:
                emu = O.bf16x3_f32(p, 0)
                ex, nrm = O.exact_f64(p, 0)
                got = p.c_view(C, 0).astype(np.float64)
                assert np.max(np.abs(got - emu) / nrm) <= 4 * p.k * U32, p.name
                assert np.max(np.abs(got - ex) / nrm) <= 2.0 ** -14, p.name


@pytest.mark.parametrize("tol,slices", [(0.0, 7), (2.0 ** -30, 5), (2.0 ** -20, 3), (2.0 ** -56, 8)])
@pytest.mark.parametrize("ta,tb", [(0, 1), (1, 0), (0, 0), (1, 1)])
def test_ozaki_stated_bound_on_wide_rows(S, tol, slices, ta, tb):
    from ssblasex_b200 import runner, workloads as W
    from bounds import check_ozaki
    p = W.make_problem("f64", ta, tb, 300, 260, 1030, 2, -0.75, 0.5, seed=70 + ta + 2 * tb, dist="expspread30")
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
    assert S.set_ozaki_tolerance(tol) == 0
    st, C = runner.call(p, mode="device_array")
    assert st == 0 and S.last_run_info()["slices"] == slices
    # same digits and operation order as the CPU restatement
    np.testing.assert_array_equal(C.view(np.uint64), O.ozaki_f64(p, slices)[1].view(np.uint64))
    check_ozaki(p, C, slices, range(p.batch), np.arange(0, p.m, 7), O.exact_f64)
