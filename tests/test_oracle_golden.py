"""The CPU oracle is pinned against golden vectors produced by the reference library itself
(tests/golden/make_golden.py runs oracle/_ref, the reference compiled from its own sources)."""
import dataclasses

import numpy as np
import pytest

from golden_cases import fp_tolerance, load_cases, load_status_cases
from oracle import oracle as O


def test_golden_file_is_complete(golden):
    cases = list(load_cases(golden))
    assert len(cases) >= 70
    rows = {p.row for p, _, _ in cases}
    assert rows == {"f32", "f64", "i8"}
    combos = {(p.row, p.transa, p.transb) for p, _, _ in cases}
    assert len(combos) == 12                      # every row x every N/T combination
    assert any(p.k > 512 for p, _, _ in cases)    # crosses the reference's K blocks


def test_restatement_matches_reference(golden):
    for p, ref_C, ref_st in load_cases(golden):
        st, C = O.restated_gemm(p)
        assert st == ref_st == 0, p.name
        if p.row == "i8":
            np.testing.assert_array_equal(C, ref_C, err_msg=p.name)
        else:
            tol = fp_tolerance(p)
            e_ref = O.normalized_error(p, ref_C)
            e_us = O.normalized_error(p, C)
            assert e_ref <= tol and e_us <= tol, (p.name, e_ref, e_us, tol)


def test_reference_untouched_padding(golden):
    """Entries between m and ldc of every C column keep their input value in the reference."""
    for p, ref_C, _ in load_cases(golden):
        if p.ldc > p.m:
            pad = ref_C.reshape(p.batch, p.n, p.ldc)[:, :, p.m:]
            src = p.C.reshape(p.batch, p.n, p.ldc)[:, :, p.m:]
            np.testing.assert_array_equal(pad, src, err_msg=p.name)


def test_status_conventions(golden):
    """m, n or batchCount <= 0 -> INTERNAL_ERROR (3); k = 0 -> SUCCESS with C untouched;
    op C on the fp rows -> INVALID_VALUE (2). The restatement reproduces each status and effect."""
    seen = {}
    for p, over, ref_C, ref_st in load_status_cases(golden):
        seen[p.name] = ref_st
        if "types" in over:
            continue                               # type-row selection is tested on the ABI
        q = dataclasses.replace(p, **over)
        st, C = O.restated_gemm(q, C=p.C.copy())
        assert st == ref_st, (p.name, st, ref_st)
        np.testing.assert_array_equal(C, ref_C, err_msg=p.name)
    assert seen["m0"] == 3 and seen["n0"] == 3 and seen["batch0"] == 3
    assert seen["k0"] == 0 and seen["opC_f32"] == 2 and seen["bad_types"] == 2


def test_exact_oracle_against_longdouble():
    from ssblasex_b200 import workloads as W
    p = W.make_problem("f64", 0, 1, 7, 6, 50, 1, alpha=0.75, beta=-2.0, seed=4, dist="expspread")
    ex, nrm = O.exact_f64(p, 0)
    a = p.op_a(0).astype(np.longdouble)
    b = p.op_b(0).astype(np.longdouble)
    c0 = p.c_view(p.C, 0).astype(np.longdouble)
    want = np.longdouble(p.alpha) * (a @ b) + np.longdouble(p.beta) * c0
    assert np.max(np.abs(ex - want.astype(np.float64)) / nrm) < 2.0 ** -52


@pytest.fixture(scope="module")
def config_fixtures():
    import pathlib
    return np.load(pathlib.Path(__file__).resolve().parent / "golden" / "config_cases.npz")


@pytest.mark.parametrize("name", ["fp32_batch64_128", "f64_batch32_1024", "i8_batch512_512", "fp32_batch4096_64"])
def test_restatement_matches_reference_at_benchmark_shapes(config_fixtures, name):
    """The reference's output at the benchmark configurations' full shapes (all of 64 x 128^3, a
    slice of the others) against the C restatement on regenerated inputs: pins the restatement at
    those sizes and that the seeded inputs are the ones the reference saw."""
    from golden_cases import check_against_config_fixture, load_config_case
    p, rows, ref_rows, ref_colsum = load_config_case(config_fixtures, name)
    st, C = O.restated_gemm(p)
    assert st == 0
    tol = 0.0 if p.row == "i8" else fp_tolerance(p)
    check_against_config_fixture(p, C, rows, ref_rows, ref_colsum, O.exact_f64, tol)
