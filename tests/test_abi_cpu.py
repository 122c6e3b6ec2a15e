"""The C-ABI library loads on a CPU-only host, exports every entry point of include/*.h, and
applies the reference's argument conventions before touching a GPU."""
import ctypes as ct
import os
import pathlib
import re
import subprocess
import sys

import numpy as np
import pytest

from golden_cases import load_status_cases

ROOT = pathlib.Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*ssblasStatus_t\s+(ssblas\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_entry_point():
    import ssblasex_b200 as S
    names = declared_functions()
    assert {"ssblasGemmBatchedEx", "ssblasGemmBatchedEx_64", "ssblasGemmGroupedBatchedEx"} <= names
    L = S.lib()
    for n in names:
        assert hasattr(L, n), n
    assert set(S.EXPORTED_SYMBOLS) >= names
    out = subprocess.run(["nm", "-D", "--defined-only", str(S.LIB_PATH)], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert names <= exported
    assert all(e.startswith("ssblas") for e in exported)   # nothing else leaks out


def test_enums_match_reference_values():
    hdr = (ROOT / "include" / "ssblasBatch_type.h").read_text()
    for name in ["SSBLAS_STATUS_SUCCESS = 0", "SSBLAS_OP_N = 0", "SSBLAS_OP_T = 1", "SSBLAS_OP_C = 2"]:
        assert name in hdr
    order = ["SSBLAS_R_8I", "SSBLAS_R_8U", "SSBLAS_R_16F", "SSBLAS_R_32I", "SSBLAS_R_32F", "SSBLAS_R_64F"]
    pos = [hdr.index(o + ",") if o + "," in hdr else hdr.index(o + "\n") for o in order]
    assert pos == sorted(pos)


@pytest.mark.parametrize("use_64", [False, True])
def test_status_codes_before_any_device_work(golden, use_64):
    """Degenerate calls return the reference's status without a GPU (they never reach CUDA)."""
    from ssblasex_b200 import runner
    for p, over, ref_C, ref_st in load_status_cases(golden):
        st, C = runner.call(p, mode="host_matrices", use_64=use_64, **over)
        assert st == ref_st, (p.name, st, ref_st)
        np.testing.assert_array_equal(C, ref_C, err_msg=p.name)


def test_invalid_arguments_the_reference_does_not_check():
    from ssblasex_b200 import runner, workloads as W
    import ssblasex_b200 as S
    p = W.make_problem("f32", 0, 0, 9, 8, 7, 2, 1.0, 0.0, seed=1)
    assert runner.call(p, mode="host_matrices", lda=8)[0] == S.SSBLAS_STATUS_INVALID_VALUE
    assert runner.call(p, mode="host_matrices", ldc=3)[0] == S.SSBLAS_STATUS_INVALID_VALUE
    q = W.make_problem("i8", 2, 0, 9, 8, 7, 2, 1, 0, seed=1) if False else None
    # op C on the int8 row: the reference reads through NULL; here it is rejected
    p8 = W.make_problem("i8", 0, 0, 9, 8, 7, 2, 1, 0, seed=1)
    assert runner.call(p8, mode="host_matrices", transa=2)[0] == S.SSBLAS_STATUS_INVALID_VALUE
    al = np.array([1.0], np.float32)
    arr = (ct.c_void_p * 2)()
    st = S.lib().ssblasGemmBatchedEx(0, 0, 4, 4, 4, None, arr, 4, 4, arr, 4, 4, al.ctypes.data, arr, 4, 4, 2, 0, 0)
    assert st == S.SSBLAS_STATUS_INVALID_VALUE


def test_math_mode_and_settings():
    import ssblasex_b200 as S
    assert S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI | S.SSBLAS_MATH_FP32_BF16X3) == 0
    assert S.get_math_mode() == 3
    assert S.set_math_mode(8) == S.SSBLAS_STATUS_INVALID_VALUE
    assert S.set_math_mode(0) == 0
    assert S.set_ozaki_slices(2) == S.SSBLAS_STATUS_INVALID_VALUE
    assert S.set_ozaki_slices(0) == 0


def test_debug_dump_is_the_reference_text():
    spec_path = ROOT / "tests" / "golden" / "make_golden.py"
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", spec_path)
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    import ssblasex_b200 as S
    got = mg.dump_text(str(S.LIB_PATH))
    want = (ROOT / "tests" / "golden" / "debug_dump.txt").read_text()
    assert got == want
