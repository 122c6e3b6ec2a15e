"""Host matrices the way the reference's example allocates them: every instance its own pageable
allocation (example/main.cpp:58-66). Above 4 MB these go through pinned staging packed and
unpacked by host threads (hostcopy.cpp); the result must equal the device-array call's bit for bit,
and the caller's C padding rows must keep their values."""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture
def S():
    import torch
    assert torch.cuda.is_available()
    import ssblasex_b200 as S
    yield S
    S.set_math_mode(S.SSBLAS_MATH_PLAIN)


@pytest.mark.parametrize("layout", ["scattered", "dense"])
@pytest.mark.parametrize("row,mode,ta,tb,beta", [("f64", "ozaki", 0, 1, 0.0), ("f64", "plain", 1, 0, 0.5),
                                                 ("i8", "plain", 1, 0, 1), ("f32", "bf16x3", 0, 0, 0.25)])
def test_scattered_pageable_instances(S, row, mode, ta, tb, beta, layout):
    """scattered: one allocation per instance; dense: the instances are equally spaced views of one
    pageable array (the layout the chunked pipeline would take if the memory were page-locked)."""
    from ssblasex_b200 import runner, workloads as W
    m, n, k, batch = 300, 260, 200, 20
    arows, brows = (m if ta == 0 else k), (k if tb == 0 else n)
    p = W.make_problem(row, ta, tb, m, n, k, batch, 1 if row == "i8" else 0.75, beta, lda=arows + 3,
                       ldb=brows + 2, ldc=m + 5, seed=7 + ta, dist="expspread" if row == "f64" else "uniform")
    S.set_math_mode({"ozaki": S.SSBLAS_MATH_FP64_OZAKI, "bf16x3": S.SSBLAS_MATH_FP32_BF16X3,
                     "plain": S.SSBLAS_MATH_PLAIN}[mode])
    st, C_dev = runner.call(p, mode="device_array")
    assert st == 0
    # one allocation per instance, created in reverse order so their addresses are not spaced
    A = [None] * batch
    B = [None] * batch
    C = [None] * batch
    if layout == "dense":
        A, B, C = list(np.array(p.A, copy=True)), list(np.array(p.B, copy=True)), list(np.array(p.C, copy=True))
    for b in reversed(range(batch) if layout == "scattered" else []):
        A[b] = np.array(p.A[b], copy=True)
        B[b] = np.array(p.B[b], copy=True)
        C[b] = np.array(p.C[b], copy=True)
    ptrs = lambda arrs: (ct.c_void_p * batch)(*[a.ctypes.data for a in arrs])
    al, be = np.array([p.alpha], p.scale_dtype), np.array([p.beta], p.scale_dtype)
    t_a, t_b, t_c = p.types
    st = S.lib().ssblasGemmBatchedEx(ta, tb, m, n, k, al.ctypes.data, ptrs(A), t_a, p.lda, ptrs(B), t_b, p.ldb,
                                     be.ctypes.data, ptrs(C), t_c, p.ldc, batch, 0, 0)
    assert st == 0
    got = np.stack(C)
    want = C_dev.reshape(got.shape)
    if mode == "ozaki" or row == "i8":
        # the Ozaki emulation and int8 give the same bits whichever kernel the layout selects
        np.testing.assert_array_equal(got.view(np.uint8), want.view(np.uint8))
    else:
        from oracle import oracle as O
        u = {"f32": 2.0 ** -24, "f64": 2.0 ** -53}[row]
        bound = 2.0 ** -14 if mode == "bf16x3" else 4 * k * u
        assert O.normalized_error(p, got.reshape(p.C.shape), instances=range(0, batch, 4)) <= bound
    # padding rows m..ldc-1 of every column untouched
    np.testing.assert_array_equal(got.reshape(batch, n, -1)[:, :, m:], p.C.reshape(batch, n, -1)[:, :, m:])
    # the operands are the caller's and stay as they were
    for b in range(batch):
        np.testing.assert_array_equal(A[b], p.A[b])
        np.testing.assert_array_equal(B[b], p.B[b])
