"""Canary bytes around every operand and result on the device, in place of a memory sanitizer.

Each instance of A, B and C sits in one device buffer with a 256-byte gap of canary bytes before,
between and after the instances, and C's leading-dimension padding holds canaries too. After a
call on each main path -- the tensor-memory paths with their bulk tensor stores included -- the
operand buffers must be byte-for-byte unchanged and C may differ only inside the m x n block of
each instance.
"""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GAP = 256
CANARY = 0x5A


@pytest.fixture
def S():
    import torch
    assert torch.cuda.is_available()
    import ssblasex_b200 as S
    yield S
    S.set_math_mode(S.SSBLAS_MATH_PLAIN)
    S.set_kernel_config("bf16x3_tcgen05", -1)


def _pack(torch, mats, dtype):
    """One device buffer: gap, instance 0, gap, instance 1, ..., gap (canary bytes in the gaps).
    Returns the buffer and the device address of every instance."""
    per = mats[0].size * mats[0].itemsize
    per_slot = (per + 15) // 16 * 16 + GAP
    buf = torch.full((GAP + per_slot * len(mats),), CANARY, dtype=torch.uint8, device="cuda")
    for b, m in enumerate(mats):
        raw = torch.from_numpy(np.ascontiguousarray(m).reshape(-1).view(np.uint8).copy())
        buf[GAP + b * per_slot: GAP + b * per_slot + per] = raw.cuda()
    ptrs = [buf.data_ptr() + GAP + b * per_slot for b in range(len(mats))]
    return buf, ptrs, per_slot


CASES = [
    # (row, mode, transa, transb, m, n, k, padded)
    ("f64", "ozaki", 0, 1, 77, 45, 70, True),      # Ozaki, bulk tensor stores of C (beta = 0)
    ("f64", "ozaki", 1, 0, 130, 66, 300, True),
    ("f64", "plain", 0, 1, 77, 45, 70, True),      # DMMA
    ("f32", "bf16x3", 1, 1, 50, 61, 70, True),     # fused 3xBF16: TMA C tiles and bulk stores
    ("f32", "bf16x3", 0, 0, 150, 70, 33, False),   # split pass + tiled GEMM
    ("f32", "plain", 1, 1, 64, 64, 64, True),      # 8 x 8 FFMA blocks
    ("f32", "plain", 0, 0, 130, 129, 128, True),
    ("i8", "plain", 1, 0, 77, 45, 64, True),       # direct TMA staging of int8
    ("i8", "plain", 0, 0, 77, 45, 70, False),
]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("beta", [0.0, 0.5])
def test_canaries_stay_untouched(S, case, beta):
    import torch
    from ssblasex_b200 import workloads as W
    row, mode, ta, tb, m, n, k, padded = case
    if row == "i8" and beta != 0.0:
        beta = 1
    arows, brows = (m if ta == 0 else k), (k if tb == 0 else n)
    # padded: leading dimensions a multiple of 16 elements (the tensor-map paths), else odd
    ld = (lambda r: (r + 15) // 16 * 16 + 16) if padded else (lambda r: r + 3)
    lda, ldb, ldc = ld(arows), ld(brows), ld(m)
    p = W.make_problem(row, ta, tb, m, n, k, 5, 1 if row == "i8" else 0.75, beta, lda=lda, ldb=ldb, ldc=ldc,
                       seed=m + n + k + ta, dist="expspread" if row == "f64" else "uniform")
    S.set_math_mode({"ozaki": S.SSBLAS_MATH_FP64_OZAKI, "bf16x3": S.SSBLAS_MATH_FP32_BF16X3,
                     "plain": S.SSBLAS_MATH_PLAIN}[mode])
    bufA, pA, _ = _pack(torch, list(p.A), p.A.dtype)
    bufB, pB, _ = _pack(torch, list(p.B), p.B.dtype)
    bufC, pC, slotC = _pack(torch, list(p.C), p.C.dtype)
    A0, B0, C0 = bufA.clone(), bufB.clone(), bufC.clone()
    arr = lambda ptrs: (ct.c_void_p * len(ptrs))(*ptrs)
    al, be = np.array([p.alpha], p.scale_dtype), np.array([p.beta], p.scale_dtype)
    ta_, tb_, tc_ = p.types
    st = S.lib().ssblasGemmBatchedEx(ta, tb, m, n, k, al.ctypes.data, arr(pA), ta_, lda, arr(pB), tb_, ldb,
                                     be.ctypes.data, arr(pC), tc_, ldc, p.batch, 0, 0)
    torch.cuda.synchronize()
    assert st == 0
    assert torch.equal(bufA, A0), "an operand of A was written"
    assert torch.equal(bufB, B0), "an operand of B was written"
    # C: only the m x n block of each instance may change
    esz = p.C.itemsize
    allowed = torch.zeros_like(bufC, dtype=torch.bool)
    for b in range(p.batch):
        base = GAP + b * slotC
        for j in range(n):
            allowed[base + j * ldc * esz: base + (j * ldc + m) * esz] = True
    changed = bufC != C0
    assert not bool((changed & ~allowed).any()), "C was written outside its m x n blocks"
