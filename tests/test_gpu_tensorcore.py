"""The tcgen05 paths against their CPU restatements, through the C ABI, on a B200.

  * int8 -> int32 (kind::i8): bit-exact against the reference semantics, on the direct TMA path
    (every layout with 16-byte aligned leading dimensions and equally spaced instances: K-major
    staging for op(A) = A^T and op(B) = B, MN-major staging for op(A) = A and op(B) = B^T) and
    through the pack pre-pass (unequal spacing, leading dimensions not a multiple of 16);
  * FP64 Ozaki emulation: bit-exact against oracle.ozaki_f64 (the same algorithm on the CPU) for
    every slice count, and its error against the FP64-exact oracle;
  * FP32 three-BF16 emulation: within FP32 accumulation error of the FP64-exact value of the
    same three products, and its stated error against the FP64-exact oracle.
"""
import ctypes as ct

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture()
def S():
    import torch
    assert torch.cuda.is_available()
    import ssblasex_b200 as S
    S.set_math_mode(S.SSBLAS_MATH_PLAIN)
    S.set_ozaki_slices(0)
    yield S
    S.set_math_mode(S.SSBLAS_MATH_PLAIN)
    S.set_ozaki_slices(0)


def run(p, mode="device_array", **kw):
    from ssblasex_b200 import runner
    st, C = runner.call(p, mode=mode, **kw)
    assert st == 0, st
    return C


# ------------------------------------------------------------------------- int8 ------------
@pytest.mark.parametrize("shape", [(128, 256, 128), (200, 300, 520), (512, 512, 512), (37, 29, 45), (1, 1, 1),
                                   (130, 40, 2048)])
def test_i8_direct_tn(S, shape):
    from ssblasex_b200 import workloads as W
    m, n, k = shape
    lda = -(-k // 16) * 16
    p = W.make_problem("i8", 1, 0, m, n, k, 3, 1, 1, lda=lda, ldb=lda, seed=m + n)
    C = run(p)
    assert S.last_run_info()["path"] == "i8_tcgen05"
    np.testing.assert_array_equal(C, O.restated_gemm(p)[1])


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 1), (1, 0)])
@pytest.mark.parametrize("m,n,k", [(128, 256, 128), (130, 201, 300), (257, 64, 129), (37, 29, 45), (1, 1, 1),
                                   (300, 520, 1040)])
@pytest.mark.parametrize("cfg", [0, 1])
def test_i8_direct_every_layout(S, ta, tb, m, n, k, cfg):
    """Direct staging from the caller's matrices in all four layouts (MN-major tiles where op(A)
    or op(B) is stored M- or N-contiguous), both tile widths, ragged shapes: one kernel launch,
    bit-exact."""
    from ssblasex_b200 import workloads as W
    al = lambda x: -(-x // 16) * 16
    lda = al(m if ta == 0 else k)
    ldb = al(k if tb == 0 else n)
    p = W.make_problem("i8", ta, tb, m, n, k, 3, -2, 3, lda=lda, ldb=ldb, ldc=m + 1, seed=m + k + 5 * ta + 7 * tb)
    S.set_kernel_config("i8_tcgen05", cfg)
    try:
        C = run(p)
        info = S.last_run_info()
    finally:
        S.set_kernel_config("i8_tcgen05", -1)
    assert info["path"] == "i8_tcgen05" and info["kernel_launches"] == 1
    np.testing.assert_array_equal(C, O.restated_gemm(p)[1])


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("m,n,k", [(130, 201, 300), (257, 64, 129)])
def test_i8_pack_aligned(S, ta, tb, m, n, k):
    """The pack pre-pass with 4-byte aligned instances and leading dimensions (word loads of
    4 x 4 byte blocks, transposed in registers) and row counts that leave a partial group of 4
    rows: bit-exact."""
    from ssblasex_b200 import workloads as W
    # multiples of 4 but not of 16: not eligible for direct staging
    al = lambda x: -(-x // 4) * 4 + (4 if -(-x // 4) * 4 % 16 == 0 else 0)
    lda = al(m if ta == 0 else k)
    ldb = al(k if tb == 0 else n)
    p = W.make_problem("i8", ta, tb, m, n, k, 3, 2, -1, lda=lda, ldb=ldb, ldc=m + 3, seed=m + 3 * ta + tb)
    C = run(p)
    assert S.last_run_info()["path"] == "i8_tcgen05"
    np.testing.assert_array_equal(C, O.restated_gemm(p)[1])


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 1), (1, 0)])
def test_i8_packed_layouts(S, ta, tb):
    from ssblasex_b200 import workloads as W
    p = W.make_problem("i8", ta, tb, 150, 270, 333, 2, -3, 2, seed=7 + ta + 2 * tb)   # odd ld -> pack path
    C = run(p)
    assert S.last_run_info()["path"] == "i8_tcgen05"
    np.testing.assert_array_equal(C, O.restated_gemm(p)[1])


def test_i8_unequally_spaced_instances(S):
    """Host array of device pointers in shuffled order: no uniform stride, so the pack path."""
    import torch
    from ssblasex_b200 import runner, workloads as W
    p = W.make_problem("i8", 1, 0, 64, 96, 256, 4, 1, 0, lda=256, ldb=256, seed=3)
    dp = runner.DeviceProblem(p)
    order = [2, 0, 3, 1]
    A, B, C = (dp.ptrs(t) for t in (dp.A, dp.B, dp.C))
    arr = [(ct.c_void_p * 4)(*[x[o] for o in order]) for x in (A, B, C)]
    al, be = np.array([1], np.int32), np.array([0], np.int32)
    st = S.lib().ssblasGemmBatchedEx(1, 0, 64, 96, 256, al.ctypes.data, arr[0], 0, 256, arr[1], 0, 256,
                                     be.ctypes.data, arr[2], 3, 64, 4, 0, 0)
    assert st == 0
    np.testing.assert_array_equal(dp.C.cpu().numpy(), O.restated_gemm(p)[1])


# ------------------------------------------------------------------------- Ozaki -----------
@pytest.mark.parametrize("k", [1000, 3000])
@pytest.mark.parametrize("form", [3, 7])
def test_ozaki_unequally_spaced_instances(S, k, form):
    """Host array of device pointers in shuffled order: no uniform stride, so both slicing forms
    (one pass with clusters; row maxima then slab digits) load their tiles by cp.async instead of
    TMA, and the product is bit-exact against the CPU restatement."""
    from ssblasex_b200 import runner, workloads as W
    m, n, batch = 96, 80, 4
    p = W.make_problem("f64", 0, 1, m, n, k, batch, 1.5, 0.5, seed=k + form, dist="expspread")
    dp = runner.DeviceProblem(p)
    order = [2, 0, 3, 1]
    A, B, C = (dp.ptrs(t) for t in (dp.A, dp.B, dp.C))
    arr = [(ct.c_void_p * batch)(*[x[o] for o in order]) for x in (A, B, C)]
    al, be = np.array([1.5]), np.array([0.5])
    ta, tb, tc = p.types
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
    S.set_kernel_config("ozaki_slicer", form)
    try:
        st = S.lib().ssblasGemmBatchedEx(0, 1, m, n, k, al.ctypes.data, arr[0], ta, p.lda, arr[1], tb, p.ldb,
                                         be.ctypes.data, arr[2], tc, p.ldc, batch, 0, 0)
    finally:
        S.set_kernel_config("ozaki_slicer", -1)
    assert st == 0
    assert S.last_run_info()["path"] == "ozaki_tcgen05"
    C_o = O.ozaki_f64(p, 7)[1]
    np.testing.assert_array_equal(dp.C.cpu().numpy().view(np.uint64), C_o.view(np.uint64))


@pytest.mark.parametrize("slices", [3, 4, 5, 6, 7, 8])
def test_ozaki_bit_exact_per_slice_count(S, slices):
    from ssblasex_b200 import workloads as W
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
    S.set_ozaki_slices(slices)
    p = W.make_problem("f64", 0, 1, 140, 90, 200, 2, 0.75, -1.25, seed=slices, dist="expspread")
    C = run(p)
    info = S.last_run_info()
    assert info["path"] == "ozaki_tcgen05" and info["slices"] == slices
    st, C_o = O.ozaki_f64(p, slices)
    assert st == 0
    np.testing.assert_array_equal(C.view(np.uint64), C_o.view(np.uint64))


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_ozaki_layouts_and_error(S, ta, tb):
    from ssblasex_b200 import workloads as W
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
    p = W.make_problem("f64", ta, tb, 257, 70, 1030, 2, 1.0, 0.5, seed=20 + ta + 2 * tb, dist="expspread")
    C = run(p)
    st, C_o = O.ozaki_f64(p, 7)
    np.testing.assert_array_equal(C.view(np.uint64), C_o.view(np.uint64))
    # the default slice count keeps the FP64 bound of the plain path: 4 k u
    assert O.normalized_error(p, C) <= 4 * p.k * 2.0 ** -53


@pytest.mark.parametrize("form", [1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("ta,tb,m,n,k,batch", [
    (1, 0, 200, 96, 2048, 2),     # single pass, clusters of 8 (4) CTAs, K contiguous, 16-byte loads
    (1, 0, 67, 45, 257, 3),       # single pass, clusters of 2 (1), odd ld (8-byte loads)
    (0, 1, 300, 33, 1030, 2),     # single pass, rows contiguous, ragged last row block
    (0, 1, 64, 48, 2500, 2),      # K > 2048 with few rows: K-parallel row maxima, digit chunks
    (0, 0, 1984, 9, 2101, 5),     # K > 2048 with many rows
    (1, 1, 40, 200, 9000, 1),     # K > 2048, several row-maximum parts per row, ragged last part
    (1, 0, 48, 17, 4608, 3),      # K > 2048, K-contiguous, 9 whole 512-k slabs, odd column count
    (1, 0, 77, 50, 200, 3),       # k <= 256: clusters of one CTA in every one-pass form, K contiguous
    (0, 1, 90, 64, 64, 2),        # the same with rows contiguous
])
def test_ozaki_slicer_paths(S, form, ta, tb, m, n, k, batch):
    """Every slicing kernel (the two-pass form 1 -- row maxima per (32 rows, 256 k) part, then
    digits per (32 rows, 128 k) chunk -- and the one-pass item shapes: form 2 = 32 rows x 256 k
    per CTA, 3 = 16 rows x 512 k, 4 = 8 rows x 1024 k, 5 = 16 rows x 256 k with two 256-thread
    CTAs per SM, 6 = 4 rows x 256 k per 128-thread CTA, the slim form that runs beside the GEMM;
    form 7, and form 3 for k > 2048, is the row-maximum pass followed by persistent CTAs over
    16 rows x 512 k slabs that take their exponents from the maxima) produces the planes the CPU
    restatement produces: the product is bit-exact against oracle.ozaki_f64 whichever kernel
    sliced the operands."""
    from ssblasex_b200 import workloads as W
    if k > 2048 and form in (2, 4, 5, 6):
        pytest.skip("the one-pass forms apply to k <= 2048")
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
    S.set_kernel_config("ozaki_slicer", form)
    p = W.make_problem("f64", ta, tb, m, n, k, batch, 1.5, -0.5, seed=m + k, dist="expspread")
    try:
        C = run(p)
    finally:
        S.set_kernel_config("ozaki_slicer", -1)
    assert S.last_run_info()["path"] == "ozaki_tcgen05"
    st, C_o = O.ozaki_f64(p, 7)
    assert st == 0
    np.testing.assert_array_equal(C.view(np.uint64), C_o.view(np.uint64))


def test_ozaki_zero_rows_and_tiny_shapes(S):
    from ssblasex_b200 import workloads as W
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
    for (m, n, k) in [(1, 1, 1), (3, 5, 7), (129, 65, 33)]:
        p = W.make_problem("f64", 1, 1, m, n, k, 2, 2.0, 0.0, seed=m, dist="expspread")
        p.A[0][: p.lda] = 0.0      # first stored column of A[0] is zero
        C = run(p)
        np.testing.assert_array_equal(C.view(np.uint64), O.ozaki_f64(p, 7)[1].view(np.uint64))


@pytest.mark.parametrize("form", [2, 3, 4, 5, 6])
@pytest.mark.parametrize("ta,tb,k", [(1, 0, 200), (0, 1, 200), (1, 0, 700), (0, 1, 700)])
def test_ozaki_slicer_rows_below_one(S, form, ta, tb, k):
    """Entries in [-1, 1) (every row exponent <= 0) with k short of the item width, so part of
    each item is zero fill: the threads that hold only zeros must not raise a row's exponent to
    0 (the clusters-of-one path reduces per-thread exponents with a sentinel for zero). Bit-exact
    against the CPU restatement."""
    from ssblasex_b200 import workloads as W
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
    S.set_kernel_config("ozaki_slicer", form)
    p = W.make_problem("f64", ta, tb, 70, 45, k, 2, 1.0, 0.0, seed=k + form, dist="uniform")
    p.op_a(0)[3, :] = 0.0                       # a zero row
    p.op_a(1)[5, :] *= 2.0 ** -900              # a row far below 1
    try:
        C = run(p)
    finally:
        S.set_kernel_config("ozaki_slicer", -1)
    st, C_o = O.ozaki_f64(p, 7)
    assert st == 0
    np.testing.assert_array_equal(C.view(np.uint64), C_o.view(np.uint64))


@pytest.mark.parametrize("form", [1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("ta,tb", [(0, 1), (1, 0)])
def test_ozaki_subnormal_rows(S, form, ta, tb):
    """Rows of op(A) and columns of op(B) made of subnormals: below 2^-1042 (every high word
    zero, so the row maximum comes from the low words), between 2^-1042 and 2^-1022, one normal
    value among tiny subnormals, and negative tiny subnormals only; a column of op(B) near 2^1000
    keeps some products representable. Every slicing form gives the exponents and digits of the
    CPU restatement (bit-exact product)."""
    from ssblasex_b200 import workloads as W
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
    S.set_kernel_config("ozaki_slicer", form)
    m, n, k, batch = 70, 40, 600, 2
    p = W.make_problem("f64", ta, tb, m, n, k, batch, 1.0, 0.0, seed=11, dist="expspread")
    rng = np.random.default_rng(5)
    tiny = 2.0 ** -1074
    for b in range(batch):
        opa, opb = p.op_a(b), p.op_b(b)
        opa[0, :] = rng.integers(-2 ** 31, 2 ** 31, k) * tiny
        opa[1, :] = rng.integers(-2 ** 50, 2 ** 50, k) * tiny
        opa[2, :] = rng.integers(-2 ** 20, 2 ** 20, k) * tiny
        opa[2, 17 + b] = 3.0
        opa[3, :] = -(rng.integers(0, 2 ** 10, k) * tiny)
        opb[:, 0] = rng.integers(-2 ** 31, 2 ** 31, k) * tiny
        opb[:, 1] = rng.integers(-2 ** 45, 2 ** 45, k) * tiny
        opb[:, 5] = rng.standard_normal(k) * 2.0 ** 1000
    try:
        C = run(p)
    finally:
        S.set_kernel_config("ozaki_slicer", -1)
    st, C_o = O.ozaki_f64(p, 7)
    assert st == 0
    np.testing.assert_array_equal(C.view(np.uint64), C_o.view(np.uint64))


# ------------------------------------------------------------------------- 3 x BF16 --------
@pytest.mark.parametrize("ta,tb,shape", [(1, 1, (64, 64, 64)), (0, 0, (200, 150, 300)), (0, 1, (129, 257, 96)),
                                         (1, 0, (33, 17, 513))])
def test_bf16x3_against_emulation_oracle(S, ta, tb, shape):
    from ssblasex_b200 import workloads as W
    S.set_math_mode(S.SSBLAS_MATH_FP32_BF16X3)
    m, n, k = shape
    p = W.make_problem("f32", ta, tb, m, n, k, 2, 0.75, 0.25, seed=k, dist="outliers")
    C = run(p)
    assert S.last_run_info()["path"] == "bf16x3_tcgen05"
    for b in range(p.batch):
        emu = O.bf16x3_f32(p, b)
        ex, nrm = O.exact_f64(p, b)
        got = p.c_view(C, b).astype(np.float64)
        # same products, FP32 accumulation on the tensor cores
        assert np.max(np.abs(got - emu) / nrm) <= 4 * k * 2.0 ** -24
        # stated error of the mode against the FP64-exact result
        assert np.max(np.abs(got - ex) / nrm) <= 2.0 ** -14


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("shape", [(64, 64, 64), (128, 128, 200), (37, 29, 45), (100, 20, 300), (64, 100, 65),
                                   (1, 1, 1), (50, 128, 130)])
@pytest.mark.parametrize("beta", [0.0, 0.25])
@pytest.mark.parametrize("aligned", [True, False])
def test_bf16x3_small_fused(S, ta, tb, shape, beta, aligned):
    """Configuration 2: instances of at most 128 x 128 that are equally spaced with leading
    dimensions a multiple of 4 run as one kernel that splits hi/lo in shared memory (no split
    pass): one launch (odd leading dimensions take the split pass and the tiled GEMM), within FP32
    accumulation error of the exact value of the three BF16 products and within the mode's stated
    2^-14 of the exact product; more instances than SMs, so every CTA streams several."""
    from ssblasex_b200 import workloads as W
    S.set_math_mode(S.SSBLAS_MATH_FP32_BF16X3)
    m, n, k = shape
    arows, brows = (m if ta == 0 else k), (k if tb == 0 else n)
    lda, ldb = ((arows + 3) // 4 * 4 + 4, (brows + 3) // 4 * 4 + 4) if aligned else (arows | 1, brows | 1)
    batch = 300 if shape == (64, 64, 64) else 5
    p = W.make_problem("f32", ta, tb, m, n, k, batch, 0.75, beta, lda=lda, ldb=ldb, ldc=m + 3,
                       seed=m + n + k + ta, dist="outliers")
    S.set_kernel_config("bf16x3_tcgen05", 2)
    try:
        C = run(p)
        info = S.last_run_info()
    finally:
        S.set_kernel_config("bf16x3_tcgen05", -1)
    assert info["path"] == "bf16x3_tcgen05" and info["kernel_launches"] == (1 if aligned else 2)
    for b in range(p.batch):
        emu = O.bf16x3_f32(p, b)
        ex, nrm = O.exact_f64(p, b)
        got = p.c_view(C, b).astype(np.float64)
        assert np.max(np.abs(got - emu) / nrm) <= 4 * k * 2.0 ** -24
        assert np.max(np.abs(got - ex) / nrm) <= 2.0 ** -14
    np.testing.assert_array_equal(C.reshape(p.batch, n, m + 3)[:, :, m:], p.C.reshape(p.batch, n, m + 3)[:, :, m:])


@pytest.mark.parametrize("cfg", [10, 11])
@pytest.mark.parametrize("shape,beta,splits", [((300, 170, 333, 3), 0.0, 0), ((129, 65, 64, 2), 0.5, 0),
                                               ((256, 128, 2000, 2), 0.0, 3), ((200, 300, 4100, 1), -1.5, 2),
                                               ((1024, 512, 1024, 2), 0.0, 0)])
def test_ozaki_two_part_release(S, cfg, shape, beta, splits):
    """Configurations 10 and 11 hand the accumulator back in two parts (the top three / two levels
    first) and issue the next tile's top-level products before the bottom levels are drained: bit-exact
    against the restatement with one K block per tile (k = 64, fewer blocks than stages), many
    blocks, forced split-K pieces (whose epilogue releases both parts at once), and enough tiles
    that every CTA runs several in a row."""
    from ssblasex_b200 import workloads as W
    m, n, k, batch = shape
    p = W.make_problem("f64", 0, 1, m, n, k, batch, 0.75, beta, seed=m + k + cfg, dist="expspread")
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
    S.set_kernel_config("ozaki_tcgen05", cfg)
    S.set_kernel_config("splitk_ozaki", splits)
    try:
        C = run(p)
        info = S.last_run_info()
    finally:
        S.set_kernel_config("ozaki_tcgen05", -1)
        S.set_kernel_config("splitk_ozaki", -1)
    assert info["path"] == "ozaki_tcgen05" and info["slices"] == 7
    if splits:
        assert info["split_k"] == splits
    np.testing.assert_array_equal(C.view(np.uint64), O.ozaki_f64(p, 7)[1].view(np.uint64))


@pytest.mark.parametrize("mode", ["device_array", "host_array"])
@pytest.mark.parametrize("shape", [(300, 170, 333, 3), (1, 17, 40, 2), (130, 200, 1030, 2), (256, 64, 64, 5)])
@pytest.mark.parametrize("extreme", [False, True])
def test_ozaki_bulk_store_epilogue(S, mode, shape, extreme):
    """Configuration 9 writes C with bulk tensor stores (beta = 0, equally spaced instances):
    bit-exact against the restatement, C's ld padding untouched; regions holding a scale factor
    outside the normal range (rows scaled by 2^-1060 and 2^1010) take the per-element path instead."""
    from ssblasex_b200 import workloads as W
    m, n, k, batch = shape
    p = W.make_problem("f64", 0, 1, m, n, k, batch, 0.75, 0.0, ldc=m + 5, seed=m + n + k, dist="expspread")
    if extreme:
        for b in range(batch):
            p.op_a(b)[0, :] *= 2.0 ** -1060
            p.op_a(b)[m - 1, :] *= 2.0 ** 1010 if m > 1 else 1.0
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
    S.set_kernel_config("ozaki_tcgen05", 9)
    try:
        C = run(p, mode=mode)
    finally:
        S.set_kernel_config("ozaki_tcgen05", -1)
    np.testing.assert_array_equal(C.view(np.uint64), O.ozaki_f64(p, 7)[1].view(np.uint64))
    pad = C.reshape(batch, n, m + 5)[:, :, m:]
    np.testing.assert_array_equal(pad, p.C.reshape(batch, n, m + 5)[:, :, m:])


# ------------------------------------------------------------------------- configurations ---
@pytest.mark.parametrize("family,cfg", [("ozaki_tcgen05", 0), ("ozaki_tcgen05", 1), ("ozaki_tcgen05", 2), ("ozaki_tcgen05", 3), ("ozaki_tcgen05", 4), ("ozaki_tcgen05", 5), ("ozaki_tcgen05", 6), ("ozaki_tcgen05", 7), ("ozaki_tcgen05", 8), ("ozaki_tcgen05", 9), ("ozaki_tcgen05", 10), ("ozaki_tcgen05", 11),
                                        ("i8_tcgen05", 0), ("i8_tcgen05", 1),
                                        ("bf16x3_tcgen05", 0), ("bf16x3_tcgen05", 1), ("bf16x3_tcgen05", 2),
                                        ("dmma", 0), ("dmma", 1), ("dmma", 2), ("dmma", 3), ("dmma", 4)])
def test_every_kernel_configuration(S, family, cfg):
    """Each configuration the autotuner may pick gives the right answer on a ragged problem."""
    from ssblasex_b200 import workloads as W
    S.set_kernel_config(family, cfg)
    try:
        if family == "ozaki_tcgen05":
            S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
            p = W.make_problem("f64", 0, 1, 300, 170, 333, 3, 0.5, 2.0, seed=40 + cfg, dist="expspread")
            C = run(p)
            np.testing.assert_array_equal(C.view(np.uint64), O.ozaki_f64(p, 7)[1].view(np.uint64))
        elif family == "i8_tcgen05":
            p = W.make_problem("i8", 1, 0, 300, 170, 336, 3, 3, -1, lda=336, ldb=336, seed=50 + cfg)
            C = run(p)
            np.testing.assert_array_equal(C, O.restated_gemm(p)[1])
        elif family == "dmma":
            # plain fp64: DMMA tiles (0: 64x64, 1, 3, 4: 128x128) or the DFMA SIMT kernel (2)
            S.set_math_mode(S.SSBLAS_MATH_PLAIN)
            p = W.make_problem("f64", 1, 1, 300, 170, 333, 3, 0.5, 2.0, seed=70 + cfg, dist="expspread")
            C = run(p)
            assert O.normalized_error(p, C) <= 4 * p.k * 2.0 ** -53
            assert S.last_run_info()["path"] == ("simt" if cfg == 2 else "dmma")
            return
        else:
            S.set_math_mode(S.SSBLAS_MATH_FP32_BF16X3)
            p = W.make_problem("f32", 1, 0, 300, 170, 200, 2, 0.75, 0.25, seed=60 + cfg)
            C = run(p)
            for b in range(p.batch):
                emu = O.bf16x3_f32(p, b)
                ex, nrm = O.exact_f64(p, b)
                assert np.max(np.abs(p.c_view(C, b) - emu) / nrm) <= 4 * p.k * 2.0 ** -24
        assert S.last_run_info()["path"] == family
    finally:
        S.set_kernel_config(family, -1)


# ------------------------------------------------------------------------- plain fp64 (DMMA)
@pytest.mark.parametrize("transa,transb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("aligned", [True, False])
def test_dmma_layouts_and_alignment(S, transa, transb, aligned):
    """Plain fp64 on the DMMA tiles for every op(A)/op(B) pair, with 16-byte aligned instances and
    even leading dimensions (16-byte copies) or instances at odd 8-byte offsets with odd leading
    dimensions (8-byte copies), ragged edges in m, n and k, beta != 0."""
    import torch
    from ssblasex_b200 import workloads as W
    m, n, k, batch = 131, 77, 203, 3
    arows, brows = (m if transa == 0 else k), (k if transb == 0 else n)
    pad = 0 if aligned else 1
    lda, ldb, ldc = arows + (2 if aligned else 1), brows + (2 if aligned else 1), m + 3
    p = W.make_problem("f64", transa, transb, m, n, k, batch, -1.25, 0.5, lda=lda, ldb=ldb, ldc=ldc,
                       seed=80 + 2 * transa + transb)
    bufs, ptrs = [], []
    for X in (p.A, p.B, p.C):
        per = X[0].size + pad
        flat = torch.zeros(pad + per * batch, dtype=torch.float64, device="cuda")
        for b in range(batch):
            flat[pad + b * per: pad + b * per + X[b].size] = torch.from_numpy(X[b].reshape(-1))
        bufs.append(flat)
        ptrs.append((ct.c_void_p * batch)(*[flat.data_ptr() + 8 * (pad + b * per) for b in range(batch)]))
    al, be = np.array([p.alpha]), np.array([p.beta])
    st = S.lib().ssblasGemmBatchedEx(p.transa, p.transb, m, n, k, al.ctypes.data, ptrs[0], S.SSBLAS_R_64F, lda,
                                     ptrs[1], S.SSBLAS_R_64F, ldb, be.ctypes.data, ptrs[2], S.SSBLAS_R_64F, ldc,
                                     batch, 0, 0)
    assert st == 0 and S.last_run_info()["path"] == "dmma"
    flat = bufs[2].cpu().numpy()
    per = p.C[0].size + pad
    C = np.stack([flat[pad + b * per: pad + b * per + p.C[0].size] for b in range(batch)]).reshape(p.C.shape)
    assert O.normalized_error(p, C) <= 4 * k * 2.0 ** -53
    # rows m..ldc-1 of every column keep their value
    np.testing.assert_array_equal(C.reshape(batch, n, ldc)[:, :, m:], p.C.reshape(batch, n, ldc)[:, :, m:])


# ------------------------------------------------------------------------- plain fp32 (cp.async)
@pytest.mark.parametrize("cfg", [3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13])
@pytest.mark.parametrize("transa,transb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("aligned", [True, False])
def test_sgemm_layouts_and_alignment(S, cfg, transa, transb, aligned):
    """Plain fp32 on the cp.async-pipelined kernels (configuration 3: 64 x 64 tiles, 4: 128 x 128,
    7: 32 x 64, 8: 32 x 32; 5 and 6: persistent 64 x 64 CTAs that double-buffer their (tile,
    instance) items, for k <= 64 -- run with 300 instances, so every CTA walks several items; 9
    and 10: 64-thread CTAs of 8 x 8 blocks holding all of k <= 64 / k <= 128; 11: four such
    groups over quarters of k <= 128, summed in shared memory; 12 and 13: TMA-staged 64 x 64
    tiles, which the unaligned layouts leave for configuration 3) for every
    op(A)/op(B) pair, with 16-byte aligned instances and leading dimensions that are multiples of
    4 (16-byte copies) or instances at odd 4-byte offsets with odd leading dimensions (4-byte
    copies), ragged edges in m, n and k, beta != 0."""
    import torch
    from ssblasex_b200 import workloads as W
    m, n, k, batch = {5: (141, 77, 61, 300), 6: (141, 77, 61, 300), 9: (141, 77, 61, 300),
                      10: (141, 77, 127, 40), 11: (141, 77, 126, 40)}.get(cfg, (141, 77, 203, 3))
    arows, brows = (m if transa == 0 else k), (k if transb == 0 else n)
    pad = 0 if aligned else 1
    lda, ldb, ldc = arows + (3 if aligned else 2), brows + (1 if aligned else 2), m + (3 if aligned else 2)
    lda, ldb, ldc = ((lda + 3) // 4 * 4, (ldb + 3) // 4 * 4, (ldc + 3) // 4 * 4) if aligned else (lda | 1, ldb | 1, ldc | 1)
    p = W.make_problem("f32", transa, transb, m, n, k, batch, 0.75, 0.25, lda=lda, ldb=ldb, ldc=ldc,
                       seed=90 + 2 * transa + transb + 4 * cfg, dist="outliers")
    bufs, ptrs = [], []
    for X in (p.A, p.B, p.C):
        per = X[0].size + pad
        flat = torch.zeros(pad + per * batch, dtype=torch.float32, device="cuda")
        for b in range(batch):
            flat[pad + b * per: pad + b * per + X[b].size] = torch.from_numpy(X[b].reshape(-1))
        bufs.append(flat)
        ptrs.append((ct.c_void_p * batch)(*[flat.data_ptr() + 4 * (pad + b * per) for b in range(batch)]))
    al, be = np.array([p.alpha], np.float32), np.array([p.beta], np.float32)
    S.set_kernel_config("simt", cfg)
    try:
        st = S.lib().ssblasGemmBatchedEx(p.transa, p.transb, m, n, k, al.ctypes.data, ptrs[0], S.SSBLAS_R_32F, lda,
                                         ptrs[1], S.SSBLAS_R_32F, ldb, be.ctypes.data, ptrs[2], S.SSBLAS_R_32F, ldc,
                                         batch, 0, 0)
        assert st == 0 and S.last_run_info()["path"] == "simt"
    finally:
        S.set_kernel_config("simt", -1)
    flat = bufs[2].cpu().numpy()
    per = p.C[0].size + pad
    C = np.stack([flat[pad + b * per: pad + b * per + p.C[0].size] for b in range(batch)]).reshape(p.C.shape)
    assert O.normalized_error(p, C) <= 4 * k * 2.0 ** -24
    np.testing.assert_array_equal(C.reshape(batch, n, ldc)[:, :, m:], p.C.reshape(batch, n, ldc)[:, :, m:])


@pytest.mark.parametrize("cfg", [12, 13])
@pytest.mark.parametrize("transa,transb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("shape", [(64, 64, 64, 300, 0.0), (64, 64, 64, 300, 0.5), (50, 70, 20, 97, 0.0),
                                   (128, 128, 128, 64, 0.5), (200, 65, 257, 5, -1.0), (1, 1, 1, 3, 0.5),
                                   (64, 64, 64, 2000, 0.25), (64, 64, 64, 2000, 0.0), (70, 40, 130, 700, 0.5)])
def test_sgemm_tma_items(S, cfg, transa, transb, shape):
    """The TMA-staged FFMA kernel (configurations 12 and 13), from one work item per CTA to about
    seven and five per CTA (2000 and 700 instances: the stage and C-tile rings wrap several
    times), with beta = 0 (C holds NaN and must not be read),
    ragged m, n and k (zero-filled tiles, clipped stores), k below one 64-deep chunk, and several
    chunks; the launch must be the TMA kernel, the result within 4 k u of the FP64-exact oracle,
    and the ld padding of C untouched."""
    import torch
    from ssblasex_b200 import runner, workloads as W
    m, n, k, batch, beta = shape
    arows, brows = (m if transa == 0 else k), (k if transb == 0 else n)
    r4 = lambda x: (x + 3) // 4 * 4
    p = W.make_problem("f32", transa, transb, m, n, k, batch, 0.75, beta, lda=r4(arows + 1), ldb=r4(brows),
                       ldc=r4(m + 2), seed=700 + 4 * cfg + 2 * transa + transb + m, dist="outliers")
    C0 = p.C.copy()
    if beta == 0.0:
        C0.reshape(batch, n, -1)[:, :, :m] = np.nan
    dp = runner.DeviceProblem(p, C=C0)
    S.set_kernel_config("simt", cfg)
    S.set_profiling(True)
    try:
        st, C = runner.call(p, mode="host_array", dp=dp)
        prof = S.get_profile()
        assert st == 0 and S.last_run_info()["path"] == "simt"
    finally:
        S.set_profiling(False)
        S.set_kernel_config("simt", -1)
    assert list(prof) == ["sgemm_tma"], prof
    C = C.reshape(p.C.shape)
    assert np.isfinite(C.reshape(batch, n, -1)[:, :, :m]).all()
    assert O.normalized_error(p, C) <= 4 * max(k, 1) * 2.0 ** -24
    np.testing.assert_array_equal(C.reshape(batch, n, -1)[:, :, m:], C0.reshape(batch, n, -1)[:, :, m:])


# ------------------------------------------------------------------------- Ozaki: Inf / NaN ---
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("k", [300, 1030, 2500])
def test_ozaki_nonfinite_inputs(S, ta, tb, k):
    """Ozaki mode with Inf and NaN entries: rows of op(A) and columns of op(B) that hold one
    get zero digits, and exactly the C(i, j) they touch become the quiet NaN; every other entry
    is bit-exact against the CPU restatement (which follows the same rule), for the one-pass
    (k <= 2048) and two-pass slicing forms."""
    from ssblasex_b200 import workloads as W
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
    m, n, batch = 150, 70, 2
    p = W.make_problem("f64", ta, tb, m, n, k, batch, 1.0, 0.5, seed=ta + 2 * tb + k, dist="expspread")
    bad_rows, bad_cols = {0: [3, 97], 1: [0]}, {0: [5], 1: [40, 69]}
    for b in range(batch):
        opa, opb = p.op_a(b), p.op_b(b)
        for i, val in zip(bad_rows[b], [np.inf, np.nan]):
            opa[i, (7 * i) % k] = val
        for j, val in zip(bad_cols[b], [-np.inf, np.nan]):
            opb[(11 * j) % k, j] = val
    C = run(p)
    st, C_o = O.ozaki_f64(p, 7)
    assert st == 0
    np.testing.assert_array_equal(C.view(np.uint64), C_o.view(np.uint64))
    for b in range(batch):
        got = p.c_view(C, b)
        want_nan = np.zeros((m, n), bool)
        want_nan[bad_rows[b], :] = True
        want_nan[:, bad_cols[b]] = True
        np.testing.assert_array_equal(np.isnan(got), want_nan)


# ------------------------------------------------------------------------- split-K ---------
def pieces(k, k_block, want):
    """K pieces the library makes of `want`: equal K-block counts, none empty."""
    nk = -(-k // k_block)
    per = -(-nk // min(want, nk))
    return -(-nk // per)


@pytest.mark.parametrize("splits", [0, 1, 2, 3, 7, 16])
@pytest.mark.parametrize("ta,tb,m,n,k,batch,alpha,beta", [
    (1, 0, 200, 300, 5000, 2, 2, -1),    # direct TMA path (op(A) = T, op(B) = N), ragged tiles
    (0, 0, 70, 90, 3000, 3, -3, 2),      # pack pre-pass, one tile per instance
])
def test_split_k_i8(S, splits, ta, tb, m, n, k, batch, alpha, beta):
    """int8 split-K: every K-piece count (0 = automatic) gives the unsplit result bit for bit --
    the pieces' int32 sums wrap the same way in any order."""
    from ssblasex_b200 import workloads as W
    lda = -(-k // 16) * 16 if ta == 1 else m
    ldb = -(-k // 16) * 16 if tb == 0 else n
    p = W.make_problem("i8", ta, tb, m, n, k, batch, alpha, beta, lda=lda, ldb=ldb, seed=k + splits)
    S.set_kernel_config("splitk_i8", splits)
    try:
        C = run(p)
        info = S.last_run_info()
    finally:
        S.set_kernel_config("splitk_i8", -1)
    assert info["path"] == "i8_tcgen05"
    if splits > 1:
        assert info["split_k"] == pieces(k, 128, splits)
    np.testing.assert_array_equal(C, O.restated_gemm(p)[1])


@pytest.mark.parametrize("splits", [0, 1, 2, 5, 9])
@pytest.mark.parametrize("ta,tb", [(0, 1), (1, 0)])
def test_split_k_ozaki(S, splits, ta, tb):
    """Ozaki split-K: the level sums of the pieces are added exactly, so the result is bit-exact
    against the CPU restatement whatever the piece count."""
    from ssblasex_b200 import workloads as W
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
    p = W.make_problem("f64", ta, tb, 130, 70, 4100, 2, 0.75, -0.5, seed=splits + 3 * ta, dist="expspread")
    S.set_kernel_config("splitk_ozaki", splits)
    try:
        C = run(p)
        info = S.last_run_info()
    finally:
        S.set_kernel_config("splitk_ozaki", -1)
    assert info["path"] == "ozaki_tcgen05"
    if splits > 1:
        assert info["split_k"] == pieces(p.k, 64, splits)
    st, C_o = O.ozaki_f64(p, 7)
    assert st == 0
    np.testing.assert_array_equal(C.view(np.uint64), C_o.view(np.uint64))


def test_ozaki_long_k_is_split(S):
    """k > 16384 stays on the Ozaki path: the GEMM is cut into K pieces of at most 16384, each
    exact in int32, added in 64 bits."""
    from ssblasex_b200 import workloads as W
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
    p = W.make_problem("f64", 1, 0, 40, 33, 40000, 2, 1.0, 0.25, seed=5, dist="expspread")
    C = run(p)
    info = S.last_run_info()
    assert info["path"] == "ozaki_tcgen05" and info["split_k"] >= 3
    st, C_o = O.ozaki_f64(p, 7)
    assert st == 0
    np.testing.assert_array_equal(C.view(np.uint64), C_o.view(np.uint64))
    assert O.normalized_error(p, C) <= 4 * p.k * 2.0 ** -53


def test_ozaki_level_sum_beyond_int32(S):
    """Constant operands make every product of leading digits equal, so the leading level's sum
    over k = 600000 exceeds the int32 range (the CPU restatement reports that with status -1);
    the split pieces are added in 64 bits and the result is still bit-exact."""
    from ssblasex_b200 import workloads as W
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
    p = W.make_problem("f64", 1, 0, 3, 2, 600000, 1, 1.0, 0.0, seed=1)
    for b in range(p.batch):
        p.op_a(b)[:] = 0.99
        p.op_b(b)[:] = -0.97
    C = run(p)
    assert S.last_run_info()["path"] == "ozaki_tcgen05"
    st, C_o = O.ozaki_f64(p, 7)
    assert st == -1
    np.testing.assert_array_equal(C.view(np.uint64), C_o.view(np.uint64))
    np.testing.assert_allclose(p.c_view(C, 0), 600000 * 0.99 * -0.97, rtol=1e-12)


# ------------------------------------------------------------------------- slicing / GEMM pipeline
@pytest.mark.parametrize("chunks", [2, 3, 4])
@pytest.mark.parametrize("ta,tb,m,n,k,batch", [
    (0, 1, 300, 200, 1030, 7),    # uneven chunks, rows contiguous, ragged tiles
    (1, 0, 256, 130, 512, 9),     # k contiguous (TMA boxes along k)
])
def test_ozaki_pipeline(S, chunks, ta, tb, m, n, k, batch):
    """The batch cut into chunks, the slicing of chunk c + 1 (slim kernel, side stream) beside the
    GEMM of chunk c: bit-exact against the CPU restatement, and equal to the unpipelined result."""
    from ssblasex_b200 import workloads as W
    S.set_math_mode(S.SSBLAS_MATH_FP64_OZAKI)
    p = W.make_problem("f64", ta, tb, m, n, k, batch, 0.5, -1.5, seed=chunks + m, dist="expspread")
    S.set_kernel_config("ozaki_pipeline", chunks)
    try:
        C = run(p)
        C_again = run(p)
        S.set_kernel_config("ozaki_pipeline", 1)
        C_plain = run(p)
    finally:
        S.set_kernel_config("ozaki_pipeline", -1)
    assert S.last_run_info()["path"] == "ozaki_tcgen05"
    st, C_o = O.ozaki_f64(p, 7)
    assert st == 0
    np.testing.assert_array_equal(C.view(np.uint64), C_o.view(np.uint64))
    np.testing.assert_array_equal(C_again.view(np.uint64), C_o.view(np.uint64))
    np.testing.assert_array_equal(C_plain.view(np.uint64), C_o.view(np.uint64))
