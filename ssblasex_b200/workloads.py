"""Seeded synthetic problems for ssblasGemmBatchedEx (numpy only).

A problem is one batched GEMM C[b] <- alpha * op(A[b]) * op(B[b]) + beta * C[b] in the reference's
column-major convention: element (r, c) of op(X) is X[r + c*ld] for op N and X[r*ld + c] for op T
(reference src/include/Utils/ssblas_BatchMat.hpp:31-39). Each operand is held as one contiguous
array of shape (batch, ld * stored_cols), so instance b starts at a fixed stride.

The five named workloads follow the benchmark configurations of this project:

  fp32_batch64_128   plain fp32, 64 x 128^3, NN, ld 128, alpha 1, beta 0.5, U[-1,1), seed 0
  i8_batch512_512    int8->int32, 512 x 512^3, TN, ld 512, A/B U{-128..127}, C U{-2^20..2^20},
                     alpha = beta = 1 (int32 scale type)
  f64_batch32_1024   fp64, 32 x 1024^3, NT, ld 1032, sign * U[1,2) * 2^U{-8..8}, alpha 1, beta 0
  fp32_batch4096_64  fp32, 4096 x 64^3, TT, ld 64, U[-1,1) with 1% of entries x 1e4,
                     alpha 0.75, beta 0.25
  grouped_10000      10,000 uneven instances (see grouped_problem)
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

OP_N, OP_T, OP_C = 0, 1, 2
R_8I, R_8U, R_16F, R_32I, R_32F, R_64F = 0, 1, 2, 3, 4, 5

ROW_TYPES = {
    "f32": (R_32F, R_32F, R_32F, np.float32, np.float32, np.float32),
    "f64": (R_64F, R_64F, R_64F, np.float64, np.float64, np.float64),
    "i8": (R_8I, R_8I, R_32I, np.int8, np.int32, np.int32),
    # rows of the type extensions (ssblasSetExtensions): fp16 inputs with fp16 or fp32 C (float
    # scale), and unsigned int8 operands (int32 scale and C)
    "f16": (R_16F, R_16F, R_16F, np.float16, np.float32, np.float16),
    "f16c32": (R_16F, R_16F, R_32F, np.float16, np.float32, np.float32),
    "u8": (R_8U, R_8U, R_32I, np.uint8, np.int32, np.int32),
    "u8s8": (R_8U, R_8I, R_32I, np.uint8, np.int32, np.int32),
    "s8u8": (R_8I, R_8U, R_32I, np.int8, np.int32, np.int32),
}
# element type of op(B) where it differs from op(A)'s
B_DTYPE = {"u8s8": np.int8, "s8u8": np.uint8}
INT_ROWS = ("i8", "u8", "u8s8", "s8u8")


def stored_shape(trans: int, rows: int, cols: int) -> tuple[int, int]:
    """(stored rows, stored cols) of X such that op(X) is rows x cols."""
    return (rows, cols) if trans == OP_N else (cols, rows)


@dataclasses.dataclass
class Problem:
    row: str                 # "f32", "f64" or "i8"
    transa: int
    transb: int
    m: int
    n: int
    k: int
    lda: int
    ldb: int
    ldc: int
    batch: int
    alpha: float
    beta: float
    A: np.ndarray            # (batch, lda * stored cols of A)
    B: np.ndarray
    C: np.ndarray            # (batch, ldc * n); the input C (beta * C term)
    name: str = ""

    @property
    def types(self):
        return ROW_TYPES[self.row][:3]

    @property
    def ab_dtype(self):
        return ROW_TYPES[self.row][3]

    @property
    def scale_dtype(self):
        return ROW_TYPES[self.row][4]

    @property
    def c_dtype(self):
        return ROW_TYPES[self.row][5]

    def op_a(self, b: int) -> np.ndarray:
        """op(A[b]) as an m x k array (a view)."""
        return _op_view(self.A[b], self.transa, self.m, self.k, self.lda)

    def op_b(self, b: int) -> np.ndarray:
        return _op_view(self.B[b], self.transb, self.k, self.n, self.ldb)

    def c_view(self, C: np.ndarray, b: int) -> np.ndarray:
        return _op_view(C[b], OP_N, self.m, self.n, self.ldc)

    def flops(self) -> float:
        return 2.0 * self.m * self.n * self.k * self.batch

    def algorithmic_bytes(self) -> float:
        """Bytes that must move once: op(A), op(B), C write, and C read when beta != 0
        (ld padding excluded)."""
        ab = np.dtype(self.ab_dtype).itemsize
        cb = np.dtype(self.c_dtype).itemsize
        per = ab * (self.m * self.k + self.k * self.n) + cb * self.m * self.n * (2 if self.beta != 0 else 1)
        return float(per * self.batch)


def _op_view(flat: np.ndarray, trans: int, rows: int, cols: int, ld: int) -> np.ndarray:
    srows, scols = stored_shape(trans, rows, cols)
    stored = flat[: ld * scols].reshape(scols, ld)[:, :srows].T   # srows x scols, column-major view
    return stored if trans == OP_N else stored.T


def _alloc(rng, dtype, batch, ld, scols, fill):
    arr = np.zeros((batch, ld * scols), dtype=dtype)
    fill(arr)
    return arr


def make_problem(row: str, transa: int, transb: int, m: int, n: int, k: int, batch: int,
                 alpha, beta, lda: int | None = None, ldb: int | None = None,
                 ldc: int | None = None, seed: int = 0, dist: str = "uniform",
                 name: str = "") -> Problem:
    """Seeded problem. dist: "uniform" (U[-1,1) for fp, U{-128..127}/U{-2^20..2^20} for int8),
    "expspread" (sign * U[1,2) * 2^U{-8..8}; "expspreadN" for 2^U{-N..N}), "outliers" (U[-1,1)
    with 1% of entries x 1e4), "small_int" (int8 in {-3..3}, C in {-64..64})."""
    rng = np.random.default_rng(seed)
    ar, ac = stored_shape(transa, m, k)
    br, bc = stored_shape(transb, k, n)
    lda = lda if lda is not None else max(1, ar)
    ldb = ldb if ldb is not None else max(1, br)
    ldc = ldc if ldc is not None else max(1, m)
    _, _, _, abt, st, ct = ROW_TYPES[row]

    def gen_ab(shape, dtype=abt):
        if row in INT_ROWS:
            if dtype == np.uint8:
                return rng.integers(0, 4 if dist == "small_int" else 256, size=shape, dtype=np.uint8)
            lo, hi = (-3, 4) if dist == "small_int" else (-128, 128)
            return rng.integers(lo, hi, size=shape, dtype=np.int8)
        if dist.startswith("expspread"):
            span = int(dist[len("expspread"):] or 8)
            # sign * U[1,2) as one uniform draw on (-2,-1] u [1,2), times 2^U{-span..span}
            u = rng.uniform(-1.0, 1.0, size=shape)
            mant = u + np.copysign(1.0, u)
            ex = rng.integers(-span, span + 1, size=shape, dtype=np.int32)
            return np.ldexp(mant, ex).astype(abt, copy=False)
        x = rng.uniform(-1.0, 1.0, size=shape)
        if dist == "outliers":
            mask = rng.random(shape) < 0.01
            x = np.where(mask, x * 1e4, x)
        return x.astype(abt)

    def gen_c(shape):
        if row in INT_ROWS:
            lim = 64 if dist == "small_int" else (1 << 20)
            return rng.integers(-lim, lim + 1, size=shape, dtype=np.int32)
        return gen_ab(shape).astype(ct)

    def fill_operand(arr, srows, scols, ld, gen):
        view = arr.reshape(arr.shape[0], scols, ld)
        view[:, :, :srows] = gen((arr.shape[0], scols, srows))

    A = np.zeros((batch, lda * ac), dtype=abt)
    fill_operand(A, ar, ac, lda, gen_ab)
    bbt = B_DTYPE.get(row, abt)
    B = np.zeros((batch, ldb * bc), dtype=bbt)
    fill_operand(B, br, bc, ldb, lambda shape: gen_ab(shape, bbt))
    C = np.zeros((batch, ldc * n), dtype=ct)
    fill_operand(C, m, n, ldc, gen_c)
    return Problem(row, transa, transb, m, n, k, lda, ldb, ldc, batch,
                   st(alpha).item(), st(beta).item(), A, B, C, name)


# ------------------------------------------------------------------------------------------
# named benchmark workloads
# ------------------------------------------------------------------------------------------
WORKLOADS = {
    "fp32_batch64_128": dict(row="f32", transa=OP_N, transb=OP_N, m=128, n=128, k=128, batch=64,
                             alpha=1.0, beta=0.5, lda=128, ldb=128, ldc=128, seed=0),
    "i8_batch512_512": dict(row="i8", transa=OP_T, transb=OP_N, m=512, n=512, k=512, batch=512,
                            alpha=1, beta=1, lda=512, ldb=512, ldc=512, seed=1),
    "f64_batch32_1024": dict(row="f64", transa=OP_N, transb=OP_T, m=1024, n=1024, k=1024,
                             batch=32, alpha=1.0, beta=0.0, lda=1032, ldb=1032, ldc=1032,
                             seed=2, dist="expspread"),
    "fp32_batch4096_64": dict(row="f32", transa=OP_T, transb=OP_T, m=64, n=64, k=64, batch=4096,
                              alpha=0.75, beta=0.25, lda=64, ldb=64, ldc=64, seed=3,
                              dist="outliers"),
    # not a configuration of the task: a compute-bound shape for the int8 tensor-core kernel
    # (the 512^3 beta=1 batch is bound by HBM bandwidth)
    "i8_batch8_4096": dict(row="i8", transa=OP_T, transb=OP_N, m=4096, n=4096, k=4096, batch=8,
                           alpha=1, beta=0, lda=4096, ldb=4096, ldc=4096, seed=4),
    # not configurations of the task either: few output tiles and a long k (two-pass slicing and
    # split-K of the Ozaki path), and int8 in the N/N layout (the pack pre-pass ahead of the
    # tensor-core kernel)
    "f64_batch2_256_8192": dict(row="f64", transa=OP_T, transb=OP_N, m=256, n=256, k=8192, batch=2,
                                alpha=1.0, beta=0.0, seed=5, dist="expspread"),
    "i8_batch64_512_nn": dict(row="i8", transa=OP_N, transb=OP_N, m=512, n=512, k=512, batch=64,
                              alpha=1, beta=1, seed=6),
}


def workload(name: str, batch: int | None = None) -> Problem:
    kw = dict(WORKLOADS[name])
    if batch is not None:
        kw["batch"] = batch
    return make_problem(name=name, **kw)


def grouped_sizes(count: int = 10000, seed: int = 5, lo: int = 8, hi: int = 512):
    """Per-instance (m, n, k) drawn log-uniform integers in [lo, hi], transposes uniform in
    {N, T}; ld = stored rows rounded up to a multiple of 8; the first half of the instances is
    fp64, the second half fp32."""
    rng = np.random.default_rng(seed)
    dims = np.floor(np.exp(rng.uniform(math.log(lo), math.log(hi + 1), size=(count, 3)))).astype(np.int64)
    dims = np.clip(dims, lo, hi)
    trans = rng.integers(0, 2, size=(count, 2))
    return dims, trans


def grouped_problems(count: int = 10000, seed: int = 5, lo: int = 8, hi: int = 512,
                     fp64_fraction: float = 0.5) -> list[Problem]:
    """The uneven grouped workload: `count` single-instance problems with m, n, k log-uniform
    integers in [lo, hi], op N/T uniform, ld = stored rows rounded up to a multiple of 8, entries
    U[-1,1), alpha 1, beta 0; the first fp64_fraction of them fp64, the rest fp32."""
    dims, trans = grouped_sizes(count, seed, lo, hi)
    out = []
    n64 = int(round(count * fp64_fraction))
    for i in range(count):
        m, n, k = (int(x) for x in dims[i])
        ta, tb = (int(x) for x in trans[i])
        ar, _ = stored_shape(ta, m, k)
        br, _ = stored_shape(tb, k, n)
        r8 = lambda x: (x + 7) // 8 * 8
        out.append(make_problem("f64" if i < n64 else "f32", ta, tb, m, n, k, 1, 1.0, 0.0,
                                lda=r8(ar), ldb=r8(br), ldc=r8(m), seed=seed * 100003 + i,
                                name=f"g{i}"))
    return out
