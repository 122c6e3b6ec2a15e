"""ctypes bindings for the CPU checkers -- TEST INFRASTRUCTURE ONLY.

Imported only by tests/, bench.py (CPU baseline / reference arm) and __graft_entry__.smoke(), and
only to check or time against; the library in ssblasex_b200/ never imports this module.

  restated_gemm(p)       the plain-C restatement of the reference semantics (liboracle.so)
  reference_gemm(p)      the reference library itself, built from its own sources
                         (_ref/libssblas_ref.so, see ref_x86_build.cpp)
  exact_f64(p, b, rows)  FP64-exact result rows (double-double) and the error normaliser
  normalized_error(...)  max |C - C*| / (|alpha| |op(A)| |op(B)| + |beta| |C0|)
"""
from __future__ import annotations

import ctypes as ct
import os
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
_ORACLE = None
_REF = None

c_long, c_int, c_double, c_float, c_vp = ct.c_long, ct.c_int, ct.c_double, ct.c_float, ct.c_void_p


def _load_oracle():
    global _ORACLE
    if _ORACLE is None:
        lib = ct.CDLL(str(HERE / "liboracle.so"))
        common = [c_int, c_int, c_long, c_long, c_long]
        lib.oracle_gemm_f32.argtypes = common + [c_float, c_vp, c_long, c_vp, c_long, c_float, c_vp, c_long, c_long]
        lib.oracle_gemm_f64.argtypes = common + [c_double, c_vp, c_long, c_vp, c_long, c_double, c_vp, c_long, c_long]
        lib.oracle_gemm_i8.argtypes = common + [ct.c_int32, c_vp, c_long, c_vp, c_long, ct.c_int32, c_vp, c_long, c_long]
        for f in (lib.oracle_gemm_f32, lib.oracle_gemm_f64, lib.oracle_gemm_i8):
            f.restype = c_int
        lib.oracle_exact_f64.argtypes = common + [c_double, c_vp, c_long, c_vp, c_long, c_double, c_vp, c_long, c_vp, c_long, c_vp, c_vp]
        lib.oracle_exact_f64.restype = None
        _ORACLE = lib
    return _ORACLE


def reference_available() -> bool:
    return (HERE / "_ref" / "libssblas_ref.so").exists()


def _load_reference():
    """The reference reads OMP_NUM_THREADS at first use; counts 2, 3, 4 and 6 crash it with a
    division by zero (src/include/Utils/ssblas_threads.hpp:26-52 lets them through to the tune
    launchers), so callers must not use them."""
    global _REF
    if _REF is None:
        nt = os.environ.get("OMP_NUM_THREADS")
        if nt is not None and nt.strip() in {"2", "3", "4", "6"}:
            raise RuntimeError("OMP_NUM_THREADS in {2,3,4,6} crashes the reference build")
        lib = ct.CDLL(str(HERE / "_ref" / "libssblas_ref.so"))
        lib.ssblasGemmBatchedEx.argtypes = [c_int, c_int, c_long, c_long, c_long, c_vp, c_vp, c_int,
                                            c_long, c_vp, c_int, c_long, c_vp, c_vp, c_int, c_long,
                                            c_long, c_int, c_int]
        lib.ssblasGemmBatchedEx.restype = c_int
        _REF = lib
    return _REF


def _ptr_array(arr: np.ndarray, batch: int):
    base = arr.ctypes.data
    stride = arr.strides[0]
    return (c_vp * max(batch, 1))(*[base + b * stride for b in range(batch)])


def _scalar(p, v):
    return np.array([v], dtype=p.scale_dtype)


def restated_gemm(p, C: np.ndarray | None = None):
    """Run the C restatement in place on a copy of p.C (or on C). Returns (status, C)."""
    lib = _load_oracle()
    C = p.C.copy() if C is None else C
    A_ = _ptr_array(p.A, p.batch)
    B_ = _ptr_array(p.B, p.batch)
    C_ = _ptr_array(C, p.batch)
    f = {"f32": lib.oracle_gemm_f32, "f64": lib.oracle_gemm_f64, "i8": lib.oracle_gemm_i8}[p.row]
    alpha = int(p.alpha) if p.row == "i8" else p.alpha
    beta = int(p.beta) if p.row == "i8" else p.beta
    st = f(p.transa, p.transb, p.m, p.n, p.k, alpha, A_, p.lda, B_, p.ldb, beta, C_, p.ldc, p.batch)
    return st, C


def reference_gemm(p, C: np.ndarray | None = None, m=None, n=None, k=None, batch=None,
                   transa=None, transb=None, types=None):
    """Run the reference library itself (host pointers, synchronous). Overrides let tests pass
    the degenerate arguments the reference's status conventions are pinned on."""
    lib = _load_reference()
    C = p.C.copy() if C is None else C
    nb = p.batch if batch is None else batch
    A_ = _ptr_array(p.A, max(p.batch, 1))
    B_ = _ptr_array(p.B, max(p.batch, 1))
    C_ = _ptr_array(C, max(p.batch, 1))
    al = _scalar(p, p.alpha)
    be = _scalar(p, p.beta)
    ta, tb, tc = p.types if types is None else types
    st = lib.ssblasGemmBatchedEx(
        p.transa if transa is None else transa, p.transb if transb is None else transb,
        p.m if m is None else m, p.n if n is None else n, p.k if k is None else k,
        al.ctypes.data, A_, ta, p.lda, B_, tb, p.ldb, be.ctypes.data, C_, tc, p.ldc, nb, 0, 0)
    return st, C


def exact_f64(p, b: int, rows=None):
    """FP64-exact alpha*op(A)*op(B) + beta*C0 for instance b on the given rows (default all).
    Returns (C_exact[len(rows), n], norm[len(rows), n])."""
    lib = _load_oracle()
    rows = np.arange(p.m, dtype=np.int64) if rows is None else np.asarray(rows, dtype=np.int64)
    A = np.ascontiguousarray(p.A[b], dtype=np.float64)
    B = np.ascontiguousarray(p.B[b], dtype=np.float64)
    C0 = np.ascontiguousarray(p.C[b], dtype=np.float64)
    nr = len(rows)
    out = np.empty(nr * p.n, dtype=np.float64)
    nrm = np.empty(nr * p.n, dtype=np.float64)
    lib.oracle_exact_f64(p.transa, p.transb, p.m, p.n, p.k, float(p.alpha), A.ctypes.data, p.lda,
                         B.ctypes.data, p.ldb, float(p.beta), C0.ctypes.data, p.ldc,
                         rows.ctypes.data, nr, out.ctypes.data, nrm.ctypes.data)
    return out.reshape(p.n, nr).T, nrm.reshape(p.n, nr).T


def normalized_error(p, C: np.ndarray, instances=None, rows=None) -> float:
    """max over the sampled entries of |C - C*| / (|alpha| |op(A)| |op(B)| + |beta| |C0|)."""
    instances = range(p.batch) if instances is None else instances
    worst = 0.0
    for b in instances:
        r = np.arange(p.m) if rows is None else np.asarray(rows)
        ex, nrm = exact_f64(p, b, r)
        got = p.c_view(C, b)[r, :].astype(np.float64)
        with np.errstate(invalid="ignore", divide="ignore"):
            err = np.abs(got - ex) / np.where(nrm > 0, nrm, 1.0)
        worst = max(worst, float(np.max(err)) if err.size else 0.0)
    return worst


def unit_roundoff(row: str) -> float:
    return {"f32": 2.0 ** -24, "f64": 2.0 ** -53}[row]


def ozaki_f64(p, slices: int, C: np.ndarray | None = None):
    """The library's Ozaki FP64 emulation restated on the CPU (bit-exact target), all instances.
    Returns (status, C) -- status -1 if an int32 accumulator would have overflowed."""
    lib = _load_oracle()
    f = lib.oracle_ozaki_f64
    f.argtypes = [c_int, c_int, c_long, c_long, c_long, c_double, c_vp, c_long, c_vp, c_long,
                  c_double, c_vp, c_long, c_int]
    f.restype = c_int
    C = p.C.copy() if C is None else C
    st = 0
    for b in range(p.batch):
        A = np.ascontiguousarray(p.A[b]); B = np.ascontiguousarray(p.B[b])
        Cb = np.ascontiguousarray(C[b])
        st |= f(p.transa, p.transb, p.m, p.n, p.k, float(p.alpha), A.ctypes.data, p.lda, B.ctypes.data,
                p.ldb, float(p.beta), Cb.ctypes.data, p.ldc, slices)
        C[b] = Cb
    return st, C


def bf16x3_f32(p, b: int):
    """FP64-exact value of the three-BF16-product emulation for instance b (m x n array)."""
    lib = _load_oracle()
    f = lib.oracle_bf16x3_f32
    f.argtypes = [c_int, c_int, c_long, c_long, c_long, c_float, c_vp, c_long, c_vp, c_long,
                  c_float, c_vp, c_long, c_vp]
    f.restype = None
    out = np.empty(p.m * p.n, dtype=np.float64)
    A = np.ascontiguousarray(p.A[b]); B = np.ascontiguousarray(p.B[b]); Cb = np.ascontiguousarray(p.C[b])
    f(p.transa, p.transb, p.m, p.n, p.k, float(p.alpha), A.ctypes.data, p.lda, B.ctypes.data, p.ldb,
      float(p.beta), Cb.ctypes.data, p.ldc, out.ctypes.data)
    return out.reshape(p.n, p.m).T
