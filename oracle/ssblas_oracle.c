/*
 * CPU oracle for ssblasGemmBatchedEx -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, bench.py (its CPU-baseline leg) and the smoke check load this code, and only to
 * check or time against it. The shipped library (ssblasex_b200/) never links, loads or calls it;
 * there is no CPU fallback in the product path.
 *
 * Two kinds of oracle live here:
 *
 *  (1) oracle_gemm_{f32,f64,i8}: a plain-C restatement of the reference's batched GEMM semantics
 *      (hirokitokura/ssblasEx), used to pin behaviour and as the parity target:
 *        - status: m, n or batchCount <= 0 -> SSBLAS_STATUS_INTERNAL_ERROR, because the launcher
 *          rejects an empty task grid (src/include/Launcher/launcher.hpp:174-176; the task counts
 *          are ceil(m/BM)*ceil(n/BN)*batch, launch_kernels/..._single_kernel_BMNK.hpp:380-384);
 *          op C on the fp32/fp64 rows -> SSBLAS_STATUS_INVALID_VALUE
 *          (Impl/GemmBatchedEx/ssblasGemmBatchedEx_ALLDATASIZESAME.hpp:50-88, 91-120);
 *        - k <= 0 -> SUCCESS with C untouched: beta is applied inside the K-block loop, which
 *          runs zero times (launch_kernels/..._single_kernel_BMNK.hpp:200-213);
 *        - C is scaled by beta before the first K block, and beta == 0 stores zero without
 *          reading C (src/include/CScale/Xgemm_scale_kernel.hpp:164-176);
 *        - each K block of 512 (..._single_kernel_BMNK.hpp:378) is accumulated from zero in the
 *          element type, k in order (fused multiply-add, src/include/asm/SVE/def_sve_asm_float.h:38-47),
 *          then added as C <- C + acc * alpha with one fused multiply-add
 *          (src/include/GemmCore/Xgemm_kernel_sve_v4x5_1.hpp:93-127, FMAD at
 *          def_sve_asm_float.h:50-59);
 *        - int8 x int8 products accumulate in int32 with two's-complement wrap (sdot,
 *          def_sve_asm_float.h:46) and the epilogue wraps too (mad, :58);
 *        - element (r, c) of op(X) is X[r + c*ld] for N and X[r*ld + c] for T
 *          (src/include/Utils/ssblas_BatchMat.hpp:31-39).
 *
 *  (2) oracle_exact_f64: an FP64-exact reference (double-double accumulation) of
 *      alpha*op(A)*op(B) + beta*C for one instance, with the normaliser
 *      |alpha|*|op(A)|*|op(B)| + |beta|*|C| used for the componentwise error metric.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { ST_SUCCESS = 0, ST_ALLOC_FAILED = 1, ST_INVALID = 2, ST_INTERNAL = 3 };
enum { OP_N = 0, OP_T = 1, OP_C = 2 };

#define REF_BLOCK_K 512

static inline long at(int trans, long r, long c, long ld) {
  return trans == OP_N ? r + c * ld : r * ld + c;
}

/* Only N and T are accepted. The reference rejects op C on the fp rows; on the int8 row it
 * accepts op C and reads through a NULL pointer (src/include/Utils/ssblas_BatchMat.hpp:38), which
 * the library turns into SSBLAS_STATUS_INVALID_VALUE as well. */
static int check_common(int transa, int transb, long m, long n, long batch) {
  if ((transa != OP_N && transa != OP_T) || (transb != OP_N && transb != OP_T)) return ST_INVALID;
  if (m <= 0 || n <= 0 || batch <= 0) return ST_INTERNAL;
  return -1;
}

int oracle_gemm_f32(int transa, int transb, long m, long n, long k, float alpha,
                    const float* const* A, long lda, const float* const* B, long ldb, float beta,
                    float* const* C, long ldc, long batch) {
  int st = check_common(transa, transb, m, n, batch);
  if (st >= 0) return st;
  if (k <= 0) return ST_SUCCESS;
  for (long b = 0; b < batch; ++b)
    for (long j = 0; j < n; ++j)
      for (long i = 0; i < m; ++i) {
        float c = (beta == 0.0f) ? 0.0f : beta * C[b][i + j * ldc];
        for (long k0 = 0; k0 < k; k0 += REF_BLOCK_K) {
          long k1 = k0 + REF_BLOCK_K < k ? k0 + REF_BLOCK_K : k;
          float acc = 0.0f;
          for (long kk = k0; kk < k1; ++kk)
            acc = fmaf(A[b][at(transa, i, kk, lda)], B[b][at(transb, kk, j, ldb)], acc);
          c = fmaf(acc, alpha, c);
        }
        C[b][i + j * ldc] = c;
      }
  return ST_SUCCESS;
}

int oracle_gemm_f64(int transa, int transb, long m, long n, long k, double alpha,
                    const double* const* A, long lda, const double* const* B, long ldb,
                    double beta, double* const* C, long ldc, long batch) {
  int st = check_common(transa, transb, m, n, batch);
  if (st >= 0) return st;
  if (k <= 0) return ST_SUCCESS;
  for (long b = 0; b < batch; ++b)
    for (long j = 0; j < n; ++j)
      for (long i = 0; i < m; ++i) {
        double c = (beta == 0.0) ? 0.0 : beta * C[b][i + j * ldc];
        for (long k0 = 0; k0 < k; k0 += REF_BLOCK_K) {
          long k1 = k0 + REF_BLOCK_K < k ? k0 + REF_BLOCK_K : k;
          double acc = 0.0;
          for (long kk = k0; kk < k1; ++kk)
            acc = fma(A[b][at(transa, i, kk, lda)], B[b][at(transb, kk, j, ldb)], acc);
          c = fma(acc, alpha, c);
        }
        C[b][i + j * ldc] = c;
      }
  return ST_SUCCESS;
}

/* int8 row: alpha/beta are int32 (Impl/GemmBatchedEx/ssblasGemmBatchedEx_ALLDATASIZESAME_impl.hpp:146-147
 * read them as T_SCALE = int for this row, ssblasGemmBatchedExSelector.hpp:38-39). All arithmetic
 * is done in uint32 so that overflow wraps exactly as the int32 vector instructions do. */
int oracle_gemm_i8(int transa, int transb, long m, long n, long k, int32_t alpha,
                   const int8_t* const* A, long lda, const int8_t* const* B, long ldb,
                   int32_t beta, int32_t* const* C, long ldc, long batch) {
  int st = check_common(transa, transb, m, n, batch);
  if (st >= 0) return st;
  if (k <= 0) return ST_SUCCESS;
  for (long b = 0; b < batch; ++b)
    for (long j = 0; j < n; ++j)
      for (long i = 0; i < m; ++i) {
        uint32_t c = (beta == 0) ? 0u : (uint32_t)beta * (uint32_t)C[b][i + j * ldc];
        for (long k0 = 0; k0 < k; k0 += REF_BLOCK_K) {
          long k1 = k0 + REF_BLOCK_K < k ? k0 + REF_BLOCK_K : k;
          uint32_t acc = 0u;
          for (long kk = k0; kk < k1; ++kk)
            acc += (uint32_t)((int32_t)A[b][at(transa, i, kk, lda)] *
                              (int32_t)B[b][at(transb, kk, j, ldb)]);
          c += acc * (uint32_t)alpha;
        }
        C[b][i + j * ldc] = (int32_t)c;
      }
  return ST_SUCCESS;
}

/* ---------------------------------------------------------------- double-double helpers ---- */
typedef struct { double hi, lo; } dd_t;

static inline dd_t dd_two_sum(double a, double b) {
  double s = a + b;
  double bb = s - a;
  double e = (a - (s - bb)) + (b - bb);
  dd_t r = {s, e};
  return r;
}
static inline dd_t dd_add(dd_t x, dd_t y) {
  dd_t s = dd_two_sum(x.hi, y.hi);
  dd_t t = dd_two_sum(x.lo, y.lo);
  s.lo += t.hi;
  s = dd_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return dd_two_sum(s.hi, s.lo);
}
static inline dd_t dd_prod(double a, double b) {
  double p = a * b;
  dd_t r = {p, fma(a, b, -p)};
  return r;
}
static inline dd_t dd_mul_d(dd_t x, double a) {
  dd_t p = dd_prod(x.hi, a);
  p.lo = fma(x.lo, a, p.lo);
  return dd_two_sum(p.hi, p.lo);
}

/* FP64-exact oracle for one instance, rows rows[0..nrows) of the m x n result (all n columns).
 * out_c and out_norm are nrows x n, column-major with leading dimension nrows.
 * C0 may be NULL when beta == 0 (C is not read, as in the library). */
void oracle_exact_f64(int transa, int transb, long m, long n, long k, double alpha,
                      const double* A, long lda, const double* B, long ldb, double beta,
                      const double* C0, long ldc, const long* rows, long nrows, double* out_c,
                      double* out_norm) {
  (void)m;
#pragma omp parallel for schedule(dynamic, 1)
  for (long r = 0; r < nrows; ++r) {
    long i = rows[r];
    for (long j = 0; j < n; ++j) {
      dd_t s = {0.0, 0.0};
      double sabs = 0.0;
      for (long kk = 0; kk < k; ++kk) {
        double a = A[at(transa, i, kk, lda)];
        double b = B[at(transb, kk, j, ldb)];
        s = dd_add(s, dd_prod(a, b));
        sabs += fabs(a) * fabs(b);
      }
      dd_t res = dd_mul_d(s, alpha);
      double nrm = fabs(alpha) * sabs;
      if (beta != 0.0) {
        double c0 = C0[i + j * ldc];
        res = dd_add(res, dd_prod(beta, c0));
        nrm += fabs(beta) * fabs(c0);
      }
      out_c[r + j * nrows] = res.hi + res.lo;
      out_norm[r + j * nrows] = nrm;
    }
  }
}
