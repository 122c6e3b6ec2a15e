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

/* --------------------------------------------------------------- Ozaki int8-slice FP64 ---- */
/* CPU restatement of the library's FP64 emulation (SSBLAS_MATH_FP64_OZAKI), operation for
 * operation, so the device result must match it bit for bit:
 *   per row i of op(A): e_i with max_k |a_ik| < 2^e_i (0 for a zero row),
 *     X = rint(a * 2^(8S-2-e_i)), balanced base-256 digits d_0..d_{S-1} (low digits in
 *     [-128,127], d_0 = the rest); the same per column j of op(B) with f_j;
 *   acc_l = sum_{p+q=l, l<S} sum_k dA_p[i,k] dB_q[j,k]  (exact integers);
 *   v = Horner over l = S-1..0 of v*2^-8 + acc_l (FP64); w = v * 2^(e_i+f_j-12);
 *   C = fma(w, alpha, beta==0 ? 0 : beta*C).
 * Returns 0, or -1 if an accumulator left the int32 range the device uses. */
static void oz_digits(long long X, int S, int8_t* d) {
  for (int p = S - 1; p >= 1; --p) {
    long long lo = ((X + 128) & 255) - 128;
    d[p] = (int8_t)lo;
    X = (X - lo) >> 8;
  }
  d[0] = (int8_t)X;
}

/* Rows (columns of op(B)) holding an Inf or a NaN get exponent OZ_NONFINITE and zero digits, and
 * every C(i, j) they touch is the quiet NaN 0x7ff8000000000000 (the library's policy). */
#define OZ_NONFINITE 4096

static void oz_slice(int trans, long rows, long k, const double* X, long ld, int rows_are_cols, int S,
                     int8_t* dig /* [S][rows][k] */, int* ex) {
  for (long r = 0; r < rows; ++r) {
    double mx = 0.0;
    int finite = 1;
    for (long kk = 0; kk < k; ++kk) {
      double v = rows_are_cols ? X[at(trans, kk, r, ld)] : X[at(trans, r, kk, ld)];
      if (!isfinite(v)) finite = 0;
      else mx = fmax(mx, fabs(v));
    }
    int e = 0;
    if (mx > 0.0) frexp(mx, &e);
    ex[r] = finite ? e : OZ_NONFINITE;
    for (long kk = 0; kk < k; ++kk) {
      double v = rows_are_cols ? X[at(trans, kk, r, ld)] : X[at(trans, r, kk, ld)];
      if (!finite) v = 0.0;
      long long Xi = llrint(scalbn(v, 8 * S - 2 - e));
      int8_t d[8];
      oz_digits(Xi, S, d);
      for (int p = 0; p < S; ++p) dig[((long)p * rows + r) * k + kk] = d[p];
    }
  }
}

int oracle_ozaki_f64(int transa, int transb, long m, long n, long k, double alpha, const double* A,
                     long lda, const double* B, long ldb, double beta, double* C, long ldc, int S) {
  int8_t* da = (int8_t*)malloc((size_t)S * m * k);
  int8_t* db = (int8_t*)malloc((size_t)S * n * k);
  int* ea = (int*)malloc(sizeof(int) * m);
  int* eb = (int*)malloc(sizeof(int) * n);
  int status = 0;
  oz_slice(transa, m, k, A, lda, 0, S, da, ea);
  oz_slice(transb, n, k, B, ldb, 1, S, db, eb);
#pragma omp parallel for schedule(dynamic, 4) reduction(| : status)
  for (long j = 0; j < n; ++j) {
    long long acc[8];
    for (long i = 0; i < m; ++i) {
      for (int l = 0; l < S; ++l) acc[l] = 0;
      for (int p = 0; p < S; ++p)
        for (int q = 0; p + q < S; ++q) {
          const int8_t* x = da + ((long)p * m + i) * k;
          const int8_t* y = db + ((long)q * n + j) * k;
          long long s = 0;
          for (long kk = 0; kk < k; ++kk) s += (long long)x[kk] * (long long)y[kk];
          acc[p + q] += s;
        }
      double v = 0.0;
      for (int l = S - 1; l >= 0; --l) {
        if (acc[l] > 2147483647LL || acc[l] < -2147483648LL) status = -1;
        v = v * 0x1p-8 + (double)acc[l];
      }
      if (ea[i] == OZ_NONFINITE || eb[j] == OZ_NONFINITE) {
        const uint64_t qnan = 0x7ff8000000000000ull;
        memcpy(&C[i + j * ldc], &qnan, 8);
        continue;
      }
      double w = scalbn(v, ea[i] + eb[j] - 12);
      double t = (beta == 0.0) ? 0.0 : beta * C[i + j * ldc];
      C[i + j * ldc] = fma(w, alpha, t);
    }
  }
  free(da); free(db); free(ea); free(eb);
  return status;
}

/* ---------------------------------------------------------------- 3 x BF16 FP32 ---------- */
static float bf16_rn(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return x; /* inf / nan unchanged */
  u += 0x7fffu + ((u >> 16) & 1u);
  u &= 0xffff0000u;
  float r;
  memcpy(&r, &u, 4);
  return r;
}

/* The value the library's SSBLAS_MATH_FP32_BF16X3 mode approximates, computed exactly in FP64:
 * hi = bf16(x), lo = bf16(x - hi) for each entry; out = alpha * sum_k (ha hb + ha lb + la hb)
 * + beta * C (the device accumulates the same products in FP32). */
void oracle_bf16x3_f32(int transa, int transb, long m, long n, long k, float alpha, const float* A,
                       long lda, const float* B, long ldb, float beta, const float* C, long ldc,
                       double* out /* m x n, ld m */) {
#pragma omp parallel for schedule(dynamic, 4)
  for (long j = 0; j < n; ++j)
    for (long i = 0; i < m; ++i) {
      double s = 0.0;
      for (long kk = 0; kk < k; ++kk) {
        float a = A[at(transa, i, kk, lda)], b = B[at(transb, kk, j, ldb)];
        float ha = bf16_rn(a), la = bf16_rn(a - ha), hb = bf16_rn(b), lb = bf16_rn(b - hb);
        s += (double)ha * hb + (double)ha * lb + (double)la * hb;
      }
      double r = (double)alpha * s;
      if (beta != 0.0f) r += (double)beta * C[i + j * ldc];
      out[i + j * m] = r;
    }
}
