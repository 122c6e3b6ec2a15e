// Plain FP32 batched GEMM (FFMA) with a cp.async pipeline, for the fp32 row in its plain form.
//
// Semantics follow the reference (hirokitokura/ssblasEx): C <- beta*C, not read when beta == 0
// (src/include/CScale/Xgemm_scale_kernel.hpp:164-176), then C <- C + acc*alpha with one fused
// multiply-add (src/include/GemmCore/Xgemm_kernel_sve_v4x5_1.hpp:93-127). The reference adds
// alpha*acc once per 512-wide K block; here it is added once, which differs only by rounding.
//
// Design: one CTA per (BM x BN tile, instance). op(A) and op(B) tiles reach shared memory through
// a STAGES-deep cp.async ring, always staged [k][mn] (mn contiguous) so that every thread reads
// its TM (TN) consecutive values with 16-byte loads:
//   - an operand whose rows (m or n) are contiguous in global memory is copied in 16-byte chunks
//     along mn (when 16-byte aligned; 4-byte copies otherwise);
//   - an operand whose K is contiguous is transposed by the copy itself: one 4-byte cp.async per
//     element, consecutive threads taking consecutive k of one row.
// Small problems (the 64^3 instances of a 4096-instance batch) keep the whole K in flight from
// the start: with K <= STAGES * BK every stage is issued in the prologue.
// Each thread owns a TM x TN block of C (rows tx*TM.., columns ty*TN..); a warp covers 4 x 8
// threads, so its A reads are 4 distinct 16-byte vectors and its B reads 8 (broadcasts).
#include <cuda_runtime.h>
#include <stdint.h>

#include "grouped.h"
#include "internal.h"

namespace ssb {
namespace {

struct SgemmArgs {
  long m, n, k, lda, ldb, ldc, batch;
  const float* const* A;
  const float* const* B;
  float* const* C;
  float alpha, beta;
};

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp16s(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp4s(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void commit_s() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void wait_s() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Copies the (ROWS x BK) slab of one operand at (r0, k0) into a stage buffer staged [k][r]
// (pitch ROWS + 4 floats). MN: element (r, k) at X[r + k*ld]; otherwise at X[r*ld + k].
// Each thread's chunks keep one position along the contiguous dimension and step a fixed number
// of rows (or k) per iteration, so the source pointer advances by a constant: no per-element
// index arithmetic.
template <int ROWS, int BK, int NT, bool MN>
__device__ __forceinline__ void sload(float* dst, const float* __restrict__ X, long nrows, long K, long ld, long r0,
                                      long k0, bool vec) {
  constexpr int P = ROWS + 4;
  const int t = threadIdx.x;
  if (MN) {
    if (vec) {
      // 16-byte chunks along r: thread t takes r = 4 (t % (ROWS/4)), k = t / (ROWS/4) + q KSTEP
      constexpr int CPR = ROWS / 4, KSTEP = NT / CPR, NQ = BK / KSTEP;
      static_assert(NT % CPR == 0 && BK % KSTEP == 0, "copy shape");
      const int rr = 4 * (t % CPR), kk0 = t / CPR;
      const long gr = r0 + rr;
      long nv = nrows - gr;
      nv = nv < 0 ? 0 : (nv > 4 ? 4 : nv);
      const float* src = X + gr + (k0 + kk0) * ld;
      const uint32_t d0 = saddr(dst + kk0 * P + rr);
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const bool ok = nv > 0 && k0 + kk0 + q * KSTEP < K;
        cp16s(d0 + 4u * (uint32_t)(q * KSTEP * P), ok ? src + (long)q * KSTEP * ld : X, ok ? (int)(4 * nv) : 0);
      }
    } else {
      constexpr int KSTEP = NT / ROWS, NQ = BK / KSTEP;
      static_assert(NT % ROWS == 0 && BK % KSTEP == 0, "copy shape");
      const int rr = t % ROWS, kk0 = t / ROWS;
      const bool rok = r0 + rr < nrows;
      const float* src = X + (r0 + rr) + (k0 + kk0) * ld;
      const uint32_t d0 = saddr(dst + kk0 * P + rr);
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const bool ok = rok && k0 + kk0 + q * KSTEP < K;
        cp4s(d0 + 4u * (uint32_t)(q * KSTEP * P), ok ? src + (long)q * KSTEP * ld : X, ok ? 4 : 0);
      }
    }
  } else {
    // Transpose by the copy. A warp instruction covers 8 consecutive k of 4 consecutive rows
    // (lane = 4 * (k % 8) + r % 4): the reads are whole 32-byte sectors, and the [k][r] stores
    // land in banks (4 k + r) mod 32 (pitch = 4 mod 32), all 32 distinct. Instruction u = warp + W q
    // of the stage takes k group u % KG and row group u / KG, so each thread keeps its k and
    // steps RSTEP rows per iteration.
    constexpr int W = NT / 32, KG = BK / 8, RSTEP = 4 * (W / KG), NQ = ROWS / RSTEP;
    static_assert(BK % 8 == 0 && W % KG == 0 && ROWS % RSTEP == 0 && P % 32 == 4, "copy shape");
    const int lane = t % 32, warp = t / 32;
    const int kk = 8 * (warp % KG) + lane / 4, rr0 = 4 * (warp / KG) + lane % 4;
    const bool kok = k0 + kk < K;
    const float* src = X + (r0 + rr0) * ld + (k0 + kk);
    const uint32_t d0 = saddr(dst + kk * P + rr0);
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const bool ok = kok && r0 + rr0 + q * RSTEP < nrows;
      cp4s(d0 + 4u * (uint32_t)(q * RSTEP), ok ? src + (long)q * RSTEP * ld : X, ok ? 4 : 0);
    }
  }
}

// One BM x BN tile of C = alpha op(A) op(B) + beta C for one instance, by the whole CTA: the K loop
// over the stage ring, then the epilogue. Leaves the stage buffers free.
template <int BM, int BN, int BK, int TM, int TN, int STAGES, bool A_MN, bool B_MN>
__device__ __forceinline__ void sgemm_tile(const float* __restrict__ A, const float* __restrict__ B,
                                           float* __restrict__ C, long m, long n, long k, long lda, long ldb,
                                           long ldc, float alpha, float beta, long m0, long n0, float* sm) {
  constexpr int TX = BM / TM, TY = BN / TN, NT = TX * TY;
  constexpr int PA = BM + 4, PB = BN + 4;
  constexpr int STAGE = BK * (PA + PB);
  // warp = 4 (m) x 8 (n) threads
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
  constexpr int WX = TX / 4;   // warps along m
  const int tx = (warp % WX) * 4 + lane % 4;
  const int ty = (warp / WX) * 8 + lane / 4;
  const bool vecA = ((uintptr_t)A % 16 == 0) && (lda % 4 == 0);
  const bool vecB = ((uintptr_t)B % 16 == 0) && (ldb % 4 == 0);
  float acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = 0.0f;

  const long ktiles = (k + BK - 1) / BK;
  auto issue = [&](long kt) {
    float* sa = sm + (kt % STAGES) * STAGE;
    float* sb = sa + BK * PA;
    sload<BM, BK, NT, A_MN>(sa, A, m, k, lda, m0, kt * BK, vecA);
    sload<BN, BK, NT, B_MN>(sb, B, n, k, ldb, n0, kt * BK, vecB);
  };
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < ktiles) issue(s);
    commit_s();
  }
  for (long kt = 0; kt < ktiles; ++kt) {
    wait_s<STAGES - 2>();
    __syncthreads();
    if (kt + STAGES - 1 < ktiles) issue(kt + STAGES - 1);
    commit_s();
    const float* sa = sm + (kt % STAGES) * STAGE;
    const float* sb = sa + BK * PA;
#pragma unroll 4
    for (int kk = 0; kk < BK; ++kk) {
      float av[TM], bv[TN];
#pragma unroll
      for (int i = 0; i < TM; i += 4) {
        const float4 x = *(const float4*)(sa + kk * PA + tx * TM + i);
        av[i] = x.x; av[i + 1] = x.y; av[i + 2] = x.z; av[i + 3] = x.w;
      }
#pragma unroll
      for (int j = 0; j < TN; j += 4) {
        const float4 x = *(const float4*)(sb + kk * PB + ty * TN + j);
        bv[j] = x.x; bv[j + 1] = x.y; bv[j + 2] = x.z; bv[j + 3] = x.w;
      }
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
  }
  wait_s<0>();
  __syncthreads();   // the next tile's copies reuse the stage buffers

  // epilogue: C rows m0 + tx*TM + i (contiguous per thread), columns n0 + ty*TN + j; 16-byte
  // reads and writes when the thread's rows are inside C and C is 16-byte aligned
  const bool read_c = beta != 0.0f;
  const long gi0 = m0 + tx * TM;
  const bool cvec = (((uintptr_t)C) % 16 == 0) && (ldc % 4 == 0) && gi0 + TM <= m;
#pragma unroll
  for (int j = 0; j < TN; ++j) {
    const long gj = n0 + ty * TN + j;
    if (gj >= n) continue;
    float* cp = C + gi0 + gj * ldc;
    if (cvec) {
      float4 cv[TM / 4];
#pragma unroll
      for (int i = 0; i < TM; i += 4) cv[i / 4] = read_c ? *(const float4*)(cp + i) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int i = 0; i < TM; i += 4) {
        float4 o;
        o.x = fmaf(acc[i][j], alpha, read_c ? beta * cv[i / 4].x : 0.0f);
        o.y = fmaf(acc[i + 1][j], alpha, read_c ? beta * cv[i / 4].y : 0.0f);
        o.z = fmaf(acc[i + 2][j], alpha, read_c ? beta * cv[i / 4].z : 0.0f);
        o.w = fmaf(acc[i + 3][j], alpha, read_c ? beta * cv[i / 4].w : 0.0f);
        *(float4*)(cp + i) = o;
      }
    } else {
      float cv[TM];
#pragma unroll
      for (int i = 0; i < TM; ++i) cv[i] = (read_c && gi0 + i < m) ? cp[i] : 0.0f;
#pragma unroll
      for (int i = 0; i < TM; ++i)
        if (gi0 + i < m) cp[i] = fmaf(acc[i][j], alpha, read_c ? beta * cv[i] : 0.0f);
    }
  }
}

template <int BM, int BN, int BK, int TM, int TN, int STAGES, int MINB, bool A_MN, bool B_MN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN), MINB) sgemm_async_kernel(SgemmArgs args) {
  extern __shared__ __align__(16) float sm[];
  const long tiles_m = (args.m + BM - 1) / BM;
  const long m0 = (blockIdx.x % tiles_m) * BM;
  const long n0 = (blockIdx.x / tiles_m) * BN;
  for (long b = blockIdx.y; b < args.batch; b += gridDim.y)
    sgemm_tile<BM, BN, BK, TM, TN, STAGES, A_MN, B_MN>(args.A[b], args.B[b], args.C[b], args.m, args.n, args.k,
                                                       args.lda, args.ldb, args.ldc, args.alpha, args.beta, m0, n0,
                                                       sm);
}

// Grouped form (plain fp32 instances of ssblasGemmGroupedBatchedEx): one CTA per (instance,
// 64 x 64 tile) entry of a tile table whose instances all have this op(A) / op(B) layout; the tile
// shape of configuration 3.
constexpr int kGT = 64, kGBK = 32, kGTM = 4, kGST = 2;
template <bool A_MN, bool B_MN>
__global__ void __launch_bounds__((kGT / kGTM) * (kGT / kGTM), 3)
sgemm_grouped_kernel(const SimtGInst* __restrict__ inst, const int* __restrict__ tiles, const float* const* A,
                     const float* const* B, float* const* C) {
  extern __shared__ __align__(16) float sm[];
  const int* t = tiles + 3 * (long)blockIdx.x;
  const SimtGInst g = inst[t[0]];
  sgemm_tile<kGT, kGT, kGBK, kGTM, kGTM, kGST, A_MN, B_MN>(A[g.idx], B[g.idx], C[g.idx], g.m, g.n, g.k, g.lda, g.ldb,
                                                         g.ldc, g.alpha_f, g.beta_f, (long)t[1] * kGT,
                                                         (long)t[2] * kGT, sm);
}

// Persistent form for K <= KS * BK (the whole K of a work item fits the KS stages of one buffer):
// work item w = (instance w / tiles, tile w % tiles), CTA c takes items c, c + G, c + 2G, ... and
// double-buffers them -- the next item's operands are in flight while the current one is computed
// and written -- so a batch of thousands of small instances keeps HBM busy instead of paying one
// load latency per CTA. C of the item (when beta != 0) is read into registers before the
// products, so that read overlaps them too.
template <int BM, int BN, int BK, int TM, int TN, int KS, int MINB, bool A_MN, bool B_MN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN), MINB) sgemm_small_kernel(SgemmArgs args, uint32_t tiles_m,
                                                                                   uint32_t tiles, uint32_t total) {
  constexpr int TX = BM / TM, TY = BN / TN, NT = TX * TY;
  constexpr int PA = BM + 4, PB = BN + 4;
  constexpr int STAGE = BK * (PA + PB);
  constexpr int BUF = KS * STAGE;
  extern __shared__ __align__(16) float sm[];
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
  constexpr int WX = TX / 4;   // warps along m (a warp = 4 (m) x 8 (n) threads)
  const int tx = (warp % WX) * 4 + lane % 4;
  const int ty = (warp / WX) * 8 + lane / 4;
  const long ktiles = (args.k + BK - 1) / BK;   // <= KS (checked by the launcher)
  const bool read_c = args.beta != 0.0f;

  // work item w -> (instance b, tile t) -> (m0, n0), in 32-bit arithmetic (the launcher keeps the
  // item count below 2^31): a 64-bit division costs dozens of instructions per item
  auto item = [&](uint32_t w, long& b, long& m0, long& n0) {
    const uint32_t bb = w / tiles, t = w - bb * tiles;
    const uint32_t tn = t / tiles_m;
    b = bb;
    m0 = (long)(t - tn * tiles_m) * BM;
    n0 = (long)tn * BN;
  };
  auto issue = [&](uint32_t w, int buf) {
    long b, m0, n0;
    item(w, b, m0, n0);
    const float* __restrict__ A = args.A[b];
    const float* __restrict__ B = args.B[b];
    const bool vecA = ((uintptr_t)A % 16 == 0) && (args.lda % 4 == 0);
    const bool vecB = ((uintptr_t)B % 16 == 0) && (args.ldb % 4 == 0);
#pragma unroll
    for (int kt = 0; kt < KS; ++kt) {
      if (kt >= ktiles) break;
      float* sa = sm + buf * BUF + kt * STAGE;
      sload<BM, BK, NT, A_MN>(sa, A, args.m, args.k, args.lda, m0, kt * BK, vecA);
      sload<BN, BK, NT, B_MN>(sa + BK * PA, B, args.n, args.k, args.ldb, n0, kt * BK, vecB);
    }
  };

  uint32_t w = blockIdx.x;
  if (w < total) issue(w, 0);
  commit_s();
  for (int buf = 0; w < total; w += gridDim.x, buf ^= 1) {
    // the next item's operands go into the other buffer (free since the previous iteration's
    // closing barrier)
    if (w + gridDim.x < total) issue(w + gridDim.x, buf ^ 1);
    commit_s();
    long b, m0, n0;
    item(w, b, m0, n0);
    float* __restrict__ C = args.C[b];
    const long gi0 = m0 + tx * TM;
    const bool cvec = (((uintptr_t)C) % 16 == 0) && (args.ldc % 4 == 0) && gi0 + TM <= args.m;
    float cv[TN][TM];
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const long gj = n0 + ty * TN + j;
      const float* cp = C + gi0 + gj * args.ldc;
#pragma unroll
      for (int i = 0; i < TM; i += 4) {
        if (read_c && gj < args.n && cvec) {
          const float4 x = *(const float4*)(cp + i);
          cv[j][i] = x.x; cv[j][i + 1] = x.y; cv[j][i + 2] = x.z; cv[j][i + 3] = x.w;
        } else {
#pragma unroll
          for (int q = 0; q < 4; ++q) cv[j][i + q] = (read_c && gj < args.n && gi0 + i + q < args.m) ? cp[i + q] : 0.0f;
        }
      }
    }
    wait_s<1>();   // this item's group has landed (the next item's may still be in flight)
    __syncthreads();
    float acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) acc[i][j] = 0.0f;
    for (int kt = 0; kt < ktiles; ++kt) {
      const float* sa = sm + buf * BUF + kt * STAGE;
      const float* sb = sa + BK * PA;
#pragma unroll 4
      for (int kk = 0; kk < BK; ++kk) {
        float av[TM], bv[TN];
#pragma unroll
        for (int i = 0; i < TM; i += 4) {
          const float4 x = *(const float4*)(sa + kk * PA + tx * TM + i);
          av[i] = x.x; av[i + 1] = x.y; av[i + 2] = x.z; av[i + 3] = x.w;
        }
#pragma unroll
        for (int j = 0; j < TN; j += 4) {
          const float4 x = *(const float4*)(sb + kk * PB + ty * TN + j);
          bv[j] = x.x; bv[j + 1] = x.y; bv[j + 2] = x.z; bv[j + 3] = x.w;
        }
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
          for (int j = 0; j < TN; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
      }
    }
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const long gj = n0 + ty * TN + j;
      if (gj >= args.n) continue;
      float* cp = C + gi0 + gj * args.ldc;
      if (cvec) {
#pragma unroll
        for (int i = 0; i < TM; i += 4) {
          float4 o;
          o.x = fmaf(acc[i][j], args.alpha, read_c ? args.beta * cv[j][i] : 0.0f);
          o.y = fmaf(acc[i + 1][j], args.alpha, read_c ? args.beta * cv[j][i + 1] : 0.0f);
          o.z = fmaf(acc[i + 2][j], args.alpha, read_c ? args.beta * cv[j][i + 2] : 0.0f);
          o.w = fmaf(acc[i + 3][j], args.alpha, read_c ? args.beta * cv[j][i + 3] : 0.0f);
          *(float4*)(cp + i) = o;
        }
      } else {
#pragma unroll
        for (int i = 0; i < TM; ++i)
          if (gi0 + i < args.m) cp[i] = fmaf(acc[i][j], args.alpha, read_c ? args.beta * cv[j][i] : 0.0f);
      }
    }
    __syncthreads();   // this buffer is refilled by the next iteration's copies
  }
  wait_s<0>();
}

// Register-heavy form for K <= KMAX: one 64 x 64 tile of one instance per CTA of 64 threads, each
// thread an 8 x 8 block of C (rows 8 tx.., columns 8 ty.., tx = t % 8, ty = t / 8). The whole K of
// the tile is requested at once (16-deep slices of the cp.async copies above, both operands
// staged [k][rows]), C (beta != 0) is read into registers while the copies land, and the inner
// loop issues 4 shared-memory vector loads per 64 FFMAs -- a quarter of the per-product overhead
// of the 4 x 4 threads. Several CTAs per SM overlap one tile's loads with another's products.
// (Staging a K-contiguous operand as it lies, [rows][k] with 16-byte copies, measured slower on
// 4096 x 64^3 TT: 0.105 ms against 0.084 ms -- its rows 8 apart per thread turn the C stores
// into 4-byte ones.)
template <int KMAX, int MINB, bool A_MN, bool B_MN>
__global__ void __launch_bounds__(64, MINB) sgemm_reg8_kernel(SgemmArgs args, uint32_t tiles_m, uint32_t tiles) {
  constexpr int P = 64 + 4;
  extern __shared__ __align__(16) float sm[];
  float* sa = sm;                 // [KMAX][P] op(A): k, then m
  float* sb = sm + KMAX * P;      // [KMAX][P] op(B): k, then n
  const uint32_t w = blockIdx.x;
  const uint32_t bb = w / tiles, t = w - bb * tiles;
  const uint32_t tn = t / tiles_m;
  const long b = bb;
  const long m0 = (long)(t - tn * tiles_m) * 64, n0 = (long)tn * 64;
  const float* __restrict__ A = args.A[b];
  const float* __restrict__ B = args.B[b];
  float* __restrict__ C = args.C[b];
  const bool vecA = ((uintptr_t)A % 16 == 0) && (args.lda % 4 == 0);
  const bool vecB = ((uintptr_t)B % 16 == 0) && (args.ldb % 4 == 0);
  const int K = (int)args.k;   // <= KMAX (checked by the launcher)
  const int slices = (K + 15) / 16;
  for (int sl = 0; sl < slices; ++sl) {
    sload<64, 16, 64, A_MN>(sa + sl * 16 * P, A, args.m, args.k, args.lda, m0, sl * 16, vecA);
    sload<64, 16, 64, B_MN>(sb + sl * 16 * P, B, args.n, args.k, args.ldb, n0, sl * 16, vecB);
  }
  commit_s();

  const int tx = threadIdx.x % 8, ty = threadIdx.x / 8;
  const long gi0 = m0 + tx * 8;
  const bool read_c = args.beta != 0.0f;
  const bool cvec = (((uintptr_t)C) % 16 == 0) && (args.ldc % 4 == 0) && gi0 + 8 <= args.m;
  // C of this thread's block, in flight while the operand copies land
  float cv[8][8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const long gj = n0 + ty * 8 + j;
    const float* cp = C + gi0 + gj * args.ldc;
    if (read_c && gj < args.n && cvec) {
      const float4 x0 = *(const float4*)cp, x1 = *(const float4*)(cp + 4);
      cv[j][0] = x0.x; cv[j][1] = x0.y; cv[j][2] = x0.z; cv[j][3] = x0.w;
      cv[j][4] = x1.x; cv[j][5] = x1.y; cv[j][6] = x1.z; cv[j][7] = x1.w;
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i) cv[j][i] = (read_c && gj < args.n && gi0 + i < args.m) ? cp[i] : 0.0f;
    }
  }
  wait_s<0>();
  __syncthreads();

  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;
#pragma unroll 4
  for (int kk = 0; kk < K; ++kk) {
    const float4 a0 = *(const float4*)(sa + kk * P + tx * 8), a1 = *(const float4*)(sa + kk * P + tx * 8 + 4);
    const float4 b0 = *(const float4*)(sb + kk * P + ty * 8), b1 = *(const float4*)(sb + kk * P + ty * 8 + 4);
    const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
    const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
  }

#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const long gj = n0 + ty * 8 + j;
    if (gj >= args.n) continue;
    float* cp = C + gi0 + gj * args.ldc;
    float o[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) o[i] = fmaf(acc[i][j], args.alpha, read_c ? args.beta * cv[j][i] : 0.0f);
    if (cvec) {
      *(float4*)cp = make_float4(o[0], o[1], o[2], o[3]);
      *(float4*)(cp + 4) = make_float4(o[4], o[5], o[6], o[7]);
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i)
        if (gi0 + i < args.m) cp[i] = o[i];
    }
  }
}

template <int KMAX, int MINB, bool A_MN, bool B_MN>
cudaError_t launch_reg8(const SgemmArgs& a, cudaStream_t st) {
  constexpr int SMEM = 2 * KMAX * (64 + 4) * 4;
  auto kern = sgemm_reg8_kernel<KMAX, MINB, A_MN, B_MN>;
  static bool attr[kMaxDevices] = {};
  if (cudaError_t e = smem_attr_once(attr, kern, SMEM)) return e;
  const long tiles_m = (a.m + 63) / 64;
  const long tiles = tiles_m * ((a.n + 63) / 64);
  const long total = tiles * a.batch;
  if (total >= (1L << 31)) return cudaErrorNotSupported;
  kern<<<(unsigned)total, 64, SMEM, st>>>(a, (uint32_t)tiles_m, (uint32_t)tiles);
  return cudaGetLastError();
}

template <int KMAX, int MINB>
cudaError_t launch_reg8_l(const SgemmArgs& a, bool a_mn, bool b_mn, cudaStream_t st) {
  if (a_mn && b_mn) return launch_reg8<KMAX, MINB, true, true>(a, st);
  if (a_mn) return launch_reg8<KMAX, MINB, true, false>(a, st);
  if (b_mn) return launch_reg8<KMAX, MINB, false, true>(a, st);
  return launch_reg8<KMAX, MINB, false, false>(a, st);
}

// K split inside the CTA, for k <= KMAX: one 64 x 64 tile per CTA of 256 threads, four groups of
// 64 threads, each group an 8 x 8 block per thread over a quarter of K (as the 64-thread form
// above), then the four partial tiles meet in shared memory (over the operand buffers) and every
// thread adds its 16 outputs' parts in a fixed order (group 0 + 1 + 2 + 3) and applies alpha and
// beta. Four times the warps of the 64-thread form per tile, so batches of few large-K tiles
// (64 x 128^3: 256 tiles for 148 SMs) keep every scheduler fed.
template <int KMAX, int MINB, bool A_MN, bool B_MN>
__global__ void __launch_bounds__(256, MINB) sgemm_ksplit_kernel(SgemmArgs args, uint32_t tiles_m, uint32_t tiles) {
  constexpr int P = 64 + 4;
  extern __shared__ __align__(16) float sm[];
  float* sa = sm;                 // [KMAX][P] op(A): k, then m
  float* sb = sm + KMAX * P;      // [KMAX][P] op(B): k, then n
  float* red = sm;                // after the products: [4 groups][64 columns][P] partial tiles
  float* sc = sm + 2 * KMAX * P;  // [64 columns][P] C (beta != 0)
  static_assert(2 * KMAX >= 4 * 64, "the partial tiles reuse the operand buffers");
  const uint32_t w = blockIdx.x;
  const uint32_t bb = w / tiles, t = w - bb * tiles;
  const uint32_t tn = t / tiles_m;
  const long b = bb;
  const long m0 = (long)(t - tn * tiles_m) * 64, n0 = (long)tn * 64;
  const float* __restrict__ A = args.A[b];
  const float* __restrict__ B = args.B[b];
  float* __restrict__ C = args.C[b];
  const bool vecA = ((uintptr_t)A % 16 == 0) && (args.lda % 4 == 0);
  const bool vecB = ((uintptr_t)B % 16 == 0) && (args.ldb % 4 == 0);
  const int K = (int)args.k;   // <= KMAX (checked by the launcher)
  const bool read_c = args.beta != 0.0f;
  const bool vecC = ((uintptr_t)C % 16 == 0) && (args.ldc % 4 == 0);
  for (int sl = 0; sl < (K + 15) / 16; ++sl) {
    sload<64, 16, 256, A_MN>(sa + sl * 16 * P, A, args.m, args.k, args.lda, m0, sl * 16, vecA);
    sload<64, 16, 256, B_MN>(sb + sl * 16 * P, B, args.n, args.k, args.ldb, n0, sl * 16, vecB);
  }
  // C tile (columns n0.., rows m0..) staged [column][row], in flight with the operands
  if (read_c)
    for (int sl = 0; sl < 4; ++sl)
      sload<64, 16, 256, true>(sc + sl * 16 * P, C, args.m, args.n, args.ldc, m0, n0 + sl * 16, vecC);
  commit_s();

  // output mapping of the final sum: thread t takes rows 4 (t % 16).., columns 4 (t / 16)..
  const int orow = 4 * (threadIdx.x % 16), ocol = 4 * (threadIdx.x / 16);
  const long gi0 = m0 + orow;
  const bool cvec = vecC && gi0 + 4 <= args.m;
  wait_s<0>();
  __syncthreads();

  const int g = threadIdx.x / 64, t64 = threadIdx.x % 64;
  const int tx = t64 % 8, ty = t64 / 8;
  const int kq = (K + 3) / 4;
  const int k0 = g * kq, k1 = (k0 + kq < K) ? k0 + kq : K;
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;
#pragma unroll 2
  for (int kk = k0; kk < k1; ++kk) {
    const float4 a0 = *(const float4*)(sa + kk * P + tx * 8), a1 = *(const float4*)(sa + kk * P + tx * 8 + 4);
    const float4 b0 = *(const float4*)(sb + kk * P + ty * 8), b1 = *(const float4*)(sb + kk * P + ty * 8 + 4);
    const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
    const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
  }
  __syncthreads();   // every group is done with the operand buffers
  float* part = red + g * 64 * P;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    float* q = part + (ty * 8 + j) * P + tx * 8;
    *(float4*)q = make_float4(acc[0][j], acc[1][j], acc[2][j], acc[3][j]);
    *(float4*)(q + 4) = make_float4(acc[4][j], acc[5][j], acc[6][j], acc[7][j]);
  }
  __syncthreads();

#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const long gj = n0 + ocol + j;
    if (gj >= args.n) continue;
    float4 s = *(const float4*)(red + (ocol + j) * P + orow);
#pragma unroll
    for (int gg = 1; gg < 4; ++gg) {
      const float4 x = *(const float4*)(red + gg * 64 * P + (ocol + j) * P + orow);
      s.x += x.x; s.y += x.y; s.z += x.z; s.w += x.w;
    }
    const float sv[4] = {s.x, s.y, s.z, s.w};
    float4 c4 = make_float4(0.f, 0.f, 0.f, 0.f);
    if (read_c) c4 = *(const float4*)(sc + (ocol + j) * P + orow);
    const float cv[4] = {c4.x, c4.y, c4.z, c4.w};
    float o[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) o[i] = fmaf(sv[i], args.alpha, read_c ? args.beta * cv[i] : 0.0f);
    float* cp = C + gi0 + gj * args.ldc;
    if (cvec) {
      *(float4*)cp = make_float4(o[0], o[1], o[2], o[3]);
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (gi0 + i < args.m) cp[i] = o[i];
    }
  }
}

template <int KMAX, int MINB, bool A_MN, bool B_MN>
cudaError_t launch_ksplit(const SgemmArgs& a, cudaStream_t st) {
  constexpr int SMEM = (2 * KMAX + 64) * (64 + 4) * 4;
  auto kern = sgemm_ksplit_kernel<KMAX, MINB, A_MN, B_MN>;
  static bool attr[kMaxDevices] = {};
  if (cudaError_t e = smem_attr_once(attr, kern, SMEM)) return e;
  const long tiles_m = (a.m + 63) / 64;
  const long tiles = tiles_m * ((a.n + 63) / 64);
  const long total = tiles * a.batch;
  if (total >= (1L << 31)) return cudaErrorNotSupported;
  kern<<<(unsigned)total, 256, SMEM, st>>>(a, (uint32_t)tiles_m, (uint32_t)tiles);
  return cudaGetLastError();
}

template <int KMAX, int MINB>
cudaError_t launch_ksplit_l(const SgemmArgs& a, bool a_mn, bool b_mn, cudaStream_t st) {
  if (a_mn && b_mn) return launch_ksplit<KMAX, MINB, true, true>(a, st);
  if (a_mn) return launch_ksplit<KMAX, MINB, true, false>(a, st);
  if (b_mn) return launch_ksplit<KMAX, MINB, false, true>(a, st);
  return launch_ksplit<KMAX, MINB, false, false>(a, st);
}

template <int BM, int BN, int BK, int TM, int TN, int KS, int MINB, bool A_MN, bool B_MN>
cudaError_t launch_small(const SgemmArgs& a, cudaStream_t st) {
  constexpr int NT = (BM / TM) * (BN / TN);
  constexpr int SMEM = 2 * KS * BK * (BM + 4 + BN + 4) * 4;
  auto kern = sgemm_small_kernel<BM, BN, BK, TM, TN, KS, MINB, A_MN, B_MN>;
  static int per_sm_dev[kMaxDevices] = {};
  const int dev = current_device();
  if (dev < 0) return cudaErrorInvalidDevice;
  int& per_sm = per_sm_dev[dev];
  if (!per_sm) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, SMEM);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
  }
  const long tiles_m = (a.m + BM - 1) / BM;
  const long tiles = tiles_m * ((a.n + BN - 1) / BN);
  const long total = tiles * a.batch;
  if (total >= (1L << 31)) return cudaErrorNotSupported;   // the caller takes the tiled kernel
  const long cap = (long)per_sm * num_sms();
  kern<<<(unsigned)(total < cap ? total : cap), NT, SMEM, st>>>(a, (uint32_t)tiles_m, (uint32_t)tiles,
                                                                 (uint32_t)total);
  return cudaGetLastError();
}

template <int BM, int BN, int BK, int TM, int TN, int STAGES, int MINB, bool A_MN, bool B_MN>
cudaError_t launch_s(const SgemmArgs& a, cudaStream_t st) {
  constexpr int NT = (BM / TM) * (BN / TN);
  constexpr int SMEM = STAGES * BK * (BM + 4 + BN + 4) * 4;
  auto kern = sgemm_async_kernel<BM, BN, BK, TM, TN, STAGES, MINB, A_MN, B_MN>;
  static bool attr[kMaxDevices] = {};
  if (cudaError_t e = smem_attr_once(attr, kern, SMEM)) return e;
  const long tiles = ((a.m + BM - 1) / BM) * ((a.n + BN - 1) / BN);
  if (tiles > 0x7fffffffL) return cudaErrorInvalidValue;
  dim3 grid((unsigned)tiles, (unsigned)(a.batch < 65535 ? a.batch : 65535));
  kern<<<grid, NT, SMEM, st>>>(a);
  return cudaGetLastError();
}

template <int BM, int BN, int BK, int TM, int TN, int STAGES, int MINB>
cudaError_t launch_sl(const SgemmArgs& a, bool a_mn, bool b_mn, cudaStream_t st) {
  if (a_mn && b_mn) return launch_s<BM, BN, BK, TM, TN, STAGES, MINB, true, true>(a, st);
  if (a_mn) return launch_s<BM, BN, BK, TM, TN, STAGES, MINB, true, false>(a, st);
  if (b_mn) return launch_s<BM, BN, BK, TM, TN, STAGES, MINB, false, true>(a, st);
  return launch_s<BM, BN, BK, TM, TN, STAGES, MINB, false, false>(a, st);
}

}  // namespace

template <bool A_MN, bool B_MN>
cudaError_t launch_sgemm_grouped_layout(const GroupedSimt& s, int lay, cudaStream_t st) {
  constexpr int SMEM = kGST * kGBK * (2 * kGT + 8) * 4;
  auto kern = sgemm_grouped_kernel<A_MN, B_MN>;
  static bool attr[kMaxDevices] = {};
  if (cudaError_t e = smem_attr_once(attr, kern, SMEM)) return e;
  kern<<<(unsigned)s.nsg[lay], (kGT / kGTM) * (kGT / kGTM), SMEM, st>>>(
      (const SimtGInst*)s.inst32, (const int*)s.sg_tiles[lay], (const float* const*)s.A, (const float* const*)s.B,
      (float* const*)s.C);
  note_launch();
  return cudaGetLastError();
}

// The plain fp32 tiles of a grouped call, one launch per op(A) / op(B) layout present (layout
// index = 2 * (op(A) rows contiguous) + (op(B) columns contiguous)).
cudaError_t launch_sgemm_grouped(const GroupedSimt& s, cudaStream_t st) {
  if (!s.nsg[0] && !s.nsg[1] && !s.nsg[2] && !s.nsg[3]) return cudaSuccess;
  ProfScope prof("sgemm_grouped", st);
  cudaError_t e = cudaSuccess;
  for (int lay = 0; lay < 4 && e == cudaSuccess; ++lay) {
    if (!s.nsg[lay]) continue;
    switch (lay) {
      case 3: e = launch_sgemm_grouped_layout<true, true>(s, lay, st); break;
      case 2: e = launch_sgemm_grouped_layout<true, false>(s, lay, st); break;
      case 1: e = launch_sgemm_grouped_layout<false, true>(s, lay, st); break;
      default: e = launch_sgemm_grouped_layout<false, false>(s, lay, st); break;
    }
  }
  return e;
}

cudaError_t launch_sgemm_async(const BatchDesc& d, int config, cudaStream_t st) {
  SgemmArgs a;
  a.m = d.m; a.n = d.n; a.k = d.k; a.lda = d.lda; a.ldb = d.ldb; a.ldc = d.ldc; a.batch = d.batch;
  a.A = (const float* const*)d.A;
  a.B = (const float* const*)d.B;
  a.C = (float* const*)d.C;
  a.alpha = d.alpha_f;
  a.beta = d.beta_f;
  const bool a_mn = d.transa == SSBLAS_OP_N;   // op(A) rows (m) contiguous
  const bool b_mn = d.transb == SSBLAS_OP_T;   // op(B) columns (n) contiguous
  cudaError_t e;
  // 12 / 13: 64 x 64 tiles, TMA staging and bulk stores (equally spaced, 16-byte aligned
  //   instances): two stages and two C tiles, two CTAs per SM / three and three, one CTA per SM
  if (config == 12 || config == 13) {
    e = launch_sgemm_tma(d, config - 12, st);
    if (e != cudaErrorNotSupported) return e;
  }
  ProfScope prof("sgemm_async", st);
  // 3: 64 x 64 tiles, 256 threads of 4 x 4, 32-deep K stages x 2 (k <= 64 entirely in flight)
  // 4: 128 x 128 tiles, 256 threads of 8 x 8, 16-deep K stages x 3
  // 5 (k <= 64): 64 x 64 tiles, persistent CTAs that double-buffer their work items, 256 threads
  //   of 4 x 4
  // 6 (k <= 64): as 5 with 128 threads of 8 x 4 (twice the products per thread for the same
  //   per-item index, copy and epilogue work)
  // 7: 32 x 64 tiles, 128 threads of 4 x 4, 32-deep K stages x 4 (k <= 128 entirely in flight):
  //   four times the CTAs of configuration 3, for batches whose 64 x 64 tiles fill under a wave
  // 8: 32 x 32 tiles, 64 threads of 4 x 4, 16-deep K stages x 8
  // 9 (k <= 64) / 10 (k <= 128): 64 x 64 tiles, 64 threads of 8 x 8, the whole K at once
  // 11 (k <= 128): 64 x 64 tiles, 256 threads: four 8 x 8 groups over quarters of K, summed in
  //   shared memory
  e = cudaErrorNotSupported;
  if (config == 9 && d.k <= 64) {
    e = launch_reg8_l<64, 4>(a, a_mn, b_mn, st);
  } else if (config == 10 && d.k <= 128) {
    e = launch_reg8_l<128, 3>(a, a_mn, b_mn, st);
  } else if (config == 11 && d.k <= 128) {
    e = launch_ksplit_l<128, 2>(a, a_mn, b_mn, st);
  } else if (config == 5 && d.k <= 64) {
    if (a_mn && b_mn) e = launch_small<64, 64, 32, 4, 4, 2, 3, true, true>(a, st);
    else if (a_mn) e = launch_small<64, 64, 32, 4, 4, 2, 3, true, false>(a, st);
    else if (b_mn) e = launch_small<64, 64, 32, 4, 4, 2, 3, false, true>(a, st);
    else e = launch_small<64, 64, 32, 4, 4, 2, 3, false, false>(a, st);
  } else if (config == 6 && d.k <= 64) {
    if (a_mn && b_mn) e = launch_small<64, 64, 32, 8, 4, 2, 3, true, true>(a, st);
    else if (a_mn) e = launch_small<64, 64, 32, 8, 4, 2, 3, true, false>(a, st);
    else if (b_mn) e = launch_small<64, 64, 32, 8, 4, 2, 3, false, true>(a, st);
    else e = launch_small<64, 64, 32, 8, 4, 2, 3, false, false>(a, st);
  } else if (config == 4) {
    e = launch_sl<128, 128, 16, 8, 8, 3, 1>(a, a_mn, b_mn, st);
  } else if (config == 7) {
    e = launch_sl<32, 64, 32, 4, 4, 4, 4>(a, a_mn, b_mn, st);
  } else if (config == 8) {
    e = launch_sl<32, 32, 16, 4, 4, 8, 8>(a, a_mn, b_mn, st);
  }
  // configuration 3 serves the rest (and item counts of 2^31 or more for 5 and 6)
  if (e == cudaErrorNotSupported) e = launch_sl<64, 64, 32, 4, 4, 2, 3>(a, a_mn, b_mn, st);
  note_launch();
  return e;
}

}  // namespace ssb
