// FP32 batched GEMM as three BF16 products for instances that fit one output tile (m, n <= 128),
// with the hi/lo split done in shared memory: the operands cross HBM once, as fp32, instead of
// being read, split into BF16 planes in HBM by a separate pass and read again.
//
// The reference's fp32 row (src/include/GemmCore/Xgemm_kernel_sve_v4x5_1.hpp, FMLA in fp32) is
// emulated as in the tiled 3xBF16 path: x = hi + lo with hi = bf16(x), lo = bf16(x - hi), and
// C = alpha * (Ahi Bhi + Ahi Blo + Alo Bhi) + beta * C with FP32 accumulation on the tensor cores
// (tcgen05.mma kind::f16, bf16 inputs) -- the same split and the same three products, so the
// results agree with the tiled path to FP32 accumulation order.
//
// Design: persistent CTAs (one per SM), one instance per item, the items of a CTA streamed
// through a warp-specialised pipeline so that several are in flight at once:
//   warp 0     TMA: each 64-wide K chunk of op(A) and op(B), as it lies in memory (K or M/N
//              contiguous), into an fp32 stage (F32S stages); a second lane brings each item's C
//              tile (beta != 0) into its own ring
//   warps 2-9  converters: fp32 stage -> BF16 hi and lo planes in the 128-byte-swizzled layout the
//              tensor core reads (K-major for an operand whose K is contiguous in memory, MN-major
//              otherwise, so every thread reads 16 contiguous bytes and writes 8 + 8), BFS stages
//   warp 1     MMA: 4 K steps x 3 products per chunk into a tensor-memory accumulator of
//              128 lanes x NB columns, two accumulators alternating between items
//   warps 10-13 epilogue: a lane per row combines alpha * acc + beta * C over the item's C tile
//              (brought in by TMA while the products run) and one bulk tensor store writes it;
//              where C is not addressable by a tensor map the lanes read and write C themselves
// Rows past m of the A planes and columns past n of the B planes hold zeros (TMA fill) or are
// never read back; the epilogue writes only the m x n block. The instances must be equally
// spaced with 16-byte-aligned rows (tensor maps); other batches take the tiled path. Every wait
// is bounded and reports through the device error flag.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "internal.h"
#include "ptx.cuh"

namespace ssb {
namespace {

constexpr int kKC = 64;          // K elements per chunk (one 128-byte swizzle span of bf16)
constexpr int kConvWarps = 8;                  // converter warps (warps 2 .. 2 + kConvWarps - 1)
constexpr int kEpiWarp0 = 2 + kConvWarps;      // first of the 4 epilogue warps
constexpr int kFusedThreads = 32 * (kEpiWarp0 + 4);

// MB, NB: the instance's row / column extent rounded up to 64 or 128; F32S, BFS: stage counts;
// CST: stages of C tiles (beta != 0), 0 = the epilogue reads C itself
template <int MB_, int NB_, int F32S_, int BFS_, int CST_>
struct Fused {
  static constexpr int MB = MB_, NB = NB_, F32S = F32S_, BFS = BFS_, CST = CST_;
  static constexpr int C_STAGE = MB * NB * 4;         // fp32 C tile, [NB columns][MB rows]
  static constexpr int F32_A = MB * kKC * 4;          // fp32 chunk of op(A)
  static constexpr int F32_STAGE = (MB + NB) * kKC * 4;
  static constexpr int A_PLANE = 128 * 128;           // bf16, 128 rows (the MMA's M) x 64 k
  static constexpr int B_PLANE = NB * 128;            // bf16, NB columns x 64 k
  static constexpr int BF_STAGE = 2 * A_PLANE + 2 * B_PLANE;   // A hi, A lo, B hi, B lo
  static constexpr int BARS = 256;
  static constexpr int SMEM = 1024 + F32S * F32_STAGE + BFS * BF_STAGE + CST * C_STAGE + BARS;
  static constexpr int TMEM_COLS = 2 * NB;            // two accumulators
  static_assert(F32_STAGE % 1024 == 0 && BF_STAGE % 1024 == 0, "stage alignment");
  static_assert(SMEM <= 232448, "shared memory");
};

struct FusedArgs {
  long m, n, k, ldc, batch;
  long strideC;            // elements between instances of C
  float* C0;
  float alpha, beta;
  int a_kcontig, b_kcontig;
  int c_tma;               // C through the tile ring by TMA (CST > 0, C addressable by a map)
  int* err;
  uint32_t wait_limit;
};

// byte offset of 8-byte group g (4 bf16 values, g in [0, 16)) of line `line` of a
// 128-byte-swizzled plane: 16-byte chunk g / 2 of the line sits at chunk (g / 2) ^ (line % 8)
__device__ __forceinline__ uint32_t swz(uint32_t line, uint32_t g) {
  return line * 128u + ((((g >> 1) ^ (line & 7u)) << 4) | ((g & 1u) << 3));
}

// hi = bf16(x), lo = bf16(x - hi) of 4 fp32 values, packed 2 per word
__device__ __forceinline__ void split4(const float4 x, uint2& hi, uint2& lo) {
  // paired conversions (one instruction per two values, each rounded to nearest even as a
  // single conversion would be); bf16 -> fp32 is exact, so x - float(hi) is the split's residue
  const __nv_bfloat162 h01 = __floats2bfloat162_rn(x.x, x.y), h23 = __floats2bfloat162_rn(x.z, x.w);
  const float2 f01 = __bfloat1622float2(h01), f23 = __bfloat1622float2(h23);
  const __nv_bfloat162 l01 = __floats2bfloat162_rn(x.x - f01.x, x.y - f01.y);
  const __nv_bfloat162 l23 = __floats2bfloat162_rn(x.z - f23.x, x.w - f23.y);
  hi.x = *(const uint32_t*)&h01;
  hi.y = *(const uint32_t*)&h23;
  lo.x = *(const uint32_t*)&l01;
  lo.y = *(const uint32_t*)&l23;
}

// One operand's fp32 chunk of ROWS x 64 k -> its hi / lo planes. K contiguous: the chunk is
// [ROWS][64 k] and the planes K-major (a line = one row's 64 k); otherwise the chunk is
// [64 k][ROWS] and the planes MN-major (a line = 64 rows at one k, blocks of 64 rows 8 KB apart).
// Unit = 4 consecutive fp32 values; the 256 converter threads take consecutive units, so a warp
// reads 512 contiguous bytes and writes whole lines.
template <int ROWS>
__device__ __forceinline__ void convert(const float* __restrict__ src, uint8_t* hi, uint8_t* lo, bool kcontig, int ct) {
  constexpr int CT = 32 * kConvWarps;
  constexpr int UNITS = ROWS * kKC / 4;
  static_assert(UNITS % CT == 0, "converter shape");
#pragma unroll 4
  for (int u = ct; u < UNITS; u += CT) {
    const float4 x = *(const float4*)(src + 4 * u);
    uint2 h, l;
    split4(x, h, l);
    uint32_t off;
    if (kcontig) {
      off = swz((uint32_t)(u >> 4), (uint32_t)(u & 15));   // row u / 16, k group u % 16
    } else {
      // k line u / (ROWS / 4), row group u % (ROWS / 4)
      const uint32_t line = (uint32_t)(u / (ROWS / 4)), rg = (uint32_t)(u % (ROWS / 4));
      off = (rg >> 4) * 8192u + swz(line, rg & 15u);
    }
    *(uint2*)(hi + off) = h;
    *(uint2*)(lo + off) = l;
  }
}

// AND of `v` over the 128 epilogue threads (named barrier 1)
__device__ __forceinline__ bool epi_all(bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.and.pred p, 1, 128, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

template <class F>
__global__ void __launch_bounds__(kFusedThreads, 1)
bf16x3_fused_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                    const __grid_constant__ CUtensorMap tmC, const FusedArgs a) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* f32 = smem;                                        // [F32S][F32_STAGE]
  uint8_t* bf = smem + F::F32S * F::F32_STAGE;                // [BFS][BF_STAGE]
  uint8_t* cst = bf + F::BFS * F::BF_STAGE;                   // [CST][C_STAGE]
  uint64_t* bars = (uint64_t*)(cst + F::CST * F::C_STAGE);
  uint64_t* f_full = bars;                                    // fp32 chunk landed (TMA bytes)
  uint64_t* f_empty = f_full + F::F32S;                       // fp32 chunk converted (converter warps)
  uint64_t* b_full = f_empty + F::F32S;                       // planes written (converter warps)
  uint64_t* b_empty = b_full + F::BFS;                        // planes read by the MMAs (commit)
  uint64_t* acc_full = b_empty + F::BFS;                      // [2] accumulator complete (commit)
  uint64_t* acc_empty = acc_full + 2;                         // [2] accumulator drained (4 warps)
  uint64_t* drain = acc_empty + 2;
  uint64_t* c_full = drain + 1;                               // [CST] C tile landed (TMA bytes)
  uint64_t* c_empty = c_full + F::CST;                        // [CST] C tile stored (bulk store read it)
  uint32_t* tmem_slot = (uint32_t*)(c_empty + F::CST);
  static_assert((2 * F::F32S + 2 * F::BFS + 2 * F::CST + 5) * 8 + 4 <= F::BARS, "barrier area");
  const bool use_c = a.c_tma && a.beta != 0.0f;

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  int* err = a.err;
  const uint32_t wl = a.wait_limit ? a.wait_limit : ptx::kWaitLimit;
  if (threadIdx.x == 0) {
    for (int s = 0; s < F::F32S; ++s) {
      ptx::mbar_init(ptx::smem_u32(&f_full[s]), 1);
      ptx::mbar_init(ptx::smem_u32(&f_empty[s]), kConvWarps);
    }
    for (int t = 0; t < F::BFS; ++t) {
      ptx::mbar_init(ptx::smem_u32(&b_full[t]), kConvWarps);
      ptx::mbar_init(ptx::smem_u32(&b_empty[t]), 1);
    }
    for (int q = 0; q < 2; ++q) {
      ptx::mbar_init(ptx::smem_u32(&acc_full[q]), 1);
      ptx::mbar_init(ptx::smem_u32(&acc_empty[q]), 4);
    }
    ptx::mbar_init(ptx::smem_u32(drain), 1);
    for (int q = 0; q < F::CST; ++q) {
      ptx::mbar_init(ptx::smem_u32(&c_full[q]), 1);
      ptx::mbar_init(ptx::smem_u32(&c_empty[q]), 1);
    }
    ptx::fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    ptx::prefetch_tmap(&tmA);
    ptx::prefetch_tmap(&tmB);
    if (use_c) ptx::prefetch_tmap(&tmC);
  }
  if (warp == 1) {
    ptx::tmem_alloc(ptx::smem_u32(tmem_slot), F::TMEM_COLS);
    ptx::tmem_relinquish();
  }
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const long nkc = (a.k + kKC - 1) / kKC;

  if (warp == 0) {
    // ------------------------------------------------------------------ TMA ---------------
    if constexpr (F::CST > 0) {
    if (lane == 1 && use_c) {
      // C tiles, on their own ring: this lane waits only for the epilogue, never holds up the
      // operand copies
      long i = 0;
      for (long b = blockIdx.x; b < a.batch; b += gridDim.x, ++i) {
        const int cs = (int)(i % F::CST);
        if (!ptx::mbar_wait(ptx::smem_u32(&c_empty[cs]), (uint32_t)(((i / F::CST) & 1) ^ 1), err, 69, wl)) break;
        const uint32_t bar = ptx::smem_u32(&c_full[cs]);
        ptx::mbar_arrive_expect_tx(bar, F::C_STAGE);
        tma_load_3d(ptx::smem_u32(cst + (size_t)cs * F::C_STAGE), &tmC, bar, 0, 0, (int)b);
      }
      // no copy may still be landing in shared memory when the CTA exits
      for (long j = (i > F::CST ? i - F::CST : 0); j < i; ++j)
        ptx::mbar_wait(ptx::smem_u32(&c_full[j % F::CST]), (uint32_t)((j / F::CST) & 1), err, 62, wl);
    }
    }
    if (lane == 0) {
      long c = 0;
      bool ok = true;
      for (long b = blockIdx.x; b < a.batch && ok; b += gridDim.x) {
        for (long kc = 0; kc < nkc; ++kc, ++c) {
          const int s = (int)(c % F::F32S);
          if (!ptx::mbar_wait(ptx::smem_u32(&f_empty[s]), (uint32_t)(((c / F::F32S) & 1) ^ 1), err, 61, wl)) {
            ok = false;
            break;
          }
          const uint32_t bar = ptx::smem_u32(&f_full[s]);
          const uint32_t fa = ptx::smem_u32(f32 + (size_t)s * F::F32_STAGE), fb = fa + F::F32_A;
          ptx::mbar_arrive_expect_tx(bar, F::F32_STAGE);
          const int k0 = (int)(kc * kKC), bi = (int)b;
          if (a.a_kcontig) tma_load_3d(fa, &tmA, bar, k0, 0, bi);
          else tma_load_3d(fa, &tmA, bar, 0, k0, bi);
          if (a.b_kcontig) tma_load_3d(fb, &tmB, bar, k0, 0, bi);
          else tma_load_3d(fb, &tmB, bar, 0, k0, bi);
        }
      }
      // no copy may still be landing in shared memory when the CTA exits
      for (long j = (c > F::F32S ? c - F::F32S : 0); j < c; ++j)
        ptx::mbar_wait(ptx::smem_u32(&f_full[j % F::F32S]), (uint32_t)((j / F::F32S) & 1), err, 62, wl);
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------------ MMA ---------------
    if (lane == 0) {
      constexpr uint32_t IDESC_KK = ptx::idesc_bf16(128, F::NB, false, false);
      const uint32_t idesc = IDESC_KK | (a.a_kcontig ? 0u : (1u << 15)) | (a.b_kcontig ? 0u : (1u << 16));
      long c = 0, i = 0;
      bool ok = true;
      for (long b = blockIdx.x; b < a.batch && ok; b += gridDim.x, ++i) {
        const int acc = (int)(i & 1);
        if (!ptx::mbar_wait(ptx::smem_u32(&acc_empty[acc]), (uint32_t)(((i >> 1) & 1) ^ 1), err, 63, wl)) break;
        ptx::tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(acc * F::NB);
        for (long kc = 0; kc < nkc; ++kc, ++c) {
          const int t = (int)(c % F::BFS);
          if (!ptx::mbar_wait(ptx::smem_u32(&b_full[t]), (uint32_t)((c / F::BFS) & 1), err, 64, wl)) {
            ok = false;
            break;
          }
          ptx::tc_fence_after();
          const uint32_t ahi = ptx::smem_u32(bf + (size_t)t * F::BF_STAGE);
          const uint32_t pa[2] = {ahi, ahi + F::A_PLANE};
          const uint32_t pb[2] = {ahi + 2 * F::A_PLANE, ahi + 2 * F::A_PLANE + F::B_PLANE};
#pragma unroll
          for (int pq = 0; pq < 3; ++pq) {             // (hi, hi), (hi, lo), (lo, hi)
            const int p = pq == 2 ? 1 : 0, q = pq == 1 ? 1 : 0;
#pragma unroll
            for (int kk = 0; kk < kKC / 16; ++kk) {
              // a K step of 16: 32 bytes along a K-major line, 16 lines of an MN-major plane
              const uint64_t ad = a.a_kcontig ? ptx::smem_desc_kmajor(pa[p] + kk * 32, 128)
                                              : ptx::smem_desc_mnmajor(pa[p] + kk * 2048, 8192);
              const uint64_t bd = a.b_kcontig ? ptx::smem_desc_kmajor(pb[q] + kk * 32, 128)
                                              : ptx::smem_desc_mnmajor(pb[q] + kk * 2048, 8192);
              ptx::mma_f16(d, ad, bd, idesc, (kc > 0 || pq > 0 || kk > 0) ? 1u : 0u);
            }
          }
          ptx::mma_commit(ptx::smem_u32(&b_empty[t]));   // the planes are free when these finish
        }
        if (!ok) break;
        ptx::mma_commit(ptx::smem_u32(&acc_full[acc]));
      }
      // every MMA issued has finished before the tensor memory is released
      ptx::mma_commit(ptx::smem_u32(drain));
      ptx::mbar_wait(ptx::smem_u32(drain), 0, err, 65, wl);
    }
  } else if (warp < kEpiWarp0) {
    // ------------------------------------------------------------------ converters --------
    const int ct = threadIdx.x - 64;
    long c = 0;
    bool ok = true;
    for (long b = blockIdx.x; b < a.batch && ok; b += gridDim.x) {
      for (long kc = 0; kc < nkc; ++kc, ++c) {
        const int s = (int)(c % F::F32S), t = (int)(c % F::BFS);
        if (!ptx::mbar_wait(ptx::smem_u32(&f_full[s]), (uint32_t)((c / F::F32S) & 1), err, 66, wl) ||
            !ptx::mbar_wait(ptx::smem_u32(&b_empty[t]), (uint32_t)(((c / F::BFS) & 1) ^ 1), err, 67, wl)) {
          ok = false;
          break;
        }
        const float* fa = (const float*)(f32 + (size_t)s * F::F32_STAGE);
        const float* fb = (const float*)(f32 + (size_t)s * F::F32_STAGE + F::F32_A);
        uint8_t* ahi = bf + (size_t)t * F::BF_STAGE;
        convert<F::MB>(fa, ahi, ahi + F::A_PLANE, a.a_kcontig != 0, ct);
        convert<F::NB>(fb, ahi + 2 * F::A_PLANE, ahi + 2 * F::A_PLANE + F::B_PLANE, a.b_kcontig != 0, ct);
        ptx::fence_proxy_async_smem();   // generic-proxy writes -> the tensor core's reads
        __syncwarp();
        if (lane == 0) {
          ptx::mbar_arrive(ptx::smem_u32(&b_full[t]));
          ptx::mbar_arrive(ptx::smem_u32(&f_empty[s]));
        }
      }
    }
  } else {
    // ------------------------------------------------------------------ epilogue ----------
    const int quarter = warp % 4;   // tensor-memory lanes 32 quarter .. + 31 = rows of C
    const long row = quarter * 32 + lane;
    const bool rok = row < a.m;
    const bool read_c = a.beta != 0.0f;
    constexpr int G = 32;            // columns per group
    constexpr int NG = F::NB / G;
    long i = 0;
    bool staged = false;
    if constexpr (F::CST > 0) staged = a.c_tma != 0;
    if (staged) {
      if constexpr (F::CST > 0) {
        // C through the tile ring: alpha * acc + beta * C is written over the staged C tile (or
        // into the free tile when beta == 0) and leaves as one bulk tensor store per item; rows
        // and columns outside C are dropped by the store
        for (long b = blockIdx.x; b < a.batch; b += gridDim.x, ++i) {
          const int acc = (int)(i & 1), cs = (int)(i % F::CST);
          float* tile = (float*)(cst + (size_t)cs * F::C_STAGE);
          bool ok = !use_c || ptx::mbar_wait(ptx::smem_u32(&c_full[cs]), (uint32_t)((i / F::CST) & 1), err, 70, wl);
          ok = ok && ptx::mbar_wait(ptx::smem_u32(&acc_full[acc]), (uint32_t)((i >> 1) & 1), err, 68, wl);
          // the four epilogue warps leave together if any wait gave up: they share the named
          // barriers below
          if (!epi_all(ok)) break;
          ptx::tc_fence_after();
#pragma unroll 1
          for (int g = 0; g < NG; ++g) {
            uint32_t raw[G / 16][16];
            const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * F::NB + g * G);
#pragma unroll
            for (int q = 0; q < G / 16; ++q) ptx::tmem_ld16(taddr + (uint32_t)(16 * q), raw[q]);
            ptx::tmem_wait_ld();
            if (row < F::MB) {
#pragma unroll
              for (int j = 0; j < G; ++j) {
                float* e = tile + (g * G + j) * F::MB + row;
                const float tb = read_c ? a.beta * *e : 0.0f;
                *e = fmaf(__uint_as_float(raw[j / 16][j % 16]), a.alpha, tb);
              }
            }
          }
          ptx::tc_fence_before();
          __syncwarp();
          if (lane == 0) ptx::mbar_arrive(ptx::smem_u32(&acc_empty[acc]));
          ptx::fence_proxy_async_smem();   // the tile's generic writes -> the bulk store
          asm volatile("bar.sync 1, 128;" ::: "memory");
          if (warp == kEpiWarp0 && lane == 0) {
            ptx::tma_store_3d(&tmC, ptx::smem_u32(tile), 0, 0, (int)b);
            ptx::bulk_commit();
            ptx::bulk_wait_read();         // the store has read the tile: it may be refilled
            if (use_c) ptx::mbar_arrive(ptx::smem_u32(&c_empty[cs]));
          }
          asm volatile("bar.sync 1, 128;" ::: "memory");
        }
        if (warp == kEpiWarp0 && lane == 0) ptx::bulk_wait_all();
      }
    } else {
      // C read and written by the epilogue threads (C not addressable by a tensor map, or tiles
      // of 128 x 128, which leave no room for a tile ring); the first group's C values are
      // requested before the accumulator is waited for
      for (long b = blockIdx.x; b < a.batch; b += gridDim.x, ++i) {
        const int acc = (int)(i & 1);
        float* __restrict__ C = (float*)((char*)a.C0 + b * a.strideC);
        auto load_c = [&](int g, float (&cv)[G]) {
#pragma unroll
          for (int j = 0; j < G; ++j) {
            const long col = g * G + j;
            cv[j] = (read_c && rok && col < a.n) ? __ldcs(C + row + col * a.ldc) : 0.0f;
          }
        };
        float cv[G];
        load_c(0, cv);
        if (!ptx::mbar_wait(ptx::smem_u32(&acc_full[acc]), (uint32_t)((i >> 1) & 1), err, 68, wl)) break;
        ptx::tc_fence_after();
#pragma unroll 1
        for (int g = 0; g < NG; ++g) {
          uint32_t raw[G / 16][16];
          const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * F::NB + g * G);
#pragma unroll
          for (int q = 0; q < G / 16; ++q) ptx::tmem_ld16(taddr + (uint32_t)(16 * q), raw[q]);
          ptx::tmem_wait_ld();
          if (rok) {
            float* cp = C + row + (long)g * G * a.ldc;
#pragma unroll
            for (int j = 0; j < G; ++j) {
              if (g * G + j < a.n) {
                const float tb = read_c ? a.beta * cv[j] : 0.0f;
                __stcs(cp, fmaf(__uint_as_float(raw[j / 16][j % 16]), a.alpha, tb));
              }
              cp += a.ldc;
            }
          }
          if (g + 1 < NG) load_c(g + 1, cv);
        }
        ptx::tc_fence_before();
        __syncwarp();
        if (lane == 0) ptx::mbar_arrive(ptx::smem_u32(&acc_empty[acc]));
      }
    }
  }
  ptx::tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    ptx::tc_fence_after();
    ptx::tmem_dealloc(tmem, F::TMEM_COLS);
  }
}

// 3-D fp32 map (innermost dimension first) over an equally spaced operand: dims {inner, outer,
// batch}, box {box_in, box_out, 1}, no swizzle, zero fill outside.
bool fp32_map(CUtensorMap* map, const void* base, long inner, long outer, long batch, long ld, long stride_bytes,
              int box_in, int box_out) {
  const long dims[3] = {inner, outer, batch};
  const long strides[2] = {ld * 4, batch > 1 ? stride_bytes : ((ld * outer * 4 + 15) / 16) * 16};
  const int box[3] = {box_in, box_out, 1};
  return make_tiled_map(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, 0);
}

template <class F>
cudaError_t launch_fused(const BatchDesc& d, cudaStream_t st) {
  const bool akc = d.transa == SSBLAS_OP_T, bkc = d.transb == SSBLAS_OP_N;
  CUtensorMap ta, tb;
  // op(A) = A^T: K contiguous (A is k x m); op(A) = A: M contiguous. op(B) = B: K contiguous.
  const bool ok_a = akc ? fp32_map(&ta, d.A0, d.k, d.m, d.batch, d.lda, d.strideA, kKC, F::MB)
                        : fp32_map(&ta, d.A0, d.m, d.k, d.batch, d.lda, d.strideA, F::MB, kKC);
  const bool ok_b = bkc ? fp32_map(&tb, d.B0, d.k, d.n, d.batch, d.ldb, d.strideB, kKC, F::NB)
                        : fp32_map(&tb, d.B0, d.n, d.k, d.batch, d.ldb, d.strideB, F::NB, kKC);
  if (!ok_a || !ok_b) return cudaErrorNotSupported;
  // C tiles by TMA (loads when beta != 0, stores always) when C is 16-byte aligned per column and
  // instance
  CUtensorMap tc;
  memset(&tc, 0, sizeof(tc));
  bool c_tma = false;
  if (F::CST > 0 && (uintptr_t)d.C0 % 16 == 0 && d.ldc % 4 == 0 && (d.batch == 1 || d.strideC % 16 == 0))
    c_tma = fp32_map(&tc, d.C0, d.m, d.n, d.batch, d.ldc, d.strideC, F::MB, F::NB);
  auto kern = bf16x3_fused_kernel<F>;
  static bool attr[kMaxDevices] = {};
  if (cudaError_t e = smem_attr_once(attr, kern, F::SMEM)) return e;
  FusedArgs a;
  a.m = d.m; a.n = d.n; a.k = d.k; a.ldc = d.ldc; a.batch = d.batch;
  a.C0 = (float*)d.C0;
  a.strideC = d.strideC;
  a.alpha = d.alpha_f;
  a.beta = d.beta_f;
  a.a_kcontig = akc;
  a.b_kcontig = bkc;
  a.c_tma = c_tma ? 1 : 0;
  a.err = device_error_flag();
  a.wait_limit = 0;
  const long grid = d.batch < num_sms() ? d.batch : num_sms();
  ProfScope prof("bf16x3_fused", st);
  kern<<<(unsigned)grid, kFusedThreads, F::SMEM, st>>>(ta, tb, tc, a);
  note_launch();
  return cudaGetLastError();
}

}  // namespace

bool bf16x3_small_fits(const BatchDesc& d) {
  if (d.m < 1 || d.n < 1 || d.k < 1 || d.m > 128 || d.n > 128 || d.batch < 1 || d.batch >= (1L << 31) ||
      d.k >= (1L << 31))
    return false;
  // equally spaced instances, rows and instances 16-byte aligned (tensor maps)
  if (!d.A0 || !d.B0 || !d.C0) return false;
  if (d.batch > 1 && (d.strideA <= 0 || d.strideB <= 0 || d.strideC <= 0)) return false;
  if ((uintptr_t)d.A0 % 16 || (uintptr_t)d.B0 % 16 || (uintptr_t)d.C0 % 4) return false;
  if (d.lda % 4 || d.ldb % 4 || (d.batch > 1 && (d.strideA % 16 || d.strideB % 16 || d.strideC % 4))) return false;
  return true;
}

cudaError_t launch_bf16x3_small(const BatchDesc& d, cudaStream_t st) {
  if (!bf16x3_small_fits(d)) return cudaErrorNotSupported;
  // stages: three fp32 and two BF16 where they fit, fewer for the larger tiles
  if (d.m <= 64) {
    if (d.n <= 64) return launch_fused<Fused<64, 64, 3, 2, 2>>(d, st);
    return launch_fused<Fused<64, 128, 2, 1, 2>>(d, st);
  }
  if (d.n <= 64) return launch_fused<Fused<128, 64, 2, 1, 2>>(d, st);
  return launch_fused<Fused<128, 128, 2, 1, 0>>(d, st);
}

}  // namespace ssb
