// Plain FP32 batched GEMM (FFMA) with TMA staging, for equally spaced instances whose rows are
// 16-byte aligned: the operand tiles and the C tile reach shared memory by tensor-map copies
// issued from one thread, and C leaves by bulk tensor stores, so the compute warps spend their
// issue slots on FFMA and shared-memory operand loads only.
//
// Semantics are those of the fp32 row in its plain form (reference
// src/include/GemmCore/Xgemm_kernel_sve_v4x5_1.hpp:93-127, FMLA in fp32; C scaled by beta, not read
// when beta == 0: src/include/CScale/Xgemm_scale_kernel.hpp:164-176): every output is the FP32
// sum of the k products, rounded at each step, then alpha * acc + beta * C with one fused
// multiply-add. The summation order is k = 0, 1, ..., k - 1, as in the other FFMA kernels.
//
// Design: work item = (instance, 64 x 64 tile of C); persistent CTAs take items
// blockIdx.x, blockIdx.x + gridDim.x, ... Warps 0-7 compute (256 threads, a 4 x 4 block of the
// tile each); warp 8 lane 0 copies each 64-deep K chunk of op(A) and op(B) into a stage ring, warp 9
// lane 0 each item's C tile (beta != 0) into a tile ring. (Two lanes of one warp would not do: a
// lane spinning on a stage that the compute warps free only after their C tile has landed keeps
// the lane that issues that C copy from being scheduled.) An operand whose K is contiguous in
// memory is copied as two 128-byte-swizzled boxes of 32 k x 64 rows, and a thread reads 4
// consecutive k of one row with one 16-byte load (its rows are tx + 16 i, so the 8 rows a
// quarter-warp reads sit in 8 different 16-byte bank groups); an operand whose rows are
// contiguous is copied as one box of 64 rows x 64 k and a thread reads 4 consecutive rows at one
// k (rows 4 tx + i). The C tile is two swizzled boxes of 32 rows x 64 columns; the compute threads
// write alpha * acc + beta * C over it and thread 0 issues the two bulk stores. Rows and columns
// outside C are zero-filled by the loads and dropped by the stores. Every wait is bounded and
// reports through the device error flag.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "internal.h"
#include "ptx.cuh"

namespace ssb {
namespace {

constexpr int kT = 64;                 // tile rows and columns
constexpr int kKC = 64;                // K per stage
constexpr int kComputeThreads = 256;   // warps 0-7
constexpr int kThreads = kComputeThreads + 64;   // + warp 8 (operands) and warp 9 (C tiles)
constexpr int kOpBytes = kT * kKC * 4; // one operand's chunk (16 KB)
constexpr int kStage = 2 * kOpBytes;
constexpr int kCTile = kT * kT * 4;

template <int ST_, int CST_, int MINB_>
struct TmaCfg {
  static constexpr int ST = ST_, CST = CST_, MINB = MINB_;
  static constexpr int BARS = 128;
  static constexpr int SMEM = 1024 + ST * kStage + CST * kCTile + BARS;
  static_assert((2 * ST + 2 * CST) * 8 <= BARS, "barrier area");
  static_assert(CST >= 2, "a C tile is rewritten only after the store of the item before last");
};

struct TmaArgs {
  long m, n, k, batch;
  uint32_t tiles_m, tiles, total;   // 64 x 64 tiles along m, per instance, and items in all
  float alpha, beta;
  int* err;
};

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
// the bulk stores of all but the newest group have read their shared memory
__device__ __forceinline__ void bulk_wait_read_all_but_one() {
  asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
}
// AND of v over the 256 compute threads (named barrier 1)
__device__ __forceinline__ bool compute_all(bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.and.pred p, 1, 256, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void compute_sync() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

__device__ __forceinline__ float4 lds4(const uint8_t* p) { return *(const float4*)p; }

// byte offset of (row r, k 4q .. 4q + 3) in a K-contiguous chunk: box h = q / 8 of 32 k, rows of
// 128 bytes, 16-byte group (q % 8) ^ (r % 8)
__device__ __forceinline__ uint32_t kmaj(uint32_t r, uint32_t q) {
  return (q >> 3) * 8192u + r * 128u + ((((q & 7u) ^ (r & 7u))) << 4);
}
// byte offset of C(r, c) in the tile: box r / 32 of 32 rows, a 128-byte line per column
__device__ __forceinline__ uint32_t ctile(uint32_t r, uint32_t c) {
  return (r >> 5) * 8192u + c * 128u + (((((r & 31u) >> 2) ^ (c & 7u))) << 4) + (r & 3u) * 4u;
}

template <class F, bool AK, bool BK>
__global__ void __launch_bounds__(kThreads, F::MINB)
sgemm_tma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                 const __grid_constant__ CUtensorMap tmC, const TmaArgs a) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* stages = smem;                               // [ST][A 16 KB | B 16 KB]
  uint8_t* ctiles = smem + F::ST * kStage;              // [CST][16 KB]
  uint64_t* bars = (uint64_t*)(ctiles + F::CST * kCTile);
  uint64_t* f_full = bars;                              // chunk landed (TMA bytes)
  uint64_t* f_empty = f_full + F::ST;                   // chunk read (8 compute warps)
  uint64_t* c_full = f_empty + F::ST;                   // C tile landed (TMA bytes)
  uint64_t* c_empty = c_full + F::CST;                  // C tile stored (store thread)
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  int* err = a.err;
  const bool read_c = a.beta != 0.0f;
  if (threadIdx.x == 0) {
    for (int s = 0; s < F::ST; ++s) {
      ptx::mbar_init(ptx::smem_u32(&f_full[s]), 1);
      ptx::mbar_init(ptx::smem_u32(&f_empty[s]), kComputeThreads / 32);
    }
    for (int s = 0; s < F::CST; ++s) {
      ptx::mbar_init(ptx::smem_u32(&c_full[s]), 1);
      ptx::mbar_init(ptx::smem_u32(&c_empty[s]), 1);
    }
    ptx::fence_mbar_init();
  }
  if (warp == kComputeThreads / 32 && lane == 0) {
    ptx::prefetch_tmap(&tmA);
    ptx::prefetch_tmap(&tmB);
  }
  if (warp == kComputeThreads / 32 + 1 && lane == 0) ptx::prefetch_tmap(&tmC);
  __syncthreads();
  const int nkc = (int)((a.k + kKC - 1) / kKC);

  if (warp == kComputeThreads / 32) {
    // ---------------------------------------------------------------- copies --------------
    if (lane == 0) {
      uint32_t c = 0;
      bool ok = true;
      for (uint32_t w = blockIdx.x; w < a.total && ok; w += gridDim.x) {
        const uint32_t b = w / a.tiles, t = w - b * a.tiles;
        const int m0 = (int)((t % a.tiles_m) * kT), n0 = (int)((t / a.tiles_m) * kT);
        for (int kc = 0; kc < nkc; ++kc, ++c) {
          const uint32_t s = c % F::ST;
          if (!ptx::mbar_wait(ptx::smem_u32(&f_empty[s]), ((c / F::ST) & 1u) ^ 1u, err, 81)) {
            ok = false;
            break;
          }
          const uint32_t bar = ptx::smem_u32(&f_full[s]);
          const uint32_t sa = ptx::smem_u32(stages + (size_t)s * kStage), sb = sa + kOpBytes;
          ptx::mbar_arrive_expect_tx(bar, kStage);
          const int k0 = kc * kKC;
          if (AK) {
            tma_load_3d(sa, &tmA, bar, k0, m0, (int)b);
            tma_load_3d(sa + 8192, &tmA, bar, k0 + 32, m0, (int)b);
          } else {
            tma_load_3d(sa, &tmA, bar, m0, k0, (int)b);
          }
          if (BK) {
            tma_load_3d(sb, &tmB, bar, k0, n0, (int)b);
            tma_load_3d(sb + 8192, &tmB, bar, k0 + 32, n0, (int)b);
          } else {
            tma_load_3d(sb, &tmB, bar, n0, k0, (int)b);
          }
        }
      }
      // no copy may still be landing in shared memory when the CTA exits
      for (uint32_t j = (c > (uint32_t)F::ST ? c - F::ST : 0); j < c; ++j)
        ptx::mbar_wait(ptx::smem_u32(&f_full[j % F::ST]), (j / F::ST) & 1u, err, 82);
    }
  } else if (warp == kComputeThreads / 32 + 1) {
    if (lane == 0 && read_c) {
      uint32_t i = 0;
      for (uint32_t w = blockIdx.x; w < a.total; w += gridDim.x, ++i) {
        const uint32_t b = w / a.tiles, t = w - b * a.tiles;
        const int m0 = (int)((t % a.tiles_m) * kT), n0 = (int)((t / a.tiles_m) * kT);
        const uint32_t cs = i % F::CST;
        if (!ptx::mbar_wait(ptx::smem_u32(&c_empty[cs]), ((i / F::CST) & 1u) ^ 1u, err, 83)) break;
        const uint32_t bar = ptx::smem_u32(&c_full[cs]);
        const uint32_t dst = ptx::smem_u32(ctiles + (size_t)cs * kCTile);
        ptx::mbar_arrive_expect_tx(bar, kCTile);
        tma_load_3d(dst, &tmC, bar, m0, n0, (int)b);
        tma_load_3d(dst + 8192, &tmC, bar, m0 + 32, n0, (int)b);
      }
      for (uint32_t j = (i > (uint32_t)F::CST ? i - F::CST : 0); j < i; ++j)
        ptx::mbar_wait(ptx::smem_u32(&c_full[j % F::CST]), (j / F::CST) & 1u, err, 84);
    }
  } else {
    // ---------------------------------------------------------------- compute -------------
    const int tx = (warp % 4) * 4 + lane % 4, ty = (warp / 4) * 8 + lane / 4;   // 16 x 16 threads
    uint32_t c = 0, i = 0;
    for (uint32_t w = blockIdx.x; w < a.total; w += gridDim.x, ++i) {
      const uint32_t b = w / a.tiles, t = w - b * a.tiles;
      const int m0 = (int)((t % a.tiles_m) * kT), n0 = (int)((t / a.tiles_m) * kT);
      float acc[4][4];
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) acc[x][y] = 0.0f;
      bool ok = true;
      for (int kc = 0; kc < nkc; ++kc, ++c) {
        const uint32_t s = c % F::ST;
        ok = ptx::mbar_wait(ptx::smem_u32(&f_full[s]), (c / F::ST) & 1u, err, 85);
        if (!__all_sync(0xffffffffu, ok)) {
          ok = false;
          break;
        }
        const uint8_t* sa = stages + (size_t)s * kStage;
        const uint8_t* sb = sa + kOpBytes;
#pragma unroll 4
        for (int q = 0; q < kKC / 4; ++q) {   // 4 k per step
          float av[4][4], bv[4][4];           // [row i][k], [column j][k]
          if (AK) {
#pragma unroll
            for (int x = 0; x < 4; ++x) {
              const float4 v = lds4(sa + kmaj((uint32_t)(tx + 16 * x), (uint32_t)q));
              av[x][0] = v.x; av[x][1] = v.y; av[x][2] = v.z; av[x][3] = v.w;
            }
          } else {
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
              const float4 v = lds4(sa + (4 * q + kk) * 256 + tx * 16);
              av[0][kk] = v.x; av[1][kk] = v.y; av[2][kk] = v.z; av[3][kk] = v.w;
            }
          }
          if (BK) {
#pragma unroll
            for (int y = 0; y < 4; ++y) {
              const float4 v = lds4(sb + kmaj((uint32_t)(ty + 16 * y), (uint32_t)q));
              bv[y][0] = v.x; bv[y][1] = v.y; bv[y][2] = v.z; bv[y][3] = v.w;
            }
          } else {
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
              const float4 v = lds4(sb + (4 * q + kk) * 256 + ty * 16);
              bv[0][kk] = v.x; bv[1][kk] = v.y; bv[2][kk] = v.z; bv[3][kk] = v.w;
            }
          }
#pragma unroll
          for (int kk = 0; kk < 4; ++kk)
#pragma unroll
            for (int x = 0; x < 4; ++x)
#pragma unroll
              for (int y = 0; y < 4; ++y) acc[x][y] = fmaf(av[x][kk], bv[y][kk], acc[x][y]);
        }
        __syncwarp();
        if (lane == 0) ptx::mbar_arrive(ptx::smem_u32(&f_empty[s]));
      }
      // ------------------------------------------------------------ epilogue ----------------
      const uint32_t cs = i % F::CST;
      if (read_c && ok) ok = ptx::mbar_wait(ptx::smem_u32(&c_full[cs]), (i / F::CST) & 1u, err, 86);
      // the compute threads leave together if any wait gave up: they share the named barrier.
      // The tile's previous store (item i - CST, CST >= 2) has read it: thread 0 reaches this
      // barrier only after waiting for every store but its newest (item i - 1); with beta != 0
      // the load of this item's C came after that read as well (c_empty)
      if (!compute_all(ok)) break;
      uint8_t* tile = ctiles + (size_t)cs * kCTile;
#pragma unroll
      for (int y = 0; y < 4; ++y) {
        const uint32_t col = BK ? (uint32_t)(ty + 16 * y) : (uint32_t)(4 * ty + y);
        if (AK) {
#pragma unroll
          for (int x = 0; x < 4; ++x) {
            float* e = (float*)(tile + ctile((uint32_t)(tx + 16 * x), col));
            *e = fmaf(acc[x][y], a.alpha, read_c ? a.beta * *e : 0.0f);
          }
        } else {
          float4* e = (float4*)(tile + ctile((uint32_t)(4 * tx), col));
          float4 v = read_c ? *e : make_float4(0.f, 0.f, 0.f, 0.f);
          v.x = fmaf(acc[0][y], a.alpha, read_c ? a.beta * v.x : 0.0f);
          v.y = fmaf(acc[1][y], a.alpha, read_c ? a.beta * v.y : 0.0f);
          v.z = fmaf(acc[2][y], a.alpha, read_c ? a.beta * v.z : 0.0f);
          v.w = fmaf(acc[3][y], a.alpha, read_c ? a.beta * v.w : 0.0f);
          *e = v;
        }
      }
      ptx::fence_proxy_async_smem();   // the tile's generic writes -> the bulk stores
      compute_sync();
      if (threadIdx.x == 0) {
        const uint32_t src = ptx::smem_u32(tile);
        ptx::tma_store_3d(&tmC, src, m0, n0, (int)b);
        ptx::tma_store_3d(&tmC, src + 8192, m0 + 32, n0, (int)b);
        ptx::bulk_commit();
        // the previous item's stores have read their tile: its slot may be loaded again
        bulk_wait_read_all_but_one();
        if (read_c && i > 0) ptx::mbar_arrive(ptx::smem_u32(&c_empty[(i - 1) % F::CST]));
      }
    }
    if (threadIdx.x == 0) ptx::bulk_wait_all();
  }
}

// 3-D fp32 map {inner, outer, batch} with box {box_in, box_out, 1}; zero fill outside.
bool map3(CUtensorMap* map, const void* base, long inner, long outer, long batch, long ld, long stride_bytes,
          int box_in, int box_out, int swz) {
  const long dims[3] = {inner, outer, batch};
  const long strides[2] = {ld * 4, batch > 1 ? stride_bytes : ((ld * outer * 4 + 15) / 16) * 16};
  const int box[3] = {box_in, box_out, 1};
  return make_tiled_map(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, swz);
}

template <class F, bool AK, bool BK>
cudaError_t launch_cfg(const CUtensorMap& ta, const CUtensorMap& tb, const CUtensorMap& tc, const TmaArgs& a,
                       cudaStream_t st) {
  auto kern = sgemm_tma_kernel<F, AK, BK>;
  static bool attr[kMaxDevices] = {};
  if (cudaError_t e = smem_attr_once(attr, kern, F::SMEM)) return e;
  const long slots = (long)num_sms() * F::MINB;
  const long grid = (long)a.total < slots ? (long)a.total : slots;
  kern<<<(unsigned)grid, kThreads, F::SMEM, st>>>(ta, tb, tc, a);
  return cudaGetLastError();
}

template <class F>
cudaError_t launch_layout(const CUtensorMap& ta, const CUtensorMap& tb, const CUtensorMap& tc, const TmaArgs& a,
                          bool ak, bool bk, cudaStream_t st) {
  if (ak && bk) return launch_cfg<F, true, true>(ta, tb, tc, a, st);
  if (ak) return launch_cfg<F, true, false>(ta, tb, tc, a, st);
  if (bk) return launch_cfg<F, false, true>(ta, tb, tc, a, st);
  return launch_cfg<F, false, false>(ta, tb, tc, a, st);
}

}  // namespace

bool sgemm_tma_fits(const BatchDesc& d) {
  if (d.m < 1 || d.n < 1 || d.k < 1 || d.batch < 1 || d.m >= (1L << 30) || d.n >= (1L << 30) ||
      d.k >= (1L << 30))
    return false;
  const long tiles = ((d.m + kT - 1) / kT) * ((d.n + kT - 1) / kT);
  if (tiles * d.batch >= (1L << 31)) return false;
  if (!d.A0 || !d.B0 || !d.C0) return false;
  if (d.batch > 1 && (d.strideA <= 0 || d.strideB <= 0 || d.strideC <= 0)) return false;
  if ((uintptr_t)d.A0 % 16 || (uintptr_t)d.B0 % 16 || (uintptr_t)d.C0 % 16) return false;
  if (d.lda % 4 || d.ldb % 4 || d.ldc % 4) return false;
  if (d.batch > 1 && (d.strideA % 16 || d.strideB % 16 || d.strideC % 16)) return false;
  return true;
}

// variant 0: two stages and two C tiles, two CTAs per SM; 1: three and three, one CTA per SM
cudaError_t launch_sgemm_tma(const BatchDesc& d, int variant, cudaStream_t st) {
  if (!sgemm_tma_fits(d)) return cudaErrorNotSupported;
  const bool ak = d.transa == SSBLAS_OP_T, bk = d.transb == SSBLAS_OP_N;   // K contiguous
  CUtensorMap ta, tb, tc;
  const bool ok_a = ak ? map3(&ta, d.A0, d.k, d.m, d.batch, d.lda, d.strideA, 32, kT, 128)
                       : map3(&ta, d.A0, d.m, d.k, d.batch, d.lda, d.strideA, kT, kKC, 0);
  const bool ok_b = bk ? map3(&tb, d.B0, d.k, d.n, d.batch, d.ldb, d.strideB, 32, kT, 128)
                       : map3(&tb, d.B0, d.n, d.k, d.batch, d.ldb, d.strideB, kT, kKC, 0);
  const bool ok_c = map3(&tc, d.C0, d.m, d.n, d.batch, d.ldc, d.strideC, 32, kT, 128);
  if (!ok_a || !ok_b || !ok_c) return cudaErrorNotSupported;
  TmaArgs a;
  a.m = d.m; a.n = d.n; a.k = d.k; a.batch = d.batch;
  a.tiles_m = (uint32_t)((d.m + kT - 1) / kT);
  a.tiles = a.tiles_m * (uint32_t)((d.n + kT - 1) / kT);
  a.total = a.tiles * (uint32_t)d.batch;
  a.alpha = d.alpha_f;
  a.beta = d.beta_f;
  a.err = device_error_flag();
  ProfScope prof("sgemm_tma", st);
  cudaError_t e = variant == 1 ? launch_layout<TmaCfg<3, 3, 1>>(ta, tb, tc, a, ak, bk, st)
                               : launch_layout<TmaCfg<2, 2, 2>>(ta, tb, tc, a, ak, bk, st);
  note_launch();
  return e;
}

}  // namespace ssb
