// FP32 batched GEMM as three BF16 products for instances that fit one output tile (m, n <= 128),
// with the hi/lo split done in the kernel: no separate split pass over the operands through HBM.
//
// The reference's fp32 row (src/include/GemmCore/Xgemm_kernel_sve_v4x5_1.hpp, FMLA in fp32) is
// emulated as in the tiled 3xBF16 path: x = hi + lo with hi = bf16(x), lo = bf16(x - hi), and
// C = alpha * (Ahi Bhi + Ahi Blo + Alo Bhi) + beta * C with FP32 accumulation on the tensor cores
// (tcgen05.mma kind::f16, bf16 inputs) -- the same split and the same three products, so the
// results agree with the tiled path to FP32 accumulation order.
//
// Design: persistent CTAs of 256 threads, one instance per item. For each 64-wide K chunk every
// thread loads its share of op(A) and op(B) (coalesced along whichever dimension is contiguous in
// memory), splits each value into hi and lo and stores them into the 128-byte-swizzled K-major
// planes the tensor core reads; the chunk's values for the next chunk (or the next item) are
// already in flight in registers while the MMAs of this one run. One thread issues the 12 MMAs of
// a chunk (3 products x 4 K steps of 16) into a tensor-memory accumulator of 128 lanes x N
// columns; eight warps drain it (lane quarter w % 4, column half w / 4) and apply alpha and beta
// (C read only when beta != 0). Rows m..127 of the A planes are zero from the start; columns past n
// of the B planes likewise. Every wait is bounded and reports through the device error flag.
//
// Measured on 4096 x 64^3 TT: 0.38 ms against 0.156 ms for the split pass plus the tiled GEMM --
// with one instance in flight per CTA the kernel is bound by memory latency (12.5% achieved
// occupancy, 7% of DRAM bandwidth in ncu) -- so it is configuration 2 of the 3xBF16 path, not
// its default.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "internal.h"
#include "ptx.cuh"

namespace ssb {
namespace {

constexpr int kThreads = 256;
constexpr int kKC = 64;                   // K elements per chunk: one 128-byte swizzle span of bf16
constexpr int kPlane = 128 * 128;         // bytes of one 128-row plane
constexpr int kSmem = 4 * kPlane + 1024 + 64;   // A hi, A lo, B hi, B lo; alignment; barrier + TMEM slot

struct SmallArgs {
  long m, n, k, lda, ldb, ldc, batch;
  int a_kcontig, b_kcontig;               // op(A) (op(B)) has K contiguous in memory
  const float* const* A;
  const float* const* B;
  float* const* C;
  float alpha, beta;
  int* err;
};

// byte offset of element (row r, k kk) of a K-major 128-byte-swizzled bf16 plane
__device__ __forceinline__ uint32_t plane_off(int r, int kk) {
  const uint32_t chunk = (uint32_t)(kk >> 3) ^ (uint32_t)(r & 7);
  return (uint32_t)r * 128u + chunk * 16u + (uint32_t)(kk & 7) * 2u;
}

// The values of one operand chunk held by a thread: R rows (R = 32, 64 or 128, the rows the
// instance can have) x 64 k, R * 64 / 256 per thread; element e at (row, kk) given by chunk_coord.
// Coordinates: consecutive threads take consecutive positions along the dimension that is
// contiguous in memory, so the loads coalesce.
template <int R>
__device__ __forceinline__ void chunk_coord(bool kcontig, int e, int& r, int& kk) {
  const int idx = threadIdx.x + e * kThreads;
  if (kcontig) { kk = idx % kKC; r = idx / kKC; }
  else { r = idx % R; kk = idx / R; }
}

template <int R>
__device__ __forceinline__ void load_chunk(float (&v)[R * kKC / kThreads], const float* __restrict__ X, bool kcontig,
                                           long rows, long K, long ld, long k0) {
#pragma unroll
  for (int e = 0; e < R * kKC / kThreads; ++e) {
    int r, kk;
    chunk_coord<R>(kcontig, e, r, kk);
    const long gk = k0 + kk;
    v[e] = (r < rows && gk < K) ? __ldg(kcontig ? X + (long)r * ld + gk : X + r + gk * ld) : 0.0f;
  }
}

template <int R>
__device__ __forceinline__ void store_chunk(const float (&v)[R * kKC / kThreads], uint8_t* hi, uint8_t* lo,
                                            bool kcontig) {
#pragma unroll
  for (int e = 0; e < R * kKC / kThreads; ++e) {
    int r, kk;
    chunk_coord<R>(kcontig, e, r, kk);
    const __nv_bfloat16 h = __float2bfloat16_rn(v[e]);
    const __nv_bfloat16 l = __float2bfloat16_rn(v[e] - __bfloat162float(h));
    const uint32_t o = plane_off(r, kk);
    *(__nv_bfloat16*)(hi + o) = h;
    *(__nv_bfloat16*)(lo + o) = l;
  }
}

// MR: rows of op(A) the instances can have (64 or 128); N: columns of C and rows of op(B) (32, 64
// or 128), also the MMA's N.
// Two CTAs per SM where the operands of a chunk fit the 128 registers that leaves a thread.
template <int MR, int N>
constexpr int min_blocks() { return MR * N <= 64 * 64 || N <= 32 ? 2 : 1; }

template <int MR, int N>
__global__ void __launch_bounds__(kThreads, min_blocks<MR, N>()) bf16x3_small_kernel(const SmallArgs a) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* a_hi = smem;
  uint8_t* a_lo = smem + kPlane;
  uint8_t* b_hi = smem + 2 * kPlane;
  uint8_t* b_lo = smem + 3 * kPlane;
  uint64_t* done = (uint64_t*)(smem + 4 * kPlane);
  uint32_t* tmem_slot = (uint32_t*)(done + 1);
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;

  // zero the planes once: rows past m (n) and K past k stay zero in every chunk that does not
  // write them
  for (int i = threadIdx.x; i < 4 * kPlane / 16; i += kThreads) ((uint4*)smem)[i] = make_uint4(0, 0, 0, 0);
  if (threadIdx.x == 0) {
    ptx::mbar_init(ptx::smem_u32(done), 1);
    ptx::fence_mbar_init();
  }
  if (warp == 0) {
    ptx::tmem_alloc(ptx::smem_u32(tmem_slot), N < 32 ? 32 : N);
    ptx::tmem_relinquish();
  }
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  constexpr uint32_t IDESC = ptx::idesc_bf16(128, N);
  const long kchunks = (a.k + kKC - 1) / kKC;
  uint32_t phase = 0;
  bool ok = true;

  float va[MR * kKC / kThreads], vb[N * kKC / kThreads];
  long item = blockIdx.x;
  long c = 0;                                      // chunk of the current item
  if (item < a.batch) {
    load_chunk<MR>(va, a.A[item], a.a_kcontig, a.m, a.k, a.lda, 0);
    load_chunk<N>(vb, a.B[item], a.b_kcontig, a.n, a.k, a.ldb, 0);
  }
  while (item < a.batch && ok) {
    // the previous chunk's MMAs are done (waited below), so the planes can be overwritten
    store_chunk<MR>(va, a_hi, a_lo, a.a_kcontig);
    store_chunk<N>(vb, b_hi, b_lo, a.b_kcontig);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // generic stores -> tensor core
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const bool last = c + 1 == kchunks;
    if (threadIdx.x == 0) {
      const uint32_t sa[2] = {ptx::smem_u32(a_hi), ptx::smem_u32(a_lo)};
      const uint32_t sb[2] = {ptx::smem_u32(b_hi), ptx::smem_u32(b_lo)};
#pragma unroll
      for (int pq = 0; pq < 3; ++pq) {               // (hi, hi), (hi, lo), (lo, hi)
        const int p = pq == 2 ? 1 : 0, q = pq == 1 ? 1 : 0;
#pragma unroll
        for (int kk = 0; kk < kKC / 16; ++kk)
          ptx::mma_f16(tmem, ptx::smem_desc_kmajor(sa[p] + kk * 32, 128), ptx::smem_desc_kmajor(sb[q] + kk * 32, 128),
                       IDESC, (c > 0 || pq > 0 || kk > 0) ? 1u : 0u);
      }
      ptx::mma_commit(ptx::smem_u32(done));
    }
    // the next chunk (or the next item's first chunk) loads while the MMAs run
    const long next_item = last ? item + gridDim.x : item;
    const long next_c = last ? 0 : c + 1;
    if (next_item < a.batch) {
      load_chunk<MR>(va, a.A[next_item], a.a_kcontig, a.m, a.k, a.lda, next_c * kKC);
      load_chunk<N>(vb, a.B[next_item], a.b_kcontig, a.n, a.k, a.ldb, next_c * kKC);
    }
    // every thread leaves the loop together if the wait gives up (the barriers below stay matched)
    ok = __syncthreads_and(ptx::mbar_poll(ptx::smem_u32(done), phase, a.err, 51) ? 1 : 0) != 0;
    phase ^= 1;
    ptx::tc_fence_after();
    if (last && ok) {
      // epilogue: warp w drains lanes 32 (w % 4) .. +31 (rows), columns [h N/2, (h+1) N/2)
      constexpr int HALF = N / 2;
      const int quarter = warp % 4, h = warp / 4;
      const long row = quarter * 32 + lane;
      float* __restrict__ C = a.C[item];
#pragma unroll
      for (int c0 = 0; c0 < HALF; c0 += 16) {
        uint32_t raw[16];
        ptx::tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(h * HALF + c0), raw);
        ptx::tmem_wait_ld();
        if (row < a.m) {
          // all reads of C first (when beta != 0), then the stores: the reads stay in flight together
          float cv[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const long col = h * HALF + c0 + j;
            cv[j] = (a.beta != 0.0f && col < a.n) ? __ldcs(C + row + col * a.ldc) : 0.0f;
          }
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const long col = h * HALF + c0 + j;
            if (col < a.n) {
              const float t = (a.beta == 0.0f) ? 0.0f : a.beta * cv[j];
              __stcs(C + row + col * a.ldc, fmaf(__uint_as_float(raw[j]), a.alpha, t));
            }
          }
        }
      }
      ptx::tc_fence_before();
      __syncthreads();   // the accumulator is read before the next item's first MMAs overwrite it
    }
    item = next_item;
    c = next_c;
  }
  ptx::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    ptx::tc_fence_after();
    ptx::tmem_dealloc(tmem, N < 32 ? 32 : N);
  }
}

template <int MR, int N>
cudaError_t launch_n(const SmallArgs& a, cudaStream_t st) {
  auto kern = bf16x3_small_kernel<MR, N>;
  static bool attr[kMaxDevices] = {};
  if (cudaError_t e = smem_attr_once(attr, kern, kSmem)) return e;
  static int per_sm_dev[kMaxDevices] = {};
  const int dev = current_device();
  if (dev < 0) return cudaErrorInvalidDevice;
  if (!per_sm_dev[dev]) {
    int v = 0;
    if (cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kern, kThreads, kSmem)) return e;
    per_sm_dev[dev] = v < 1 ? 1 : (v > 3 ? 3 : v);   // at most 3 x 128 tensor-memory columns per SM
  }
  const long cap = (long)per_sm_dev[dev] * num_sms();
  const long grid = a.batch < cap ? a.batch : cap;
  ProfScope prof("bf16x3_small", st);
  kern<<<(unsigned)grid, kThreads, kSmem, st>>>(a);
  note_launch();
  return cudaGetLastError();
}

}  // namespace

bool bf16x3_small_fits(const BatchDesc& d) { return d.m <= 128 && d.n <= 128; }

cudaError_t launch_bf16x3_small(const BatchDesc& d, cudaStream_t st) {
  if (!bf16x3_small_fits(d)) return cudaErrorNotSupported;
  SmallArgs a;
  a.m = d.m; a.n = d.n; a.k = d.k; a.lda = d.lda; a.ldb = d.ldb; a.ldc = d.ldc; a.batch = d.batch;
  a.a_kcontig = d.transa == SSBLAS_OP_T;
  a.b_kcontig = d.transb == SSBLAS_OP_N;
  a.A = (const float* const*)d.A;
  a.B = (const float* const*)d.B;
  a.C = (float* const*)d.C;
  a.alpha = d.alpha_f;
  a.beta = d.beta_f;
  a.err = device_error_flag();
  if (d.m <= 64) {
    if (d.n <= 32) return launch_n<64, 32>(a, st);
    if (d.n <= 64) return launch_n<64, 64>(a, st);
    return launch_n<64, 128>(a, st);
  }
  if (d.n <= 32) return launch_n<128, 32>(a, st);
  if (d.n <= 64) return launch_n<128, 64>(a, st);
  return launch_n<128, 128>(a, st);
}

}  // namespace ssb
