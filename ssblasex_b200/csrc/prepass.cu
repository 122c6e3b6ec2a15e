// Operand pre-passes for the tensor-core paths (HBM-bound): each reads op(X) of every instance
// through the caller's pointer array -- any transpose, any leading dimension -- and writes
// K-major "planes" [instance][plane][rows][Kp] that the GEMM kernel stages with TMA.
//
//   pack_i8      one plane: the int8 values themselves (int8 row, layouts other than TN)
//   split_bf16   two planes: hi = bf16(x), lo = bf16(x - hi) of an fp32 value
//   ozaki_slice  S planes of balanced int8 digits of an fp64 value under a per-row power-of-two
//                exponent, plus that exponent (Ozaki scheme):
//                  e   = exponent with max_k |x[r,k]| < 2^e  (0 for an all-zero row)
//                  X   = rint(x * 2^(8S-2-e))            |X| < 2^(8S-2)
//                  X   = sum_p d_p 256^(S-1-p),  d_p in [-128,127] (low digits balanced), |d_0| <= 64
//                so x ~= 2^(e+2-8S) * sum_p d_p 256^(S-1-p).
//
// "Rows" are the rows of op(A) (m of them) or the columns of op(B) (n of them); K runs along
// each row. The reference's packers play the same role for its SVE microkernel
// (src/include/ACopy/Xgemm_ncopy_sve_v4.hpp, src/include/BCopy/Xgemm_ncopy_sve_1.hpp), but they
// run per K block inside the tile loop; here each operand is converted once per call.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "internal.h"
#include "prepass.h"

namespace ssb {
namespace {

constexpr int RT = 32;   // rows per tile
constexpr int KT = 64;   // k per tile
constexpr int NTH = 256;

// Loads the RT x KT tile at (row0, k0) of one instance into smem (zero outside the matrix).
// kcontig: element (r, k) is X[r*ld + k]; else X[r + k*ld].
template <typename T>
__device__ __forceinline__ void load_tile(T (&tile)[RT][KT + 1], const T* __restrict__ X, long rows, long K,
                                          long ld, bool kcontig, long row0, long k0) {
  constexpr int PER = RT * KT / NTH;
  T v[PER];   // all loads first, then the smem stores, so the loads overlap
#pragma unroll
  for (int e = 0; e < PER; ++e) {
    const int idx = threadIdx.x + e * NTH;
    int r, kk;
    if (kcontig) { r = idx / KT; kk = idx % KT; }
    else { kk = idx / RT; r = idx % RT; }
    const long gr = row0 + r, gk = k0 + kk;
    v[e] = (gr < rows && gk < K) ? __ldg(kcontig ? X + gr * ld + gk : X + gr + gk * ld) : T(0);
  }
#pragma unroll
  for (int e = 0; e < PER; ++e) {
    const int idx = threadIdx.x + e * NTH;
    int r, kk;
    if (kcontig) { r = idx / KT; kk = idx % KT; }
    else { kk = idx / RT; r = idx % RT; }
    tile[r][kk] = v[e];
  }
}

__global__ void __launch_bounds__(NTH) pack_i8_kernel(PlaneArgs a) {
  __shared__ int8_t tile[RT][KT + 1];
  const long b = blockIdx.y;
  const long row0 = (long)blockIdx.x * RT;
  const int8_t* X = (const int8_t*)a.X[b];
  int8_t* out = (int8_t*)a.out + b * a.batch_stride;
  for (long k0 = 0; k0 < a.K; k0 += KT) {
    load_tile<int8_t>(tile, X, a.rows, a.K, a.ld, a.kcontig, row0, k0);
    __syncthreads();
    // 32 rows x 16 groups of 4 k -> 512 items, 4-byte stores
    for (int it = threadIdx.x; it < RT * (KT / 4); it += NTH) {
      const int r = it / (KT / 4), g = it % (KT / 4);
      const long gr = row0 + r, gk = k0 + 4 * g;
      if (gr < a.rows && gk < a.Kp) {
        uint32_t w = (uint32_t)(uint8_t)tile[r][4 * g] | ((uint32_t)(uint8_t)tile[r][4 * g + 1] << 8) |
                     ((uint32_t)(uint8_t)tile[r][4 * g + 2] << 16) | ((uint32_t)(uint8_t)tile[r][4 * g + 3] << 24);
        *(uint32_t*)(out + gr * a.Kp + gk) = w;
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(NTH) split_bf16_kernel(PlaneArgs a) {
  __shared__ float tile[RT][KT + 1];
  const long b = blockIdx.y;
  const long row0 = (long)blockIdx.x * RT;
  const float* X = (const float*)a.X[b];
  __nv_bfloat16* hi = (__nv_bfloat16*)((int8_t*)a.out + b * a.batch_stride);
  __nv_bfloat16* lo = hi + a.plane_stride / 2;
  for (long k0 = 0; k0 < a.K; k0 += KT) {
    load_tile<float>(tile, X, a.rows, a.K, a.ld, a.kcontig, row0, k0);
    __syncthreads();
    for (int it = threadIdx.x; it < RT * (KT / 2); it += NTH) {
      const int r = it / (KT / 2), g = it % (KT / 2);
      const long gr = row0 + r, gk = k0 + 2 * g;
      if (gr < a.rows && gk < a.Kp) {
        const float x0 = tile[r][2 * g], x1 = tile[r][2 * g + 1];
        const __nv_bfloat16 h0 = __float2bfloat16_rn(x0), h1 = __float2bfloat16_rn(x1);
        const __nv_bfloat16 l0 = __float2bfloat16_rn(x0 - __bfloat162float(h0));
        const __nv_bfloat16 l1 = __float2bfloat16_rn(x1 - __bfloat162float(h1));
        __nv_bfloat162 hv, lv;
        hv.x = h0; hv.y = h1; lv.x = l0; lv.y = l1;
        *(__nv_bfloat162*)(hi + gr * a.Kp + gk) = hv;
        *(__nv_bfloat162*)(lo + gr * a.Kp + gk) = lv;
      }
    }
    __syncthreads();
  }
}

// Ozaki slicing. With Y = X + 0x80..80 (128 added to each of the S-1 low bytes), the balanced
// base-256 digits of X are: d_p = byte_{S-1-p}(Y) - 128 for p >= 1 (that is, the byte with its
// top bit flipped, read as int8), and d_0 = byte_{S-1}(Y) read as int8 -- the carries of the
// digit-by-digit recurrence d = ((X + 128) mod 256) - 128, X <- (X - d) / 256 are exactly the
// carries of the single addition.
constexpr int ORT = 32;    // rows per work item
constexpr int OKT = 128;   // k per smem tile

template <int S>
__global__ void __launch_bounds__(NTH, 2) ozaki_slice_kernel(PlaneArgs a, int32_t* __restrict__ exps) {
  __shared__ double tile[ORT][OKT + 1];
  __shared__ double rmax[ORT];
  __shared__ double rscale[ORT][2];
  const long blocks_per_inst = (a.rows + ORT - 1) / ORT;
  const long total = blocks_per_inst * a.batch;
  unsigned long long bias = 0;
#pragma unroll
  for (int j = 0; j < S - 1; ++j) bias |= 0x80ull << (8 * j);

  // persistent loop: ~2 work items per SM in flight keeps both passes of an item inside L2
  for (long w = blockIdx.x; w < total; w += gridDim.x) {
    const long b = w / blocks_per_inst;
    const long row0 = (w % blocks_per_inst) * ORT;
    const double* X = (const double*)a.X[b];
    int8_t* out = (int8_t*)a.out + b * a.batch_stride;
    if (threadIdx.x < ORT) rmax[threadIdx.x] = 0.0;
    __syncthreads();
    // Loads the ORT x OKT tile at k0 into smem: all loads are issued before any smem store so
    // that they are in flight together (a store to smem between them would serialise them).
    auto load_tile = [&](long k0, bool absval) {
      constexpr int PER = ORT * OKT / NTH;
      double v[PER];
#pragma unroll
      for (int e = 0; e < PER; ++e) {
        const int idx = threadIdx.x + e * NTH;
        int r, kk;
        if (a.kcontig) { r = idx / OKT; kk = idx % OKT; }
        else { kk = idx / ORT; r = idx % ORT; }
        const long gr = row0 + r, gk = k0 + kk;
        v[e] = (gr < a.rows && gk < a.K) ? __ldg(a.kcontig ? X + gr * a.ld + gk : X + gr + gk * a.ld) : 0.0;
      }
#pragma unroll
      for (int e = 0; e < PER; ++e) {
        const int idx = threadIdx.x + e * NTH;
        int r, kk;
        if (a.kcontig) { r = idx / OKT; kk = idx % OKT; }
        else { kk = idx / ORT; r = idx % ORT; }
        tile[r][kk] = absval ? fabs(v[e]) : v[e];
      }
    };
    // pass 1: row maxima of |x|
    for (long k0 = 0; k0 < a.K; k0 += OKT) {
      load_tile(k0, true);
      __syncthreads();
      {
        const int r = threadIdx.x / 8, part = threadIdx.x % 8;   // 8 threads per row
        double mx = 0.0;
#pragma unroll
        for (int j = 0; j < OKT / 8; ++j) mx = fmax(mx, tile[r][part * (OKT / 8) + j]);
#pragma unroll
        for (int off = 4; off >= 1; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        if (part == 0) rmax[r] = fmax(rmax[r], mx);
      }
      __syncthreads();
    }
    if (threadIdx.x < ORT) {
      int e = 0;
      if (rmax[threadIdx.x] > 0.0) frexp(rmax[threadIdx.x], &e);
      const long gr = row0 + threadIdx.x;
      if (gr < a.rows) exps[b * a.rows + gr] = e;
      // x * 2^(8S-2-e) as two exact power-of-two factors (each within the double range)
      const int sh = 8 * S - 2 - e;
      const int h1 = sh / 2;
      rscale[threadIdx.x][0] = ldexp(1.0, h1);
      rscale[threadIdx.x][1] = ldexp(1.0, sh - h1);
    }
    __syncthreads();
    // pass 2: digits (this item's rows were just read, so this pass is served from L2)
    for (long k0 = 0; k0 < a.K; k0 += OKT) {
      load_tile(k0, false);
      __syncthreads();
#pragma unroll
      for (int it0 = 0; it0 < ORT * (OKT / 4) / NTH; ++it0) {
        const int it = threadIdx.x + it0 * NTH;
        const int r = it / (OKT / 4), g = it % (OKT / 4);
        const long gr = row0 + r, gk = k0 + 4 * g;
        if (gr < a.rows && gk < a.Kp) {
          const double s0 = rscale[r][0], s1 = rscale[r][1];
          uint32_t lo[4], hi[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const unsigned long long Y = (unsigned long long)__double2ll_rn(tile[r][4 * g + j] * s0 * s1) + bias;
            lo[j] = (uint32_t)Y;
            hi[j] = (uint32_t)(Y >> 32);
          }
#pragma unroll
          for (int p = 0; p < S; ++p) {
            const int byte = S - 1 - p;
            const uint32_t flip = (p == 0) ? 0u : 0x80808080u;
            uint32_t wv = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const uint32_t src = byte < 4 ? (lo[j] >> (8 * byte)) : (hi[j] >> (8 * (byte - 4)));
              wv |= (src & 255u) << (8 * j);
            }
            *(uint32_t*)(out + p * a.plane_stride + gr * a.Kp + gk) = wv ^ flip;
          }
        }
      }
      __syncthreads();
    }
  }
}

dim3 grid_of(const PlaneArgs& a) {
  return dim3((unsigned)((a.rows + RT - 1) / RT), (unsigned)a.batch);
}

}  // namespace

cudaError_t launch_pack_i8(const PlaneArgs& a, cudaStream_t st) {
  ProfScope prof("pack_i8", st);
  pack_i8_kernel<<<grid_of(a), NTH, 0, st>>>(a);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_split_bf16(const PlaneArgs& a, cudaStream_t st) {
  ProfScope prof("split_bf16", st);
  split_bf16_kernel<<<grid_of(a), NTH, 0, st>>>(a);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_ozaki_slice(const PlaneArgs& a, int slices, int32_t* exps, cudaStream_t st) {
  ProfScope prof("ozaki_slice", st);
  const long items = (a.rows + ORT - 1) / ORT * a.batch;
  const unsigned grid = (unsigned)(items < 2L * num_sms() ? items : 2L * num_sms());
  switch (slices) {
    case 3: ozaki_slice_kernel<3><<<grid, NTH, 0, st>>>(a, exps); break;
    case 4: ozaki_slice_kernel<4><<<grid, NTH, 0, st>>>(a, exps); break;
    case 5: ozaki_slice_kernel<5><<<grid, NTH, 0, st>>>(a, exps); break;
    case 6: ozaki_slice_kernel<6><<<grid, NTH, 0, st>>>(a, exps); break;
    case 7: ozaki_slice_kernel<7><<<grid, NTH, 0, st>>>(a, exps); break;
    case 8: ozaki_slice_kernel<8><<<grid, NTH, 0, st>>>(a, exps); break;
    default: return cudaErrorInvalidValue;
  }
  note_launch();
  return cudaGetLastError();
}

}  // namespace ssb
