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
#pragma unroll
  for (int e = 0; e < RT * KT / NTH; ++e) {
    const int idx = threadIdx.x + e * NTH;
    int r, kk;
    if (kcontig) { r = idx / KT; kk = idx % KT; }
    else { kk = idx / RT; r = idx % RT; }
    const long gr = row0 + r, gk = k0 + kk;
    T v = T(0);
    if (gr < rows && gk < K) v = kcontig ? X[gr * ld + gk] : X[gr + gk * ld];
    tile[r][kk] = v;
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

// Balanced base-256 digits of X (|X| < 2^(8S-2)), most significant first.
template <int S>
__device__ __forceinline__ void digits(long long X, int8_t (&d)[S]) {
#pragma unroll
  for (int p = S - 1; p >= 1; --p) {
    const long long lo = ((X + 128) & 255) - 128;
    d[p] = (int8_t)lo;
    X = (X - lo) >> 8;
  }
  d[0] = (int8_t)X;
}

template <int S>
__global__ void __launch_bounds__(NTH) ozaki_slice_kernel(PlaneArgs a, int32_t* __restrict__ exps) {
  __shared__ double tile[RT][KT + 1];
  __shared__ double rmax[RT];
  __shared__ int rexp[RT];
  const long b = blockIdx.y;
  const long row0 = (long)blockIdx.x * RT;
  const double* X = (const double*)a.X[b];
  int8_t* out = (int8_t*)a.out + b * a.batch_stride;
  if (threadIdx.x < RT) rmax[threadIdx.x] = 0.0;
  __syncthreads();
  // pass 1: row maxima of |x|
  for (long k0 = 0; k0 < a.K; k0 += KT) {
    load_tile<double>(tile, X, a.rows, a.K, a.ld, a.kcontig, row0, k0);
    __syncthreads();
    {
      const int r = threadIdx.x / 8, part = threadIdx.x % 8;   // 8 threads per row
      double mx = 0.0;
#pragma unroll
      for (int j = 0; j < KT / 8; ++j) mx = fmax(mx, fabs(tile[r][part * (KT / 8) + j]));
#pragma unroll
      for (int off = 4; off >= 1; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
      if (part == 0) rmax[r] = fmax(rmax[r], mx);
    }
    __syncthreads();
  }
  if (threadIdx.x < RT) {
    int e = 0;
    if (rmax[threadIdx.x] > 0.0) frexp(rmax[threadIdx.x], &e);
    rexp[threadIdx.x] = e;
    const long gr = row0 + threadIdx.x;
    if (gr < a.rows) exps[b * a.rows + gr] = e;
  }
  __syncthreads();
  // pass 2: digits (the rows were just read, so this pass is served from L2)
  for (long k0 = 0; k0 < a.K; k0 += KT) {
    load_tile<double>(tile, X, a.rows, a.K, a.ld, a.kcontig, row0, k0);
    __syncthreads();
    for (int it = threadIdx.x; it < RT * (KT / 4); it += NTH) {
      const int r = it / (KT / 4), g = it % (KT / 4);
      const long gr = row0 + r, gk = k0 + 4 * g;
      if (gr < a.rows && gk < a.Kp) {
        const int sh = 8 * S - 2 - rexp[r];
        int8_t dg[4][S];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const long long Xi = __double2ll_rn(scalbn(tile[r][4 * g + j], sh));
          digits<S>(Xi, dg[j]);
        }
#pragma unroll
        for (int p = 0; p < S; ++p) {
          const uint32_t w = (uint32_t)(uint8_t)dg[0][p] | ((uint32_t)(uint8_t)dg[1][p] << 8) |
                             ((uint32_t)(uint8_t)dg[2][p] << 16) | ((uint32_t)(uint8_t)dg[3][p] << 24);
          *(uint32_t*)(out + p * a.plane_stride + gr * a.Kp + gk) = w;
        }
      }
    }
    __syncthreads();
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
  switch (slices) {
    case 3: ozaki_slice_kernel<3><<<grid_of(a), NTH, 0, st>>>(a, exps); break;
    case 4: ozaki_slice_kernel<4><<<grid_of(a), NTH, 0, st>>>(a, exps); break;
    case 5: ozaki_slice_kernel<5><<<grid_of(a), NTH, 0, st>>>(a, exps); break;
    case 6: ozaki_slice_kernel<6><<<grid_of(a), NTH, 0, st>>>(a, exps); break;
    case 7: ozaki_slice_kernel<7><<<grid_of(a), NTH, 0, st>>>(a, exps); break;
    case 8: ozaki_slice_kernel<8><<<grid_of(a), NTH, 0, st>>>(a, exps); break;
    default: return cudaErrorInvalidValue;
  }
  note_launch();
  return cudaGetLastError();
}

}  // namespace ssb
