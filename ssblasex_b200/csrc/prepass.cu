// Operand pre-passes for the tensor-core paths (HBM-bound): each reads op(X) of every instance
// through the caller's pointer array -- any transpose, any leading dimension -- and writes
// K-major "planes" [instance][plane][rows][Kp] that the GEMM kernel stages with TMA.
//
//   pack_i8      one plane: the int8 values themselves (int8 row, layouts other than TN)
//   split_bf16   two planes: hi = bf16(x), lo = bf16(x - hi) of an fp32 value (both operands of a
//                call in one launch)
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
//
// Memory plan: every thread issues all of its global loads for a tile back to back (coalesced
// along whichever of rows / k is contiguous), converts in registers, transposes the output bytes
// through shared memory, and writes 16-byte vectors along K. Several CTAs per SM keep enough
// loads in flight to run at HBM speed.
//
// Ozaki slicing has three forms:
//   K <= 2048   ozaki_cluster_kernel: one pass, persistent thread-block clusters. The ceil(K/256)
//               CTAs of a cluster share 32 rows, exchange their partial row maxima through
//               distributed shared memory and write the digits; tiles arrive by TMA (equally
//               spaced instances) or cp.async two items ahead, digit rows leave as 16-byte stores.
//               Each operand is read once.
//   K > 2048    ozaki_rowmax_kernel (row maxima of |x| per 32 rows x 256 k part, combined by
//               atomicMax) then ozaki_cluster_kernel in its BITS form (clusters of one CTA,
//               persistent over 16 rows x 512 k slabs, exponents from the maxima); or (the
//               allocation-free entry point, which has no room for the maxima)
//               ozaki_rowexp_kernel (row exponents) then ozaki_digits_kernel (one CTA per
//               32 rows x 128 k chunk) when there are enough rows to fill the GPU, else
//               ozaki_slice_kernel (both passes inside one CTA per 32 rows).
// All forms pack the 4 digits of 4 consecutive k into one word per plane with a 4 x 4 byte
// transpose (byte_perm), and produce identical planes.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>

#include "internal.h"
#include "ozaki_digits.cuh"
#include "prepass.h"
#include "ptx.cuh"

namespace ssb {
namespace {

constexpr int RT = 32;    // rows per tile
constexpr int KT = 64;    // k per tile
constexpr int NTH = 256;
constexpr int PER = RT * KT / NTH;   // elements per thread per tile (8)
constexpr int OPITCH = 68;           // smem bytes per staged output row (17 words: conflict-free)

// element e of this thread's share of the tile: (row r, column kk)
__device__ __forceinline__ void tile_coord(bool kcontig, int e, int& r, int& kk) {
  if (kcontig) {           // 8 threads per row, 8 consecutive k each
    r = threadIdx.x / 8;
    kk = (threadIdx.x % 8) * 8 + e;
  } else {                 // a warp covers 32 consecutive rows at one k
    r = threadIdx.x % 32;
    kk = threadIdx.x / 32 + 8 * e;
  }
}

template <typename T>
__device__ __forceinline__ void load_regs(T (&v)[PER], const T* __restrict__ X, long rows, long K, long ld,
                                          bool kcontig, long row0, long k0) {
#pragma unroll
  for (int e = 0; e < PER; ++e) {
    int r, kk;
    tile_coord(kcontig, e, r, kk);
    const long gr = row0 + r, gk = k0 + kk;
    v[e] = (gr < rows && gk < K) ? __ldg(kcontig ? X + gr * ld + gk : X + gr + gk * ld) : T(0);
  }
}

// Writes staged bytes st[p][r][0..ROWB) (row pitch ROWB + 4) of P planes as 16-byte vectors.
template <int P, int ROWB>
__device__ __forceinline__ void write_rows(const uint8_t* st, uint8_t* out, long plane_stride, long rows,
                                           long Kp_bytes, long row0, long kbyte0) {
  constexpr int SEGS = ROWB / 16;
  for (int it = threadIdx.x; it < P * RT * SEGS; it += NTH) {
    const int p = it / (RT * SEGS), rem = it % (RT * SEGS), r = rem / SEGS, sg = rem % SEGS;
    const long gr = row0 + r, gb = kbyte0 + 16 * sg;
    if (gr < rows && gb < Kp_bytes) {
      const uint32_t* src = (const uint32_t*)(st + (p * RT + r) * (ROWB + 4) + 16 * sg);
      uint4 w = make_uint4(src[0], src[1], src[2], src[3]);
      *(uint4*)(out + p * plane_stride + gr * Kp_bytes + gb) = w;
    }
  }
}

template <int P, int BPE>
__device__ __forceinline__ void write_out(const uint8_t* st, uint8_t* out, long plane_stride, long rows,
                                          long Kp_bytes, long row0, long kbyte0) {
  write_rows<P, KT * BPE>(st, out, plane_stride, rows, Kp_bytes, row0, kbyte0);
}

// int8 -> K-major plane. A CTA takes 128 rows x 128 k of one instance (blocks: k tile fastest,
// then row tile, then instance). K contiguous: already K-major, each thread copies 16-byte row
// segments to the plane's pitch. Rows contiguous (element (r, k) at X[r + k*ld]): each thread
// loads four 4 x 4 byte blocks as 32-bit words -- lane l of a warp takes rows 4l .. 4l+3, so one
// load instruction reads 128 contiguous bytes -- transposes them in registers (byte permutes),
// stages the 4-byte k runs of its rows in shared memory, and the CTA writes 16-byte row segments.
// Positions past K (up to Kp) get zero bytes.
constexpr int PKR = 128, PKK = 128;          // rows and k per CTA
constexpr int PKP = PKK + 4;                 // staged row pitch (bytes)
__global__ void __launch_bounds__(NTH) pack_i8_kernel(PlaneArgs a, long ktiles, long rtiles) {
  __shared__ __align__(16) uint8_t st[PKR * PKP];
  const long blk = blockIdx.x;
  const long kt = blk % ktiles, rt = (blk / ktiles) % rtiles, b = blk / (ktiles * rtiles);
  const long r0 = rt * PKR, k0 = kt * PKK;
  const int8_t* X = (const int8_t*)a.X[b];
  uint8_t* out = (uint8_t*)a.out + b * a.batch_stride;
  const int t = threadIdx.x;
  if (a.kcontig) {
    const bool vec = ((uintptr_t)X % 16) == 0 && a.ld % 16 == 0;
#pragma unroll
    for (int q = 0; q < PKR * PKK / 16 / NTH; ++q) {
      const int id = t + q * NTH, r = id / (PKK / 16), c = id % (PKK / 16);
      const long gr = r0 + r, gk = k0 + 16 * c;
      if (gr >= a.rows || gk >= a.Kp) continue;
      uint4 w = make_uint4(0u, 0u, 0u, 0u);
      const int8_t* src = X + gr * a.ld + gk;
      if (vec && gk + 16 <= a.K) {
        w = __ldg((const uint4*)src);
      } else {
        uint8_t by[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) by[i] = gk + i < a.K ? (uint8_t)__ldg(src + i) : 0;
        memcpy(&w, by, 16);
      }
      *(uint4*)(out + gr * a.Kp + gk) = w;
    }
    return;
  }
  const bool vec = ((uintptr_t)X % 4) == 0 && a.ld % 4 == 0;
  const int rg = t % 32;                       // rows 4 rg .. 4 rg + 3 of the tile
  const long gr = r0 + 4 * rg;
#pragma unroll
  for (int q = 0; q < PKK / 4 / (NTH / 32); ++q) {
    const int kg = t / 32 + (NTH / 32) * q;    // k 4 kg .. 4 kg + 3 of the tile
    uint32_t w[4], o[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const long gk = k0 + 4 * kg + i;
      const int8_t* src = X + gr + gk * a.ld;
      w[i] = 0u;
      if (gk < a.K) {
        if (vec && gr + 4 <= a.rows) {
          w[i] = __ldg((const uint32_t*)src);
        } else {
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (gr + j < a.rows) w[i] |= (uint32_t)(uint8_t)__ldg(src + j) << (8 * j);
        }
      }
    }
    byte_transpose4(w, o);                     // o[j]: k 4 kg .. 4 kg + 3 of row 4 rg + j
#pragma unroll
    for (int j = 0; j < 4; ++j) *(uint32_t*)(st + (4 * rg + j) * PKP + 4 * kg) = o[j];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < PKR * PKK / 16 / NTH; ++q) {
    const int id = t + q * NTH, r = id / (PKK / 16), c = id % (PKK / 16);
    const long gr2 = r0 + r, gk = k0 + 16 * c;
    if (gr2 >= a.rows || gk >= a.Kp) continue;
    const uint32_t* src = (const uint32_t*)(st + r * PKP + 16 * c);
    *(uint4*)(out + gr2 * a.Kp + gk) = make_uint4(src[0], src[1], src[2], src[3]);
  }
}

// Both operands in one launch: work item = (operand, instance, 32 rows, 64 k); each CTA takes
// SPLIT_ITEMS consecutive items and issues all of their loads before converting the first. One
// item per CTA measured best on 4096 x 64^3 (0.081 ms for both operands; 4 items per CTA took
// 0.115 ms: twice the registers, half the resident CTAs).
constexpr int SPLIT_ITEMS = 1;

__global__ void __launch_bounds__(NTH) split_bf16_pair_kernel(PlaneArgs a0, long n0, PlaneArgs a1, long n_items) {
  __shared__ __align__(16) uint8_t st[2 * RT * (2 * KT + 4)];
  float v[SPLIT_ITEMS][PER];
  long item_b[SPLIT_ITEMS], item_row0[SPLIT_ITEMS], item_k0[SPLIT_ITEMS];
  bool item_second[SPLIT_ITEMS];
  const long first = (long)blockIdx.x * SPLIT_ITEMS;
#pragma unroll
  for (int q = 0; q < SPLIT_ITEMS; ++q) {
    const long item = first + q;
    item_second[q] = item >= n0;
    const PlaneArgs& a = item_second[q] ? a1 : a0;
    const long it = item_second[q] ? item - n0 : item;
    const long kch = (a.K + KT - 1) / KT, rbl = (a.rows + RT - 1) / RT;
    item_k0[q] = (it % kch) * KT;
    item_row0[q] = ((it / kch) % rbl) * RT;
    item_b[q] = (it / kch) / rbl;
    if (item < n_items) {
      load_regs<float>(v[q], (const float*)a.X[item_b[q]], a.rows, a.K, a.ld, a.kcontig, item_row0[q], item_k0[q]);
    }
  }
#pragma unroll
  for (int q = 0; q < SPLIT_ITEMS; ++q) {
    if (first + q >= n_items) break;
    const PlaneArgs& a = item_second[q] ? a1 : a0;
    uint8_t* out = (uint8_t*)a.out + item_b[q] * a.batch_stride;
#pragma unroll
    for (int e = 0; e < PER; ++e) {
      int r, kk;
      tile_coord(a.kcontig, e, r, kk);
      const __nv_bfloat16 h = __float2bfloat16_rn(v[q][e]);
      const __nv_bfloat16 l = __float2bfloat16_rn(v[q][e] - __bfloat162float(h));
      *(__nv_bfloat16*)(st + (0 * RT + r) * (2 * KT + 4) + 2 * kk) = h;
      *(__nv_bfloat16*)(st + (1 * RT + r) * (2 * KT + 4) + 2 * kk) = l;
    }
    __syncthreads();
    write_out<2, 2>(st, out, a.plane_stride, a.rows, a.Kp * 2, item_row0[q], item_k0[q] * 2);
    __syncthreads();
  }
}

// Ozaki slicing. With Y = X + 0x80..80 (128 added to each of the S-1 low bytes), the balanced
// base-256 digits of X are: d_p = byte_{S-1-p}(Y) - 128 for p >= 1 (that is, the byte with its
// top bit flipped, read as int8), and d_0 = byte_{S-1}(Y) read as int8 -- the carries of the
// digit-by-digit recurrence d = ((X + 128) mod 256) - 128, X <- (X - d) / 256 are exactly the
// carries of the single addition.
template <int S>
__global__ void __launch_bounds__(NTH, 4) ozaki_slice_kernel(PlaneArgs a, int32_t* __restrict__ exps) {
  __shared__ __align__(16) uint8_t st[S * RT * OPITCH];
  __shared__ double red[8][RT];
  __shared__ double rscale[RT][2];
  const long blocks_per_inst = (a.rows + RT - 1) / RT;
  const long total = blocks_per_inst * a.batch;
  unsigned long long bias = 0;
#pragma unroll
  for (int j = 0; j < S - 1; ++j) bias |= 0x80ull << (8 * j);

  for (long w = blockIdx.x; w < total; w += gridDim.x) {
    const long b = w / blocks_per_inst;
    const long row0 = (w % blocks_per_inst) * RT;
    const double* X = (const double*)a.X[b];
    uint8_t* out = (uint8_t*)a.out + b * a.batch_stride;
    // pass 1: row maxima of |x| straight from global memory (8 loads in flight per thread)
    {
      unsigned long long mx = 0;
      if (a.kcontig) {
        const int r = threadIdx.x / 8, part = threadIdx.x % 8;
        const long gr = row0 + r;
        if (gr < a.rows) {
          const double* row = X + gr * a.ld;
          long k = part;
          for (; k + 56 < a.K; k += 64) {
            double t[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) t[j] = __ldg(row + k + 8 * j);
#pragma unroll
            for (int j = 0; j < 8; ++j) mx = max_u64(mx, abs_bits(t[j]));
          }
          for (; k < a.K; k += 8) mx = max_u64(mx, abs_bits(__ldg(row + k)));
        }
#pragma unroll
        for (int off = 4; off >= 1; off >>= 1) mx = max_u64(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        if (part == 0) red[0][r] = __longlong_as_double((long long)mx);
      } else {
        const int r = threadIdx.x % 32, part = threadIdx.x / 32;
        const long gr = row0 + r;
        if (gr < a.rows) {
          const double* col = X + gr;
          long k = part;
          for (; k + 56 < a.K; k += 64) {
            double t[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) t[j] = __ldg(col + (k + 8 * j) * a.ld);
#pragma unroll
            for (int j = 0; j < 8; ++j) mx = max_u64(mx, abs_bits(t[j]));
          }
          for (; k < a.K; k += 8) mx = max_u64(mx, abs_bits(__ldg(col + k * a.ld)));
        }
        red[part][r] = __longlong_as_double((long long)mx);
      }
    }
    __syncthreads();
    if (threadIdx.x < RT) {
      unsigned long long mx = (unsigned long long)__double_as_longlong(red[0][threadIdx.x]);
      if (!a.kcontig)
        for (int q = 1; q < 8; ++q) mx = max_u64(mx, (unsigned long long)__double_as_longlong(red[q][threadIdx.x]));
      const int e = row_exponent(mx);
      const long gr = row0 + threadIdx.x;
      if (gr < a.rows) exps[b * a.rows + gr] = e;
      // x * 2^(8S-2-e) as two exact power-of-two factors (each within the double range)
      row_scale(S, e, rscale[threadIdx.x][0], rscale[threadIdx.x][1]);
    }
    __syncthreads();
    // pass 2: digits, transposed through smem, written as 16-byte vectors along K
    for (long k0 = 0; k0 < a.K; k0 += KT) {
      double v[PER];
      load_regs<double>(v, X, a.rows, a.K, a.ld, a.kcontig, row0, k0);
#pragma unroll
      for (int e = 0; e < PER; ++e) {
        int r, kk;
        tile_coord(a.kcontig, e, r, kk);
        // a non-finite row (zero scale) has zero digits
        const unsigned long long Y = slice_y(rscale[r][0] == 0.0 ? 0.0 : v[e], rscale[r][0], rscale[r][1], bias);
        const uint32_t lo = (uint32_t)Y, hi = (uint32_t)(Y >> 32);
#pragma unroll
        for (int p = 0; p < S; ++p) {
          const int byte = S - 1 - p;
          uint32_t d = (byte < 4 ? (lo >> (8 * byte)) : (hi >> (8 * (byte - 4)))) & 255u;
          if (p > 0) d ^= 0x80u;
          st[(p * RT + r) * OPITCH + kk] = (uint8_t)d;
        }
      }
      __syncthreads();
      write_out<S, 1>(st, out, a.plane_stride, a.rows, a.Kp, row0, k0);
      __syncthreads();
    }
  }
}

// Two-kernel form of the slicing for large operands: a streaming pass that only finds the row
// exponents, then one CTA per (instance, 32 rows, 128 k) chunk for the digits, so that every
// chunk's loads are in flight at once instead of walking K inside a CTA. Both kernels take two
// operands (op(A) and op(B)): blocks [0, n0) work on the first, the rest on the second.
__global__ void __launch_bounds__(NTH) ozaki_rowexp_kernel(PlaneArgs a0, int32_t* e0, long n0, PlaneArgs a1,
                                                           int32_t* e1) {
  __shared__ double red[8][RT];
  const bool second = blockIdx.x >= n0;
  const PlaneArgs a = second ? a1 : a0;
  int32_t* __restrict__ exps = second ? e1 : e0;
  const long blk = second ? blockIdx.x - n0 : blockIdx.x;
  const long blocks_per_inst = (a.rows + RT - 1) / RT;
  const long b = blk / blocks_per_inst;
  const long row0 = (blk % blocks_per_inst) * RT;
  const double* X = (const double*)a.X[b];
  unsigned long long mx = 0;
  if (a.kcontig) {
    const int r = threadIdx.x / 8, part = threadIdx.x % 8;
    const long gr = row0 + r;
    if (gr < a.rows) {
      const double* row = X + gr * a.ld;
      long k = part;
      for (; k + 120 < a.K; k += 128) {
        double t[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) t[j] = __ldg(row + k + 8 * j);
#pragma unroll
        for (int j = 0; j < 16; ++j) mx = max_u64(mx, abs_bits(t[j]));
      }
      for (; k < a.K; k += 8) mx = max_u64(mx, abs_bits(__ldg(row + k)));
    }
#pragma unroll
    for (int off = 4; off >= 1; off >>= 1) mx = max_u64(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    if (part == 0) red[0][r] = __longlong_as_double((long long)mx);
  } else {
    const int r = threadIdx.x % 32, part = threadIdx.x / 32;
    const long gr = row0 + r;
    if (gr < a.rows) {
      const double* col = X + gr;
      long k = part;
      for (; k + 120 < a.K; k += 128) {
        double t[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) t[j] = __ldg(col + (k + 8 * j) * a.ld);
#pragma unroll
        for (int j = 0; j < 16; ++j) mx = max_u64(mx, abs_bits(t[j]));
      }
      for (; k < a.K; k += 8) mx = max_u64(mx, abs_bits(__ldg(col + k * a.ld)));
    }
    red[part][r] = __longlong_as_double((long long)mx);
  }
  __syncthreads();
  if (threadIdx.x < RT) {
    unsigned long long m2 = (unsigned long long)__double_as_longlong(red[0][threadIdx.x]);
    if (!a.kcontig)
      for (int q = 1; q < 8; ++q) m2 = max_u64(m2, (unsigned long long)__double_as_longlong(red[q][threadIdx.x]));
    const long gr = row0 + threadIdx.x;
    if (gr < a.rows) exps[b * a.rows + gr] = row_exponent(m2);
  }
}

// K-parallel form of the exponent pass: one CTA per (instance, 32 rows, MKT k) part; each row's
// maximum of the |x| bit patterns over the part goes to bits[b * rows + r] by atomicMax (bits zero
// at launch), so problems with few rows and long K still spread over all SMs.
constexpr int MKT = 256;   // short parts: several CTAs per SM keep enough loads in flight
__global__ void __launch_bounds__(NTH) ozaki_rowmax_kernel(PlaneArgs a0, unsigned long long* m0, long n0,
                                                           PlaneArgs a1, unsigned long long* m1) {
  __shared__ unsigned long long red[8][RT];
  const bool second = blockIdx.x >= n0;
  const PlaneArgs a = second ? a1 : a0;
  unsigned long long* __restrict__ bits = second ? m1 : m0;
  const long blk = second ? blockIdx.x - n0 : blockIdx.x;
  const long blocks_per_inst = (a.rows + RT - 1) / RT;
  const long kparts = (a.K + MKT - 1) / MKT;
  const long item = blk / kparts;
  const long klo = (blk % kparts) * MKT;
  const long khi = klo + MKT < a.K ? klo + MKT : a.K;
  const long b = item / blocks_per_inst;
  const long row0 = (item % blocks_per_inst) * RT;
  const double* X = (const double*)a.X[b];
  unsigned long long mx = 0;
  if (a.kcontig) {
    // 8 threads per row, 16 loads in flight each
    const int r = threadIdx.x / 8, part = threadIdx.x % 8;
    const long gr = row0 + r;
    if (gr < a.rows) {
      const double* row = X + gr * a.ld;
      long k = klo + part;
      for (; k + 120 < khi; k += 128) {
        double t[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) t[j] = __ldg(row + k + 8 * j);
#pragma unroll
        for (int j = 0; j < 16; ++j) mx = max_u64(mx, abs_bits(t[j]));
      }
      for (; k < khi; k += 8) mx = max_u64(mx, abs_bits(__ldg(row + k)));
    }
#pragma unroll
    for (int off = 4; off >= 1; off >>= 1) mx = max_u64(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    if (part == 0) red[0][r] = mx;
  } else {
    // a warp reads 32 adjacent rows of one k; 8 warps split the k range
    const int r = threadIdx.x % 32, part = threadIdx.x / 32;
    const long gr = row0 + r;
    if (gr < a.rows) {
      const double* col = X + gr;
      long k = klo + part;
      for (; k + 120 < khi; k += 128) {
        double t[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) t[j] = __ldg(col + (k + 8 * j) * a.ld);
#pragma unroll
        for (int j = 0; j < 16; ++j) mx = max_u64(mx, abs_bits(t[j]));
      }
      for (; k < khi; k += 8) mx = max_u64(mx, abs_bits(__ldg(col + k * a.ld)));
    }
    red[part][r] = mx;
  }
  __syncthreads();
  if (threadIdx.x < RT) {
    unsigned long long m2 = red[0][threadIdx.x];
    if (!a.kcontig)
      for (int q = 1; q < 8; ++q) m2 = max_u64(m2, red[q][threadIdx.x]);
    const long gr = row0 + threadIdx.x;
    if (gr < a.rows && m2 != 0) atomicMax(bits + b * a.rows + gr, m2);
  }
}

constexpr int DKT = 128;                // k per digits chunk
constexpr int DPER = RT * DKT / NTH;     // 16 elements per thread
constexpr int DPITCH = DKT + 4;          // 33 words per staged row: conflict-free

// FROM_BITS: the row maxima come as |x| bit patterns (ozaki_rowmax_kernel) in bits0/bits1; the
// exponents are derived here and the chunks at k0 = 0 store them to e0/e1. Otherwise e0/e1 hold
// the exponents already (ozaki_rowexp_kernel).
template <int S, bool FROM_BITS>
__global__ void __launch_bounds__(NTH) ozaki_digits_kernel(PlaneArgs a0, int32_t* e0, long n0, PlaneArgs a1,
                                                           int32_t* e1, const unsigned long long* bits0,
                                                           const unsigned long long* bits1) {
  __shared__ __align__(16) uint8_t st[S * RT * DPITCH];
  __shared__ double rscale[RT][2];
  const bool second = blockIdx.x >= n0;
  const PlaneArgs a = second ? a1 : a0;
  int32_t* __restrict__ exps = second ? e1 : e0;
  const long blk = second ? blockIdx.x - n0 : blockIdx.x;
  const long blocks_per_inst = (a.rows + RT - 1) / RT;
  const long kchunks = (a.K + DKT - 1) / DKT;
  const long item = blk / kchunks;
  const long k0 = (blk % kchunks) * DKT;
  const long b = item / blocks_per_inst;
  const long row0 = (item % blocks_per_inst) * RT;
  const double* X = (const double*)a.X[b];
  uint8_t* out = (uint8_t*)a.out + b * a.batch_stride;
  // this thread's 16 elements: one row, four runs of 4 consecutive k, so that the 4 digits of a
  // run pack into one 32-bit shared-memory store per plane
  const int r = a.kcontig ? threadIdx.x / 8 : threadIdx.x % 32;
  auto kk_of = [&](int e) {
    return a.kcontig ? (threadIdx.x % 8) * 16 + e : (threadIdx.x / 32) * 4 + (e % 4) + 32 * (e / 4);
  };
  constexpr int PER = DPER;
  constexpr int OPITCH = DPITCH;
  double v[PER];
  {
    const long gr = row0 + r;
#pragma unroll
    for (int e = 0; e < PER; ++e) {
      const long gk = k0 + kk_of(e);
      v[e] = (gr < a.rows && gk < a.K) ? __ldg(a.kcontig ? X + gr * a.ld + gk : X + gr + gk * a.ld) : 0.0;
    }
  }
  if (threadIdx.x < RT) {
    const long gr = row0 + threadIdx.x;
    int e = 0;
    if (gr < a.rows) {
      if constexpr (FROM_BITS) {
        e = row_exponent((second ? bits1 : bits0)[b * a.rows + gr]);
        if (k0 == 0) exps[b * a.rows + gr] = e;
      } else {
        e = exps[b * a.rows + gr];
      }
    }
    row_scale(S, e, rscale[threadIdx.x][0], rscale[threadIdx.x][1]);
  }
  __syncthreads();
  const double s0 = rscale[r][0], s1 = rscale[r][1];
  if (s0 == 0.0) {   // a non-finite row has zero digits
#pragma unroll
    for (int e = 0; e < PER; ++e) v[e] = 0.0;
  }
#pragma unroll
  for (int g = 0; g < PER / 4; ++g) {
    uint32_t wd[S];
    const double x[4] = {v[4 * g], v[4 * g + 1], v[4 * g + 2], v[4 * g + 3]};
    digit_words_rs<S>(x, s0, s1, wd);
    const int kk = kk_of(4 * g);
#pragma unroll
    for (int p = 0; p < S; ++p) *(uint32_t*)(st + (p * RT + r) * OPITCH + kk) = wd[p];
  }
  __syncthreads();
  write_rows<S, DKT>(st, out, a.plane_stride, a.rows, a.Kp, row0, k0);
}

// Single-pass slicing with thread-block clusters. An item is R rows of one instance; the
// CS = ceil(K/KC) CTAs of a cluster share it, CTA q taking k in [KC q, KC q + KC), and the clusters
// are persistent (one 512-thread CTA per SM, items strided over the clusters). Two item shapes,
// both 8192 fp64 values (64 KB) per CTA: 32 rows x 256 k (256-byte row segments when the rows are
// contiguous in memory) and 16 rows x 512 k (half the cluster size, so clusters fit on all SMs).
// Per item:
//   the R x KC fp64 tile -- brought into shared memory two items ahead, by TMA when the
//   instances are equally spaced and 16-byte aligned, else by cp.async -- is read into registers
//   (16 values per thread); partial row maxima go to this CTA's pmax[item parity]; a cluster
//   barrier; every CTA reads all CS partial maxima through distributed shared memory and derives
//   the row exponents; the copies of the item two ahead are issued into the stage just read; the
//   digits are staged [plane][row][k] in shared memory and leave as 16-byte stores spread over
//   all threads, a warp per 512 contiguous bytes of a plane row (bulk copies per plane row, tried
//   before, needed a proxy fence in every thread and left 112 threads doing the write-out).
// Each operand is read from HBM once, and the next item's tile is in flight while the current
// one is converted.
// BITS form (k > 2048, after ozaki_rowmax_kernel): clusters of one CTA, items = (row block, KC
// slab) pairs, and the row exponents come from the maxima instead of the partial-maximum
// exchange; the rest of the item sequence is the same.
//
// Thread t (warp w, lane l) owns row r and 4 runs of 4 consecutive k: k = KC q + 4c + 4 NC j + i
// (j < 4, i < 4, NC = KC / 16 runs per row), with
//   rows contiguous in memory (element (r, k) at X[r + k*ld]): r = l % 16 + 16 (w % (R/16)),
//     c = l / 16 + 2 (w / (R/16)); the tile is staged [k][R rows], so a half-warp reads 16
//     consecutive rows: no bank conflicts;
//   k contiguous (element (r, k) at X[r*ld + k]): r = t / NC, c = t % NC; the tile is staged
//     [k / 256][R rows][256 k] (one TMA box per 256 k).
constexpr int CL_NTH = 512;
// Row-exponent reduction of the clusters-of-one path: a thread whose values are all zero takes
// kRowZeroKey (below every exponent); with rows spread over several warps, the row maxima meet in
// 64 words past the reduction buffer's [W][32] doubles (32 per parity of the item counter)
constexpr int kRowZeroKey = -0x40000000;

template <int R, int KC, int NTH, int RUNS = 4>
struct ClShape {
  static constexpr int TILE = R * KC;                // fp64 values per stage (4 RUNS per thread)
  static constexpr int W = NTH / 32;                 // warps
  static constexpr int NC = KC / (4 * RUNS);         // run positions per row (threads sharing a row)
  static constexpr int LR = R < 16 ? R : 16;         // rows per half-warp (rows contiguous)
  static constexpr int RG = R / LR;                  // row groups
  static constexpr int NW = W / RG;                  // warps sharing a row (rows contiguous)
  static constexpr int PW = KC / 4 + 4;              // staged digit words per row (16-byte aligned)
  static_assert(TILE / NTH == 4 * RUNS && TILE % NTH == 0, "tile shape");
  static_assert(W % RG == 0 && (32 / LR) * NW == NC && NTH % NC == 0, "thread mapping");
  template <int S>
  static constexpr int smem_bytes() {
    return 2 * TILE * 8 + S * R * PW * 4 + (W * 32 + 32) * 8 + 2 * R * 8 + R * 16 + 16;
  }
  // position of element (r, k) of a tile staged with K contiguous
  static __device__ __forceinline__ int kc_index(int r, int k) { return (k / 256) * R * 256 + r * 256 + (k % 256); }
};

__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void cluster_arrive_relaxed() {
  asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory"); }
__device__ __forceinline__ double ld_cluster_f64(const double* local, uint32_t rank) {
  uint32_t a = (uint32_t)__cvta_generic_to_shared(local), remote;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(remote) : "r"(a), "r"(rank));
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];\n" : "=d"(v) : "r"(remote) : "memory");
  return v;
}
__device__ __forceinline__ void cpa16(void* dst, const void* src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cpa8(void* dst, const void* src, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cpa_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cpa_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

struct ClusterItem {
  bool second;     // the item belongs to the second operand
  long b, row0;
};

// item -> (operand, instance, first row); 32-bit division (item counts are below 2^31)
template <int R>
__device__ __forceinline__ ClusterItem cluster_item(long item, long n0, uint32_t bpi0, uint32_t bpi1) {
  ClusterItem ci;
  ci.second = item >= n0;
  const uint32_t rb = (uint32_t)(ci.second ? item - n0 : item);
  const uint32_t bpi = ci.second ? bpi1 : bpi0;
  const uint32_t b = rb / bpi;
  ci.b = b;
  ci.row0 = (long)(rb - b * bpi) * R;
  return ci;
}

// cp.async: this CTA's R x KC slab of an item into a stage (zero outside the matrix).
template <int R, int KC, int NTH, int RUNS>
__device__ __forceinline__ void cluster_load(double* stage, const PlaneArgs a, const ClusterItem& ci, long kbase) {
  using Sh = ClShape<R, KC, NTH, RUNS>;
  const double* X = (const double*)a.X[ci.b];
  const int t = threadIdx.x;
  const bool vec = (((uintptr_t)X) % 16 == 0) && (a.ld % 2 == 0);
  if (!a.kcontig) {
    // [k][R rows]: chunk = 2 rows at one k
#pragma unroll 4
    for (int q = 0; q < Sh::TILE / 2 / NTH; ++q) {
      const int ch = t + q * NTH, kl = ch / (R / 2), rp = 2 * (ch % (R / 2));
      const long gr = ci.row0 + rp, gk = kbase + kl;
      const long nr = (gk < a.K) ? (a.rows - gr >= 2 ? 2 : (a.rows - gr > 0 ? a.rows - gr : 0)) : 0;
      const double* src = nr > 0 ? X + gr + gk * a.ld : X;
      double* dst = stage + kl * R + rp;
      if (vec) {
        cpa16(dst, src, (int)(8 * nr));
      } else {
        cpa8(dst, src, nr > 0 ? 8 : 0);
        cpa8(dst + 1, nr > 1 ? src + 1 : X, nr > 1 ? 8 : 0);
      }
    }
  } else {
    // [k / 256][R rows][256 k]: chunk = 2 consecutive k of one row
#pragma unroll 4
    for (int q = 0; q < Sh::TILE / 2 / NTH; ++q) {
      const int ch = t + q * NTH, rl = ch / (KC / 2), kp = 2 * (ch % (KC / 2));
      const long gr = ci.row0 + rl, gk = kbase + kp;
      const long nk = (gr < a.rows) ? (a.K - gk >= 2 ? 2 : (a.K - gk > 0 ? a.K - gk : 0)) : 0;
      const double* src = nk > 0 ? X + gr * a.ld + gk : X;
      double* dst = stage + Sh::kc_index(rl, kp);
      if (vec) {
        cpa16(dst, src, (int)(8 * nk));
      } else {
        cpa8(dst, src, nk > 0 ? 8 : 0);
        cpa8(dst + 1, nk > 1 ? src + 1 : X, nk > 1 ? 8 : 0);
      }
    }
  }
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

// TMA: the item's R x KC tile of one operand through its 3-D tensor map (box: R rows x 256 k,
// zero outside), one box per 256 k.
template <int R, int KC, int NTH, int RUNS>
__device__ __forceinline__ void cluster_tma(double* stage, uint64_t* bar, const CUtensorMap* tm, bool kcontig,
                                            const ClusterItem& ci, long kbase) {
  const uint32_t b = ptx::smem_u32(bar);
  ptx::mbar_arrive_expect_tx(b, ClShape<R, KC, NTH, RUNS>::TILE * 8);
#pragma unroll
  for (int h = 0; h < KC / 256; ++h) {
    const uint32_t dst = ptx::smem_u32(stage + h * R * 256);
    if (kcontig) tma_load_3d(dst, tm, b, (int)(kbase + 256 * h), (int)ci.row0, (int)ci.b);
    else tma_load_3d(dst, tm, b, (int)ci.row0, (int)(kbase + 256 * h), (int)ci.b);
  }
}

template <int S, bool TMA, int R, int KC, int NTH, int RUNS, bool BITS>
__global__ void __launch_bounds__(NTH, RUNS == 4 ? CL_NTH / NTH : 6) ozaki_cluster_kernel(const __grid_constant__ CUtensorMap tm0,
                                                                  const __grid_constant__ CUtensorMap tm1, PlaneArgs a0,
                                                                  int32_t* e0, long n0, PlaneArgs a1, int32_t* e1,
                                                                  long n_items, int CS, int* err,
                                                                  const unsigned long long* bits0,
                                                                  const unsigned long long* bits1, int KB) {
  using Sh = ClShape<R, KC, NTH, RUNS>;
  constexpr int NC = Sh::NC, LR = Sh::LR, RG = Sh::RG, NW = Sh::NW, PW = Sh::PW, TILE = Sh::TILE;
  extern __shared__ __align__(16) uint8_t dyn[];
  double* stages = (double*)dyn;                                                   // [2][TILE]
  uint32_t* st = (uint32_t*)(dyn + 2 * TILE * 8);                                  // [S][R][PW]
  double* red = (double*)(dyn + 2 * TILE * 8 + S * R * PW * 4);                    // [W][32] + 32
  double* pmax = red + Sh::W * 32 + 32;                                               // [2][R]
  constexpr int kRowMaxWords = Sh::W * 64;   // int words of red past the [W][32] doubles
  double* rscale = pmax + 2 * R;                                                   // [R][2]
  uint64_t* full = (uint64_t*)(rscale + 2 * R);                                    // [2] (TMA)

  const int rank = (int)(blockIdx.x % CS);           // rank in the cluster (cluster dims CS x 1 x 1)
  const long cluster = blockIdx.x / CS, nclusters = gridDim.x / CS;
  const int t = threadIdx.x, lane = t % 32, warp = t / 32;
  const uint32_t bpi0 = (uint32_t)((a0.rows + R - 1) / R);
  const uint32_t bpi1 = (uint32_t)((a1.rows + R - 1) / R);
  // item -> (operand, instance, first row) and the first k of this CTA's slab: the cluster rank's
  // KC-wide slab, or with BITS (clusters of one CTA, items = row blocks x KB slabs) the item's own
  auto item_at = [&](long item, long& kbase) -> ClusterItem {
    if constexpr (BITS) {
      const uint32_t rb = (uint32_t)item / (uint32_t)KB;
      kbase = (long)((uint32_t)item - rb * (uint32_t)KB) * KC;
      return cluster_item<R>(rb, n0, bpi0, bpi1);
    } else {
      kbase = (long)rank * KC;
      return cluster_item<R>(item, n0, bpi0, bpi1);
    }
  };

  if (TMA && t == 0) {
    ptx::mbar_init(ptx::smem_u32(&full[0]), 1);
    ptx::mbar_init(ptx::smem_u32(&full[1]), 1);
    ptx::fence_mbar_init();
  }
  // per-row maximum words of the clusters-of-one path (rows not contiguous in K), two parities
  if (t < 64) ((int*)red)[kRowMaxWords + t] = kRowZeroKey;
  __syncthreads();
  // under a programmatic launch the set-up above overlaps the end of the kernel before; the
  // operands, planes and exponents are touched only after it has completed
  ptx::grid_dep_wait();
  ptx::grid_dep_launch();

  // prologue: the first two items of this cluster
  for (int s = 0; s < 2; ++s) {
    const long item = cluster + s * nclusters;
    if (item < n_items) {
      long kbase;
      const ClusterItem ci = item_at(item, kbase);
      if (TMA) {
        if (t == 0) cluster_tma<R, KC, NTH, RUNS>(stages + s * TILE, &full[s], ci.second ? &tm1 : &tm0,
                                       ci.second ? a1.kcontig : a0.kcontig, ci, kbase);
      } else {
        cluster_load<R, KC, NTH, RUNS>(stages + s * TILE, ci.second ? a1 : a0, ci, kbase);
      }
    }
    if (!TMA) cpa_commit();
  }

  long iter = 0;
  for (long item = cluster; item < n_items; item += nclusters, ++iter) {
    const int s = (int)(iter & 1);
    long kbase;
    const ClusterItem ci = item_at(item, kbase);
    const PlaneArgs a = ci.second ? a1 : a0;
    int32_t* __restrict__ exps = ci.second ? e1 : e0;
    const int r = a.kcontig ? t / NC : lane % LR + LR * (warp % RG);
    const int c = a.kcontig ? t % NC : lane / LR + (32 / LR) * (warp / RG);
    if (TMA) {
      // a wait that gives up records the error and carries on (every CTA of the cluster must
      // take the same barriers, and every copy is waited for); the host reports the call as failed
      ptx::mbar_wait(ptx::smem_u32(&full[s]), (uint32_t)((iter >> 1) & 1), err, 41);
    } else {
      cpa_wait1();
    }
    // Every thread has waited for the TMA tile itself. The barrier is needed for cp.async tiles
    // (other threads' copies); otherwise the barrier after the row maxima (or the cluster
    // barrier) separates the previous item's reads of st, red and rscale from this item's writes.
    if (!TMA) __syncthreads();
    const double* tile = stages + s * TILE;
    double v[4 * RUNS];
    if (a.kcontig) {
#pragma unroll
      for (int j = 0; j < RUNS; ++j) {
        const int k = 4 * c + 4 * NC * j;
        const double2 x0 = *(const double2*)(tile + Sh::kc_index(r, k));
        const double2 x1 = *(const double2*)(tile + Sh::kc_index(r, k) + 2);
        v[4 * j] = x0.x; v[4 * j + 1] = x0.y; v[4 * j + 2] = x1.x; v[4 * j + 3] = x1.y;
      }
    } else {
#pragma unroll
      for (int j = 0; j < RUNS; ++j)
#pragma unroll
        for (int i = 0; i < 4; ++i) v[4 * j + i] = tile[(4 * c + 4 * NC * j + i) * R + r];
    }

    // A cluster of one CTA (k <= KC) holds whole rows: every thread takes its row's maximum from
    // the reduction itself and derives the scale in registers -- no cluster exchange, no
    // rscale buffer, two barriers per item instead of four. The BITS form does the same with
    // the maxima of the K-parallel pass.
    const bool local = BITS || CS == 1;
    double s0 = 0.0, s1 = 0.0;
    if constexpr (BITS) {
      // the row maxima of the whole K range come from the K-parallel pass
      const long gr = ci.row0 + r;
      const unsigned long long m2 = gr < a.rows ? (ci.second ? bits1 : bits0)[ci.b * a.rows + gr] : 0ull;
      const int e = row_exponent(m2);
      if (kbase == 0 && c == 0 && gr < a.rows) exps[ci.b * a.rows + gr] = e;
      row_scale(S, e, s0, s1);
      __syncthreads();   // stage s fully read; the previous item's st reads done
    } else if (local) {
      // row_exponent is monotonic in nonzero keys, so the row's exponent is the maximum of the
      // threads' exponents: 32-bit reductions instead of 64-bit keys. A thread whose values are
      // all zero (the fill past k, or zeros) takes a sentinel below every exponent (-1073 is the
      // smallest), and a row that is zero throughout gets 0 back.
      constexpr int kZeroKey = kRowZeroKey;
      const unsigned long long key = row_key(v);
      int e = key ? row_exponent(key) : kZeroKey;
      int* const redi = (int*)red;
      if (a.kcontig && NC <= 32) {
        // the NC threads of row r are consecutive lanes: the xor reduction leaves the maximum in
        // all of them
#pragma unroll
        for (int off = 1; off < NC; off <<= 1) e = max(e, __shfl_xor_sync(0xffffffffu, e, off));
      } else if (a.kcontig) {
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) e = max(e, __shfl_xor_sync(0xffffffffu, e, off));
        if (lane == 0) redi[warp] = e;
      } else {
        // rows spread over NW warps: each warp's maxima meet in one word per row by a shared-
        // memory atomicMax (the words of this item's parity; the other parity's are reset below
        // for the next item), so every thread then reads one word instead of NW
#pragma unroll
        for (int off = LR; off < 32; off <<= 1) e = max(e, __shfl_xor_sync(0xffffffffu, e, off));
        if (lane < LR) atomicMax(&redi[kRowMaxWords + (int)(iter & 1) * 32 + r], e);
      }
      __syncthreads();   // red visible; stage s fully read; the previous item's st reads done
      if (a.kcontig && NC > 32) {
        e = redi[r * (NC / 32)];
        for (int w = 1; w < NC / 32; ++w) e = max(e, redi[r * (NC / 32) + w]);
      } else if (!a.kcontig) {
        e = redi[kRowMaxWords + (int)(iter & 1) * 32 + r];
        // the other parity was last read in the previous item, before its second barrier
        if (t < R) redi[kRowMaxWords + (int)((iter + 1) & 1) * 32 + t] = kZeroKey;
      }
      if (e == kZeroKey) e = 0;
      if (c == 0 && ci.row0 + r < a.rows) exps[ci.b * a.rows + ci.row0 + r] = e;
      row_scale(S, e, s0, s1);
    } else {
      // partial row maxima of this CTA's K range (row_key of |x|; the shared-memory buffers hold
      // them as doubles, bit for bit)
      unsigned long long mx = row_key(v);
      double* pm = pmax + s * R;
      auto as_d = [](unsigned long long u) { return __longlong_as_double((long long)u); };
      auto as_u = [](double d) { return (unsigned long long)__double_as_longlong(d); };
      if (a.kcontig && NC <= 32) {
        // the NC threads of row r are consecutive lanes
#pragma unroll
        for (int off = 1; off < NC; off <<= 1) mx = max_u64(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        if (c == 0) pm[r] = as_d(mx);
      } else if (a.kcontig) {
        // row r spans the NC / 32 warps r * NC / 32 ..
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) mx = max_u64(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        if (lane == 0) red[warp] = as_d(mx);
        __syncthreads();
        if (t < R) {
          unsigned long long m2 = as_u(red[t * (NC / 32)]);
          for (int w = 1; w < NC / 32; ++w) m2 = max_u64(m2, as_u(red[t * (NC / 32) + w]));
          pm[t] = as_d(m2);
        }
      } else {
        // row r: lanes with lane % LR == r % LR of the NW warps with w % RG == r / LR
#pragma unroll
        for (int off = LR; off < 32; off <<= 1) mx = max_u64(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        if (lane < LR) red[(warp / RG) * 32 + r] = as_d(mx);
        __syncthreads();
        if (t < R) {
          unsigned long long m2 = as_u(red[t]);
#pragma unroll
          for (int w = 1; w < NW; ++w) m2 = max_u64(m2, as_u(red[w * 32 + t]));
          pm[t] = as_d(m2);
        }
      }
      cluster_arrive();   // every CTA's pmax[s] is visible after the wait
      cluster_wait();
      if (t < R) {
        unsigned long long m2 = 0;
        for (int q = 0; q < CS; ++q) m2 = max_u64(m2, as_u(ld_cluster_f64(pm + t, (uint32_t)q)));
        const int e = row_exponent(m2);
        if (rank == 0 && ci.row0 + t < a.rows) exps[ci.b * a.rows + ci.row0 + t] = e;
        // x * 2^(8S-2-e) as two exact power-of-two factors (each within the double range)
        row_scale(S, e, rscale[2 * t], rscale[2 * t + 1]);
      }
    }
    if (!local) {
      __syncthreads();   // rscale visible; stage s fully read into registers
      s0 = rscale[2 * r];
      s1 = rscale[2 * r + 1];
    }

    // the item two ahead goes into the stage just read
    {
      const long nxt = item + 2 * nclusters;
      if (nxt < n_items) {
        long kn;
        const ClusterItem cn = item_at(nxt, kn);
        if (TMA) {
          if (t == 0) cluster_tma<R, KC, NTH, RUNS>(stages + s * TILE, &full[s], cn.second ? &tm1 : &tm0,
                                         cn.second ? a1.kcontig : a0.kcontig, cn, kn);
        } else {
          cluster_load<R, KC, NTH, RUNS>(stages + s * TILE, cn.second ? a1 : a0, cn, kn);
        }
      }
      if (!TMA) cpa_commit();
    }

    // digits: one 32-bit word per plane per run of 4 k, staged [p][r][k/4]
    if (s0 == 0.0) {   // a non-finite row has zero digits
#pragma unroll
      for (int e = 0; e < 4 * RUNS; ++e) v[e] = 0.0;
    }
#pragma unroll
    for (int j = 0; j < RUNS; ++j) {
      uint32_t wd[S];
      const double x[4] = {v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]};
      digit_words_rs<S>(x, s0, s1, wd);
#pragma unroll
      for (int p = 0; p < S; ++p) st[(p * R + r) * PW + c + NC * j] = wd[p];
    }
    __syncthreads();

    // write-out: each (plane, row) of this CTA's KC bytes of K (k >= K holds zero digits, up to
    // Kp) as 16-byte stores, a warp per 512 contiguous bytes, spread over all threads
    {
      constexpr int CPRW = KC / 16;                       // 16-byte chunks per staged row
      constexpr int NCH = S * R * CPRW;                   // chunks of the item
      const long bytes = a.Kp - kbase < KC ? a.Kp - kbase : KC;
      uint8_t* const out0 = (uint8_t*)a.out + ci.b * a.batch_stride + ci.row0 * a.Kp + kbase;
#pragma unroll
      for (int q = 0; q < (NCH + NTH - 1) / NTH; ++q) {
        const int ch = t + q * NTH, pr = ch / CPRW, cc = ch % CPRW;
        const int p = pr / R, rr = pr % R;
        if (ch < NCH && ci.row0 + rr < a.rows && 16L * cc < bytes) {
          const uint4 w = *(const uint4*)(st + pr * PW + 4 * cc);
          *(uint4*)(out0 + p * a.plane_stride + (long)rr * a.Kp + 16 * cc) = w;
        }
      }
    }
  }
  if (!TMA) cpa_wait0();
  if (TMA && t == 0) {
    // no copy may still be in flight when the CTA exits (bounded, like every wait here)
    for (long j = iter; j < iter + 2; ++j) {
      const long item = cluster + j * nclusters;
      if (item < n_items) ptx::mbar_wait(ptx::smem_u32(&full[j & 1]), (uint32_t)((j >> 1) & 1), err, 42);
    }
  }
  // no CTA leaves while another may still read its pmax
  cluster_arrive_relaxed();
  cluster_wait();
}

// BITS: row maxima in bits0/bits1, CS = 1 and KB k slabs per row block
template <int S, bool TMA, int R, int KC, int NTH, int RUNS, bool BITS = false>
cudaError_t launch_cluster_st(const CUtensorMap& tm0, const CUtensorMap& tm1, const PlaneArgs& a0, int32_t* e0,
                              long n0, const PlaneArgs& a1, int32_t* e1, long n1, int CS, cudaStream_t st,
                              const unsigned long long* bits0 = nullptr, const unsigned long long* bits1 = nullptr,
                              int KB = 1) {
  constexpr int SMEM = ClShape<R, KC, NTH, RUNS>::template smem_bytes<S>();
  auto kern = ozaki_cluster_kernel<S, TMA, R, KC, NTH, RUNS, BITS>;
  static bool attr[kMaxDevices] = {};
  if (cudaError_t e = smem_attr_once(attr, kern, SMEM)) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.blockDim = dim3(NTH, 1, 1);
  cfg.dynamicSmemBytes = SMEM;
  cfg.stream = st;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)CS;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  // persistent clusters: as many as fit at once (CL_NTH / NTH CTAs per SM), at most one per item
  static int max_clusters_dev[kMaxDevices][9] = {};
  const int dev = current_device();
  if (dev < 0) return cudaErrorInvalidDevice;
  int (&max_clusters)[9] = max_clusters_dev[dev];
  if (max_clusters[CS] == 0) {
    cfg.gridDim = dim3((unsigned)(CS * num_sms() * (CL_NTH / NTH)), 1, 1);
    int nc = 0;
    cudaError_t e = cudaOccupancyMaxActiveClusters(&nc, kern, &cfg);
    if (e != cudaSuccess || nc <= 0) {
      cudaGetLastError();
      nc = num_sms() * (CL_NTH / NTH) / CS;
    }
    max_clusters[CS] = nc > 0 ? nc : 1;
  }
  const long n_items = (n0 + n1) * KB;
  const long nclusters = n_items < max_clusters[CS] ? n_items : max_clusters[CS];
  cfg.gridDim = dim3((unsigned)(nclusters * CS), 1, 1);
  // programmatic launch: the CTAs' set-up overlaps the end of the kernel before (the kernel waits
  // for it before touching global memory)
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.numAttrs = 2;
  return cudaLaunchKernelEx(&cfg, kern, tm0, tm1, a0, e0, n0, a1, e1, n_items, CS, device_error_flag(), bits0,
                            bits1, KB);
}

// 3-D map (innermost dimension first) over an equally spaced fp64 operand with an R x 256 box.
bool slicer_map(CUtensorMap* m, const PlaneArgs& a, int R) {
  if (!a.X0 || a.xstride <= 0 || ((uintptr_t)a.X0 % 16) != 0 || (a.ld * 8) % 16 != 0 || a.xstride % 16 != 0)
    return false;
  if (a.rows >= (1L << 31) || a.K >= (1L << 31) || a.batch >= (1L << 31)) return false;
  long dims[3], strides[2];
  int box[3];
  if (a.kcontig) {
    dims[0] = a.K; dims[1] = a.rows; box[0] = 256; box[1] = R;
  } else {
    dims[0] = a.rows; dims[1] = a.K; box[0] = R; box[1] = 256;
  }
  dims[2] = a.batch; box[2] = 1;
  strides[0] = a.ld * 8;
  strides[1] = a.xstride;
  return make_tiled_map(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, a.X0, dims, strides, box, 0);
}

template <int S, int R, int KC, int NTH = CL_NTH, int RUNS = 4>
cudaError_t launch_cluster_shape(const PlaneArgs& a0, int32_t* e0, const PlaneArgs& a1, int32_t* e1, bool two,
                                 cudaStream_t st) {
  const int CS = (int)((a0.Kp + KC - 1) / KC);
  const long n0 = (a0.rows + R - 1) / R * a0.batch;
  const long n1 = two ? (a1.rows + R - 1) / R * a1.batch : 0;
  if ((n0 + n1) * CS >= (1L << 31) || CS < 1 || CS > 8) return cudaErrorInvalidValue;
  CUtensorMap tm0, tm1;
  const bool tma = slicer_map(&tm0, a0, R) && (!two || slicer_map(&tm1, a1, R));
  if (!two) tm1 = tm0;
  if (tma) return launch_cluster_st<S, true, R, KC, NTH, RUNS>(tm0, tm1, a0, e0, n0, a1, e1, n1, CS, st);
  return launch_cluster_st<S, false, R, KC, NTH, RUNS>(tm0, tm1, a0, e0, n0, a1, e1, n1, CS, st);
}

// Item shape: 16 x 512 (configuration 3, the default), 32 x 256 (2) or 8 x 1024 (4), all with
// 512-thread CTAs (one per SM); or 16 x 256 with 256-thread CTAs, two per SM (5), so that one
// CTA converts while the other waits at its cluster barrier.
template <int S>
cudaError_t launch_cluster_s(const PlaneArgs& a0, int32_t* e0, const PlaneArgs& a1, int32_t* e1, bool two, int shape,
                             cudaStream_t st) {
  if (shape == 5) return launch_cluster_shape<S, 16, 256, 256>(a0, e0, a1, e1, two, st);
  if (shape == 6) return launch_cluster_shape<S, 4, 256, 128, 2>(a0, e0, a1, e1, two, st);
  if (shape == 2) return launch_cluster_shape<S, 32, 256>(a0, e0, a1, e1, two, st);
  if (shape == 4) return launch_cluster_shape<S, 8, 1024>(a0, e0, a1, e1, two, st);
  return launch_cluster_shape<S, 16, 512>(a0, e0, a1, e1, two, st);
}

// Digits of one or two operands (same Kp) whose row maxima are in bits0/bits1: persistent CTAs
// over (16 rows, 512 k) items, tiles by TMA or cp.async two items ahead, no cluster exchange.
template <int S>
cudaError_t launch_digits_from_bits(const PlaneArgs& a0, int32_t* e0, const unsigned long long* bits0,
                                    const PlaneArgs& a1, int32_t* e1, const unsigned long long* bits1,
                                    cudaStream_t st) {
  constexpr int R = 16, KC = 512;
  const long KB = (a0.Kp + KC - 1) / KC;
  const long n0 = (a0.rows + R - 1) / R * a0.batch, n1 = (a1.rows + R - 1) / R * a1.batch;
  if ((n0 + n1) * KB >= (1L << 31)) return cudaErrorInvalidValue;
  CUtensorMap tm0, tm1;
  if (slicer_map(&tm0, a0, R) && slicer_map(&tm1, a1, R))
    return launch_cluster_st<S, true, R, KC, CL_NTH, 4, true>(tm0, tm1, a0, e0, n0, a1, e1, n1, 1, st, bits0, bits1,
                                                             (int)KB);
  return launch_cluster_st<S, false, R, KC, CL_NTH, 4, true>(tm0, tm1, a0, e0, n0, a1, e1, n1, 1, st, bits0, bits1,
                                                            (int)KB);
}

}  // namespace

// K up to 2048 with clusters of at most 8 CTAs of 256 k (at most 4 of 512 k)
bool cluster_kernel_fits(const PlaneArgs& a) { return a.K <= 2048 && a.Kp <= 2048; }

// One launch for one or two operands (with the same K).
cudaError_t launch_ozaki_cluster(const PlaneArgs& a0, int32_t* e0, const PlaneArgs& a1, int32_t* e1, bool two,
                                 int slices, int shape, cudaStream_t st) {
  ProfScope prof("ozaki_slice", st);
  cudaError_t e;
  switch (slices) {
    case 3: e = launch_cluster_s<3>(a0, e0, a1, e1, two, shape, st); break;
    case 4: e = launch_cluster_s<4>(a0, e0, a1, e1, two, shape, st); break;
    case 5: e = launch_cluster_s<5>(a0, e0, a1, e1, two, shape, st); break;
    case 6: e = launch_cluster_s<6>(a0, e0, a1, e1, two, shape, st); break;
    case 7: e = launch_cluster_s<7>(a0, e0, a1, e1, two, shape, st); break;
    case 8: e = launch_cluster_s<8>(a0, e0, a1, e1, two, shape, st); break;
    default: return cudaErrorInvalidValue;
  }
  note_launch();
  return e;
}


cudaError_t launch_pack_i8(const PlaneArgs& a, cudaStream_t st) {
  const long ktiles = (a.Kp + PKK - 1) / PKK, rtiles = (a.rows + PKR - 1) / PKR;
  const long blocks = ktiles * rtiles * a.batch;
  if (blocks >= (1L << 31)) return cudaErrorInvalidValue;
  ProfScope prof("pack_i8", st);
  pack_i8_kernel<<<(unsigned)blocks, NTH, 0, st>>>(a, ktiles, rtiles);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_split_bf16_pair(const PlaneArgs& a, const PlaneArgs& b, cudaStream_t st) {
  const long na = (a.K + KT - 1) / KT * ((a.rows + RT - 1) / RT) * a.batch;
  const long nb = (b.K + KT - 1) / KT * ((b.rows + RT - 1) / RT) * b.batch;
  const long blocks = (na + nb + SPLIT_ITEMS - 1) / SPLIT_ITEMS;
  if (blocks >= (1L << 31)) return cudaErrorInvalidValue;
  ProfScope prof("split_bf16", st);
  split_bf16_pair_kernel<<<(unsigned)blocks, NTH, 0, st>>>(a, na, b, na + nb);
  note_launch();
  return cudaGetLastError();
}


cudaError_t launch_ozaki_slice_pair(const PlaneArgs& a, int32_t* ea, const PlaneArgs& b, int32_t* eb, int slices,
                                    cudaStream_t st) {
  // K up to 2048: one pass over both operands (unless a two-pass form, 1 or 7, is configured).
  // Untuned default: 16 x 512 items while one CTA holds a whole row (k <= 512), else 8 x 1024
  // (clusters of one CTA up to k = 1024, half as many CTAs exchanging maxima above).
  const int form = choose_config(SSBLAS_PATH_OZAKI_SLICER, a.rows, b.rows, a.K, a.batch, a.Kp <= 512 ? 3 : 4);
  if (form != 1 && form != 7 && cluster_kernel_fits(a) && b.K == a.K)
    return launch_ozaki_cluster(a, ea, b, eb, true, slices, form, st);
  // two passes over both operands: row maxima per (32 rows, 256 k) part, then the digits --
  // by persistent CTAs over (16 rows, 512 k) slabs (form 7, and every form but 1 when K > 2048),
  // or (form 1) per (32 rows, 128 k) chunk; both passes spread over all SMs whatever the row count
  const long items_a = (a.rows + RT - 1) / RT * a.batch, items_b = (b.rows + RT - 1) / RT * b.batch;
  const long parts_a = items_a * ((a.K + MKT - 1) / MKT), parts_b = items_b * ((b.K + MKT - 1) / MKT);
  const long chunks_a = items_a * ((a.K + DKT - 1) / DKT), chunks_b = items_b * ((b.K + DKT - 1) / DKT);
  if (chunks_a + chunks_b >= (1L << 31)) {
    cudaError_t e = launch_ozaki_slice(a, slices, ea, st);
    return e != cudaSuccess ? e : launch_ozaki_slice(b, slices, eb, st);
  }
  cudaError_t e;
  const size_t nbits = (size_t)(a.rows * a.batch + b.rows * b.batch);
  unsigned long long* bits = (unsigned long long*)workspace(WS_ROWMAX, sizeof(unsigned long long) * nbits, &e);
  if (!bits) return e;
  unsigned long long* bits_b = bits + a.rows * a.batch;
  if ((e = cudaMemsetAsync(bits, 0, sizeof(unsigned long long) * nbits, st)) != cudaSuccess) return e;
  {
    ProfScope prof("ozaki_rowmax", st);
    ozaki_rowmax_kernel<<<(unsigned)(parts_a + parts_b), NTH, 0, st>>>(a, bits, parts_a, b, bits_b);
    note_launch();
  }
  ProfScope prof("ozaki_slice", st);
  if (form != 1 && a.Kp == b.Kp) {
    // digits by the persistent slab kernel
    switch (slices) {
      case 3: e = launch_digits_from_bits<3>(a, ea, bits, b, eb, bits_b, st); break;
      case 4: e = launch_digits_from_bits<4>(a, ea, bits, b, eb, bits_b, st); break;
      case 5: e = launch_digits_from_bits<5>(a, ea, bits, b, eb, bits_b, st); break;
      case 6: e = launch_digits_from_bits<6>(a, ea, bits, b, eb, bits_b, st); break;
      case 7: e = launch_digits_from_bits<7>(a, ea, bits, b, eb, bits_b, st); break;
      case 8: e = launch_digits_from_bits<8>(a, ea, bits, b, eb, bits_b, st); break;
      default: return cudaErrorInvalidValue;
    }
    note_launch();
    return e;
  }
  // form 1: digits per (32 rows, 128 k) chunk
  const unsigned g = (unsigned)(chunks_a + chunks_b);
  switch (slices) {
    case 3: ozaki_digits_kernel<3, true><<<g, NTH, 0, st>>>(a, ea, chunks_a, b, eb, bits, bits_b); break;
    case 4: ozaki_digits_kernel<4, true><<<g, NTH, 0, st>>>(a, ea, chunks_a, b, eb, bits, bits_b); break;
    case 5: ozaki_digits_kernel<5, true><<<g, NTH, 0, st>>>(a, ea, chunks_a, b, eb, bits, bits_b); break;
    case 6: ozaki_digits_kernel<6, true><<<g, NTH, 0, st>>>(a, ea, chunks_a, b, eb, bits, bits_b); break;
    case 7: ozaki_digits_kernel<7, true><<<g, NTH, 0, st>>>(a, ea, chunks_a, b, eb, bits, bits_b); break;
    case 8: ozaki_digits_kernel<8, true><<<g, NTH, 0, st>>>(a, ea, chunks_a, b, eb, bits, bits_b); break;
    default: return cudaErrorInvalidValue;
  }
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_ozaki_slice(const PlaneArgs& a, int slices, int32_t* exps, cudaStream_t st) {
  const int form = choose_config(SSBLAS_PATH_OZAKI_SLICER, a.rows, a.rows, a.K, a.batch, a.Kp <= 512 ? 3 : 4);
  if (form != 1 && form != 7 && cluster_kernel_fits(a))
    return launch_ozaki_cluster(a, exps, a, exps, false, slices, form, st);
  const long items = (a.rows + RT - 1) / RT * a.batch;
  const long chunks = items * ((a.K + DKT - 1) / DKT);
  if (items >= 2L * num_sms() && chunks < (1L << 31)) {
    // enough rows to fill the GPU: the two-kernel form (exponents, then digits per chunk)
    {
      ProfScope prof("ozaki_rowexp", st);
      ozaki_rowexp_kernel<<<(unsigned)items, NTH, 0, st>>>(a, exps, items, a, exps);
      note_launch();
    }
    ProfScope prof("ozaki_slice", st);
    switch (slices) {
      case 3: ozaki_digits_kernel<3, false><<<(unsigned)chunks, NTH, 0, st>>>(a, exps, chunks, a, exps, nullptr, nullptr); break;
      case 4: ozaki_digits_kernel<4, false><<<(unsigned)chunks, NTH, 0, st>>>(a, exps, chunks, a, exps, nullptr, nullptr); break;
      case 5: ozaki_digits_kernel<5, false><<<(unsigned)chunks, NTH, 0, st>>>(a, exps, chunks, a, exps, nullptr, nullptr); break;
      case 6: ozaki_digits_kernel<6, false><<<(unsigned)chunks, NTH, 0, st>>>(a, exps, chunks, a, exps, nullptr, nullptr); break;
      case 7: ozaki_digits_kernel<7, false><<<(unsigned)chunks, NTH, 0, st>>>(a, exps, chunks, a, exps, nullptr, nullptr); break;
      case 8: ozaki_digits_kernel<8, false><<<(unsigned)chunks, NTH, 0, st>>>(a, exps, chunks, a, exps, nullptr, nullptr); break;
      default: return cudaErrorInvalidValue;
    }
    note_launch();
    return cudaGetLastError();
  }
  ProfScope prof("ozaki_slice", st);
  const long cap = 4L * num_sms();
  const unsigned grid = (unsigned)(items < cap ? items : cap);
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
