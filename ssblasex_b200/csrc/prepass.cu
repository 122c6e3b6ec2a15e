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
//
// All three kernels follow the same memory plan: every thread issues its global loads for a
// 32-row x 64-k tile back to back (coalesced along whichever of rows / k is contiguous), converts
// in registers, transposes the output bytes through shared memory, and writes 16-byte vectors
// along K. Several CTAs per SM keep enough loads in flight to run at HBM speed.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "internal.h"
#include "prepass.h"

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

__global__ void __launch_bounds__(NTH) pack_i8_kernel(PlaneArgs a) {
  __shared__ __align__(16) uint8_t st[RT * (KT + 4)];
  const long b = blockIdx.y;
  const long row0 = (long)blockIdx.x * RT;
  const int8_t* X = (const int8_t*)a.X[b];
  uint8_t* out = (uint8_t*)a.out + b * a.batch_stride;
  for (long k0 = 0; k0 < a.K; k0 += KT) {
    int8_t v[PER];
    load_regs<int8_t>(v, X, a.rows, a.K, a.ld, a.kcontig, row0, k0);
#pragma unroll
    for (int e = 0; e < PER; ++e) {
      int r, kk;
      tile_coord(a.kcontig, e, r, kk);
      st[r * (KT + 4) + kk] = (uint8_t)v[e];
    }
    __syncthreads();
    write_out<1, 1>(st, out, a.plane_stride, a.rows, a.Kp, row0, k0);
    __syncthreads();
  }
}

__global__ void __launch_bounds__(NTH) split_bf16_kernel(PlaneArgs a) {
  __shared__ __align__(16) uint8_t st[2 * RT * (2 * KT + 4)];
  const long b = blockIdx.y;
  const long row0 = (long)blockIdx.x * RT;
  const float* X = (const float*)a.X[b];
  uint8_t* out = (uint8_t*)a.out + b * a.batch_stride;
  for (long k0 = 0; k0 < a.K; k0 += KT) {
    float v[PER];
    load_regs<float>(v, X, a.rows, a.K, a.ld, a.kcontig, row0, k0);
#pragma unroll
    for (int e = 0; e < PER; ++e) {
      int r, kk;
      tile_coord(a.kcontig, e, r, kk);
      const __nv_bfloat16 h = __float2bfloat16_rn(v[e]);
      const __nv_bfloat16 l = __float2bfloat16_rn(v[e] - __bfloat162float(h));
      *(__nv_bfloat16*)(st + (0 * RT + r) * (2 * KT + 4) + 2 * kk) = h;
      *(__nv_bfloat16*)(st + (1 * RT + r) * (2 * KT + 4) + 2 * kk) = l;
    }
    __syncthreads();
    write_out<2, 2>(st, out, a.plane_stride, a.rows, a.Kp * 2, row0, k0 * 2);
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
      double mx = 0.0;
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
            for (int j = 0; j < 8; ++j) mx = fmax(mx, fabs(t[j]));
          }
          for (; k < a.K; k += 8) mx = fmax(mx, fabs(__ldg(row + k)));
        }
#pragma unroll
        for (int off = 4; off >= 1; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        if (part == 0) red[0][r] = mx;
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
            for (int j = 0; j < 8; ++j) mx = fmax(mx, fabs(t[j]));
          }
          for (; k < a.K; k += 8) mx = fmax(mx, fabs(__ldg(col + k * a.ld)));
        }
        red[part][r] = mx;
      }
    }
    __syncthreads();
    if (threadIdx.x < RT) {
      double mx = red[0][threadIdx.x];
      if (!a.kcontig)
        for (int q = 1; q < 8; ++q) mx = fmax(mx, red[q][threadIdx.x]);
      int e = 0;
      if (mx > 0.0) frexp(mx, &e);
      const long gr = row0 + threadIdx.x;
      if (gr < a.rows) exps[b * a.rows + gr] = e;
      // x * 2^(8S-2-e) as two exact power-of-two factors (each within the double range)
      const int sh = 8 * S - 2 - e;
      const int h1 = sh / 2;
      rscale[threadIdx.x][0] = ldexp(1.0, h1);
      rscale[threadIdx.x][1] = ldexp(1.0, sh - h1);
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
        const unsigned long long Y =
            (unsigned long long)__double2ll_rn(v[e] * rscale[r][0] * rscale[r][1]) + bias;
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
  double mx = 0.0;
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
        for (int j = 0; j < 16; ++j) mx = fmax(mx, fabs(t[j]));
      }
      for (; k < a.K; k += 8) mx = fmax(mx, fabs(__ldg(row + k)));
    }
#pragma unroll
    for (int off = 4; off >= 1; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    if (part == 0) red[0][r] = mx;
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
        for (int j = 0; j < 16; ++j) mx = fmax(mx, fabs(t[j]));
      }
      for (; k < a.K; k += 8) mx = fmax(mx, fabs(__ldg(col + k * a.ld)));
    }
    red[part][r] = mx;
  }
  __syncthreads();
  if (threadIdx.x < RT) {
    double m2 = red[0][threadIdx.x];
    if (!a.kcontig)
      for (int q = 1; q < 8; ++q) m2 = fmax(m2, red[q][threadIdx.x]);
    int e = 0;
    if (m2 > 0.0) frexp(m2, &e);
    const long gr = row0 + threadIdx.x;
    if (gr < a.rows) exps[b * a.rows + gr] = e;
  }
}

constexpr int DKT = 128;                // k per digits chunk
constexpr int DPER = RT * DKT / NTH;     // 16 elements per thread
constexpr int DPITCH = DKT + 4;          // 33 words per staged row: conflict-free

template <int S>
__global__ void __launch_bounds__(NTH) ozaki_digits_kernel(PlaneArgs a0, const int32_t* e0, long n0, PlaneArgs a1,
                                                           const int32_t* e1) {
  __shared__ __align__(16) uint8_t st[S * RT * DPITCH];
  __shared__ double rscale[RT][2];
  const bool second = blockIdx.x >= n0;
  const PlaneArgs a = second ? a1 : a0;
  const int32_t* __restrict__ exps = second ? e1 : e0;
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
    const int e = gr < a.rows ? exps[b * a.rows + gr] : 0;
    const int sh = 8 * S - 2 - e;
    const int h1 = sh / 2;
    rscale[threadIdx.x][0] = ldexp(1.0, h1);
    rscale[threadIdx.x][1] = ldexp(1.0, sh - h1);
  }
  __syncthreads();
  unsigned long long bias = 0;
#pragma unroll
  for (int j = 0; j < S - 1; ++j) bias |= 0x80ull << (8 * j);
  const double s0 = rscale[r][0], s1 = rscale[r][1];
#pragma unroll
  for (int g = 0; g < PER / 4; ++g) {
    uint32_t lo[4], hi[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const unsigned long long Y = (unsigned long long)__double2ll_rn(v[4 * g + j] * s0 * s1) + bias;
      lo[j] = (uint32_t)Y;
      hi[j] = (uint32_t)(Y >> 32);
    }
    const int kk = kk_of(4 * g);
#pragma unroll
    for (int p = 0; p < S; ++p) {
      const int byte = S - 1 - p;
      uint32_t w = 0;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const uint32_t src = byte < 4 ? (lo[j] >> (8 * byte)) : (hi[j] >> (8 * (byte - 4)));
        w |= (src & 255u) << (8 * j);
      }
      if (p > 0) w ^= 0x80808080u;
      *(uint32_t*)(st + (p * RT + r) * OPITCH + kk) = w;
    }
  }
  __syncthreads();
  write_rows<S, DKT>(st, out, a.plane_stride, a.rows, a.Kp, row0, k0);
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

cudaError_t launch_ozaki_slice_pair(const PlaneArgs& a, int32_t* ea, const PlaneArgs& b, int32_t* eb, int slices,
                                    cudaStream_t st) {
  const long items_a = (a.rows + RT - 1) / RT * a.batch, items_b = (b.rows + RT - 1) / RT * b.batch;
  const long chunks_a = items_a * ((a.K + DKT - 1) / DKT), chunks_b = items_b * ((b.K + DKT - 1) / DKT);
  if (items_a + items_b < 2L * num_sms() || chunks_a + chunks_b >= (1L << 31)) {
    cudaError_t e = launch_ozaki_slice(a, slices, ea, st);
    return e != cudaSuccess ? e : launch_ozaki_slice(b, slices, eb, st);
  }
  // enough rows to fill the GPU: exponents of both operands, then digits of both, per chunk
  {
    ProfScope prof("ozaki_rowexp", st);
    ozaki_rowexp_kernel<<<(unsigned)(items_a + items_b), NTH, 0, st>>>(a, ea, items_a, b, eb);
    note_launch();
  }
  ProfScope prof("ozaki_slice", st);
  const unsigned g = (unsigned)(chunks_a + chunks_b);
  switch (slices) {
    case 3: ozaki_digits_kernel<3><<<g, NTH, 0, st>>>(a, ea, chunks_a, b, eb); break;
    case 4: ozaki_digits_kernel<4><<<g, NTH, 0, st>>>(a, ea, chunks_a, b, eb); break;
    case 5: ozaki_digits_kernel<5><<<g, NTH, 0, st>>>(a, ea, chunks_a, b, eb); break;
    case 6: ozaki_digits_kernel<6><<<g, NTH, 0, st>>>(a, ea, chunks_a, b, eb); break;
    case 7: ozaki_digits_kernel<7><<<g, NTH, 0, st>>>(a, ea, chunks_a, b, eb); break;
    case 8: ozaki_digits_kernel<8><<<g, NTH, 0, st>>>(a, ea, chunks_a, b, eb); break;
    default: return cudaErrorInvalidValue;
  }
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_ozaki_slice(const PlaneArgs& a, int slices, int32_t* exps, cudaStream_t st) {
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
      case 3: ozaki_digits_kernel<3><<<(unsigned)chunks, NTH, 0, st>>>(a, exps, chunks, a, exps); break;
      case 4: ozaki_digits_kernel<4><<<(unsigned)chunks, NTH, 0, st>>>(a, exps, chunks, a, exps); break;
      case 5: ozaki_digits_kernel<5><<<(unsigned)chunks, NTH, 0, st>>>(a, exps, chunks, a, exps); break;
      case 6: ozaki_digits_kernel<6><<<(unsigned)chunks, NTH, 0, st>>>(a, exps, chunks, a, exps); break;
      case 7: ozaki_digits_kernel<7><<<(unsigned)chunks, NTH, 0, st>>>(a, exps, chunks, a, exps); break;
      case 8: ozaki_digits_kernel<8><<<(unsigned)chunks, NTH, 0, st>>>(a, exps, chunks, a, exps); break;
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
