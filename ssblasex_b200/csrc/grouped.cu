// Grouped batched GEMM (ssblasGemmGroupedBatchedEx): thousands of uneven instances in one
// persistent launch per phase.
//
// Phase 1 (pre-pass, one launch per kind): every instance's op(A) and op(B) are converted -- into
//   Ozaki int8 slices (fp64 rows, SSBLAS_MATH_FP64_OZAKI), BF16 hi/lo parts (fp32 rows,
//   SSBLAS_MATH_FP32_BF16X3) or plain int8 (int8 row) -- and written as ready-to-use tensor-core
//   operand tiles: for each (row tile, K block) one contiguous chunk holding all planes, already in
//   the 128B/64B/32B-swizzled K-major layout the MMA reads, zero-padded to whole tiles. Each
//   instance's chunks start at its own offset (a prefix sum over the instances).
// Phase 2 (GEMM, one launch per kind): the persistent tcgen05 kernel walks a device-side tile
//   table (instance, row tile, column tile), longest K first; its producer stages each chunk with a
//   single plain bulk copy, so no per-instance tensor map is needed.
// Plain fp32 instances run on the cp.async FFMA tiles (gemm_sgemm.cu), plain fp64 ones on the FP64
// tensor cores (gemm_dmma.cu), one launch per op(A) / op(B) layout present.
//
// The sequence is captured once per distinct call signature into a CUDA graph and replayed.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

#include "grouped.h"
#include "internal.h"
#include "ozaki_digits.cuh"
#include "tc_gemm.cuh"

namespace ssb {
namespace {

using tc::GInst;
using tc::GTile;

// byte offset of (row r, byte c) inside a [rows][KB] tile stored with the hardware swizzle of a
// KB-byte span (16-byte chunk index XOR a function of the row, Swizzle<log2(KB/16), 4, 3>)
__device__ __forceinline__ uint32_t swz(int r, int c, int KB) {
  const int x = (KB == 128) ? (r & 7) : (KB == 64) ? ((r >> 1) & 3) : ((r >> 2) & 1);
  return (uint32_t)(r * KB + ((((c >> 4) ^ x) << 4) | (c & 15)));
}

struct GPrepInst {
  const void* const* X;  // pointer array (A or B) of the call
  long idx;              // instance position in the pointer array
  long rows, K, ld;
  int kcontig;
  int tiles;             // row tiles
  int nk;                // K blocks
  long off;              // byte offset of the instance's chunks
  long eoff;             // exponent offset (Ozaki)
};

constexpr int GRT = 32;   // rows per work item
constexpr int GNT = 256;

// One CTA per work item = (operand of an instance, block of 32 rows of it). Only rows and K
// blocks of the matrix are written; the tile padding around them was zeroed when the plan was made.
// MODE 0: int8 copy (1 plane); 1: BF16 hi/lo (2 planes); 2: Ozaki slices (S planes).
//
// The item's rows are converted in K chunks of KC elements. Each thread handles runs of 4
// consecutive k of one row; with the rows contiguous in memory (element (r, k) at X[r + k*ld]) the
// 32 lanes of a warp take the 32 rows (coalesced loads), with K contiguous the lanes take
// consecutive runs of one row. Ozaki items first find their row maxima over all of K (the second
// read, for the digits, mostly hits the caches: an item is at most 32 x 16384 values and usually
// 32 x 512). The converted words are staged per (K block, plane) as [32 rows][KB + 4 bytes]
// (conflict-free word stores) and leave as 16-byte vectors into the pre-swizzled tile layout the
// grouped GEMM stages with bulk copies: for each (row tile, K block) of the instance, P planes of
// [RTILE rows][KB bytes], 16-byte chunks permuted by the hardware swizzle of a KB-byte span.
template <int MODE> struct GElem;
template <> struct GElem<0> { using T = int8_t; };
template <> struct GElem<1> { using T = float; };
template <> struct GElem<2> { using T = double; };

template <int MODE, int S, int KB, int RTILE_A, int RTILE_B>
__global__ void __launch_bounds__(GNT, MODE == 2 ? 6 : MODE == 0 ? 6 : 8) gprep_kernel(const GPrepInst* __restrict__ items, const uint2* __restrict__ work,
                                                    uint8_t* __restrict__ outA, uint8_t* __restrict__ outB,
                                                    int32_t* __restrict__ exps) {
  using T = typename GElem<MODE>::T;
  constexpr int P = MODE == 0 ? 1 : MODE == 1 ? 2 : S;
  constexpr int OB = MODE == 1 ? 2 : 1;                     // output bytes per element and plane
  constexpr int KE = KB / OB;                               // K elements per block
  constexpr int KC = MODE == 0 ? 128 : 64;                  // K elements per chunk
  constexpr int NKB = KC / KE;                              // K blocks per chunk
  constexpr int RPR = KC / 4;                               // runs of 4 k per row and chunk
  constexpr int PER = GRT * RPR / GNT;                      // runs per thread and chunk
  constexpr int PB = KB + 4;                                // staged row pitch (bytes)
  constexpr int CPR = KB / 16;                              // 16-byte chunks per staged row
  constexpr int CHT = GRT * CPR;                            // 16-byte chunks per (K block, plane)
  constexpr int BPP = GNT / CHT;                            // (K block, plane) pairs per write pass
  constexpr int NBP = NKB * P;                              // (K block, plane) pairs per chunk
  static_assert(NKB >= 1 && PER >= 1 && RPR >= 8 && RPR <= 32 && GNT % RPR == 0 && GNT % CHT == 0, "chunk shape");
  __shared__ __align__(16) uint8_t stage[NBP * GRT * PB];
  __shared__ double red[8][GRT];
  __shared__ double rscale[GRT][2];

  const uint2 wk = work[blockIdx.x];
  const GPrepInst it = items[wk.x];
  const bool is_b = (wk.x & 1) != 0;
  const int RTILE = is_b ? RTILE_B : RTILE_A;
  uint8_t* out = (is_b ? outB : outA) + it.off;
  const T* X = (const T*)it.X[it.idx];
  const long gr0 = (long)wk.y * GRT;                        // first row (of the padded range)
  const int rt = (int)(gr0 / RTILE), rr0 = (int)(gr0 % RTILE);
  const long K = it.K, ld = it.ld;
  const bool kc = it.kcontig != 0;
  const int t = threadIdx.x, lane = t % 32, warp = t / 32;

  // This thread's runs: row r[q] of the item and first k kq[q] within a chunk. K contiguous: the
  // RPR threads of a row are consecutive lanes; rows contiguous: lane = row (coalesced loads).
  // Element (r, k) is at pq[q][(k - kq[q]) * estep]; rows past the matrix are never read.
  int rq[PER], kq[PER];
  const T* pq[PER];
  bool rv[PER];
  const long estep = kc ? 1 : ld;
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    rq[q] = kc ? t / RPR + q * (GNT / RPR) : lane;
    kq[q] = kc ? 4 * (t % RPR) : 4 * (warp + 8 * q);
    const long gr = gr0 + rq[q];
    rv[q] = gr < it.rows;
    pq[q] = rv[q] ? X + (kc ? gr * ld + kq[q] : gr + kq[q] * ld) : X;
  }
  // 4 consecutive k of a row in one vector load when the row starts are aligned for it
  const bool vec = kc && ((uintptr_t)X % (sizeof(T) == 1 ? 4 : 16)) == 0 && ld % (sizeof(T) == 8 ? 2 : 4) == 0;
  auto load4 = [&](int q, long k0, T (&x)[4]) {
#pragma unroll
    for (int i = 0; i < 4; ++i) x[i] = T(0);
    if (!rv[q]) return;
    const T* p = pq[q] + k0 * estep;
    const long kk = k0 + kq[q];
    if (kk + 4 <= K) {
      if (vec) {
        if constexpr (sizeof(T) == 8) {
          const double2 a = __ldg((const double2*)p), b = __ldg((const double2*)p + 1);
          x[0] = a.x; x[1] = a.y; x[2] = b.x; x[3] = b.y;
        } else if constexpr (sizeof(T) == 4) {
          const float4 a = __ldg((const float4*)p);
          x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
        } else {
          const char4 a = __ldg((const char4*)p);
          x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
        }
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) x[i] = __ldg(p + i * estep);
      }
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (kk + i < K) x[i] = __ldg(p + i * estep);
    }
  };

  // Ozaki: row maxima over all of K (row-maximum keys of |x|, stored in the double buffers bit
  // for bit); the digit pass reads the values again, mostly from L1/L2
  if constexpr (MODE == 2) {
    unsigned long long mx[PER];
    {
      uint32_t mh[PER], ml[PER];
#pragma unroll
      for (int q = 0; q < PER; ++q) mh[q] = ml[q] = 0;
      for (long k0 = 0; k0 < K; k0 += KC) {
#pragma unroll
        for (int q = 0; q < PER; ++q) {
          T x[4];
          load4(q, k0, x);
#pragma unroll
          for (int i = 0; i < 4; ++i) key_fold(x[i], mh[q], ml[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < PER; ++q) mx[q] = key_of(mh[q], ml[q]);
    }
    if (kc) {
      // the RPR threads of a row are consecutive lanes
#pragma unroll
      for (int q = 0; q < PER; ++q) {
#pragma unroll
        for (int off = 1; off < RPR; off <<= 1) mx[q] = max_u64(mx[q], __shfl_xor_sync(0xffffffffu, mx[q], off));
        if (kq[q] == 0) red[0][rq[q]] = __longlong_as_double((long long)mx[q]);
      }
    } else {
      unsigned long long m = mx[0];
#pragma unroll
      for (int q = 1; q < PER; ++q) m = max_u64(m, mx[q]);
      red[warp][lane] = __longlong_as_double((long long)m);
    }
    __syncthreads();
    if (t < GRT) {
      unsigned long long m2 = (unsigned long long)__double_as_longlong(red[0][t]);
      if (!kc)
        for (int w = 1; w < 8; ++w) m2 = max_u64(m2, (unsigned long long)__double_as_longlong(red[w][t]));
      const int e = row_exponent(m2);
      if (gr0 + t < it.rows) exps[it.eoff + gr0 + t] = e;
      row_scale(S, e, rscale[t][0], rscale[t][1]);
    }
    __syncthreads();
  }

  // write-out mapping: this thread's row and 16-byte chunk of a staged (K block, plane) block,
  // and that chunk's place in the hardware-swizzled tile
  const int wr = (t % CHT) / CPR, wc = t % CPR;
  const bool wrow = gr0 + wr < it.rows;
  const uint32_t soff = (uint32_t)(wr * PB + 16 * wc);
  const uint32_t doff = swz(rr0 + wr, 16 * wc, KB);
  const long tile_bytes = (long)P * RTILE * KB;             // one (row tile, K block) chunk, all planes

  // K blocks at or past K are padding, zero since the plan was created: chunks start below K
  for (long k0 = 0; k0 < K; k0 += KC) {
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int r = rq[q], kl = kq[q];
      const int kb = kl / KE, cbyte = (kl % KE) * OB;
      uint8_t* row = stage + (kb * P) * GRT * PB + r * PB + cbyte;
      // rows past the matrix are never written out; a run past K is zero in every plane (the
      // digits, BF16 parts and int8 copy of 0 are all zero bytes)
      if (!rv[q]) continue;
      if (k0 + kl >= K) {
#pragma unroll
        for (int p = 0; p < P; ++p)
#pragma unroll
          for (int w = 0; w < OB; ++w) *(uint32_t*)(row + p * GRT * PB + 4 * w) = 0u;
        continue;
      }
      T x[4];
      load4(q, k0, x);
      if constexpr (MODE == 0) {
        uint32_t w = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i) w |= ((uint32_t)(uint8_t)x[i]) << (8 * i);
        *(uint32_t*)row = w;
      } else if constexpr (MODE == 1) {
        // paired conversions, each value rounded to nearest even as a single conversion would be
        const __nv_bfloat162 h01 = __floats2bfloat162_rn(x[0], x[1]), h23 = __floats2bfloat162_rn(x[2], x[3]);
        const float2 f01 = __bfloat1622float2(h01), f23 = __bfloat1622float2(h23);
        const __nv_bfloat162 l01 = __floats2bfloat162_rn(x[0] - f01.x, x[1] - f01.y);
        const __nv_bfloat162 l23 = __floats2bfloat162_rn(x[2] - f23.x, x[3] - f23.y);
        *(__nv_bfloat162*)row = h01;
        *(__nv_bfloat162*)(row + 4) = h23;
        *(__nv_bfloat162*)(row + GRT * PB) = l01;
        *(__nv_bfloat162*)(row + GRT * PB + 4) = l23;
      } else {
        // rows holding an Inf or a NaN (zero scale) have zero digits
        double xd[4] = {x[0], x[1], x[2], x[3]};
        if (rscale[r][0] == 0.0) xd[0] = xd[1] = xd[2] = xd[3] = 0.0;
        uint32_t wd[S];
        digit_words_rs<S>(xd, rscale[r][0], rscale[r][1], wd);
#pragma unroll
        for (int p = 0; p < P; ++p) *(uint32_t*)(row + p * GRT * PB) = wd[p];
      }
    }
    __syncthreads();
    // write-out: per (K block, plane), 32 rows x KB bytes of the tile, 16-byte chunks swizzled
    if (wrow) {
#pragma unroll
      for (int bp = t / CHT; bp < NBP; bp += BPP) {
        const int kb = bp / P, pl = bp - kb * P;
        const long kbg = k0 / KE + kb;
        if (kbg * KE >= K) continue;
        const uint32_t* src = (const uint32_t*)(stage + bp * GRT * PB + soff);
        const uint4 w = make_uint4(src[0], src[1], src[2], src[3]);
        *(uint4*)(out + ((long)rt * it.nk + kbg) * tile_bytes + (long)pl * RTILE * KB + doff) = w;
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------ host side ---
template <class Cfg>
struct KindPlan {
  std::vector<GInst> inst;
  std::vector<GTile> tiles;
  std::vector<GPrepInst> prep;   // 2 per instance: A then B
  std::vector<uint2> work;       // pre-pass work items: (prep index, 32-row block)
  long bytesA = 0, bytesB = 0, nexp = 0;
};

template <class Cfg>
void plan_kind(const GroupedDesc& g, const std::vector<int>& members, KindPlan<Cfg>& kp) {
  constexpr int KE = Cfg::KB / Cfg::ELEM;
  for (int id : members) {
    const GroupedInst& in = g.inst[id];
    GInst gi{};
    gi.m = in.m; gi.n = in.n; gi.k = in.k; gi.ldc = in.ldc; gi.idx = in.idx;
    gi.alpha_d = in.alpha_d; gi.beta_d = in.beta_d; gi.alpha_f = in.alpha_f; gi.beta_f = in.beta_f;
    gi.alpha_i = in.alpha_i; gi.beta_i = in.beta_i;
    // Ozaki tiles are BM = 128 rows by BN (< BM) columns: when the transposed product C^T =
    // op(B)^T op(A)^T wastes less of its tiles (n on the 128-row side, m on the narrow side), the
    // instance is computed that way -- its rows are then n, its columns m, and the epilogue writes
    // element (i, j) of C^T to C(j, i). (The FP32 and int32 kinds keep the direct orientation: their
    // tiles hold less work per output element, and the transposed stores cost them more than the
    // padding they save.)
    auto padded = [&](long rows, long cols) {
      return ((rows + Cfg::BM - 1) / Cfg::BM) * Cfg::BM * (((cols + Cfg::BN - 1) / Cfg::BN) * Cfg::BN);
    };
    const bool swap = Cfg::EPI == tc::EPI_OZAKI && padded(in.n, in.m) < padded(in.m, in.n);
    const long rows = swap ? in.n : in.m, cols = swap ? in.m : in.n;
    gi.m = rows;
    gi.n = cols;
    gi.swap = swap ? 1 : 0;
    const int tm = (int)((rows + Cfg::BM - 1) / Cfg::BM), tn = (int)((cols + Cfg::BN - 1) / Cfg::BN);
    gi.nk = (int)((in.k + KE - 1) / KE);
    gi.tiles_n = tn;
    gi.offA = kp.bytesA;
    gi.offB = kp.bytesB;
    gi.offEA = kp.nexp;
    gi.offEB = kp.nexp + rows;
    kp.bytesA += (long)tm * gi.nk * Cfg::A_STAGE;
    kp.bytesB += (long)tn * gi.nk * Cfg::B_STAGE;
    kp.nexp += in.m + in.n;
    const int li = (int)kp.inst.size();
    kp.inst.push_back(gi);
    for (int a = 0; a < tm; ++a)
      for (int b = 0; b < tn; ++b) kp.tiles.push_back(GTile{li, a, b});
    // op(A) as rows x K (K contiguous when A is transposed), op(B)^T likewise
    const GPrepInst opa{g.A, in.idx, in.m, in.k, in.lda, in.transa == SSBLAS_OP_T, 0, gi.nk, 0, 0};
    const GPrepInst opb{(const void* const*)g.B, in.idx, in.n, in.k, in.ldb, in.transb == SSBLAS_OP_N, 0, gi.nk, 0, 0};
    GPrepInst pa = swap ? opb : opa, pb = swap ? opa : opb;   // tile rows, tile columns
    pa.tiles = tm; pa.off = gi.offA; pa.eoff = gi.offEA;
    pb.tiles = tn; pb.off = gi.offB; pb.eoff = gi.offEB;
    // only row blocks that hold rows of the matrix: the padding of the tiles is zeroed once, when
    // the plan's buffers are created, and no call writes it again
    for (long rb = 0; rb < (pa.rows + GRT - 1) / GRT; ++rb) kp.work.push_back(make_uint2((unsigned)kp.prep.size(), (unsigned)rb));
    kp.prep.push_back(pa);
    for (long rb = 0; rb < (pb.rows + GRT - 1) / GRT; ++rb) kp.work.push_back(make_uint2((unsigned)kp.prep.size(), (unsigned)rb));
    kp.prep.push_back(pb);
  }
  // longest K first: the persistent CTAs then finish close together
  std::stable_sort(kp.tiles.begin(), kp.tiles.end(),
                   [&](const GTile& x, const GTile& y) { return kp.inst[x.inst].nk > kp.inst[y.inst].nk; });
}

// Device copies of the tables of one kind, owned by a cached plan.
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t n) { return cudaMalloc(&p, n ? n : 16); }
};

struct KindDev {
  DevBuf inst, tiles, prep, work, packA, packB, exps, queue;
  long ninst = 0, ntiles = 0, nwork = 0;
};

template <class Cfg>
cudaError_t upload_kind(const KindPlan<Cfg>& kp, KindDev& kd, cudaStream_t st) {
  cudaError_t e;
  if ((e = kd.inst.alloc(sizeof(GInst) * kp.inst.size())) || (e = kd.tiles.alloc(sizeof(GTile) * kp.tiles.size())) ||
      (e = kd.prep.alloc(sizeof(GPrepInst) * kp.prep.size())) || (e = kd.work.alloc(sizeof(uint2) * kp.work.size())) ||
      (e = kd.packA.alloc(kp.bytesA)) || (e = kd.queue.alloc(sizeof(unsigned long long))) ||
      (e = kd.packB.alloc(kp.bytesB)) || (e = kd.exps.alloc(sizeof(int32_t) * (kp.nexp + 1))))
    return e;
  if ((e = cudaMemcpyAsync(kd.inst.p, kp.inst.data(), sizeof(GInst) * kp.inst.size(), cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(kd.tiles.p, kp.tiles.data(), sizeof(GTile) * kp.tiles.size(), cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(kd.prep.p, kp.prep.data(), sizeof(GPrepInst) * kp.prep.size(), cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(kd.work.p, kp.work.data(), sizeof(uint2) * kp.work.size(), cudaMemcpyHostToDevice, st)))
    return e;
  if ((e = cudaMemsetAsync(kd.packA.p, 0, kp.bytesA, st)) || (e = cudaMemsetAsync(kd.packB.p, 0, kp.bytesB, st)))
    return e;
  kd.nwork = (long)kp.work.size();
  kd.ninst = (long)kp.inst.size();
  kd.ntiles = (long)kp.tiles.size();
  return cudaStreamSynchronize(st);   // the host tables are temporaries
}

template <class Cfg, int MODE, int S>
cudaError_t launch_kind(const KindDev& kd, void* const* C, cudaStream_t st, const char* prep_name,
                        const char* gemm_name, bool dynamic_order) {
  if (kd.ninst == 0) return cudaSuccess;
  {
    ProfScope prof(prep_name, st);
    if (kd.nwork >= (1L << 31)) return cudaErrorInvalidValue;
    gprep_kernel<MODE, S, Cfg::KB, Cfg::BM, Cfg::BN><<<(unsigned)kd.nwork, GNT, 0, st>>>(
        (const GPrepInst*)kd.prep.p, (const uint2*)kd.work.p, (uint8_t*)kd.packA.p, (uint8_t*)kd.packB.p,
        (int32_t*)kd.exps.p);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  static bool attr_set[kMaxDevices] = {};
  if (cudaError_t e = smem_attr_once(attr_set, tc::tc_gemm_kernel<Cfg, true>, Cfg::SMEM)) return e;
  tc::Params prm{};
  prm.total_tiles = kd.ntiles;
  prm.tiles_m = prm.tiles_n = 1;
  prm.C = C;
  prm.exp_a = (const int32_t*)kd.exps.p;
  prm.exp_b = (const int32_t*)kd.exps.p;
  prm.exp_shift = -12;
  prm.err = device_error_flag();
  prm.splits = 1;
  prm.ginst = (const GInst*)kd.inst.p;
  prm.gtiles = (const GTile*)kd.tiles.p;
  prm.packA = (const uint8_t*)kd.packA.p;
  prm.packB = (const uint8_t*)kd.packB.p;
  prm.queue = dynamic_order ? (unsigned long long*)kd.queue.p : nullptr;
  // the device-side tile queue starts at tile 0 on every launch (a memset node when captured)
  if (dynamic_order) {
    cudaError_t e = cudaMemsetAsync(kd.queue.p, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
  }
  CUtensorMap dummy;
  memset(&dummy, 0, sizeof(dummy));
  const long grid = kd.ntiles < num_sms() ? kd.ntiles : num_sms();
  ProfScope prof(gemm_name, st);
  tc::tc_gemm_kernel<Cfg, true><<<(unsigned)grid, tc::kThreadsGrouped, Cfg::SMEM, st>>>(dummy, dummy, dummy, prm);
  note_launch();
  return cudaGetLastError();
}

// Ozaki instances: 128 x 64 tiles with one accumulator (configuration 0 of SSBLAS_PATH_GROUPED),
// or 128 x 32 tiles with two, so that a tile's epilogue overlaps the next tile's MMAs (1, the
// default: most tiles of an uneven batch are short in K, and their epilogues dominate)
using GCfgOz = tc::Config<tc::KIND_I8, 7, 7, 64, 32, 5, 7, 1, tc::EPI_OZAKI, 2>;
using GCfgOz32 = tc::Config<tc::KIND_I8, 7, 7, 32, 32, 6, 7, 2, tc::EPI_OZAKI, 2>;
using GCfgBf = tc::Config<tc::KIND_BF16, 2, 2, 64, 128, 4, 1, 2, tc::EPI_F32, 1>;
using GCfgI8 = tc::Config<tc::KIND_I8, 1, 1, 128, 128, 6, 1, 2, tc::EPI_I32, 0>;

// A prepared grouped call: device tables and packed buffers per kind, the plain-instance batch,
// and (after the first replay request) the captured CUDA graph of all its launches.
struct Plan {
  std::vector<uint64_t> key;
  bool dynamic = true;       // tiles from the device-side queue (else the static stride)
  // Ozaki instances by tile shape: oz on 128 x 32 tiles with two accumulators, oz_wide on
  // 128 x 64 tiles with one (chosen per instance size bucket)
  KindDev oz, oz_wide, bf, i8;
  std::unique_ptr<GroupedSimt> simt;
  void* const* C = nullptr;
  cudaGraphExec_t exec = nullptr;
  int launches = 0;
  ~Plan() {
    if (exec) cudaGraphExecDestroy(exec);
  }
};

std::map<int, std::unique_ptr<Plan>> g_plans;   // one cached plan per device

// Tile shape of one Ozaki instance: 128 x 64 tiles with one accumulator read the slice planes from
// shared memory a third more efficiently per product than 128 x 32 tiles with two, whose gain is
// an epilogue that overlaps the next tile's MMAs. Per size bucket (batch 1) the tuning table may
// choose (SSBLAS_PATH_GROUPED_OZAKI_TILE: 0 = 128 x 64, 1 = 128 x 32); without an entry the tiles
// are 128 x 32: on the 10,000-instance mix (m, n, k log-uniform in [8, 512]) 128 x 64 tiles for
// the instances with k >= 384 and both sides >= 48 took 1.95 ms against 1.80 ms for 128 x 32
// everywhere. The grouped configuration 0 or 2 forces one shape for all.
bool ozaki_wide_tiles(const GroupedInst& in, int gcfg) {
  if (gcfg == 0) return true;
  if (gcfg == 2) return false;
  return choose_config(SSBLAS_PATH_GROUPED_OZAKI_TILE, in.m, in.n, in.k, 1, 1) == 0;
}

std::vector<uint64_t> signature(const GroupedDesc& g, int mode, int oz_cfg) {
  std::vector<uint64_t> k;
  k.reserve(g.inst.size() * 12 + 8);
  k.push_back((uint64_t)mode | ((uint64_t)oz_cfg << 32));
  // a forced DMMA configuration decides whether plain fp64 instances take the tensor cores
  k.push_back((uint64_t)(int64_t)forced_config(SSBLAS_PATH_DMMA));
  k.push_back((uint64_t)(int64_t)forced_config(SSBLAS_PATH_SIMT));
  k.push_back((uint64_t)(uintptr_t)g.A);
  k.push_back((uint64_t)(uintptr_t)g.B);
  k.push_back((uint64_t)(uintptr_t)g.C);
  for (const auto& in : g.inst) {
    uint64_t f[12];
    f[0] = (uint64_t)in.row | ((uint64_t)in.transa << 8) | ((uint64_t)in.transb << 16);
    f[1] = in.m; f[2] = in.n; f[3] = in.k; f[4] = in.lda; f[5] = in.ldb; f[6] = in.ldc; f[7] = in.idx;
    memcpy(&f[8], &in.alpha_d, 8);
    memcpy(&f[9], &in.beta_d, 8);
    uint64_t t;
    memcpy(&t, &in.alpha_f, 4);
    f[10] = t | ((uint64_t)(uint32_t)in.alpha_i << 32);
    memcpy(&t, &in.beta_f, 4);
    f[11] = (t & 0xffffffffu) | ((uint64_t)(uint32_t)in.beta_i << 32);
    k.insert(k.end(), f, f + 12);
  }
  return k;
}

cudaError_t run_plan(Plan& pl, cudaStream_t st) {
  cudaError_t e;
  if ((e = launch_kind<GCfgOz, 2, 7>(pl.oz_wide, pl.C, st, "grouped_ozaki_slice", "grouped_ozaki_gemm", pl.dynamic)))
    return e;
  if ((e = launch_kind<GCfgOz32, 2, 7>(pl.oz, pl.C, st, "grouped_ozaki_slice", "grouped_ozaki_gemm", pl.dynamic)))
    return e;
  if ((e = launch_kind<GCfgBf, 1, 1>(pl.bf, pl.C, st, "grouped_split_bf16", "grouped_bf16x3_gemm", pl.dynamic))) return e;
  if ((e = launch_kind<GCfgI8, 0, 1>(pl.i8, pl.C, st, "grouped_pack_i8", "grouped_i8_gemm", pl.dynamic))) return e;
  if (pl.simt && (e = launch_simt_grouped(*pl.simt, st))) return e;
  if (pl.simt && (e = launch_dmma_grouped(*pl.simt, st))) return e;
  if (pl.simt && (e = launch_sgemm_grouped(*pl.simt, st))) return e;
  return cudaSuccess;
}

}  // namespace

cudaError_t grouped_run(const GroupedDesc& g, cudaStream_t st) {
  const int mode = settings().math_mode;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  // configurations: 0 = every Ozaki instance on 128 x 64 tiles, dynamic tile queue; 1 (default) =
  // the tile shape of each Ozaki instance from its size bucket (SSBLAS_PATH_GROUPED_OZAKI_TILE),
  // dynamic tile queue; 2 = every Ozaki instance on 128 x 32 tiles, static tile order
  const int gcfg = choose_config(SSBLAS_PATH_GROUPED, 0, 0, 0, 0, 1);
  const bool dynamic_order = gcfg != 2;
  std::vector<uint64_t> key = signature(g, mode, gcfg);
  auto it = g_plans.find(dev);
  if (it != g_plans.end() && it->second->key == key) {
    Plan& pl = *it->second;
    if (pl.exec == nullptr) {
      // second call with this signature: capture the launch sequence into a graph
      cudaStream_t cs;
      if ((e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking))) return e;
      cudaGraph_t graph;
      const int before = 0;
      (void)before;
      if ((e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal))) {
        cudaStreamDestroy(cs);
        return e;
      }
      cudaError_t er = run_plan(pl, cs);
      e = cudaStreamEndCapture(cs, &graph);
      cudaStreamDestroy(cs);
      if (er) return er;
      if (e) return e;
      e = cudaGraphInstantiate(&pl.exec, graph, 0);
      cudaGraphDestroy(graph);
      if (e) return e;
    }
    ProfScope prof("grouped_graph", st);
    e = cudaGraphLaunch(pl.exec, st);
    note_launch(pl.launches);
    note_path(SSBLAS_PATH_GROUPED, 7);
    return e;
  }

  // new signature: build the plan
  auto pl = std::make_unique<Plan>();
  pl->key = std::move(key);
  pl->dynamic = dynamic_order;
  pl->C = g.C;
  std::vector<int> oz, oz_wide, bf, i8, plain;
  for (int i = 0; i < (int)g.inst.size(); ++i) {
    const GroupedInst& in = g.inst[i];
    if (in.k <= 0) continue;   // C untouched, as in the reference
    if (in.row == ROW_I8) i8.push_back(i);
    else if (in.row == ROW_F64 && (mode & SSBLAS_MATH_FP64_OZAKI) && in.k <= 16384)
      (ozaki_wide_tiles(in, gcfg) ? oz_wide : oz).push_back(i);
    else if (in.row == ROW_F32 && (mode & SSBLAS_MATH_FP32_BF16X3)) bf.push_back(i);
    else plain.push_back(i);
  }
  {
    KindPlan<GCfgOz32> k1;
    plan_kind(g, oz, k1);
    if ((e = upload_kind(k1, pl->oz, st))) return e;
    KindPlan<GCfgOz> k0;
    plan_kind(g, oz_wide, k0);
    if ((e = upload_kind(k0, pl->oz_wide, st))) return e;
    KindPlan<GCfgBf> k2;
    plan_kind(g, bf, k2);
    if ((e = upload_kind(k2, pl->bf, st))) return e;
    KindPlan<GCfgI8> k3;
    plan_kind(g, i8, k3);
    if ((e = upload_kind(k3, pl->i8, st))) return e;
  }
  if (!plain.empty()) {
    pl->simt = std::make_unique<GroupedSimt>();
    if ((e = plan_simt_grouped(g, plain, *pl->simt, st))) return e;
  }
  pl->launches = (pl->oz.ninst ? 2 : 0) + (pl->oz_wide.ninst ? 2 : 0) + (pl->bf.ninst ? 2 : 0) +
                 (pl->i8.ninst ? 2 : 0) + (pl->simt ? pl->simt->launches : 0);
  g_plans[dev] = std::move(pl);
  Plan& p = *g_plans[dev];
  note_path(SSBLAS_PATH_GROUPED, (p.oz.ninst || p.oz_wide.ninst) ? 7 : 0);
  return run_plan(p, st);
}

void grouped_release() { g_plans.clear(); }

}  // namespace ssb
