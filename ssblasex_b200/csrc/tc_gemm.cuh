// Persistent, warp-specialised tcgen05 GEMM over a batch of (instance, 128 x BN tile) pairs.
//
// Replaces the reference's blocked CPU launcher + packing + SVE microkernel chain
// (launch_kernels/ssblasGemmBatchedEx_Batchgemm_tune_kernel_BMKN.hpp:157-336 for the tile loop,
// src/include/ACopy and BCopy for packing, src/include/GemmCore/Xgemm_kernel_sve_v4x5_1.hpp for
// the register-tile FMA loop, src/include/CScale for the beta pass):
//   - operand tiles are staged by TMA (cp.async.bulk.tensor) straight into the 128B/64B/32B
//     swizzled K-major layout the tensor cores read -- there is no packing pass;
//   - one elected thread issues tcgen05.mma (kind::i8 or kind::f16) accumulating in tensor memory;
//   - four epilogue warps drain tensor memory (tcgen05.ld) and apply alpha/beta in one pass
//     (C is read only when beta != 0, as in src/include/CScale/Xgemm_scale_kernel.hpp:164-176).
//
// An operand may consist of several "planes" (int8 slices of an FP64 value, or the hi/lo BF16
// parts of an FP32 value) stored as [batch][plane][rows][K]. Each stage loads all planes of a
// K block for A and for B with one 4-D TMA each, then multiplies the plane pairs the
// configuration selects; each pair accumulates into the tensor-memory "level" the configuration
// assigns to it.
//
// Warp roles (320 threads): warp 0 = TMA producer, warp 1 = MMA issuer and TMEM owner,
// warps 2-9 = epilogue (warp w reads TMEM lanes 32*(w%4) .. +31, half (w-2)/4 of the columns).
#pragma once

#include <type_traits>

#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "ptx.cuh"

namespace ssb {
namespace tc {

constexpr int kThreads = 320;
// grouped launches add a scheduler warp (warp 10) that feeds the device-side tile queue
constexpr int kThreadsGrouped = 352;
template <bool GROUPED>
constexpr int threads_of() { return GROUPED ? kThreadsGrouped : kThreads; }
// exponent the slicing pre-passes give a row of op(A) / column of op(B) that holds an Inf or a NaN
// (kNonFiniteExp of ozaki_digits.cuh)
constexpr int kOzakiNonFiniteExp = 4096;

enum Kind { KIND_I8 = 0, KIND_BF16 = 1, KIND_F16 = 2 };
enum Epi { EPI_I32 = 0, EPI_F32 = 1, EPI_OZAKI = 2, EPI_F16 = 3 };

// Grouped launches: one entry per instance ...
struct GInst {
  long m, n, k;
  long ldc;
  long idx;                 // position of the instance in the caller's A/B/C pointer arrays
  long offA, offB;          // byte offsets of its packed operand tiles
  long offEA, offEB;        // element offsets of its Ozaki exponents
  int nk;                   // K blocks (stages) per tile
  int tiles_n;
  int swap;                 // 1: the tiles compute C^T = op(B)^T op(A)^T (m and n, the exponents and
                            // the operand packs are those of the transposed product)
  int pad_;
  double alpha_d, beta_d;
  float alpha_f, beta_f;
  int32_t alpha_i, beta_i;
};
// ... and one per output tile, longest K first.
struct GTile {
  int inst;
  int mt, nt;
};

struct Params {
  long m, n, k;             // GEMM shape (k in elements)
  long batch;
  int tiles_m, tiles_n;
  long total_tiles;
  long ldc;
  void* const* C;           // device array of C pointers
  int c_batch_offset;       // instance b of this launch is C[b + c_batch_offset]
  double alpha_d, beta_d;
  float alpha_f, beta_f;
  int32_t alpha_i, beta_i;
  const int32_t* exp_a;     // Ozaki: per-row exponents of op(A), [batch][m]
  const int32_t* exp_b;     // Ozaki: per-column exponents of op(B), [batch][n]
  int exp_shift;            // Ozaki: result = alpha * 2^(ea+eb+exp_shift) * sum_l acc_l 2^(-8 l)
  int* err;                 // device error flag
  // grouped launches only: operands come pre-tiled (already swizzled) from packA/packB and are
  // staged with plain bulk copies; shapes and scalars come from the instance table
  const GInst* ginst;
  const GTile* gtiles;
  const uint8_t* packA;
  const uint8_t* packB;
  unsigned long long* queue;   // grouped launches: tile counter (zero at launch) shared by all CTAs,
                               // or nullptr for the static order (tile blockIdx.x + i * gridDim.x)
  // split-K (batched launches, integer and Ozaki epilogues): work unit u is split u % splits of
  // tile u / splits and covers K blocks [split * kb_per_split, +kb_per_split) of it. Each unit
  // stores its int32 level sums to split_ws ([tile][split][level][BN column][128 rows]); the
  // epilogue warp that arrives last at its region of the tile (split_cnt[tile * 8 + warp - 2],
  // zero at launch) adds the splits' sums in 64 bits and writes C.
  int splits;
  int kb_per_split;
  int32_t* split_ws;
  int* split_cnt;
  // fault injection (ssblasSetFaultInjection): try_wait rounds of every wait (0 = kWaitLimit), and
  // the stage (producer iteration) whose operand copy CTA 0 skips (-1 = none), so that the waits
  // on it run out and the kernel reports through the error flag
  uint32_t wait_limit;
  long skip_copy;
  // int8 kinds: bit 0 = op(A) unsigned, bit 1 = op(B) unsigned (0: both signed)
  int ab_unsigned;
  // the C tensor map (kernel argument tmC, {m, n, batch} of the instances' C) is valid: C_TMA
  // configurations store the Ozaki results with bulk tensor stores when beta == 0
  int c_tma;
};

// Grouped launches take tiles from a device-side queue: a scheduler warp (warp 10) of each CTA
// claims kSB tiles at a time with one atomic add to prm.queue, decodes their instance records
// (lane j fills record j of the batch, so the batch costs one chain of dependent loads, not kSB),
// and passes them to the TMA, MMA and epilogue warps through a ring of kTQ shared-memory slots
// (tq_full: record written; tq_empty: the TMA warp, the MMA warp and the 8 epilogue warps are done
// with it). The scheduler runs up to kTQ records ahead, so the claims and the record loads are off
// the other warps' paths. A record with valid == 0 ends the CTA's tile sequence.
constexpr int kTQ = 16;
constexpr int kSB = kTQ / 2;
struct TileDesc {
  GInst g;
  const void* cptr;         // the instance's C pointer
  int mt, nt, valid, pad;
};
constexpr int kTileQueueBytes = 4096;   // 2 x kTQ barriers + kTQ records

struct TileInfo {
  int b, mt, nt;
  int kb0, kb1;             // K blocks [kb0, kb1) of the tile
  int sp;                   // split index
};

// work unit t of a batched launch -> instance, tile, K range
__device__ __forceinline__ TileInfo tile_info(const Params& p, long t, long tiles_mn, int nk) {
  TileInfo ti;
  const long tile = p.splits > 1 ? t / p.splits : t;
  ti.sp = (int)(t - tile * p.splits);
  ti.b = (int)(tile / tiles_mn);
  const long r = tile % tiles_mn;
  ti.mt = (int)(r / p.tiles_n);
  ti.nt = (int)(r % p.tiles_n);
  ti.kb0 = ti.sp * p.kb_per_split;
  ti.kb1 = min(nk, ti.kb0 + p.kb_per_split);
  return ti;
}

template <int KIND_, int PA_, int PB_, int BN_, int KB_, int STAGES_, int NLEV_, int ACCB_, int EPI_, int PAIRS_,
          int AMN_ = 0, int BMN_ = 0, int OPT_ = 0>
struct Config {
  static constexpr int KIND = KIND_;
  static constexpr int PA = PA_;       // planes of A
  static constexpr int PB = PB_;       // planes of B
  static constexpr int BM = 128;
  static constexpr int BN = BN_;
  static constexpr int KB = KB_;       // bytes of K per stage (= swizzle span)
  static constexpr int STAGES = STAGES_;
  static constexpr int NLEV = NLEV_;   // accumulator levels
  static constexpr int ACCB = ACCB_;   // accumulator buffers (2 = epilogue overlaps next tile)
  static constexpr int EPI = EPI_;
  static constexpr int PAIRS = PAIRS_; // 0: (0,0) only; 1: p+q <= 1 (bf16x3); 2: p+q < NLEV (Ozaki)
  // Operand staging: K-major (K contiguous, the packed planes and transposed inputs) or MN-major
  // (M or N contiguous: the caller's column-major op(A) = A, op(B) = B^T staged as they lie, so
  // the transpose costs nothing). MN-major tiles are blocks of 128 bytes of M (N) by the stage's
  // K rows, each K row one 128-byte swizzled line.
  static constexpr bool AMN = AMN_ != 0;
  static constexpr bool BMN = BMN_ != 0;
  // Ozaki options (bit 0): an A slice plane whose products need two MMAs (more B planes than one
  // MMA's N) is read from shared memory once and kept in the tensor core's A collector for the
  // second; (bit 1) the epilogue drains the accumulator in four batches of tensor-memory loads,
  // each issued before the previous batch is combined, so only the first load latency is exposed
  static constexpr bool AREUSE = (OPT_ & 1) != 0;
  static constexpr bool DRAIN_PIPE = (OPT_ & 2) != 0;
  // (bit 2) the producer prefetches into L2 the tiles of the K block 2 * STAGES ahead of the one it
  // loads; (bit 3) each stage arrives in two parts with their own barriers -- A planes 0-3 with all
  // B planes, then A planes 4-7 (the A stage holds 8 plane slots, the 8th zero-filled) -- so the
  // MMAs of A planes 0-3 (79% of a stage's products for 7 slices) start before the rest lands
  static constexpr bool L2_PREFETCH = (OPT_ & 4) != 0;
  static constexpr bool SPLIT_STAGE = (OPT_ & 8) != 0;
  // (bit 4) Ozaki epilogue with beta == 0 and a C tensor map: each epilogue warp writes its
  // 32 x 16 outputs to a 4 KB shared-memory buffer and one lane hands them to a bulk tensor store,
  // so the warp is free for the next tile's accumulator instead of waiting on its global stores
  static constexpr bool C_TMA = (OPT_ & 16) != 0;
  // (bit 5) two-part accumulator release (Ozaki, one accumulator): the levels are split into a
  // top group (the last TOPN, which the Horner pass reads first) and a bottom group, and every
  // MMA stays inside one group. The epilogue hands the top group back as soon as it has read it;
  // the MMA warp then issues the next tile's top-group products of its first STAGES K blocks and
  // only waits for the bottom group after them, so the drain of the bottom levels (and their
  // conversions) overlaps tensor-core work instead of stalling it. Same products, same Horner
  // order: the results are bit for bit those of the other configurations. Measured slower than
  // the ungrouped order on 32 x 1024^3 (GEMM 0.70 against 0.62 ms): MMAs confined to a group are
  // more and narrower (11 per K step instead of 10, one N = 256 instead of four), and that costs
  // more tensor time than the hidden drain saves.
  static constexpr bool EARLY = (OPT_ & 32) != 0;
  // (bit 7, with bit 5) a top group of two levels instead of three (13 MMAs per K step; measured
  // 0.71 ms)
  static constexpr int TOPN = (OPT_ & 128) ? 2 : 3;
  static constexpr int TOP0 = NLEV_ - TOPN;           // first level of the top group
  static constexpr int C_STAGING = C_TMA ? 8 * 32 * 16 * 8 : 0;
  static constexpr int A_SLOTS = SPLIT_STAGE ? 8 : PA_;
  static_assert(!SPLIT_STAGE || (PAIRS_ == 2 && PA_ > 4 && PA_ <= 8 && !AREUSE), "split stages: Ozaki, 5-8 slices");
  static_assert(!EARLY || (PAIRS_ == 2 && ACCB_ == 1 && NLEV_ >= 4 && !AREUSE && !SPLIT_STAGE && !DRAIN_PIPE),
                "two-part release: Ozaki, one accumulator, plain MMA order");
  static constexpr int ELEM = (KIND == KIND_I8) ? 1 : 2;
  static constexpr int KROWS = KB_ / ELEM;             // K elements (MN-major: K rows) per stage
  static constexpr int MN_BLOCK = KROWS * 128;         // bytes of one 128-byte-wide MN block
  static_assert(!(AMN || BMN) || (PA_ == 1 && PB_ == 1 && PAIRS_ == 0 && KB_ == 128),
                "MN-major staging is for single-plane operands with 128-byte K stages");
  // split-K adds the pieces' sums afterwards: only exact integer sums give the unsplit result
  static constexpr bool SPLITTABLE = EPI_ == EPI_I32 || EPI_ == EPI_OZAKI;
  static constexpr int A_STAGE = A_SLOTS * BM * KB;
  static constexpr int B_STAGE = PB * BN * KB;
  static constexpr int STAGE = A_STAGE + B_STAGE;
  static constexpr int TMEM_COLS_USED = ACCB * NLEV * BN;
  static constexpr int TMEM_COLS = TMEM_COLS_USED <= 32 ? 32 : TMEM_COLS_USED <= 64 ? 64 : TMEM_COLS_USED <= 128 ? 128
                                   : TMEM_COLS_USED <= 256 ? 256 : 512;
  static constexpr int SMEM = 1024 + STAGES * STAGE + 256 + kTileQueueBytes + C_STAGING;
  static_assert(TMEM_COLS_USED <= 512, "tensor memory overflow");
  static_assert(A_STAGE % 1024 == 0 && B_STAGE % 1024 == 0, "stage alignment");
  static_assert(SMEM <= 232448, "shared memory overflow");

  __host__ __device__ static constexpr bool use_pair(int p, int q) {
    return PAIRS == 0 ? (p == 0 && q == 0) : PAIRS == 1 ? (p + q <= 1) : (p + q < NLEV);
  }
  __host__ __device__ static constexpr int level(int p, int q) { return PAIRS == 2 ? p + q : 0; }
  // the first pair (in issue order p-major) that writes a level starts it from zero
  __host__ __device__ static constexpr bool first_of_level(int p, int q) {
    return PAIRS == 2 ? (p == 0) : (p == 0 && q == 0);
  }
};

// Exact integer -> double conversions on the FP64 pipe (the magic-number method: an integer
// placed in the low mantissa bits of a large power of two, which is then subtracted), instead of
// the conversion instructions, which run on the narrow XU pipe and bounded the Horner epilogue.
//   int32 x:  2^52 + (x + 2^31) has x + 2^31 (as an unsigned word) in its low 32 mantissa bits;
//   int64 s, |s| < 2^51:  1.5 * 2^52 + s has s in its low 51 mantissa bits (two's complement).
__device__ __forceinline__ double i32_to_f64(uint32_t x) {
  return __hiloint2double(0x43300000, (int)(x ^ 0x80000000u)) - 0x1.000008p52;
}
__device__ __forceinline__ double i64_to_f64(long long s) {
  return __longlong_as_double(s + 0x4338000000000000ll) - 0x1.8p52;
}

// C value of one Ozaki output: alpha * v * 2^(ea + eb + exp_shift) + beta * old (old is only used,
// and must only be read, when beta != 0); the quiet NaN when the row or column held an Inf or NaN.
__device__ __forceinline__ double ozaki_value(double v, int ea, int eb, int exp_shift, double alpha_d, double beta_d,
                                              double old) {
  const int E = ea + eb + exp_shift;
  const double tb = (beta_d == 0.0) ? 0.0 : beta_d * old;
  // v * 2^E: one multiplication by the exact power of two when 2^E is a normal double (correctly
  // rounded, so equal to scalbn), scalbn otherwise
  if (E >= -1022 && E <= 1023) return fma(v * __longlong_as_double((long long)(E + 1023) << 52), alpha_d, tb);
  // row i of op(A) or column j of op(B) holds an Inf or a NaN
  if (ea == kOzakiNonFiniteExp || eb == kOzakiNonFiniteExp) return __longlong_as_double((long long)0x7FF8000000000000ull);
  return fma(scalbn(v, E), alpha_d, tb);
}

// Ozaki epilogue of one thread's row gi: C(gi, j) = alpha * v_j * 2^(ea + eb_j + exp_shift) + beta * C
// for the columns j = n0 + 16c + jj below n; element (i, j) of C is at Cd[i * rs + j * cs]. The
// column exponents come from exb, or (PRE) from registers loaded before the accumulator was ready.
// Each output is computed and stored with 2^E built as a normal double when E is in [-1022, 1023];
// the others (huge or tiny scale factors, and the sentinel exponent of rows/columns holding Inf or
// NaN) are only flagged, then redone through ozaki_value in a block entered only when a flag is
// set -- so the common path carries no trace of scalbn and the NaN case, and every result equals
// ozaki_value's bit for bit. When a thread's 16 outputs are adjacent in memory (cs = 1: a
// transposed grouped tile) and 16-byte aligned, they are written as 8 two-double vectors. C is
// written with evict-first (streaming) stores: nothing here reads it again, and the operand tiles
// keep L2.
template <int CH, bool PRE = false>
__device__ __forceinline__ void ozaki_store(double* Cd, long gi, long n0, long n, long rs, long cs, int32_t ea,
                                            const int32_t* exb, int exp_shift, double alpha_d, double beta_d,
                                            const double (&v)[CH][16], const int32_t (*ebp)[16] = nullptr) {
  static_assert(CH <= 2, "flag bits");
  if constexpr (PRE && CH == 1) {
    double* row = Cd + gi * rs + n0;
    if (cs == 1 && n0 + 16 <= n && ((uintptr_t)row & 15) == 0) {
      double w[16];
      bool rare = false;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int E = ea + ebp[0][j] + exp_shift;
        rare |= (unsigned)(E + 1022) > 2045u;
        const double tb = (beta_d == 0.0) ? 0.0 : beta_d * row[j];
        w[j] = fma(v[0][j] * __longlong_as_double((long long)(E + 1023) << 52), alpha_d, tb);
      }
      if (!rare) {
#pragma unroll
        for (int h = 0; h < 8; ++h) __stcs((double2*)row + h, make_double2(w[2 * h], w[2 * h + 1]));
        return;
      }
    }
  }
  uint32_t slow = 0u;   // bit 16c + j: output (c, j) needs ozaki_value
#pragma unroll
  for (int c = 0; c < CH; ++c)
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const long gj = n0 + c * 16 + j;
      if (gj < n) {
        const int E = ea + (PRE ? ebp[c][j] : exb[gj]) + exp_shift;
        double* cp = Cd + gi * rs + gj * cs;
        if ((unsigned)(E + 1022) <= 2045u) {
          const double tb = (beta_d == 0.0) ? 0.0 : beta_d * (*cp);
          __stcs(cp, fma(v[c][j] * __longlong_as_double((long long)(E + 1023) << 52), alpha_d, tb));
        } else {
          slow |= 1u << (16 * c + j);
        }
      }
    }
  if (slow) {
#pragma unroll
    for (int c = 0; c < CH; ++c)
#pragma unroll
      for (int j = 0; j < 16; ++j)
        if ((slow >> (16 * c + j)) & 1u) {
          const long gj = n0 + c * 16 + j;
          double* cp = Cd + gi * rs + gj * cs;
          __stcs(cp, ozaki_value(v[c][j], ea, PRE ? ebp[c][j] : exb[gj], exp_shift, alpha_d, beta_d,
                                 (beta_d == 0.0) ? 0.0 : *cp));
        }
  }
}

// int32 epilogue of one thread's row (Ci = &C(gi, 0)): C(gi, j) = alpha * raw + beta * C with
// wrapping int32 arithmetic, columns j = nb + 16c + jj below n. C is read (all reads first) only
// when beta != 0.
template <int GC>
__device__ __forceinline__ void i32_store(int32_t* Ci, long nb, long n, long ldc, int32_t alpha_i, int32_t beta_i,
                                          const uint32_t (&raw)[GC][16]) {
  uint32_t cv[GC][16];
  if (beta_i != 0) {
#pragma unroll
    for (int c = 0; c < GC; ++c)
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const long gj = nb + 16 * c + j;
        cv[c][j] = (gj < n) ? (uint32_t)__ldcs(Ci + gj * ldc) : 0u;
      }
  }
#pragma unroll
  for (int c = 0; c < GC; ++c)
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const long gj = nb + 16 * c + j;
      if (gj < n) {
        const uint32_t t = (beta_i == 0) ? 0u : (uint32_t)beta_i * cv[c][j];
        __stcs(Ci + gj * ldc, (int32_t)(t + raw[c][j] * (uint32_t)alpha_i));
      }
    }
}

// sum[j] += w[s * unit + j * pitch] over the pieces s < splits, four pieces' loads in flight at
// once (the sums are read once, from L2).
template <int PITCH>
__device__ __forceinline__ void add_pieces(const int32_t* w, long unit, int splits, long long (&sum)[16]) {
  int s = 0;
#pragma unroll 1
  for (; s + 4 <= splits; s += 4) {
    int32_t x[4][16];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int j = 0; j < 16; ++j) x[u][j] = __ldcg(w + (s + u) * unit + j * PITCH);
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int j = 0; j < 16; ++j) sum[j] += x[u][j];
  }
#pragma unroll 1
  for (; s < splits; ++s) {
    int32_t x[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) x[j] = __ldcg(w + s * unit + j * PITCH);
#pragma unroll
    for (int j = 0; j < 16; ++j) sum[j] += x[j];
  }
}

// Split-K epilogue of one epilogue warp's region of a tile (rows row_in_tile of the warp, columns
// [half * HALF, +HALF) of the tile) for split `sp` of `splits`: store this split's level sums from
// tensor memory to the workspace (the warp's 32 rows of one column are adjacent, so every store
// is one 128-byte line), hand the accumulator back to the MMA warp, then count the arrival. The
// warp that arrives last adds all splits' sums (64-bit, exact) and writes C. Not inlined, so its
// registers do not add to the other epilogue paths'.
template <class Cfg, int HALF>
__device__ __noinline__ void split_k_region(uint32_t t_row, int32_t* split_ws, int* split_cnt, long tile, int splits,
                                            int sp, int half, int region, int row_in_tile, int lane,
                                            uint32_t tempty_bar, bool row_ok, uint8_t* Cb, long gi, long n0, long n,
                                            long ldc, int32_t ea, const int32_t* exb, int exp_shift, double alpha_d,
                                            double beta_d, int32_t alpha_i, int32_t beta_i) {
  constexpr long UNIT = (long)Cfg::NLEV * Cfg::BN * Cfg::BM;   // int32 per (tile, split)
  const long off = (long)half * HALF * Cfg::BM + row_in_tile;
  const int32_t* wt = split_ws + tile * splits * UNIT + off;
  {
    int32_t* wm = split_ws + (tile * splits + sp) * UNIT + off;
#pragma unroll 1
    for (int l = 0; l < Cfg::NLEV; ++l) {
#pragma unroll 1
      for (int c = 0; c < HALF / 16; ++c) {
        uint32_t raw[16];
        ptx::tmem_ld16(t_row + (uint32_t)(l * Cfg::BN + c * 16), raw);
        ptx::tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 16; ++j) __stcg(wm + ((long)l * Cfg::BN + c * 16 + j) * Cfg::BM, (int)raw[j]);
      }
    }
  }
  ptx::tc_fence_before();
  __syncwarp();
  if (lane == 0) ptx::mbar_arrive(tempty_bar);
  __threadfence();   // this lane's sums are visible before the arrival is counted
  __syncwarp();
  int last = 0;
  if (lane == 0) last = atomicAdd(split_cnt + tile * 8 + region, 1) == splits - 1;
  last = __shfl_sync(0xffffffffu, last, 0);
  if (!last) return;
  __threadfence();   // the other splits' sums are read after their arrivals were seen
#pragma unroll 1
  for (int c = 0; c < HALF / 16; ++c) {
    if (n0 + c * 16 >= n) break;   // columns outside C
    if constexpr (Cfg::EPI == EPI_OZAKI) {
      // Horner over the levels (l = NLEV-1 .. 0: v = v * 2^-8 + acc_l), acc_l summed over the splits
      double v[1][16];
#pragma unroll
      for (int j = 0; j < 16; ++j) v[0][j] = 0.0;
#pragma unroll 1
      for (int l = Cfg::NLEV - 1; l >= 0; --l) {
        long long sum[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) sum[j] = 0;
        add_pieces<Cfg::BM>(wt + ((long)l * Cfg::BN + c * 16) * Cfg::BM, UNIT, splits, sum);
#pragma unroll
        for (int j = 0; j < 16; ++j) v[0][j] = fma(v[0][j], 0x1p-8, i64_to_f64(sum[j]));
      }
      if (row_ok) ozaki_store<1>((double*)Cb, gi, n0 + c * 16, n, 1, ldc, ea, exb, exp_shift, alpha_d, beta_d, v);
    } else {
      long long sum[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) sum[j] = 0;
      add_pieces<Cfg::BM>(wt + (long)c * 16 * Cfg::BM, UNIT, splits, sum);
      uint32_t raw[1][16];
#pragma unroll
      for (int j = 0; j < 16; ++j) raw[0][j] = (uint32_t)sum[j];   // the int32 sum, wrapped
      if (row_ok) i32_store<1>((int32_t*)Cb + gi, n0 + c * 16, n, ldc, alpha_i, beta_i, raw);
    }
  }
}

// SPLIT: the split-K form (batched launches with prm.splits > 1); a separate instantiation, so the
// unsplit kernels carry no trace of the split epilogue.
template <class Cfg, bool GROUPED, bool SPLIT = false>
__global__ void __launch_bounds__(threads_of<GROUPED>(), 1)
tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
               const __grid_constant__ CUtensorMap tmC, const Params prm) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* stages = smem;
  uint64_t* bars = (uint64_t*)(smem + Cfg::STAGES * Cfg::STAGE);
  uint64_t* full = bars;
  uint64_t* empty = bars + Cfg::STAGES;
  uint64_t* tfull = bars + 2 * Cfg::STAGES;
  uint64_t* tempty = tfull + 2;
  uint64_t* drain = tempty + 2;
  uint32_t* tmem_slot = (uint32_t*)(drain + 1);
  uint64_t* full_hi = drain + 2;   // split stages: second part of each stage
  uint64_t* tq_full = (uint64_t*)(smem + Cfg::STAGES * Cfg::STAGE + 256);
  uint64_t* tq_empty = tq_full + kTQ;
  TileDesc* tq = (TileDesc*)(tq_empty + kTQ);
  static_assert(2 * kTQ * 8 + kTQ * sizeof(TileDesc) <= kTileQueueBytes, "tile queue size");

  const int warp = threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  int* err = prm.err;
  const uint32_t wl = prm.wait_limit ? prm.wait_limit : ptx::kWaitLimit;

  if (threadIdx.x == 0) {
    for (int s = 0; s < Cfg::STAGES; ++s) {
      ptx::mbar_init(ptx::smem_u32(&full[s]), 1);
      ptx::mbar_init(ptx::smem_u32(&empty[s]), 1);
      if (Cfg::SPLIT_STAGE) ptx::mbar_init(ptx::smem_u32(&full_hi[s]), 1);
    }
    for (int a = 0; a < 2; ++a) {
      ptx::mbar_init(ptx::smem_u32(&tfull[a]), 1);
      ptx::mbar_init(ptx::smem_u32(&tempty[a]), 8);
    }
    ptx::mbar_init(ptx::smem_u32(drain), 1);
    if (GROUPED) {
      for (int q = 0; q < kTQ; ++q) {
        ptx::mbar_init(ptx::smem_u32(&tq_full[q]), 1);
        ptx::mbar_init(ptx::smem_u32(&tq_empty[q]), 10);
      }
    }
    ptx::fence_mbar_init();
  }
  if (!GROUPED && warp == 0 && lane == 0) {
    ptx::prefetch_tmap(&tmA);
    ptx::prefetch_tmap(&tmB);
  }
  if (warp == 1) {
    ptx::tmem_alloc(ptx::smem_u32(tmem_slot), Cfg::TMEM_COLS);
    ptx::tmem_relinquish();
  }
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  // the set-up above (barriers, tensor memory, tensor-map prefetch) touches no global data, so
  // under a programmatic launch it overlaps the end of the kernel before; every global access
  // comes after the wait
  ptx::grid_dep_wait();
  ptx::grid_dep_launch();

  const long tiles_mn = (long)prm.tiles_m * prm.tiles_n;
  const int KE = Cfg::KB / Cfg::ELEM;                       // K elements per stage
  const int nk_uniform = GROUPED ? 0 : (int)((prm.k + KE - 1) / KE);

  if (warp == 0) {
    // ------------------------------------------------------------------ producer ----------
    if (lane == 0) {
      long it = 0;
      bool ok = true;
      for (long i = 0, t = blockIdx.x; ok; ++i, t += gridDim.x) {
        TileInfo ti{};
        const uint8_t* srcA = nullptr;
        const uint8_t* srcB = nullptr;
        if constexpr (GROUPED) {
          // the next record of the tile queue
          const int slot = (int)(i % kTQ);
          if (!ptx::mbar_wait(ptx::smem_u32(&tq_full[slot]), (uint32_t)((i / kTQ) & 1), err, 13, wl)) break;
          const TileDesc& d = tq[slot];
          if (!d.valid) break;
          ti.mt = d.mt; ti.nt = d.nt; ti.kb0 = 0; ti.kb1 = d.g.nk;
          srcA = prm.packA + d.g.offA + (size_t)ti.mt * ti.kb1 * Cfg::A_STAGE;
          srcB = prm.packB + d.g.offB + (size_t)ti.nt * ti.kb1 * Cfg::B_STAGE;
          ptx::mbar_arrive(ptx::smem_u32(&tq_empty[slot]));
        } else {
          if (t >= prm.total_tiles) break;
          ti = tile_info(prm, t, tiles_mn, nk_uniform);
        }
        for (int kb = ti.kb0; kb < ti.kb1; ++kb, ++it) {
          const int s = (int)(it % Cfg::STAGES);
          const uint32_t ph = (uint32_t)((it / Cfg::STAGES) & 1);
          if (!ptx::mbar_wait(ptx::smem_u32(&empty[s]), ph ^ 1, err, 11, wl)) { ok = false; break; }
          if (!GROUPED && it == prm.skip_copy && blockIdx.x == 0) continue;   // injected fault
          const uint32_t fb = ptx::smem_u32(&full[s]);
          uint8_t* sa = stages + (size_t)s * Cfg::STAGE;
          if constexpr (Cfg::SPLIT_STAGE && !GROUPED) {
            // A planes 0-3 and all B planes, then A planes 4-7 (the A map's box holds 4 planes)
            constexpr int HALF_A = 4 * Cfg::BM * Cfg::KB;
            ptx::mbar_arrive_expect_tx(fb, HALF_A + Cfg::B_STAGE);
            ptx::tma_load_4d(ptx::smem_u32(sa), &tmA, fb, kb * KE, ti.mt * Cfg::BM, 0, ti.b);
            ptx::tma_load_4d(ptx::smem_u32(sa + Cfg::A_STAGE), &tmB, fb, kb * KE, ti.nt * Cfg::BN, 0, ti.b);
            const uint32_t fh = ptx::smem_u32(&full_hi[s]);
            ptx::mbar_arrive_expect_tx(fh, HALF_A);
            ptx::tma_load_4d(ptx::smem_u32(sa + HALF_A), &tmA, fh, kb * KE, ti.mt * Cfg::BM, 4, ti.b);
          } else {
          ptx::mbar_arrive_expect_tx(fb, Cfg::STAGE);
          if constexpr (GROUPED) {
            ptx::bulk_load(ptx::smem_u32(sa), srcA + (size_t)kb * Cfg::A_STAGE, Cfg::A_STAGE, fb);
            ptx::bulk_load(ptx::smem_u32(sa + Cfg::A_STAGE), srcB + (size_t)kb * Cfg::B_STAGE, Cfg::B_STAGE, fb);
          } else {
            if constexpr (Cfg::AMN) {
              // tensor map {M, K, 1, batch}: one 128-byte-wide M block per copy
#pragma unroll
              for (int j = 0; j < Cfg::BM * Cfg::ELEM / 128; ++j)
                ptx::tma_load_4d(ptx::smem_u32(sa + j * Cfg::MN_BLOCK), &tmA, fb, ti.mt * Cfg::BM + j * (128 / Cfg::ELEM),
                                 kb * KE, 0, ti.b);
            } else {
              ptx::tma_load_4d(ptx::smem_u32(sa), &tmA, fb, kb * KE, ti.mt * Cfg::BM, 0, ti.b);
            }
            if constexpr (Cfg::BMN) {
#pragma unroll
              for (int j = 0; j < Cfg::BN * Cfg::ELEM / 128; ++j)
                ptx::tma_load_4d(ptx::smem_u32(sa + Cfg::A_STAGE + j * Cfg::MN_BLOCK), &tmB, fb,
                                 ti.nt * Cfg::BN + j * (128 / Cfg::ELEM), kb * KE, 0, ti.b);
            } else {
              ptx::tma_load_4d(ptx::smem_u32(sa + Cfg::A_STAGE), &tmB, fb, kb * KE, ti.nt * Cfg::BN, 0, ti.b);
            }
          }
          }
          if constexpr (Cfg::L2_PREFETCH && !GROUPED) {
            // the tiles of K block kb + 2 STAGES of this output tile into L2, ahead of their loads
            const int kp = kb + 2 * Cfg::STAGES;
            if (kp < ti.kb1) {
              ptx::tma_prefetch_l2_4d(&tmA, kp * KE, ti.mt * Cfg::BM, 0, ti.b);
              ptx::tma_prefetch_l2_4d(&tmB, kp * KE, ti.nt * Cfg::BN, 0, ti.b);
              if constexpr (Cfg::SPLIT_STAGE) ptx::tma_prefetch_l2_4d(&tmA, kp * KE, ti.mt * Cfg::BM, 4, ti.b);
            }
          }
        }
      }
      // no copy may still be in flight when the CTA exits
      for (long j = (it > Cfg::STAGES ? it - Cfg::STAGES : 0); j < it; ++j) {
        ptx::mbar_wait(ptx::smem_u32(&full[j % Cfg::STAGES]), (uint32_t)((j / Cfg::STAGES) & 1), err, 12, wl);
        if (Cfg::SPLIT_STAGE)
          ptx::mbar_wait(ptx::smem_u32(&full_hi[j % Cfg::STAGES]), (uint32_t)((j / Cfg::STAGES) & 1), err, 12, wl);
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------------ MMA issuer --------
    if (lane == 0) {
      const uint32_t IDESC =
          (Cfg::KIND == KIND_I8)
              ? ptx::idesc_i8(128, Cfg::BN, !(prm.ab_unsigned & 1), !(prm.ab_unsigned & 2), Cfg::AMN, Cfg::BMN)
          : (Cfg::KIND == KIND_F16) ? ptx::idesc_f16(128, Cfg::BN, Cfg::AMN, Cfg::BMN)
                                    : ptx::idesc_bf16(128, Cfg::BN);
      long it = 0;
      int tcount = 0;
      bool ok = true;
      for (long t = blockIdx.x; ok; t += gridDim.x, ++tcount) {
        TileInfo ti{};
        int slot = 0;
        if constexpr (GROUPED) {
          slot = tcount % kTQ;
          if (!ptx::mbar_wait(ptx::smem_u32(&tq_full[slot]), (uint32_t)((tcount / kTQ) & 1), err, 24, wl)) break;
          if (!tq[slot].valid) break;
          ti.kb0 = 0;
          ti.kb1 = tq[slot].g.nk;
          ptx::mbar_arrive(ptx::smem_u32(&tq_empty[slot]));   // the MMA warp only needs nk
        } else {
          if (t >= prm.total_tiles) break;
          ti = tile_info(prm, t, tiles_mn, nk_uniform);
        }
        const int acc = tcount % Cfg::ACCB;
        const uint32_t acc_ph = (uint32_t)((tcount / Cfg::ACCB) & 1);
        if constexpr (Cfg::EARLY && !GROUPED) {
          // two-part release: tempty[0] = top group drained, tempty[1] = bottom group drained
          constexpr int MAXQ = 256 / Cfg::BN;
          const uint32_t d_base = tmem_base;
          // the MMAs of one group for one K block in stage s; first = the tile's first K block
          // (the group is a compile-time constant, so every loop below unrolls completely and
          // the descriptors fold into constants plus the stage address)
          auto issue_group = [&](auto top_c, int s, bool first) {
            constexpr bool top = decltype(top_c)::value;
            const uint32_t sa = ptx::smem_u32(stages + (size_t)s * Cfg::STAGE);
            const uint32_t sb = sa + Cfg::A_STAGE;
#pragma unroll
            for (int p = 0; p < Cfg::PA; ++p) {
              const int qlo = top ? (Cfg::TOP0 - p > 0 ? Cfg::TOP0 - p : 0) : 0;
              const int qhi = top ? Cfg::NLEV - 1 - p : Cfg::TOP0 - 1 - p;   // inclusive
#pragma unroll
              for (int q0 = qlo; q0 <= qhi; q0 += MAXQ) {
                const int nq = (qhi - q0 + 1) < MAXQ ? (qhi - q0 + 1) : MAXQ;
                const uint32_t idesc = ptx::idesc_i8(128, nq * Cfg::BN, true, true);
                const uint32_t d = d_base + (uint32_t)((p + q0) * Cfg::BN);
#pragma unroll
                for (int kk = 0; kk < Cfg::KB / 32; ++kk) {
                  const uint64_t ad = ptx::smem_desc_kmajor(sa + p * Cfg::BM * Cfg::KB + kk * 32, Cfg::KB);
                  const uint64_t bd = ptx::smem_desc_kmajor(sb + q0 * Cfg::BN * Cfg::KB + kk * 32, Cfg::KB);
                  // every level of a group is first written by its p = 0 MMA
                  ptx::mma_i8(d, ad, bd, idesc, (!first || kk > 0 || p > 0) ? 1u : 0u);
                }
              }
            }
          };
          if (!ptx::mbar_wait(ptx::smem_u32(&tempty[0]), acc_ph ^ 1, err, 21, wl)) { ok = false; break; }
          ptx::tc_fence_after();
          const long nkb = ti.kb1 - ti.kb0;
          const int D = nkb < Cfg::STAGES ? (int)nkb : Cfg::STAGES;
          // the top-group products of the first D K blocks, while the bottom group drains
          for (int j = 0; j < D; ++j) {
            const long itj = it + j;
            if (!ptx::mbar_wait(ptx::smem_u32(&full[itj % Cfg::STAGES]), (uint32_t)((itj / Cfg::STAGES) & 1), err, 22,
                                wl)) {
              ok = false;
              break;
            }
            ptx::tc_fence_after();
            issue_group(std::true_type{}, (int)(itj % Cfg::STAGES), j == 0);
          }
          if (!ok) break;
          if (!ptx::mbar_wait(ptx::smem_u32(&tempty[1]), acc_ph ^ 1, err, 26, wl)) { ok = false; break; }
          ptx::tc_fence_after();
          for (int j = 0; j < D; ++j) {
            const int s = (int)((it + j) % Cfg::STAGES);
            issue_group(std::false_type{}, s, j == 0);
            ptx::mma_commit(ptx::smem_u32(&empty[s]));
          }
          it += D;
          for (long kb = ti.kb0 + D; kb < ti.kb1; ++kb, ++it) {
            const int s = (int)(it % Cfg::STAGES);
            if (!ptx::mbar_wait(ptx::smem_u32(&full[s]), (uint32_t)((it / Cfg::STAGES) & 1), err, 22, wl)) {
              ok = false;
              break;
            }
            ptx::tc_fence_after();
            issue_group(std::true_type{}, s, false);
            issue_group(std::false_type{}, s, false);
            ptx::mma_commit(ptx::smem_u32(&empty[s]));
          }
          if (!ok) break;
          ptx::mma_commit(ptx::smem_u32(&tfull[0]));
          continue;
        }
        if (!ptx::mbar_wait(ptx::smem_u32(&tempty[acc]), acc_ph ^ 1, err, 21, wl)) { ok = false; break; }
        ptx::tc_fence_after();
        const uint32_t d_base = tmem_base + (uint32_t)(acc * Cfg::NLEV * Cfg::BN);
        for (int kb = ti.kb0; kb < ti.kb1; ++kb, ++it) {
          const int s = (int)(it % Cfg::STAGES);
          const uint32_t ph = (uint32_t)((it / Cfg::STAGES) & 1);
          const bool acc_k = kb > ti.kb0;   // this K block adds to the blocks before it
          if (!ptx::mbar_wait(ptx::smem_u32(&full[s]), ph, err, 22, wl)) { ok = false; break; }
          ptx::tc_fence_after();
          const uint32_t sa = ptx::smem_u32(stages + (size_t)s * Cfg::STAGE);
          const uint32_t sb = sa + Cfg::A_STAGE;
          if constexpr (Cfg::PAIRS == 2) {
            // Ozaki: slice planes q..q+j-1 of B are contiguous rows of one operand and levels
            // p+q..p+q+j-1 are adjacent TMEM column blocks, so one MMA with N = j*BN (<= 256)
            // multiplies A_p by j planes of B at once and adds each product into its own level.
            // Every level is first written by the p = 0 MMAs of the first K step.
            constexpr int MAXQ = 256 / Cfg::BN;
            if constexpr (Cfg::AREUSE) {
              static_assert(Cfg::NLEV <= 2 * MAXQ, "at most two MMAs per A plane");
              // per (A plane, 32-byte K step): its MMAs back to back, the first filling the A
              // collector and the second (when the plane's B planes need two) reusing it
#pragma unroll
              for (int p = 0; p < Cfg::PA; ++p) {
#pragma unroll
                for (int kk = 0; kk < Cfg::KB / 32; ++kk) {
                  const uint64_t ad = ptx::smem_desc_kmajor(sa + p * Cfg::BM * Cfg::KB + kk * 32, Cfg::KB);
                  const uint32_t accum = (acc_k || kk > 0 || p > 0) ? 1u : 0u;
                  if (Cfg::NLEV - p > MAXQ) {
                    const int nq1 = (Cfg::NLEV - p - MAXQ) < MAXQ ? (Cfg::NLEV - p - MAXQ) : MAXQ;
                    ptx::mma_i8_collect<1>(d_base + (uint32_t)(p * Cfg::BN),
                                           ad, ptx::smem_desc_kmajor(sb + kk * 32, Cfg::KB),
                                           ptx::idesc_i8(128, MAXQ * Cfg::BN, true, true), accum);
                    ptx::mma_i8_collect<2>(d_base + (uint32_t)((p + MAXQ) * Cfg::BN), ad,
                                           ptx::smem_desc_kmajor(sb + MAXQ * Cfg::BN * Cfg::KB + kk * 32, Cfg::KB),
                                           ptx::idesc_i8(128, nq1 * Cfg::BN, true, true), accum);
                  } else {
                    ptx::mma_i8(d_base + (uint32_t)(p * Cfg::BN), ad, ptx::smem_desc_kmajor(sb + kk * 32, Cfg::KB),
                                ptx::idesc_i8(128, (Cfg::NLEV - p) * Cfg::BN, true, true), accum);
                  }
                }
              }
            } else {
#pragma unroll
            for (int p = 0; p < Cfg::PA; ++p) {
              if (Cfg::SPLIT_STAGE && p == 4) {
                // the stage's second part: A planes 4-7
                if (!ptx::mbar_wait(ptx::smem_u32(&full_hi[s]), ph, err, 25, wl)) { ok = false; break; }
                ptx::tc_fence_after();
              }
#pragma unroll
              for (int q0 = 0; q0 < Cfg::NLEV - p; q0 += MAXQ) {
                const int nq = (Cfg::NLEV - p - q0) < MAXQ ? (Cfg::NLEV - p - q0) : MAXQ;
                const uint32_t idesc = ptx::idesc_i8(128, nq * Cfg::BN, true, true);
                const uint32_t d = d_base + (uint32_t)((p + q0) * Cfg::BN);
#pragma unroll
                for (int kk = 0; kk < Cfg::KB / 32; ++kk) {
                  const uint64_t ad = ptx::smem_desc_kmajor(sa + p * Cfg::BM * Cfg::KB + kk * 32, Cfg::KB);
                  const uint64_t bd = ptx::smem_desc_kmajor(sb + q0 * Cfg::BN * Cfg::KB + kk * 32, Cfg::KB);
                  ptx::mma_i8(d, ad, bd, idesc, (acc_k || kk > 0 || p > 0) ? 1u : 0u);
                }
              }
            }
            }
          } else {
#pragma unroll
          for (int p = 0; p < Cfg::PA; ++p) {
#pragma unroll
            for (int q = 0; q < Cfg::PB; ++q) {
              if (!Cfg::use_pair(p, q)) continue;
              const uint32_t d = d_base + (uint32_t)(Cfg::level(p, q) * Cfg::BN);
#pragma unroll
              for (int kk = 0; kk < Cfg::KB / 32; ++kk) {
                // one MMA covers 32 bytes of K: 32 / ELEM K rows of an MN-major tile
                const uint64_t ad = Cfg::AMN ? ptx::smem_desc_mnmajor(sa + kk * (32 / Cfg::ELEM) * 128, Cfg::MN_BLOCK)
                                             : ptx::smem_desc_kmajor(sa + p * Cfg::BM * Cfg::KB + kk * 32, Cfg::KB);
                const uint64_t bd = Cfg::BMN ? ptx::smem_desc_mnmajor(sb + kk * (32 / Cfg::ELEM) * 128, Cfg::MN_BLOCK)
                                             : ptx::smem_desc_kmajor(sb + q * Cfg::BN * Cfg::KB + kk * 32, Cfg::KB);
                const uint32_t accum = (acc_k || kk > 0 || !Cfg::first_of_level(p, q)) ? 1u : 0u;
                if (Cfg::KIND == KIND_I8) ptx::mma_i8(d, ad, bd, IDESC, accum);
                else ptx::mma_f16(d, ad, bd, IDESC, accum);
              }
            }
          }
          }
          if (!ok) break;   // a split stage's second part never arrived
          ptx::mma_commit(ptx::smem_u32(&empty[s]));   // frees the stage when these MMAs finish
        }
        if (!ok) break;
        ptx::mma_commit(ptx::smem_u32(&tfull[acc]));     // accumulator ready for the epilogue
      }
      ptx::mma_commit(ptx::smem_u32(drain));
      ptx::mbar_wait(ptx::smem_u32(drain), 0, err, 23, wl);
    }
  } else if (GROUPED && warp == 10) {
    // ------------------------------------------------------------------ scheduler ---------
    if constexpr (GROUPED) {
      // batches of kSB records: lane j < kSB fills record i + j (slot (i + j) % kTQ)
      for (long i = 0;; i += kSB) {
        const long rec = i + lane;
        const int slot = (int)(rec % kTQ);
        bool ok = true;
        if (lane < kSB) ok = ptx::mbar_wait(ptx::smem_u32(&tq_empty[slot]), (uint32_t)(((rec / kTQ) & 1) ^ 1), err, 14, wl);
        // dynamic order: kSB consecutive tiles per claim; static order: the CTA's stride
        unsigned long long base = 0;
        if (prm.queue && lane == 0) base = atomicAdd(prm.queue, (unsigned long long)kSB);
        base = __shfl_sync(0xffffffffu, base, 0);
        const long q = !ok ? prm.total_tiles
                           : prm.queue ? (long)base + lane : (long)blockIdx.x + rec * (long)gridDim.x;
        const bool last = __any_sync(0xffffffffu, lane < kSB && q >= prm.total_tiles);
        if (lane < kSB) {
          TileDesc& d = tq[slot];
          if (q >= prm.total_tiles) {
            d.valid = 0;
          } else {
            const GTile gt = prm.gtiles[q];
            d.g = prm.ginst[gt.inst];
            d.cptr = prm.C[d.g.idx];
            d.mt = gt.mt;
            d.nt = gt.nt;
            d.valid = 1;
          }
          ptx::mbar_arrive(ptx::smem_u32(&tq_full[slot]));
        }
        if (last) break;
      }
    }
  } else {
    // ------------------------------------------------------------------ epilogue ----------
    // 8 warps: warp w reads TMEM lanes 32*(w%4) .. +31 (its rows) and half (w-2)/4 of the columns
    constexpr int HALF = Cfg::BN / 2;
    const int quarter = warp % 4;
    const int half = (warp - 2) / 4;
    const int row_in_tile = quarter * 32 + lane;
    int tcount = 0;
    for (long t = blockIdx.x;; t += gridDim.x, ++tcount) {
      TileInfo ti{};
      int slot = 0;
      if constexpr (GROUPED) {
        slot = tcount % kTQ;
        if (!ptx::mbar_wait(ptx::smem_u32(&tq_full[slot]), (uint32_t)((tcount / kTQ) & 1), err, 32, wl)) break;
        if (!tq[slot].valid) break;
        ti.mt = tq[slot].mt;
        ti.nt = tq[slot].nt;
      } else {
        if (t >= prm.total_tiles) break;
        ti = tile_info(prm, t, tiles_mn, nk_uniform);
      }
      long m = prm.m, n = prm.n, ldc = prm.ldc;
      long rs = 1;   // C(i, j) at C[i * rs + j * cs]
      double alpha_d = prm.alpha_d, beta_d = prm.beta_d;
      float alpha_f = prm.alpha_f, beta_f = prm.beta_f;
      int32_t alpha_i = prm.alpha_i, beta_i = prm.beta_i;
      const int32_t* exa = prm.exp_a + (long)ti.b * prm.m;
      const int32_t* exb = prm.exp_b + (long)ti.b * prm.n;
      uint8_t* Cb;
      if constexpr (GROUPED) {
        const GInst& g = tq[slot].g;
        m = g.m; n = g.n; ldc = g.ldc;
        alpha_d = g.alpha_d; beta_d = g.beta_d; alpha_f = g.alpha_f; beta_f = g.beta_f;
        alpha_i = g.alpha_i; beta_i = g.beta_i;
        exa = prm.exp_a + g.offEA;
        exb = prm.exp_a + g.offEB;
        if (g.swap) { rs = ldc; ldc = 1; }
        Cb = (uint8_t*)tq[slot].cptr;
        // the record is copied: release the slot
        __syncwarp();
        if (lane == 0) ptx::mbar_arrive(ptx::smem_u32(&tq_empty[slot]));
      } else {
        Cb = (uint8_t*)prm.C[ti.b + prm.c_batch_offset];
      }
      // grouped Ozaki tiles are short: the exponents of a 16-column region are loaded while the
      // MMAs still run
      constexpr bool PRE = GROUPED && Cfg::EPI == EPI_OZAKI && HALF == 16;
      int32_t pre_ea = 0;
      int32_t pre_eb[1][16];
      if constexpr (PRE) {
        const long pi = (long)ti.mt * Cfg::BM + row_in_tile, pn0 = (long)ti.nt * Cfg::BN + half * HALF;
        if (pi < m) pre_ea = exa[pi];
#pragma unroll
        for (int j = 0; j < 16; ++j) pre_eb[0][j] = pn0 + j < n ? exb[pn0 + j] : 0;
      }
      const int acc = tcount % Cfg::ACCB;
      const uint32_t acc_ph = (uint32_t)((tcount / Cfg::ACCB) & 1);
      if (!ptx::mbar_wait(ptx::smem_u32(&tfull[acc]), acc_ph, err, 31, wl)) break;
      ptx::tc_fence_after();
      const long gi = (long)ti.mt * Cfg::BM + row_in_tile;
      const long n0 = (long)ti.nt * Cfg::BN + half * HALF;
      const uint32_t t_row = tmem_base + ((uint32_t)(quarter * 32) << 16) +
                             (uint32_t)(acc * Cfg::NLEV * Cfg::BN + half * HALF);
      const bool row_ok = gi < m;
      if constexpr (SPLIT && !GROUPED && Cfg::SPLITTABLE) {
        {
          split_k_region<Cfg, HALF>(t_row, prm.split_ws, prm.split_cnt, t / prm.splits, prm.splits, ti.sp, half,
                                    warp - 2, row_in_tile, lane, ptx::smem_u32(&tempty[acc]), row_ok, Cb, gi, n0, n,
                                    ldc, (Cfg::EPI == EPI_OZAKI && row_ok) ? exa[gi] : 0, exb, prm.exp_shift, alpha_d, beta_d,
                                    alpha_i, beta_i);
          if constexpr (Cfg::EARLY) {
            // the split epilogue drains the whole accumulator before its arrival on tempty[0]
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(ptx::smem_u32(&tempty[1]));
          }
          continue;
        }
      }
      if constexpr (Cfg::EPI == EPI_OZAKI) {
        // Horner over the levels (l = NLEV-1 .. 0: v = v * 2^-8 + acc_l) for this warp's columns,
        // four levels per batch of TMEM loads; then the accumulator is handed back to the MMA
        // warp before the (slower) scaling and global stores.
        constexpr int CH = HALF / 16;
        double v[CH][16];
        if constexpr (Cfg::EARLY) {
          // the top group (levels NLEV-1 .. TOP0: the first TOPN Horner steps), handed back at
          // once; then the bottom group continues the same Horner sequence
#pragma unroll
          for (int c = 0; c < CH; ++c) {
            uint32_t raw[Cfg::TOPN][16];
#pragma unroll
            for (int q = 0; q < Cfg::TOPN; ++q)
              ptx::tmem_ld16(t_row + (uint32_t)((Cfg::NLEV - 1 - q) * Cfg::BN + c * 16), raw[q]);
            ptx::tmem_wait_ld();
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              double x = 0.0;
#pragma unroll
              for (int q = 0; q < Cfg::TOPN; ++q) x = fma(x, 0x1p-8, i32_to_f64(raw[q][j]));
              v[c][j] = x;
            }
          }
          ptx::tc_fence_before();
          __syncwarp();
          if (lane == 0) ptx::mbar_arrive(ptx::smem_u32(&tempty[0]));
#pragma unroll
          for (int c = 0; c < CH; ++c) {
#pragma unroll
            for (int l0 = Cfg::TOP0 - 1; l0 >= 0; l0 -= 4) {
              uint32_t raw[4][16];
#pragma unroll
              for (int q = 0; q < 4; ++q)
                if (l0 - q >= 0) ptx::tmem_ld16(t_row + (uint32_t)((l0 - q) * Cfg::BN + c * 16), raw[q]);
              ptx::tmem_wait_ld();
#pragma unroll
              for (int q = 0; q < 4; ++q)
                if (l0 - q >= 0) {
#pragma unroll
                  for (int j = 0; j < 16; ++j) v[c][j] = fma(v[c][j], 0x1p-8, i32_to_f64(raw[q][j]));
                }
            }
          }
        } else if constexpr (Cfg::DRAIN_PIPE && CH == 2 && Cfg::NLEV == 7) {
          // batches: chunk 0 levels 6..3, chunk 1 levels 6..3, chunk 0 levels 2..0, chunk 1
          // levels 2..0; each batch's loads go out before the previous batch is combined (the
          // same Horner order and operations as below, so the same results bit for bit)
          uint32_t r0[4][16], r1[4][16];
          const uint32_t t0 = t_row, t1 = t_row + 16;
#pragma unroll
          for (int q = 0; q < 4; ++q) ptx::tmem_ld16(t0 + (uint32_t)((6 - q) * Cfg::BN), r0[q]);
          ptx::tmem_wait_ld();
#pragma unroll
          for (int q = 0; q < 4; ++q) ptx::tmem_ld16(t1 + (uint32_t)((6 - q) * Cfg::BN), r1[q]);
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            double x = fma(0.0, 0x1p-8, i32_to_f64(r0[0][j]));
#pragma unroll
            for (int q = 1; q < 4; ++q) x = fma(x, 0x1p-8, i32_to_f64(r0[q][j]));
            v[0][j] = x;
          }
          ptx::tmem_wait_ld();
#pragma unroll
          for (int q = 0; q < 3; ++q) ptx::tmem_ld16(t0 + (uint32_t)((2 - q) * Cfg::BN), r0[q]);
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            double x = fma(0.0, 0x1p-8, i32_to_f64(r1[0][j]));
#pragma unroll
            for (int q = 1; q < 4; ++q) x = fma(x, 0x1p-8, i32_to_f64(r1[q][j]));
            v[1][j] = x;
          }
          ptx::tmem_wait_ld();
#pragma unroll
          for (int q = 0; q < 3; ++q) ptx::tmem_ld16(t1 + (uint32_t)((2 - q) * Cfg::BN), r1[q]);
#pragma unroll
          for (int j = 0; j < 16; ++j)
#pragma unroll
            for (int q = 0; q < 3; ++q) v[0][j] = fma(v[0][j], 0x1p-8, i32_to_f64(r0[q][j]));
          ptx::tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 16; ++j)
#pragma unroll
            for (int q = 0; q < 3; ++q) v[1][j] = fma(v[1][j], 0x1p-8, i32_to_f64(r1[q][j]));
        } else
#pragma unroll
        for (int c = 0; c < CH; ++c) {
#pragma unroll
          for (int j = 0; j < 16; ++j) v[c][j] = 0.0;
#pragma unroll
          for (int l0 = Cfg::NLEV - 1; l0 >= 0; l0 -= 4) {
            uint32_t raw[4][16];
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (l0 - q >= 0) ptx::tmem_ld16(t_row + (uint32_t)((l0 - q) * Cfg::BN + c * 16), raw[q]);
            ptx::tmem_wait_ld();
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (l0 - q >= 0) {
#pragma unroll
                for (int j = 0; j < 16; ++j) v[c][j] = fma(v[c][j], 0x1p-8, i32_to_f64(raw[q][j]));
              }
          }
        }
        ptx::tc_fence_before();
        __syncwarp();
        if (lane == 0) ptx::mbar_arrive(ptx::smem_u32(&tempty[Cfg::EARLY ? 1 : acc]));
        if constexpr (PRE) {
          if (row_ok) ozaki_store<1, true>((double*)Cb, gi, n0, n, rs, ldc, pre_ea, exb, prm.exp_shift, alpha_d, beta_d, v, pre_eb);
        } else {
          bool stored = false;
          if constexpr (Cfg::C_TMA && !GROUPED && CH == 2) {
            if (prm.c_tma && beta_d == 0.0) {
              // every output's scale factor must be a normal double (the branch-free formula) for the
              // bulk store; otherwise the whole region takes ozaki_store's rare-value handling
              const int32_t ea = row_ok ? exa[gi] : 0;
              double w[CH][16];
              bool rare = false;
#pragma unroll
              for (int c = 0; c < CH; ++c)
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                  const long gj = n0 + c * 16 + j;
                  const int E = ea + (gj < n ? exb[gj] : 0) + prm.exp_shift;
                  rare |= row_ok && gj < n && (unsigned)(E + 1022) > 2045u;
                  w[c][j] = fma(v[c][j] * __longlong_as_double((long long)(E + 1023) << 52), alpha_d, 0.0);
                }
              if (!__any_sync(0xffffffffu, rare)) {
                // 32 rows x 16 columns per bulk store: buffer [column][row], rows and columns outside
                // C are dropped by the store
                double* stg = (double*)(stages + Cfg::STAGES * Cfg::STAGE + 256 + kTileQueueBytes) + (warp - 2) * 512;
                const int row0 = ti.mt * Cfg::BM + quarter * 32;
#pragma unroll
                for (int c = 0; c < CH; ++c) {
                  if (n0 + c * 16 >= n) break;
                  if (lane == 0) ptx::bulk_wait_read();   // the previous store has read the buffer
                  __syncwarp();
#pragma unroll
                  for (int j = 0; j < 16; ++j) stg[j * 32 + lane] = w[c][j];
                  ptx::fence_proxy_async_smem();
                  __syncwarp();
                  if (lane == 0) {
                    ptx::tma_store_3d(&tmC, ptx::smem_u32(stg), row0, (int)(n0 + c * 16), ti.b + prm.c_batch_offset);
                    ptx::bulk_commit();
                  }
                }
                stored = true;
              }
            }
          }
          if (!stored && row_ok)
            ozaki_store<CH>((double*)Cb, gi, n0, n, rs, ldc, exa[gi], exb, prm.exp_shift, alpha_d, beta_d, v);
        }
        continue;
      }
      // Groups of up to 64 columns: all TMEM loads, then all C loads (when beta != 0) are issued
      // before any use, so each thread keeps up to 64 reads of C in flight.
      constexpr int G = HALF < 64 ? HALF : 64;
      constexpr int GC = G / 16;
#pragma unroll 1
      for (int g0 = 0; g0 < HALF; g0 += G) {
        if (n0 + g0 >= n) break;   // whole group outside C: nothing to read or write
        uint32_t raw[GC][16];
#pragma unroll
        for (int c = 0; c < GC; ++c) ptx::tmem_ld16(t_row + (uint32_t)(g0 + 16 * c), raw[c]);
        ptx::tmem_wait_ld();
        if (!row_ok) continue;
        if (Cfg::EPI == EPI_I32) {
          i32_store<GC>((int32_t*)Cb + gi * rs, n0 + g0, n, ldc, alpha_i, beta_i, raw);
        } else if (Cfg::EPI == EPI_F16) {
          // fp16 C: alpha * acc + beta * C in fp32, rounded once to fp16
          __half* Ch = (__half*)Cb + gi * rs;
          float cv[GC][16];
          if (beta_f != 0.0f) {
#pragma unroll
            for (int c = 0; c < GC; ++c)
#pragma unroll
              for (int j = 0; j < 16; ++j) {
                const long gj = n0 + g0 + 16 * c + j;
                cv[c][j] = (gj < n) ? __half2float(Ch[gj * ldc]) : 0.0f;
              }
          }
#pragma unroll
          for (int c = 0; c < GC; ++c)
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const long gj = n0 + g0 + 16 * c + j;
              if (gj < n) {
                const float tb = (beta_f == 0.0f) ? 0.0f : beta_f * cv[c][j];
                Ch[gj * ldc] = __float2half_rn(fmaf(__uint_as_float(raw[c][j]), alpha_f, tb));
              }
            }
        } else {
          float* Cf = (float*)Cb + gi * rs;
          float cv[GC][16];
          if (beta_f != 0.0f) {
#pragma unroll
            for (int c = 0; c < GC; ++c)
#pragma unroll
              for (int j = 0; j < 16; ++j) {
                const long gj = n0 + g0 + 16 * c + j;
                cv[c][j] = (gj < n) ? __ldcs(Cf + gj * ldc) : 0.0f;
              }
          }
#pragma unroll
          for (int c = 0; c < GC; ++c)
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const long gj = n0 + g0 + 16 * c + j;
              if (gj < n) {
                const float tb = (beta_f == 0.0f) ? 0.0f : beta_f * cv[c][j];
                __stcs(Cf + gj * ldc, fmaf(__uint_as_float(raw[c][j]), alpha_f, tb));
              }
            }
        }
      }
      ptx::tc_fence_before();
      __syncwarp();
      if (lane == 0) ptx::mbar_arrive(ptx::smem_u32(&tempty[acc]));
    }
  }

  if constexpr (Cfg::C_TMA) {
    // the epilogue's bulk stores complete before the CTA (and its shared memory) goes away
    if (warp >= 2 && lane == 0) ptx::bulk_wait_all();
  }
  ptx::tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    ptx::tc_fence_after();
    ptx::tmem_dealloc(tmem_base, Cfg::TMEM_COLS);
  }
}

}  // namespace tc
}  // namespace ssb
