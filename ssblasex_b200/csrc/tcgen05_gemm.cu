// Host launchers of the tcgen05 paths: int8 -> int32 (direct TMA from the caller's matrices, or
// through the int8 pack pre-pass), FP64 via Ozaki int8 slices, FP32 via three BF16 products.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstring>

#include "internal.h"
#include "prepass.h"
#include "tc_gemm.cuh"

namespace ssb {
namespace {

using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encoder() {
  static EncodeFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return (EncodeFn) nullptr;
    }
    return (EncodeFn)p;
  }();
  return fn;
}

// The current device is an sm_100 part (the only target the tensor-core kernels are built for).
bool is_sm100() {
  static int ok[kMaxDevices] = {};   // 0 unknown, 1 yes, 2 no
  const int dev = current_device();
  if (dev < 0) return false;
  if (!ok[dev]) {
    int major = 0, minor = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    cudaGetLastError();
    ok[dev] = (major == 10 && minor == 0) ? 1 : 2;
  }
  return ok[dev] == 1;
}

// 4-D tiled tensor map: dims {K, rows, planes, batch} (K innermost), strides in bytes.
bool make_map(CUtensorMap* map, const void* base, CUtensorMapDataType dt, long K, long rows, long planes,
              long batch, long row_stride, long plane_stride, long batch_stride, int box_k, int box_rows,
              int box_planes, int swz_bytes) {
  EncodeFn enc = encoder();
  if (!enc) return false;
  cuuint64_t dims[4] = {(cuuint64_t)K, (cuuint64_t)rows, (cuuint64_t)planes, (cuuint64_t)batch};
  cuuint64_t strides[3] = {(cuuint64_t)row_stride, (cuuint64_t)plane_stride, (cuuint64_t)batch_stride};
  cuuint32_t box[4] = {(cuuint32_t)box_k, (cuuint32_t)box_rows, (cuuint32_t)box_planes, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUtensorMapSwizzle sw = swz_bytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                          : swz_bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B
                                            : CU_TENSOR_MAP_SWIZZLE_32B;
  CUresult r = enc(map, dt, 4, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// Split-K plan of one GEMM launch: how many K pieces per output tile.
struct SplitPlan {
  int key = -1;          // ssblasSetKernelConfig key (SSBLAS_PATH_SPLITK_*), -1 = never split
  long min_kb = 1;       // automatic choice: K blocks a piece keeps at least
  long max_kb = 0;       // K blocks a piece may hold at most (0 = no bound)
};

// Number of K pieces: forced or tuned (config = pieces, 0 = automatic), else automatic -- only
// when the tiles fill less than half of the SMs, up to one wave of (tile, piece) units, each
// piece keeping at least min_kb K blocks. A forced count is cut to four waves of units. Never
// below what max_kb requires, never above nk.
int choose_splits(const SplitPlan& sp, long m, long n, long k, long batch, long tiles, long nk) {
  if (sp.key < 0) return 1;
  const long need = sp.max_kb > 0 ? (nk + sp.max_kb - 1) / sp.max_kb : 1;
  long s = choose_config(sp.key, m, n, k, batch, 0);
  if (s > 1 && s * tiles > 4L * num_sms()) s = (4L * num_sms()) / tiles > 1 ? (4L * num_sms()) / tiles : 1;
  if (s == 0) {
    s = 1;
    if (2 * tiles <= num_sms()) {
      s = num_sms() / tiles;
      const long by_k = nk / (sp.min_kb > 0 ? sp.min_kb : 1);
      if (s > by_k) s = by_k;
      if (s > 32) s = 32;
    }
  }
  if (s < need) s = need;
  if (s > nk) s = nk;
  return s < 1 ? 1 : (int)s;
}

// pdl: launch with programmatic stream serialization (the kernel's set-up overlaps the end of the
// kernel before it in the stream; tc_gemm_kernel waits for that kernel before any global access)
template <class Cfg>
cudaError_t run_gemm(const CUtensorMap& ta, const CUtensorMap& tb, tc::Params prm, cudaStream_t st,
                     const char* name, const SplitPlan& plan = SplitPlan(), const CUtensorMap* tcmap = nullptr,
                     bool pdl = false) {
  CUtensorMap tmc;
  if (tcmap) tmc = *tcmap;
  else memset(&tmc, 0, sizeof(tmc));
  static bool attr_set[kMaxDevices] = {};
  static bool attr_set_split[kMaxDevices] = {};
  if (cudaError_t e = smem_attr_once(attr_set, tc::tc_gemm_kernel<Cfg, false, false>, Cfg::SMEM)) return e;
  if constexpr (Cfg::SPLITTABLE)
    if (cudaError_t e = smem_attr_once(attr_set_split, tc::tc_gemm_kernel<Cfg, false, true>, Cfg::SMEM)) return e;
  prm.tiles_m = (int)((prm.m + Cfg::BM - 1) / Cfg::BM);
  prm.tiles_n = (int)((prm.n + Cfg::BN - 1) / Cfg::BN);
  const long tiles = (long)prm.tiles_m * prm.tiles_n * prm.batch;
  constexpr long KE = Cfg::KB / Cfg::ELEM;
  const long nk = (prm.k + KE - 1) / KE;
  prm.splits = 1;
  prm.kb_per_split = (int)nk;
  if (Cfg::SPLITTABLE) {
    const int want = choose_splits(plan, prm.m, prm.n, prm.k, prm.batch, tiles, nk);
    if (want > 1) {
      // pieces of equal K-block count; the last may be shorter, none is empty
      const long kps = (nk + want - 1) / want;
      const int splits = (int)((nk + kps - 1) / kps);
      cudaError_t e;
      const size_t unit = (size_t)Cfg::NLEV * Cfg::BN * Cfg::BM * sizeof(int32_t);
      void* ws = workspace(WS_SPLIT, unit * (size_t)tiles * splits, &e);
      if (!ws) return e;
      void* cnt = workspace(WS_SPLIT_CNT, sizeof(int) * 8 * (size_t)tiles, &e);
      if (!cnt) return e;
      if ((e = cudaMemsetAsync(cnt, 0, sizeof(int) * 8 * (size_t)tiles, st)) != cudaSuccess) return e;
      prm.splits = splits;
      prm.kb_per_split = (int)kps;
      prm.split_ws = (int32_t*)ws;
      prm.split_cnt = (int*)cnt;
    }
  }
  prm.total_tiles = tiles * prm.splits;
  note_splits(prm.splits);
  if (settings().fault == SSBLAS_FAULT_SKIP_COPY) {
    // one-shot test fault: CTA 0 skips its first operand copy, every wait of the launch gives up
    // after a short limit, and the kernel reports through the device error flag
    settings().fault = SSBLAS_FAULT_NONE;
    prm.skip_copy = 0;
    prm.wait_limit = 1u << 10;
  }
  long grid = prm.total_tiles < num_sms() ? prm.total_tiles : num_sms();
  ProfScope prof(name, st);
  if (prm.splits > 1) {
    if constexpr (Cfg::SPLITTABLE)
      tc::tc_gemm_kernel<Cfg, false, true><<<(unsigned)grid, tc::kThreads, Cfg::SMEM, st>>>(ta, tb, tmc, prm);
  } else if (pdl) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid, 1, 1);
    cfg.blockDim = dim3(tc::kThreads, 1, 1);
    cfg.dynamicSmemBytes = Cfg::SMEM;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    note_launch();
    return cudaLaunchKernelEx(&cfg, tc::tc_gemm_kernel<Cfg, false, false>, ta, tb, tmc, prm);
  } else {
    tc::tc_gemm_kernel<Cfg, false, false><<<(unsigned)grid, tc::kThreads, Cfg::SMEM, st>>>(ta, tb, tmc, prm);
  }
  note_launch();
  return cudaGetLastError();
}

tc::Params base_params(const BatchDesc& d) {
  tc::Params p{};
  p.m = d.m; p.n = d.n; p.k = d.k; p.batch = d.batch; p.ldc = d.ldc;
  p.C = d.C;
  p.c_batch_offset = 0;
  p.alpha_d = d.alpha_d; p.beta_d = d.beta_d;
  p.alpha_f = d.alpha_f; p.beta_f = d.beta_f;
  p.alpha_i = d.alpha_i; p.beta_i = d.beta_i;
  p.err = device_error_flag();
  p.splits = 1;
  p.skip_copy = -1;
  return p;
}

inline long round_up(long x, long a) { return (x + a - 1) / a * a; }

// int8 planes of op(A) and op(B), K-major, through the pack pre-pass.
cudaError_t pack_operands_i8(const BatchDesc& d, cudaStream_t st, int8_t** pa, int8_t** pb, long* Kp) {
  cudaError_t e;
  *Kp = round_up(d.k, 16);
  const long sa = d.m * *Kp, sb = d.n * *Kp;
  *pa = (int8_t*)workspace(WS_PACK_A, (size_t)sa * d.batch, &e);
  if (!*pa) return e;
  *pb = (int8_t*)workspace(WS_PACK_B, (size_t)sb * d.batch, &e);
  if (!*pb) return e;
  PlaneArgs a{d.A, d.m, d.k, d.lda, d.transa == SSBLAS_OP_T, d.batch, *pa, *Kp, sa, sa};
  if ((e = launch_pack_i8(a, st)) != cudaSuccess) return e;
  PlaneArgs b{d.B, d.n, d.k, d.ldb, d.transb == SSBLAS_OP_N, d.batch, *pb, *Kp, sb, sb};
  return launch_pack_i8(b, st);
}

using CfgBf64 = tc::Config<tc::KIND_BF16, 2, 2, 64, 128, 4, 1, 2, tc::EPI_F32, 1>;
using CfgBf128 = tc::Config<tc::KIND_BF16, 2, 2, 128, 128, 3, 1, 2, tc::EPI_F32, 1>;
template <int S> struct OzCfg;
template <> struct OzCfg<3> { using T = tc::Config<tc::KIND_I8, 3, 3, 64, 32, 8, 3, 1, tc::EPI_OZAKI, 2>; };
template <> struct OzCfg<4> { using T = tc::Config<tc::KIND_I8, 4, 4, 64, 32, 8, 4, 1, tc::EPI_OZAKI, 2>; };
template <> struct OzCfg<5> { using T = tc::Config<tc::KIND_I8, 5, 5, 64, 32, 7, 5, 1, tc::EPI_OZAKI, 2>; };
template <> struct OzCfg<6> { using T = tc::Config<tc::KIND_I8, 6, 6, 64, 32, 6, 6, 1, tc::EPI_OZAKI, 2>; };
template <> struct OzCfg<7> { using T = tc::Config<tc::KIND_I8, 7, 7, 64, 32, 5, 7, 1, tc::EPI_OZAKI, 2>; };
template <> struct OzCfg<8> { using T = tc::Config<tc::KIND_I8, 8, 8, 64, 32, 4, 8, 1, tc::EPI_OZAKI, 2>; };

// Alternative Ozaki configurations for the default slice count (7), chosen by the autotuner:
//   1: 64-byte K stages (two MMA K steps per slice pair per stage), 2 stages
//   2: 128 x 32 tiles with a double-buffered accumulator (the epilogue overlaps the next tile)
using OzCfg7KB64 = tc::Config<tc::KIND_I8, 7, 7, 64, 64, 2, 7, 1, tc::EPI_OZAKI, 2>;
using OzCfg7N32 = tc::Config<tc::KIND_I8, 7, 7, 32, 32, 6, 7, 2, tc::EPI_OZAKI, 2>;
//   3: configuration 1 with the A collector: an A plane with two MMAs per K step is read from
//      shared memory once
//   4: configuration 1 with the accumulator drained in four overlapped batches of loads
//   5: both
using OzCfg7KB64R = tc::Config<tc::KIND_I8, 7, 7, 64, 64, 2, 7, 1, tc::EPI_OZAKI, 2, 0, 0, 1>;
using OzCfg7KB64D = tc::Config<tc::KIND_I8, 7, 7, 64, 64, 2, 7, 1, tc::EPI_OZAKI, 2, 0, 0, 2>;
using OzCfg7KB64RD = tc::Config<tc::KIND_I8, 7, 7, 64, 64, 2, 7, 1, tc::EPI_OZAKI, 2, 0, 0, 3>;
//   6: configuration 1 with an L2 prefetch of the K block two stages ahead of each load
//   7: configuration 1 with each stage in two parts (A planes 0-3 and B, then A planes 4-6)
//   8: both
using OzCfg7KB64P = tc::Config<tc::KIND_I8, 7, 7, 64, 64, 2, 7, 1, tc::EPI_OZAKI, 2, 0, 0, 4>;
using OzCfg7KB64S = tc::Config<tc::KIND_I8, 7, 7, 64, 64, 2, 7, 1, tc::EPI_OZAKI, 2, 0, 0, 8>;
using OzCfg7KB64SP = tc::Config<tc::KIND_I8, 7, 7, 64, 64, 2, 7, 1, tc::EPI_OZAKI, 2, 0, 0, 12>;
//   9: configuration 1 with the results written by bulk tensor stores (beta == 0)
using OzCfg7KB64T = tc::Config<tc::KIND_I8, 7, 7, 64, 64, 2, 7, 1, tc::EPI_OZAKI, 2, 0, 0, 16>;
//  10: configuration 9 with the accumulator handed back in two parts (the top three levels
//      first), so the next tile's top-level products overlap the drain of the bottom levels;
//  11: the same with a top group of two levels. Both are bit-exact and slower on 32 x 1024^3
//      (GEMM 0.70 / 0.71 ms against 0.62): the grouped MMA order costs more than the drain it hides
using OzCfg7KB64TE = tc::Config<tc::KIND_I8, 7, 7, 64, 64, 2, 7, 1, tc::EPI_OZAKI, 2, 0, 0, 48>;
using OzCfg7KB64TE2 = tc::Config<tc::KIND_I8, 7, 7, 64, 64, 2, 7, 1, tc::EPI_OZAKI, 2, 0, 0, 176>;

// Ozaki split-K: a piece holds at most 16384 k (its int32 level sums stay exact); automatic
// pieces keep at least 512 k.
constexpr long kOzakiMaxPieceK = 16384;
template <class Cfg>
SplitPlan ozaki_split_plan(bool allow_split) {
  SplitPlan p;
  if (!allow_split) return p;
  constexpr long KE = Cfg::KB / Cfg::ELEM;
  p.key = SSBLAS_PATH_SPLITK_OZAKI;
  p.min_kb = 512 / KE;
  p.max_kb = kOzakiMaxPieceK / KE;
  return p;
}

template <class Cfg>
cudaError_t ozaki_gemm_cfg(const BatchDesc& d, int S, const int8_t* pa, const int8_t* pb, const int32_t* exa,
                           const int32_t* exb, long Kp, bool allow_split, cudaStream_t st) {
  const long sa = d.m * Kp, sb = d.n * Kp;
  CUtensorMap ta, tb;
  // split stages load A in two boxes of 4 planes (the second reads planes 4-7; planes past S are
  // outside the tensor and arrive as zeros)
  if (!make_map(&ta, pa, CU_TENSOR_MAP_DATA_TYPE_UINT8, d.k, d.m, S, d.batch, Kp, sa, sa * S, Cfg::KB, 128,
                Cfg::SPLIT_STAGE ? 4 : S, Cfg::KB) ||
      !make_map(&tb, pb, CU_TENSOR_MAP_DATA_TYPE_UINT8, d.k, d.n, S, d.batch, Kp, sb, sb * S, Cfg::KB, Cfg::BN, S,
                Cfg::KB))
    return cudaErrorNotSupported;
  tc::Params prm = base_params(d);
  prm.exp_a = exa;
  prm.exp_b = exb;
  prm.exp_shift = -12;
  note_path(SSBLAS_PATH_OZAKI_TCGEN05, S);
  // bulk tensor stores of C: beta == 0 and C instances addressable by one 3-D map
  CUtensorMap tcm;
  const CUtensorMap* tcp = nullptr;
  if constexpr (Cfg::C_TMA) {
    const bool uniform = d.batch == 1 || d.strideC > 0;
    if (d.beta_d == 0.0 && d.C0 && uniform && ((uintptr_t)d.C0 % 16) == 0 && (d.ldc * 8) % 16 == 0 &&
        d.strideC % 16 == 0 && d.m < (1L << 31) && d.n < (1L << 31)) {
      const long dims[3] = {d.m, d.n, d.batch};
      const long strides[2] = {d.ldc * 8, d.batch > 1 ? d.strideC : round_up(d.ldc * d.n * 8, 16)};
      const int box[3] = {32, 16, 1};
      if (make_tiled_map(&tcm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, d.C0, dims, strides, box, 0)) {
        prm.c_tma = 1;
        tcp = &tcm;
      }
    }
  }
  // programmatic launch: the set-up overlaps the slicing kernel's last items
  return run_gemm<Cfg>(ta, tb, prm, st, "ozaki_gemm", ozaki_split_plan<Cfg>(allow_split), tcp, true);
}

// exa: exponents of the rows of op(A), [batch][m]; exb: of the columns of op(B), [batch][n]
cudaError_t ozaki_gemm(const BatchDesc& d, int S, const int8_t* pa, const int8_t* pb, const int32_t* exa,
                       const int32_t* exb, long Kp, bool allow_split, cudaStream_t st) {
  switch (S) {
    case 3: return ozaki_gemm_cfg<OzCfg<3>::T>(d, S, pa, pb, exa, exb, Kp, allow_split, st);
    case 4: return ozaki_gemm_cfg<OzCfg<4>::T>(d, S, pa, pb, exa, exb, Kp, allow_split, st);
    case 5: return ozaki_gemm_cfg<OzCfg<5>::T>(d, S, pa, pb, exa, exb, Kp, allow_split, st);
    case 6: return ozaki_gemm_cfg<OzCfg<6>::T>(d, S, pa, pb, exa, exb, Kp, allow_split, st);
    case 7: {
      // 64-byte K stages won every bucket the autotuner measured, so they are the default
      const int c = choose_config(SSBLAS_PATH_OZAKI_TCGEN05, d.m, d.n, d.k, d.batch, 1);
      if (c == 1) return ozaki_gemm_cfg<OzCfg7KB64>(d, S, pa, pb, exa, exb, Kp, allow_split, st);
      if (c == 2) return ozaki_gemm_cfg<OzCfg7N32>(d, S, pa, pb, exa, exb, Kp, allow_split, st);
      if (c == 3) return ozaki_gemm_cfg<OzCfg7KB64R>(d, S, pa, pb, exa, exb, Kp, allow_split, st);
      if (c == 4) return ozaki_gemm_cfg<OzCfg7KB64D>(d, S, pa, pb, exa, exb, Kp, allow_split, st);
      if (c == 5) return ozaki_gemm_cfg<OzCfg7KB64RD>(d, S, pa, pb, exa, exb, Kp, allow_split, st);
      if (c == 6) return ozaki_gemm_cfg<OzCfg7KB64P>(d, S, pa, pb, exa, exb, Kp, allow_split, st);
      if (c == 7) return ozaki_gemm_cfg<OzCfg7KB64S>(d, S, pa, pb, exa, exb, Kp, allow_split, st);
      if (c == 8) return ozaki_gemm_cfg<OzCfg7KB64SP>(d, S, pa, pb, exa, exb, Kp, allow_split, st);
      if (c == 9) return ozaki_gemm_cfg<OzCfg7KB64T>(d, S, pa, pb, exa, exb, Kp, allow_split, st);
      if (c == 10) return ozaki_gemm_cfg<OzCfg7KB64TE>(d, S, pa, pb, exa, exb, Kp, allow_split, st);
      if (c == 11) return ozaki_gemm_cfg<OzCfg7KB64TE2>(d, S, pa, pb, exa, exb, Kp, allow_split, st);
      return ozaki_gemm_cfg<OzCfg<7>::T>(d, S, pa, pb, exa, exb, Kp, allow_split, st);
    }
    default: return ozaki_gemm_cfg<OzCfg<8>::T>(d, S, pa, pb, exa, exb, Kp, allow_split, st);
  }
}

}  // namespace

bool tcgen05_available() { return is_sm100() && encoder() != nullptr; }

double ozaki_term_bound(int slices) { return (slices + 1) * std::ldexp(1.0, 2 - 8 * slices); }

int ozaki_slices_for_call() {
  const Settings& s = settings();
  if (s.ozaki_slices != 0) return s.ozaki_slices;
  const double tol = s.ozaki_tolerance > 0 ? s.ozaki_tolerance : kOzakiDefaultTolerance;
  for (int S = 3; S < 8; ++S)
    if (ozaki_term_bound(S) <= tol) return S;
  return 8;
}

bool make_tiled_map(CUtensorMap* map, CUtensorMapDataType dt, int rank, const void* base, const long* dims,
                    const long* strides_bytes, const int* box, int swz_bytes) {
  EncodeFn enc = encoder();
  if (!enc || rank < 1 || rank > 5) return false;
  cuuint64_t d[5], s[4];
  cuuint32_t b[5], es[5];
  for (int i = 0; i < rank; ++i) {
    d[i] = (cuuint64_t)dims[i];
    b[i] = (cuuint32_t)box[i];
    es[i] = 1;
    if (i + 1 < rank) s[i] = (cuuint64_t)strides_bytes[i];
  }
  CUtensorMapSwizzle sw = swz_bytes == 128  ? CU_TENSOR_MAP_SWIZZLE_128B
                          : swz_bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B
                          : swz_bytes == 32 ? CU_TENSOR_MAP_SWIZZLE_32B
                                            : CU_TENSOR_MAP_SWIZZLE_NONE;
  return enc(map, dt, (cuuint32_t)rank, const_cast<void*>(base), d, s, b, es, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

namespace {

// Operands staged straight from the caller's matrices (equally spaced instances, 16-byte aligned
// bases, strides and leading dimensions): each op(X) is K-major where it is stored K-contiguous
// (op(A) = A^T, op(B) = B) and MN-major where it is stored M- (N-)contiguous (op(A) = A,
// op(B) = B^T), so no layout needs a transposing pass. `elem` = bytes per element.
bool direct_eligible(const BatchDesc& d, int elem) {
  const bool uniform = d.batch == 1 || (d.strideA > 0 && d.strideB > 0);
  return uniform && (d.lda * elem) % 16 == 0 && (d.ldb * elem) % 16 == 0 && ((uintptr_t)d.A0 % 16) == 0 &&
         ((uintptr_t)d.B0 % 16) == 0 && d.strideA % 16 == 0 && d.strideB % 16 == 0;
}

// 4-D maps {inner, outer, 1, batch} of op(A) and op(B) for one 128-byte K stage: K-major tiles are
// (K 128 bytes) x (128 rows of A, BN rows of B); MN-major tiles are loaded as 128-byte-wide M (N)
// blocks by the stage's K rows.
bool direct_maps(const BatchDesc& d, CUtensorMapDataType dt, int elem, int BN, CUtensorMap* ta, CUtensorMap* tb) {
  const bool amn = d.transa == SSBLAS_OP_N, bmn = d.transb == SSBLAS_OP_T;
  const int kel = 128 / elem;                           // K elements (rows) per stage
  const long a_cols = amn ? d.k : d.m, b_cols = bmn ? d.k : d.n;   // stored columns
  const long psa = d.batch > 1 ? d.strideA : round_up(d.lda * a_cols * elem, 16);
  const long psb = d.batch > 1 ? d.strideB : round_up(d.ldb * b_cols * elem, 16);
  const bool okA = amn ? make_map(ta, d.A0, dt, d.m, d.k, 1, d.batch, d.lda * elem, psa, psa, kel, kel, 1, 128)
                       : make_map(ta, d.A0, dt, d.k, d.m, 1, d.batch, d.lda * elem, psa, psa, kel, 128, 1, 128);
  const bool okB = bmn ? make_map(tb, d.B0, dt, d.n, d.k, 1, d.batch, d.ldb * elem, psb, psb, kel, kel, 1, 128)
                       : make_map(tb, d.B0, dt, d.k, d.n, 1, d.batch, d.ldb * elem, psb, psb, kel, BN, 1, 128);
  return okA && okB;
}

template <int BN, int AMN, int BMN>
using CfgI8 = tc::Config<tc::KIND_I8, 1, 1, BN, 128, BN == 256 ? 4 : 6, 1, 2, tc::EPI_I32, 0, AMN, BMN>;

template <int BN>
cudaError_t run_i8(const CUtensorMap& ta, const CUtensorMap& tb, const tc::Params& prm, bool amn, bool bmn,
                   cudaStream_t st, const SplitPlan& plan) {
  if (amn && bmn) return run_gemm<CfgI8<BN, 1, 1>>(ta, tb, prm, st, "i8_gemm", plan);
  if (amn) return run_gemm<CfgI8<BN, 1, 0>>(ta, tb, prm, st, "i8_gemm", plan);
  if (bmn) return run_gemm<CfgI8<BN, 0, 1>>(ta, tb, prm, st, "i8_gemm", plan);
  return run_gemm<CfgI8<BN, 0, 0>>(ta, tb, prm, st, "i8_gemm", plan);
}

}  // namespace

cudaError_t launch_i8_tcgen05(const BatchDesc& d, cudaStream_t st) {
  if (!is_sm100() || !encoder()) return cudaErrorNotSupported;
  if (d.k > (1L << 31) || d.m > (1L << 31) || d.n > (1L << 31)) return cudaErrorNotSupported;
  CUtensorMap ta, tb;
  const int BN = choose_config(SSBLAS_PATH_I8_TCGEN05, d.m, d.n, d.k, d.batch, d.n <= 128 ? 1 : 0) == 1 ? 128 : 256;
  bool amn = false, bmn = false, ok;
  if (direct_eligible(d, 1)) {
    amn = d.transa == SSBLAS_OP_N;
    bmn = d.transb == SSBLAS_OP_T;
    ok = direct_maps(d, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, BN, &ta, &tb);
  } else {
    // odd leading dimensions or unevenly spaced instances: K-major planes from the pack pre-pass
    int8_t *pa, *pb;
    long Kp;
    cudaError_t e = pack_operands_i8(d, st, &pa, &pb, &Kp);
    if (e != cudaSuccess) return e;
    ok = make_map(&ta, pa, CU_TENSOR_MAP_DATA_TYPE_UINT8, d.k, d.m, 1, d.batch, Kp, d.m * Kp, d.m * Kp, 128, 128, 1, 128) &&
         make_map(&tb, pb, CU_TENSOR_MAP_DATA_TYPE_UINT8, d.k, d.n, 1, d.batch, Kp, d.n * Kp, d.n * Kp, 128, BN, 1, 128);
  }
  if (!ok) return cudaErrorNotSupported;
  tc::Params prm = base_params(d);
  prm.ab_unsigned = (d.a_unsigned ? 1 : 0) | (d.b_unsigned ? 2 : 0);
  note_path(SSBLAS_PATH_I8_TCGEN05);
  // split-K: int32 sums wrap identically in any order; automatic pieces keep at least 2048 k
  SplitPlan plan;
  plan.key = SSBLAS_PATH_SPLITK_I8;
  plan.min_kb = 2048 / 128;
  return BN == 128 ? run_i8<128>(ta, tb, prm, amn, bmn, st, plan) : run_i8<256>(ta, tb, prm, amn, bmn, st, plan);
}

namespace {

template <int BN, int AMN, int BMN, int EPI>
using CfgF16 = tc::Config<tc::KIND_F16, 1, 1, BN, 128, BN == 256 ? 4 : 6, 1, 2, EPI, 0, AMN, BMN>;

template <int EPI>
cudaError_t run_f16(const CUtensorMap& ta, const CUtensorMap& tb, const tc::Params& prm, bool amn, bool bmn,
                    cudaStream_t st) {
  if (amn && bmn) return run_gemm<CfgF16<256, 1, 1, EPI>>(ta, tb, prm, st, "f16_gemm");
  if (amn) return run_gemm<CfgF16<256, 1, 0, EPI>>(ta, tb, prm, st, "f16_gemm");
  if (bmn) return run_gemm<CfgF16<256, 0, 1, EPI>>(ta, tb, prm, st, "f16_gemm");
  return run_gemm<CfgF16<256, 0, 0, EPI>>(ta, tb, prm, st, "f16_gemm");
}

}  // namespace

cudaError_t launch_f16_tcgen05(const BatchDesc& d, cudaStream_t st) {
  if (!is_sm100() || !encoder()) return cudaErrorNotSupported;
  if (d.k > (1L << 31) || d.m > (1L << 31) || d.n > (1L << 31)) return cudaErrorNotSupported;
  // the fp16 row takes its operands straight from the caller's matrices only
  if (!direct_eligible(d, 2)) return cudaErrorNotSupported;
  CUtensorMap ta, tb;
  if (!direct_maps(d, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, 256, &ta, &tb)) return cudaErrorNotSupported;
  tc::Params prm = base_params(d);
  const bool amn = d.transa == SSBLAS_OP_N, bmn = d.transb == SSBLAS_OP_T;
  return d.c_f32 ? run_f16<tc::EPI_F32>(ta, tb, prm, amn, bmn, st) : run_f16<tc::EPI_F16>(ta, tb, prm, amn, bmn, st);
}

namespace {

// The instances [b0, b0 + nb) of an operand's slicing arguments.
PlaneArgs plane_chunk(const PlaneArgs& x, long b0, long nb) {
  PlaneArgs c = x;
  c.X = x.X + b0;
  c.batch = nb;
  c.out = (int8_t*)x.out + b0 * x.batch_stride;
  if (x.X0) c.X0 = (const uint8_t*)x.X0 + b0 * x.xstride;
  return c;
}

// Chunks of the slicing / GEMM pipeline (1 = none): a tuned or forced count
// (SSBLAS_PATH_OZAKI_PIPELINE); automatic means none. Measured on 32 x 1024^3: the slim slicer
// beside the GEMM slows the GEMM by a third (0.65 -> 0.87 ms for the batch) -- the GEMM streams its
// operands through shared memory near that memory's bandwidth, and the slicer needs the same --
// so the 4-chunk pipeline took 1.15 ms against 0.89 ms for slicing then multiplying.
int ozaki_pipeline_chunks(const BatchDesc& d, const PlaneArgs& a) {
  if (!cluster_kernel_fits(a) || d.batch < 2) return 1;
  int c = choose_config(SSBLAS_PATH_OZAKI_PIPELINE, d.m, d.n, d.k, d.batch, 0);
  if (c == 0) c = 1;
  if (c > d.batch) c = (int)d.batch;
  if (c > 8) c = 8;
  return c < 1 ? 1 : c;
}

// Side stream and events of the pipeline, one set per device, created on first use.
struct PipeRes {
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr;
  cudaEvent_t ready[8] = {};
};
cudaError_t pipe_res(PipeRes** out) {
  static PipeRes res[kMaxDevices];
  const int dev = current_device();
  if (dev < 0) return cudaErrorInvalidDevice;
  cudaError_t e;
  PipeRes& r = res[dev];
  if (!r.side) {
    if ((e = cudaStreamCreateWithFlags(&r.side, cudaStreamNonBlocking)) != cudaSuccess) return e;
    if ((e = cudaEventCreateWithFlags(&r.fork, cudaEventDisableTiming)) != cudaSuccess) return e;
    for (auto& ev : r.ready)
      if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return e;
  }
  *out = &r;
  return cudaSuccess;
}

// Slicing of chunk c + 1 overlaps the GEMM of chunk c: chunk 0 is sliced on the caller's stream by
// the full-size one-pass kernel; then a side stream slices chunks 1.. with the slim kernel (4 rows
// x 256 k per 128-thread CTA, 80 registers, 25 KB of shared memory), which fits on an SM beside a
// GEMM CTA, so it uses the issue slots and memory bandwidth the tensor-bound GEMM leaves free.
// GEMM chunk c waits for its chunk's event; the last wait joins the side stream back into the
// caller's.
cudaError_t ozaki_pipelined(const BatchDesc& d, int S, const PlaneArgs& a, const PlaneArgs& b, int8_t* pa,
                            int8_t* pb, int32_t* ex, long Kp, int chunks, cudaStream_t st) {
  PipeRes* r = nullptr;
  cudaError_t e = pipe_res(&r);
  if (e != cudaSuccess) return e;
  int32_t* exa = ex;
  int32_t* exb = ex + d.m * d.batch;
  auto lo = [&](int c) { return d.batch * c / chunks; };
  {
    const long b0 = lo(0), nb = lo(1) - b0;
    if ((e = launch_ozaki_slice_pair(plane_chunk(a, b0, nb), exa + b0 * d.m, plane_chunk(b, b0, nb),
                                     exb + b0 * d.n, S, st)) != cudaSuccess)
      return e;
  }
  if ((e = cudaEventRecord(r->fork, st)) != cudaSuccess) return e;
  if ((e = cudaStreamWaitEvent(r->side, r->fork, 0)) != cudaSuccess) return e;
  for (int c = 1; c < chunks; ++c) {
    const long b0 = lo(c), nb = lo(c + 1) - b0;
    if ((e = launch_ozaki_cluster(plane_chunk(a, b0, nb), exa + b0 * d.m, plane_chunk(b, b0, nb), exb + b0 * d.n,
                                  true, S, 6, r->side)) != cudaSuccess)
      return e;
    if ((e = cudaEventRecord(r->ready[c], r->side)) != cudaSuccess) return e;
  }
  for (int c = 0; c < chunks; ++c) {
    const long b0 = lo(c), nb = lo(c + 1) - b0;
    if (c > 0 && (e = cudaStreamWaitEvent(st, r->ready[c], 0)) != cudaSuccess) return e;
    BatchDesc dc = d;
    dc.batch = nb;
    dc.C = d.C + b0;
    dc.C0 = nullptr;   // a chunk's C is not addressed through the batch's C tensor map
    if ((e = ozaki_gemm(dc, S, pa + b0 * a.batch_stride, pb + b0 * b.batch_stride, exa + b0 * d.m,
                        exb + b0 * d.n, Kp, false, st)) != cudaSuccess)
      return e;
  }
  return cudaSuccess;
}

}  // namespace

cudaError_t launch_ozaki_f64(const BatchDesc& d, int slices, cudaStream_t st) {
  if (!is_sm100() || !encoder()) return cudaErrorNotSupported;
  // int32 accumulation stays exact while (pairs per level) * k * 2^14 < 2^31: longer k is cut into
  // split-K pieces of at most 16384, whose sums are added in 64 bits
  if (d.k > (1L << 30) || d.m > (1L << 31) || d.n > (1L << 31)) return cudaErrorNotSupported;
  const int S = slices;
  if (S < 3 || S > 8) return cudaErrorInvalidValue;
  cudaError_t e;
  const long Kp = round_up(d.k, 16);
  const long sa = d.m * Kp, sb = d.n * Kp;
  int8_t* pa = (int8_t*)workspace(WS_PACK_A, (size_t)sa * S * d.batch, &e);
  if (!pa) return e;
  int8_t* pb = (int8_t*)workspace(WS_PACK_B, (size_t)sb * S * d.batch, &e);
  if (!pb) return e;
  int32_t* ex = (int32_t*)workspace(WS_EXP, sizeof(int32_t) * (size_t)(d.m + d.n) * d.batch, &e);
  if (!ex) return e;
  PlaneArgs a{d.A, d.m, d.k, d.lda, d.transa == SSBLAS_OP_T, d.batch, pa, Kp, sa, sa * S};
  PlaneArgs b{d.B, d.n, d.k, d.ldb, d.transb == SSBLAS_OP_N, d.batch, pb, Kp, sb, sb * S};
  if (d.A0 && (d.batch == 1 || d.strideA > 0)) { a.X0 = d.A0; a.xstride = d.batch == 1 ? 16 : d.strideA; }
  if (d.B0 && (d.batch == 1 || d.strideB > 0)) { b.X0 = d.B0; b.xstride = d.batch == 1 ? 16 : d.strideB; }
  const int chunks = ozaki_pipeline_chunks(d, a);
  if (chunks <= 1) {
    if ((e = launch_ozaki_slice_pair(a, ex, b, ex + d.m * d.batch, S, st)) != cudaSuccess) return e;
    return ozaki_gemm(d, S, pa, pb, ex, ex + d.m * d.batch, Kp, true, st);
  }
  return ozaki_pipelined(d, S, a, b, pa, pb, ex, Kp, chunks, st);
}

cudaError_t launch_ozaki_gemm_on(const BatchDesc& d, int S, const int8_t* pa, const int8_t* pb, const int32_t* ex,
                                 long Kp, cudaStream_t st) {
  if (!is_sm100() || !encoder()) return cudaErrorNotSupported;
  if (S < 3 || S > 8) return cudaErrorInvalidValue;
  if (d.k > kOzakiMaxPieceK) return cudaErrorNotSupported;   // splitting would need workspace
  return ozaki_gemm(d, S, pa, pb, ex, ex + d.m * d.batch, Kp, false, st);
}

cudaError_t launch_bf16x3_f32(const BatchDesc& d, cudaStream_t st) {
  if (!is_sm100() || !encoder()) return cudaErrorNotSupported;
  if (d.m > (1L << 31) || d.n > (1L << 31) || d.k > (1L << 31)) return cudaErrorNotSupported;
  // configurations: 0 / 1 = split pass then tiled GEMM with 64- / 128-column tiles; 2 = one
  // kernel that splits in shared memory, for equally spaced instances of at most 128 x 128 (the
  // others take configuration 0 / 1) -- the default where it applies: on 4096 x 64^3 TT it takes
  // 0.069 ms against 0.084 + 0.072 ms for the split pass and the tiled GEMM
  const int fallback = bf16x3_small_fits(d) ? 2 : d.n <= 64 ? 0 : 1;
  const int cfg = choose_config(SSBLAS_PATH_BF16X3_TCGEN05, d.m, d.n, d.k, d.batch, fallback);
  cudaError_t e;
  if (cfg == 2 && bf16x3_small_fits(d)) {
    e = launch_bf16x3_small(d, st);
    if (e != cudaErrorNotSupported) return e;
  }
  const long Kp = round_up(d.k, 8);
  const long sa = d.m * Kp * 2, sb = d.n * Kp * 2;   // bytes per plane
  void* pa = workspace(WS_PACK_A, (size_t)sa * 2 * d.batch, &e);
  if (!pa) return e;
  void* pb = workspace(WS_PACK_B, (size_t)sb * 2 * d.batch, &e);
  if (!pb) return e;
  PlaneArgs a{d.A, d.m, d.k, d.lda, d.transa == SSBLAS_OP_T, d.batch, pa, Kp, sa, sa * 2};
  PlaneArgs b{d.B, d.n, d.k, d.ldb, d.transb == SSBLAS_OP_N, d.batch, pb, Kp, sb, sb * 2};
  if ((e = launch_split_bf16_pair(a, b, st)) != cudaSuccess) return e;
  const int BN = (cfg == 0 || (cfg == 2 && d.n <= 64)) ? 64 : 128;
  CUtensorMap ta, tb;
  if (!make_map(&ta, pa, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, d.k, d.m, 2, d.batch, Kp * 2, sa, sa * 2, 64, 128, 2, 128) ||
      !make_map(&tb, pb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, d.k, d.n, 2, d.batch, Kp * 2, sb, sb * 2, 64, BN, 2, 128))
    return cudaErrorNotSupported;
  tc::Params prm = base_params(d);
  note_path(SSBLAS_PATH_BF16X3_TCGEN05);
  return BN == 64 ? run_gemm<CfgBf64>(ta, tb, prm, st, "bf16x3_gemm") : run_gemm<CfgBf128>(ta, tb, prm, st, "bf16x3_gemm");
}

}  // namespace ssb
