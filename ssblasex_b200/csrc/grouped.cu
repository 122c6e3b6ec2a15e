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
// Plain fp32/fp64 instances run through the grouped SIMT kernel (gemm_simt.cu).
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

constexpr int GRT = 32;   // rows per pass
constexpr int GNT = 256;

// One CTA per (instance, operand). MODE 0: int8 copy; 1: BF16 hi/lo; 2: Ozaki slices (S planes).
template <int MODE, int S, int KB, int RTILE_A, int RTILE_B>
__global__ void __launch_bounds__(GNT) gprep_kernel(const GPrepInst* __restrict__ items, uint8_t* __restrict__ outA,
                                                    uint8_t* __restrict__ outB, int32_t* __restrict__ exps) {
  constexpr int P = MODE == 0 ? 1 : MODE == 1 ? 2 : S;
  constexpr int KE = MODE == 1 ? KB / 2 : KB;               // K elements per block
  const GPrepInst it = items[blockIdx.x];
  const bool is_b = (blockIdx.x & 1) != 0;
  const int RTILE = is_b ? RTILE_B : RTILE_A;
  uint8_t* out = (is_b ? outB : outA) + it.off;
  const uint8_t* X = (const uint8_t*)it.X[it.idx];
  const long rows_pad = (long)it.tiles * RTILE;
  const long kpad = (long)it.nk * KE;
  __shared__ double rmax[GRT];
  __shared__ double rscale[GRT][2];

  for (long r0 = 0; r0 < rows_pad; r0 += GRT) {
    if (MODE == 2) {
      if (threadIdx.x < GRT) rmax[threadIdx.x] = 0.0;
      __syncthreads();
      // row maxima: 8 threads per row stride over K
      const int r = threadIdx.x / 8, part = threadIdx.x % 8;
      const long gr = r0 + r;
      double mx = 0.0;
      if (gr < it.rows) {
        const double* Xd = (const double*)X;
        for (long k = part; k < it.K; k += 8)
          mx = fmax(mx, fabs(it.kcontig ? Xd[gr * it.ld + k] : Xd[gr + k * it.ld]));
      }
#pragma unroll
      for (int off = 4; off >= 1; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
      if (part == 0) rmax[r] = mx;
      __syncthreads();
      if (threadIdx.x < GRT) {
        int e = 0;
        if (rmax[threadIdx.x] > 0.0) frexp(rmax[threadIdx.x], &e);
        const long g2 = r0 + threadIdx.x;
        if (g2 < it.rows) exps[it.eoff + g2] = e;
        const int sh = 8 * S - 2 - e;
        const int h1 = sh / 2;
        rscale[threadIdx.x][0] = ldexp(1.0, h1);
        rscale[threadIdx.x][1] = ldexp(1.0, sh - h1);
      }
      __syncthreads();
    }
    // each thread emits 4 output bytes per plane: (row, 4 consecutive int8 k) or (row, 2 bf16 k)
    constexpr int EPW = MODE == 1 ? 2 : 4;          // elements per 4-byte word
    const long words_per_row = kpad / EPW;
    for (long w = threadIdx.x; w < GRT * words_per_row; w += GNT) {
      const int r = (int)(w / words_per_row);
      const long kw = w % words_per_row;
      const long gr = r0 + r;
      if (gr >= rows_pad) break;
      const long k0 = kw * EPW;
      const int rt = (int)(gr / RTILE), rr = (int)(gr % RTILE);
      const long kb = k0 / KE;
      const int cbyte = (int)((k0 % KE) * (MODE == 1 ? 2 : 1));
      uint8_t* chunk = out + ((long)rt * it.nk + kb) * (long)P * RTILE * KB;
      const uint32_t so = swz(rr, cbyte, KB);
      double vals[4];
#pragma unroll
      for (int j = 0; j < EPW; ++j) {
        const long k = k0 + j;
        double v = 0.0;
        if (gr < it.rows && k < it.K) {
          if (MODE == 0) {
            const int8_t* Xi = (const int8_t*)X;
            v = (double)(it.kcontig ? Xi[gr * it.ld + k] : Xi[gr + k * it.ld]);
          } else if (MODE == 1) {
            const float* Xf = (const float*)X;
            v = (double)(it.kcontig ? Xf[gr * it.ld + k] : Xf[gr + k * it.ld]);
          } else {
            const double* Xd = (const double*)X;
            v = it.kcontig ? Xd[gr * it.ld + k] : Xd[gr + k * it.ld];
          }
        }
        vals[j] = v;
      }
      if (MODE == 0) {
        uint32_t wv = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) wv |= ((uint32_t)(uint8_t)(int8_t)vals[j]) << (8 * j);
        *(uint32_t*)(chunk + so) = wv;
      } else if (MODE == 1) {
        const float x0 = (float)vals[0], x1 = (float)vals[1];
        const __nv_bfloat16 h0 = __float2bfloat16_rn(x0), h1 = __float2bfloat16_rn(x1);
        const __nv_bfloat16 l0 = __float2bfloat16_rn(x0 - __bfloat162float(h0));
        const __nv_bfloat16 l1 = __float2bfloat16_rn(x1 - __bfloat162float(h1));
        __nv_bfloat162 hv, lv;
        hv.x = h0; hv.y = h1; lv.x = l0; lv.y = l1;
        *(__nv_bfloat162*)(chunk + so) = hv;
        *(__nv_bfloat162*)(chunk + RTILE * KB + so) = lv;
      } else {
        const double s0 = (gr < it.rows) ? rscale[r][0] : 0.0, s1 = (gr < it.rows) ? rscale[r][1] : 0.0;
        // padding rows/columns are zero digits (value 0 gives Y = bias)
        uint32_t wd[S];
        digit_words<S>(vals, s0, s1, wd);
#pragma unroll
        for (int p = 0; p < P; ++p) *(uint32_t*)(chunk + (long)p * RTILE * KB + so) = wd[p];
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
    const int tm = (int)((in.m + Cfg::BM - 1) / Cfg::BM), tn = (int)((in.n + Cfg::BN - 1) / Cfg::BN);
    gi.nk = (int)((in.k + KE - 1) / KE);
    gi.tiles_n = tn;
    gi.offA = kp.bytesA;
    gi.offB = kp.bytesB;
    gi.offEA = kp.nexp;
    gi.offEB = kp.nexp + in.m;
    kp.bytesA += (long)tm * gi.nk * Cfg::A_STAGE;
    kp.bytesB += (long)tn * gi.nk * Cfg::B_STAGE;
    kp.nexp += in.m + in.n;
    const int li = (int)kp.inst.size();
    kp.inst.push_back(gi);
    for (int a = 0; a < tm; ++a)
      for (int b = 0; b < tn; ++b) kp.tiles.push_back(GTile{li, a, b});
    GPrepInst pa{g.A, in.idx, in.m, in.k, in.lda, in.transa == SSBLAS_OP_T, tm, gi.nk, gi.offA, gi.offEA};
    GPrepInst pb{(const void* const*)g.B, in.idx, in.n, in.k, in.ldb, in.transb == SSBLAS_OP_N, tn, gi.nk, gi.offB, gi.offEB};
    kp.prep.push_back(pa);
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
  DevBuf inst, tiles, prep, packA, packB, exps;
  long ninst = 0, ntiles = 0;
};

template <class Cfg>
cudaError_t upload_kind(const KindPlan<Cfg>& kp, KindDev& kd, cudaStream_t st) {
  cudaError_t e;
  if ((e = kd.inst.alloc(sizeof(GInst) * kp.inst.size())) || (e = kd.tiles.alloc(sizeof(GTile) * kp.tiles.size())) ||
      (e = kd.prep.alloc(sizeof(GPrepInst) * kp.prep.size())) || (e = kd.packA.alloc(kp.bytesA)) ||
      (e = kd.packB.alloc(kp.bytesB)) || (e = kd.exps.alloc(sizeof(int32_t) * (kp.nexp + 1))))
    return e;
  if ((e = cudaMemcpyAsync(kd.inst.p, kp.inst.data(), sizeof(GInst) * kp.inst.size(), cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(kd.tiles.p, kp.tiles.data(), sizeof(GTile) * kp.tiles.size(), cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(kd.prep.p, kp.prep.data(), sizeof(GPrepInst) * kp.prep.size(), cudaMemcpyHostToDevice, st)))
    return e;
  kd.ninst = (long)kp.inst.size();
  kd.ntiles = (long)kp.tiles.size();
  return cudaStreamSynchronize(st);   // the host tables are temporaries
}

template <class Cfg, int MODE, int S>
cudaError_t launch_kind(const KindDev& kd, void* const* C, cudaStream_t st, const char* prep_name,
                        const char* gemm_name) {
  if (kd.ninst == 0) return cudaSuccess;
  {
    ProfScope prof(prep_name, st);
    gprep_kernel<MODE, S, Cfg::KB, Cfg::BM, Cfg::BN><<<(unsigned)(2 * kd.ninst), GNT, 0, st>>>(
        (const GPrepInst*)kd.prep.p, (uint8_t*)kd.packA.p, (uint8_t*)kd.packB.p, (int32_t*)kd.exps.p);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(tc::tc_gemm_kernel<Cfg, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         Cfg::SMEM);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  tc::Params prm{};
  prm.total_tiles = kd.ntiles;
  prm.tiles_m = prm.tiles_n = 1;
  prm.C = C;
  prm.exp_a = (const int32_t*)kd.exps.p;
  prm.exp_b = (const int32_t*)kd.exps.p;
  prm.exp_shift = -12;
  prm.err = device_error_flag();
  prm.ginst = (const GInst*)kd.inst.p;
  prm.gtiles = (const GTile*)kd.tiles.p;
  prm.packA = (const uint8_t*)kd.packA.p;
  prm.packB = (const uint8_t*)kd.packB.p;
  CUtensorMap dummy;
  memset(&dummy, 0, sizeof(dummy));
  const long grid = kd.ntiles < num_sms() ? kd.ntiles : num_sms();
  ProfScope prof(gemm_name, st);
  tc::tc_gemm_kernel<Cfg, true><<<(unsigned)grid, tc::kThreads, Cfg::SMEM, st>>>(dummy, dummy, prm);
  note_launch();
  return cudaGetLastError();
}

using GCfgOz = tc::Config<tc::KIND_I8, 7, 7, 64, 32, 5, 7, 1, tc::EPI_OZAKI, 2>;
using GCfgBf = tc::Config<tc::KIND_BF16, 2, 2, 64, 128, 4, 1, 2, tc::EPI_F32, 1>;
using GCfgI8 = tc::Config<tc::KIND_I8, 1, 1, 128, 128, 6, 1, 2, tc::EPI_I32, 0>;

// A prepared grouped call: device tables and packed buffers per kind, the plain-instance batch,
// and (after the first replay request) the captured CUDA graph of all its launches.
struct Plan {
  std::vector<uint64_t> key;
  KindDev oz, bf, i8;
  std::unique_ptr<GroupedSimt> simt;
  void* const* C = nullptr;
  cudaGraphExec_t exec = nullptr;
  int launches = 0;
  ~Plan() {
    if (exec) cudaGraphExecDestroy(exec);
  }
};

std::map<int, std::unique_ptr<Plan>> g_plans;   // one cached plan per device

std::vector<uint64_t> signature(const GroupedDesc& g, int mode) {
  std::vector<uint64_t> k;
  k.reserve(g.inst.size() * 12 + 8);
  k.push_back((uint64_t)mode);
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
  if ((e = launch_kind<GCfgOz, 2, 7>(pl.oz, pl.C, st, "grouped_ozaki_slice", "grouped_ozaki_gemm"))) return e;
  if ((e = launch_kind<GCfgBf, 1, 1>(pl.bf, pl.C, st, "grouped_split_bf16", "grouped_bf16x3_gemm"))) return e;
  if ((e = launch_kind<GCfgI8, 0, 1>(pl.i8, pl.C, st, "grouped_pack_i8", "grouped_i8_gemm"))) return e;
  if (pl.simt && (e = launch_simt_grouped(*pl.simt, st))) return e;
  return cudaSuccess;
}

}  // namespace

cudaError_t grouped_run(const GroupedDesc& g, cudaStream_t st) {
  const int mode = settings().math_mode;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::vector<uint64_t> key = signature(g, mode);
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
  pl->C = g.C;
  std::vector<int> oz, bf, i8, plain;
  for (int i = 0; i < (int)g.inst.size(); ++i) {
    const GroupedInst& in = g.inst[i];
    if (in.k <= 0) continue;   // C untouched, as in the reference
    if (in.row == ROW_I8) i8.push_back(i);
    else if (in.row == ROW_F64 && (mode & SSBLAS_MATH_FP64_OZAKI) && in.k <= 16384) oz.push_back(i);
    else if (in.row == ROW_F32 && (mode & SSBLAS_MATH_FP32_BF16X3)) bf.push_back(i);
    else plain.push_back(i);
  }
  {
    KindPlan<GCfgOz> k1;
    plan_kind(g, oz, k1);
    if ((e = upload_kind(k1, pl->oz, st))) return e;
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
  pl->launches = (pl->oz.ninst ? 2 : 0) + (pl->bf.ninst ? 2 : 0) + (pl->i8.ninst ? 2 : 0) +
                 (pl->simt ? pl->simt->launches : 0);
  g_plans[dev] = std::move(pl);
  Plan& p = *g_plans[dev];
  note_path(SSBLAS_PATH_GROUPED, p.oz.ninst ? 7 : 0);
  return run_plan(p, st);
}

void grouped_release() { g_plans.clear(); }

}  // namespace ssb
