// Register-tiled SIMT batched GEMM: the plain fp32 (FFMA) and fp64 (DFMA) rows, and the int8 row
// for layouts the tensor-core path does not take.
//
// Semantics follow the reference (hirokitokura/ssblasEx): C <- beta*C (not read when beta == 0,
// src/include/CScale/Xgemm_scale_kernel.hpp:164-176) then C <- C + acc*alpha with one fused
// multiply-add (src/include/GemmCore/Xgemm_kernel_sve_v4x5_1.hpp:93-127); int8 products
// accumulate in int32 with wrap-around (sdot, src/include/asm/SVE/def_sve_asm_float.h:46).
// The reference adds alpha*acc once per 512-wide K block; this kernel adds it once, which
// differs only by rounding on the fp rows and not at all on the int8 row.
//
// Design: one CTA per (BM x BN tile, instance); op(A)/op(B) tiles are staged through shared
// memory k-major (the transposes are absorbed by the staging loads), double-buffered through
// registers; each thread owns a TM x TN sub-tile whose rows are spaced by BM/TM so that the
// column-major C stores of a warp are contiguous.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "grouped.h"
#include "internal.h"

namespace ssb {
namespace {

template <typename T> struct RowTraits;
template <> struct RowTraits<float> {
  using AB = float; using Acc = float; using C = float; using S = float;
  static __device__ __forceinline__ Acc mac(Acc acc, AB a, AB b) { return fmaf(a, b, acc); }
  static __device__ __forceinline__ C epi(Acc acc, S alpha, S beta, const C* cptr) {
    C t = (beta == 0.0f) ? 0.0f : beta * (*cptr);
    return fmaf(acc, alpha, t);
  }
};
template <> struct RowTraits<double> {
  using AB = double; using Acc = double; using C = double; using S = double;
  static __device__ __forceinline__ Acc mac(Acc acc, AB a, AB b) { return fma(a, b, acc); }
  static __device__ __forceinline__ C epi(Acc acc, S alpha, S beta, const C* cptr) {
    C t = (beta == 0.0) ? 0.0 : beta * (*cptr);
    return fma(acc, alpha, t);
  }
};
template <> struct RowTraits<int8_t> {
  using AB = int8_t; using Acc = uint32_t; using C = int32_t; using S = int32_t;
  static __device__ __forceinline__ Acc mac(Acc acc, AB a, AB b) {
    return acc + (uint32_t)((int32_t)a * (int32_t)b);
  }
  static __device__ __forceinline__ C epi(Acc acc, S alpha, S beta, const C* cptr) {
    uint32_t t = (beta == 0) ? 0u : (uint32_t)beta * (uint32_t)(*cptr);
    return (int32_t)(t + acc * (uint32_t)alpha);
  }
};

// fp16 row of the type extensions: fp16 inputs, fp32 scale and accumulation, C in fp16 or fp32
struct HalfC16 {};
struct HalfC32 {};
template <> struct RowTraits<HalfC16> {
  using AB = __half; using Acc = float; using C = __half; using S = float;
  static __device__ __forceinline__ Acc mac(Acc acc, AB a, AB b) { return fmaf(__half2float(a), __half2float(b), acc); }
  static __device__ __forceinline__ C epi(Acc acc, S alpha, S beta, const C* cptr) {
    const float t = (beta == 0.0f) ? 0.0f : beta * __half2float(*cptr);
    return __float2half_rn(fmaf(acc, alpha, t));
  }
};
template <> struct RowTraits<HalfC32> {
  using AB = __half; using Acc = float; using C = float; using S = float;
  static __device__ __forceinline__ Acc mac(Acc acc, AB a, AB b) { return fmaf(__half2float(a), __half2float(b), acc); }
  static __device__ __forceinline__ C epi(Acc acc, S alpha, S beta, const C* cptr) {
    const float t = (beta == 0.0f) ? 0.0f : beta * (*cptr);
    return fmaf(acc, alpha, t);
  }
};

template <typename T>
struct SimtArgs {
  int transa, transb;
  long m, n, k, lda, ldb, ldc, batch;
  const typename RowTraits<T>::AB* const* A;
  const typename RowTraits<T>::AB* const* B;
  typename RowTraits<T>::C* const* C;
  typename RowTraits<T>::S alpha, beta;
};

// One BM x BN tile of instance b at (m0, n0), BK deep; each thread computes TM x TN outputs.
// LAY = (op(A) is T) + 2 * (op(B) is T) when known at compile time (then the staging loads have
// no layout branches), or -1 to read the layout from args.
template <typename T, int BM, int BN, int BK, int TM, int TN, int LAY>
__device__ __forceinline__ void simt_tile(const SimtArgs<T>& args, long b, long m0, long n0) {
  const bool a_n = LAY >= 0 ? (LAY & 1) == 0 : args.transa == SSBLAS_OP_N;
  const bool b_n = LAY >= 0 ? (LAY & 2) == 0 : args.transb == SSBLAS_OP_N;
  using Tr = RowTraits<T>;
  using AB = typename Tr::AB;
  using Acc = typename Tr::Acc;
  constexpr int TX = BM / TM;            // threads along M (fast index -> coalesced C columns)
  constexpr int TY = BN / TN;
  constexpr int NT = TX * TY;
  constexpr int A_PER = BM * BK / NT;    // staged elements per thread per tile
  constexpr int B_PER = BK * BN / NT;
  static_assert(A_PER * NT == BM * BK && B_PER * NT == BK * BN, "tile/thread mismatch");

  __shared__ AB As[2][BK][BM];
  __shared__ AB Bs[2][BK][BN];

  const int tid = threadIdx.x;
  const int tx = tid % TX, ty = tid / TX;
  {
    const AB* __restrict__ A = args.A[b];
    const AB* __restrict__ B = args.B[b];

    AB ra[A_PER], rb[B_PER];
    // load op(A)[m0.., k0..] and op(B)[k0.., n0..] into registers (zero outside the matrix)
    auto load_tiles = [&](long k0) {
#pragma unroll
      for (int e = 0; e < A_PER; ++e) {
        int idx = tid + e * NT;
        int ii, kk;
        if (a_n) { ii = idx % BM; kk = idx / BM; }   // rows contiguous
        else { kk = idx % BK; ii = idx / BK; }                              // k contiguous
        long gi = m0 + ii, gk = k0 + kk;
        AB v = AB(0.0f);
        if (gi < args.m && gk < args.k)
          v = (a_n) ? A[gi + gk * args.lda] : A[gi * args.lda + gk];
        ra[e] = v;
      }
#pragma unroll
      for (int e = 0; e < B_PER; ++e) {
        int idx = tid + e * NT;
        int jj, kk;
        if (b_n) { kk = idx % BK; jj = idx / BK; }   // k contiguous
        else { jj = idx % BN; kk = idx / BN; }                              // cols contiguous
        long gj = n0 + jj, gk = k0 + kk;
        AB v = AB(0.0f);
        if (gj < args.n && gk < args.k)
          v = (b_n) ? B[gk + gj * args.ldb] : B[gk * args.ldb + gj];
        rb[e] = v;
      }
    };
    auto store_tiles = [&](int buf) {
#pragma unroll
      for (int e = 0; e < A_PER; ++e) {
        int idx = tid + e * NT;
        int ii, kk;
        if (a_n) { ii = idx % BM; kk = idx / BM; }
        else { kk = idx % BK; ii = idx / BK; }
        As[buf][kk][ii] = ra[e];
      }
#pragma unroll
      for (int e = 0; e < B_PER; ++e) {
        int idx = tid + e * NT;
        int jj, kk;
        if (b_n) { kk = idx % BK; jj = idx / BK; }
        else { jj = idx % BN; kk = idx / BN; }
        Bs[buf][kk][jj] = rb[e];
      }
    };

    Acc acc[TM][TN];
#pragma unroll
    for (int r = 0; r < TM; ++r)
#pragma unroll
      for (int c = 0; c < TN; ++c) acc[r][c] = Acc(0);

    const long ktiles = (args.k + BK - 1) / BK;
    load_tiles(0);
    store_tiles(0);
    __syncthreads();
    for (long kt = 0; kt < ktiles; ++kt) {
      const int buf = kt & 1;
      if (kt + 1 < ktiles) load_tiles((kt + 1) * BK);
#pragma unroll
      for (int kk = 0; kk < BK; ++kk) {
        AB av[TM], bv[TN];
#pragma unroll
        for (int r = 0; r < TM; ++r) av[r] = As[buf][kk][tx + r * TX];
#pragma unroll
        for (int c = 0; c < TN; ++c) bv[c] = Bs[buf][kk][ty + c * TY];
#pragma unroll
        for (int r = 0; r < TM; ++r)
#pragma unroll
          for (int c = 0; c < TN; ++c) acc[r][c] = Tr::mac(acc[r][c], av[r], bv[c]);
      }
      if (kt + 1 < ktiles) store_tiles(buf ^ 1);
      __syncthreads();
    }

    // epilogue, one column of the thread's sub-tile at a time: its TM reads of C (beta != 0)
    // are issued before its stores, so they overlap
    typename Tr::C* __restrict__ Cm = args.C[b];
    const bool read_c = !(args.beta == typename Tr::S(0));
#pragma unroll
    for (int c = 0; c < TN; ++c) {
      const long gj = n0 + ty + c * TY;
      if (gj >= args.n) continue;
      typename Tr::C cv[TM];
#pragma unroll
      for (int r = 0; r < TM; ++r) {
        const long gi = m0 + tx + r * TX;
        cv[r] = (read_c && gi < args.m) ? Cm[gi + gj * args.ldc] : typename Tr::C(0.0f);
      }
#pragma unroll
      for (int r = 0; r < TM; ++r) {
        const long gi = m0 + tx + r * TX;
        if (gi < args.m) Cm[gi + gj * args.ldc] = Tr::epi(acc[r][c], args.alpha, args.beta, &cv[r]);
      }
    }
  }
}

template <typename T, int BM, int BN, int BK, int TM, int TN, int LAY>
__global__ void __launch_bounds__((BM / TM) * (BN / TN), 1) simt_gemm_kernel(SimtArgs<T> args) {
  const long tiles_m = (args.m + BM - 1) / BM;
  const long m0 = (blockIdx.x % tiles_m) * BM;
  const long n0 = (blockIdx.x / tiles_m) * BN;
  for (long b = blockIdx.y; b < args.batch; b += gridDim.y) simt_tile<T, BM, BN, BK, TM, TN, LAY>(args, b, m0, n0);
}

// Grouped form: one CTA per (instance, tile) entry of the tile table.
template <typename T, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
simt_grouped_kernel(const SimtGInst* __restrict__ inst, const int* __restrict__ tiles, const T* const* A,
                    const T* const* B, typename RowTraits<T>::C* const* C) {
  const int* t = tiles + 3 * (long)blockIdx.x;
  const SimtGInst g = inst[t[0]];
  SimtArgs<T> a;
  a.transa = g.transa; a.transb = g.transb;
  a.m = g.m; a.n = g.n; a.k = g.k; a.lda = g.lda; a.ldb = g.ldb; a.ldc = g.ldc; a.batch = 1;
  a.A = A; a.B = B; a.C = C;
  if constexpr (sizeof(T) == 8) { a.alpha = g.alpha_d; a.beta = g.beta_d; }
  else { a.alpha = g.alpha_f; a.beta = g.beta_f; }
  simt_tile<T, BM, BN, BK, TM, TN, -1>(a, g.idx, (long)t[1] * BM, (long)t[2] * BN);
}

template <typename T, int BM, int BN, int BK, int TM, int TN>
cudaError_t launch_tile(const SimtArgs<T>& a, cudaStream_t stream) {
  long tiles = ((a.m + BM - 1) / BM) * ((a.n + BN - 1) / BN);
  if (tiles > 0x7fffffffL) return cudaErrorInvalidValue;
  dim3 grid((unsigned)tiles, (unsigned)(a.batch < 65535 ? a.batch : 65535));
  constexpr int NT = (BM / TM) * (BN / TN);
  ProfScope prof("simt_gemm", stream);
  switch ((a.transa == SSBLAS_OP_T ? 1 : 0) + (a.transb == SSBLAS_OP_T ? 2 : 0)) {
    case 0: simt_gemm_kernel<T, BM, BN, BK, TM, TN, 0><<<grid, NT, 0, stream>>>(a); break;
    case 1: simt_gemm_kernel<T, BM, BN, BK, TM, TN, 1><<<grid, NT, 0, stream>>>(a); break;
    case 2: simt_gemm_kernel<T, BM, BN, BK, TM, TN, 2><<<grid, NT, 0, stream>>>(a); break;
    default: simt_gemm_kernel<T, BM, BN, BK, TM, TN, 3><<<grid, NT, 0, stream>>>(a); break;
  }
  note_launch();
  return cudaGetLastError();
}

template <typename T>
SimtArgs<T> make_args(const BatchDesc& d) {
  SimtArgs<T> a;
  a.transa = d.transa; a.transb = d.transb;
  a.m = d.m; a.n = d.n; a.k = d.k; a.lda = d.lda; a.ldb = d.ldb; a.ldc = d.ldc; a.batch = d.batch;
  a.A = (const typename RowTraits<T>::AB* const*)d.A; a.B = (const typename RowTraits<T>::AB* const*)d.B;
  a.C = (typename RowTraits<T>::C* const*)d.C;
  return a;
}

}  // namespace

cudaError_t launch_simt_gemm(const BatchDesc& d, cudaStream_t stream) {
  // Large tiles when both dimensions fill them and there is enough work to occupy the GPU with
  // them, small tiles otherwise (the tuning table or a forced configuration can override).
  const long big_tiles = ((d.m + 127) / 128) * ((d.n + 127) / 128) * d.batch;
  const bool big_default = d.m >= 128 && d.n >= 128 && big_tiles >= 2L * num_sms();
  const int cfg = choose_config(SSBLAS_PATH_SIMT, d.m, d.n, d.k, d.batch,
                                d.row == ROW_F32 ? (big_default ? 4 : d.k <= 64 ? 5 : 3) : (big_default ? 1 : 0));
  // fp32: configurations 3, 4 and 5 are the cp.async-pipelined kernels (gemm_sgemm.cu)
  if (d.row == ROW_F32 && cfg >= 3) return launch_sgemm_async(d, cfg, stream);
  const bool big = cfg == 1;
  switch (d.row) {
    case ROW_F32: {
      auto a = make_args<float>(d);
      a.alpha = d.alpha_f; a.beta = d.beta_f;
      return big ? launch_tile<float, 128, 128, 16, 8, 8>(a, stream)
                 : launch_tile<float, 64, 64, 16, 4, 4>(a, stream);
    }
    case ROW_F64: {
      auto a = make_args<double>(d);
      a.alpha = d.alpha_d; a.beta = d.beta_d;
      return big ? launch_tile<double, 128, 128, 8, 8, 8>(a, stream)
                 : launch_tile<double, 64, 64, 16, 4, 4>(a, stream);
    }
    case ROW_I8: {
      // signed operands only (the unsigned ones of the type extensions take the tensor-core
      // path; with k = 0 no operand is read)
      if ((d.a_unsigned || d.b_unsigned) && d.k > 0) return cudaErrorNotSupported;
      auto a = make_args<int8_t>(d);
      a.alpha = d.alpha_i; a.beta = d.beta_i;
      return launch_tile<int8_t, 64, 64, 32, 4, 4>(a, stream);
    }
    case ROW_F16: {
      if (d.c_f32) {
        auto a = make_args<HalfC32>(d);
        a.alpha = d.alpha_f; a.beta = d.beta_f;
        return launch_tile<HalfC32, 64, 64, 16, 4, 4>(a, stream);
      }
      auto a = make_args<HalfC16>(d);
      a.alpha = d.alpha_f; a.beta = d.beta_f;
      return launch_tile<HalfC16, 64, 64, 16, 4, 4>(a, stream);
    }
  }
  return cudaErrorInvalidValue;
}

GroupedSimt::~GroupedSimt() {
  for (void* p : {inst32, tiles32, inst64, tiles64, dmma_tiles[0], dmma_tiles[1], dmma_tiles[2], dmma_tiles[3],
                  sg_tiles[0], sg_tiles[1], sg_tiles[2], sg_tiles[3]})
    if (p) cudaFree(p);
}

cudaError_t plan_simt_grouped(const GroupedDesc& g, const std::vector<int>& members, GroupedSimt& out,
                              cudaStream_t st) {
  std::vector<SimtGInst> in32, in64;
  std::vector<int> t32, t64;
  struct DTile {
    long k;
    int li, a, b;
  };
  std::vector<DTile> td[4], ts[4];   // DMMA (fp64) and cp.async FFMA (fp32) tiles per layout
  for (int id : members) {
    const GroupedInst& x = g.inst[id];
    SimtGInst s{x.transa, x.transb, x.m, x.n, x.k, x.lda, x.ldb, x.ldc, x.idx, x.alpha_d, x.beta_d, x.alpha_f, x.beta_f};
    auto& iv = (x.row == ROW_F64) ? in64 : in32;
    auto& tv = (x.row == ROW_F64) ? t64 : t32;
    const int li = (int)iv.size();
    iv.push_back(s);
    // plain fp64 on the FP64 tensor cores, as the batched call does, unless its DMMA configuration
    // for this shape is 2 (the DFMA kernel)
    const bool dmma = x.row == ROW_F64 && choose_config(SSBLAS_PATH_DMMA, x.m, x.n, x.k, 1, 0) != 2;
    // plain fp32 on the cp.async FFMA tiles unless the SIMT configuration for this shape is 0 or 1
    // (the register-tiled SIMT kernel)
    const bool sg = x.row == ROW_F32 && choose_config(SSBLAS_PATH_SIMT, x.m, x.n, x.k, 1, 3) >= 3;
    const int lay = 2 * (x.transa == SSBLAS_OP_N ? 1 : 0) + (x.transb == SSBLAS_OP_T ? 1 : 0);
    for (long a = 0; a < (x.m + 63) / 64; ++a)
      for (long b = 0; b < (x.n + 63) / 64; ++b) {
        if (dmma || sg) {
          (dmma ? td : ts)[lay].push_back({x.k, li, (int)a, (int)b});
          continue;
        }
        tv.push_back(li);
        tv.push_back((int)a);
        tv.push_back((int)b);
      }
  }
  std::vector<int> tdl[4], tsl[4];
  auto flatten = [](std::vector<DTile>& v, std::vector<int>& out) {
    std::stable_sort(v.begin(), v.end(), [](const DTile& p, const DTile& q) { return p.k > q.k; });
    for (const DTile& t : v) {
      out.push_back(t.li);
      out.push_back(t.a);
      out.push_back(t.b);
    }
  };
  for (int l = 0; l < 4; ++l) {
    flatten(td[l], tdl[l]);
    flatten(ts[l], tsl[l]);
  }
  cudaError_t e;
  auto up = [&](void** dst, const void* src, size_t n) -> cudaError_t {
    if (n == 0) return cudaSuccess;
    cudaError_t r = cudaMalloc(dst, n);
    if (r) return r;
    return cudaMemcpyAsync(*dst, src, n, cudaMemcpyHostToDevice, st);
  };
  if ((e = up(&out.inst32, in32.data(), in32.size() * sizeof(SimtGInst))) ||
      (e = up(&out.tiles32, t32.data(), t32.size() * sizeof(int))) ||
      (e = up(&out.inst64, in64.data(), in64.size() * sizeof(SimtGInst))) ||
      (e = up(&out.tiles64, t64.data(), t64.size() * sizeof(int))))
    return e;
  for (int l = 0; l < 4; ++l)
    if ((e = up(&out.dmma_tiles[l], tdl[l].data(), tdl[l].size() * sizeof(int))) ||
        (e = up(&out.sg_tiles[l], tsl[l].data(), tsl[l].size() * sizeof(int))))
      return e;
  out.ntiles32 = (long)t32.size() / 3;
  out.ntiles64 = (long)t64.size() / 3;
  out.A = g.A; out.B = g.B; out.C = g.C;
  out.launches = (out.ntiles32 ? 1 : 0) + (out.ntiles64 ? 1 : 0);
  for (int l = 0; l < 4; ++l) {
    out.ndmma[l] = (long)tdl[l].size() / 3;
    out.nsg[l] = (long)tsl[l].size() / 3;
    out.launches += (out.ndmma[l] ? 1 : 0) + (out.nsg[l] ? 1 : 0);
  }
  return cudaStreamSynchronize(st);
}

cudaError_t launch_simt_grouped(const GroupedSimt& s, cudaStream_t st) {
  if (!s.ntiles32 && !s.ntiles64) return cudaSuccess;
  ProfScope prof("simt_grouped", st);
  if (s.ntiles32) {
    simt_grouped_kernel<float, 64, 64, 16, 4, 4><<<(unsigned)s.ntiles32, 256, 0, st>>>(
        (const SimtGInst*)s.inst32, (const int*)s.tiles32, (const float* const*)s.A, (const float* const*)s.B,
        (float* const*)s.C);
    note_launch();
  }
  if (s.ntiles64) {
    simt_grouped_kernel<double, 64, 64, 16, 4, 4><<<(unsigned)s.ntiles64, 256, 0, st>>>(
        (const SimtGInst*)s.inst64, (const int*)s.tiles64, (const double* const*)s.A, (const double* const*)s.B,
        (double* const*)s.C);
    note_launch();
  }
  return cudaGetLastError();
}

}  // namespace ssb
