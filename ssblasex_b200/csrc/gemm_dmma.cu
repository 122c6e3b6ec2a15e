// Plain FP64 batched GEMM on the FP64 tensor cores (DMMA: mma.sync.m8n8k4.f64).
//
// The fp64 row of ssblasGemmBatchedEx in its plain (non-emulated) form. Semantics follow the
// reference (hirokitokura/ssblasEx): C <- beta*C, not read when beta == 0
// (src/include/CScale/Xgemm_scale_kernel.hpp:164-176), then C <- C + acc*alpha with one fused
// multiply-add (src/include/GemmCore/Xgemm_kernel_sve_v4x5_1.hpp:93-127). The reference adds
// alpha*acc once per 512-wide K block; here it is added once, which differs only by rounding.
//
// Design: one CTA per (BM x BN tile, instance). op(A) and op(B) tiles are copied into shared
// memory by cp.async in a STAGES-deep ring (the copies for K step kt + STAGES - 1 are in flight
// while step kt is multiplied), each in the orientation it has in global memory -- the copy
// absorbs op(A)/op(B): an operand whose rows (m or n) are contiguous is staged [k][mn], one whose
// K is contiguous is staged [mn][k]. Each warp owns a WM x WN block of C as (WM/8) x (WN/8)
// DMMA accumulator tiles. Row pitches are 4 (mod 16) doubles, so the fragment loads (lane l reads
// (mn = l/4, k = l%4) of an 8 x 4 block) hit 16 distinct 8-byte bank pairs per half-warp.
//
// 16-byte copies when the instance's base pointer is 16-byte aligned and its ld is even, else
// 8-byte copies; elements outside the matrix are zero-filled by the copy itself (src-size).
#include <cuda_runtime.h>
#include <stdint.h>

#include "grouped.h"
#include "internal.h"

namespace ssb {
namespace {

struct DmmaArgs {
  long m, n, k, lda, ldb, ldc, batch;
  const double* const* A;
  const double* const* B;
  double* const* C;
  double alpha, beta;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
// cp.async of `bytes` valid bytes (0, 8 or 16) into a 16- or 8-byte slot; the rest is zero-filled
__device__ __forceinline__ void cp16(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp8(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// D (8x8, two per lane) += A (8x4, row) * B (4x8, col)
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

template <int BM, int BN, int BK>
struct DmmaSmem {
  static constexpr int PMN_A = BM + 4;    // [k][m] pitch
  static constexpr int PMN_B = BN + 4;    // [k][n] pitch
  static constexpr int PK = BK + 4;       // [mn][k] pitch
  static constexpr int A_MAX = (BK * PMN_A > BM * PK) ? BK * PMN_A : BM * PK;   // doubles
  static constexpr int B_MAX = (BK * PMN_B > BN * PK) ? BK * PMN_B : BN * PK;
  static constexpr int STAGE = A_MAX + B_MAX;
};

// Copies the (rows x BK) slab of one operand at (r0, k0) into a stage buffer.
// MN: rows contiguous in global memory (element (r, k) at X[r + k*ld]) -> staged [k][r];
// otherwise element (r, k) at X[r*ld + k] -> staged [r][k].
template <int ROWS, int BK, int NT, bool MN>
__device__ __forceinline__ void load_slab(double* dst, const double* __restrict__ X, long nrows, long K, long ld,
                                          long r0, long k0, bool vec) {
  constexpr int P = MN ? ROWS + 4 : BK + 4;
  constexpr int CHUNKS = ROWS * BK / 2;   // pairs of doubles
  static_assert(CHUNKS % NT == 0, "slab/threads mismatch");
  const int t = threadIdx.x;
#pragma unroll
  for (int q = 0; q < CHUNKS / NT; ++q) {
    const int idx = t + q * NT;
    int rr, kk;       // first element of the pair: pair runs along r (MN) or along k
    if (MN) { kk = idx / (ROWS / 2); rr = 2 * (idx % (ROWS / 2)); }
    else { rr = idx / (BK / 2); kk = 2 * (idx % (BK / 2)); }
    const long gr = r0 + rr, gk = k0 + kk;
    double* s = MN ? dst + kk * P + rr : dst + rr * P + kk;
    // valid elements of the pair
    long nvalid;
    if (MN) nvalid = (gk < K) ? (nrows - gr < 2 ? nrows - gr : 2) : 0;
    else nvalid = (gr < nrows) ? (K - gk < 2 ? K - gk : 2) : 0;
    if (nvalid < 0) nvalid = 0;
    const double* g = (nvalid > 0) ? (MN ? X + gr + gk * ld : X + gr * ld + gk) : X;
    if (vec) {
      cp16(smem_addr(s), g, (int)(8 * nvalid));
    } else {
      cp8(smem_addr(s), g, nvalid > 0 ? 8 : 0);
      const double* g1 = (nvalid > 1) ? g + 1 : X;
      cp8(smem_addr(s + 1), g1, nvalid > 1 ? 8 : 0);
    }
  }
}

// One BM x BN tile of C = alpha op(A) op(B) + beta C for one instance, by the whole CTA: the K loop
// over the stage ring, then the epilogue. Leaves the stage buffers free (every copy has landed and
// every thread has passed a barrier after its last read).
template <int BM, int BN, int BK, int WM, int WN, int STAGES, bool A_MN, bool B_MN>
__device__ __forceinline__ void dmma_tile(const double* __restrict__ A, const double* __restrict__ B,
                                          double* __restrict__ C, long m, long n, long k, long lda, long ldb,
                                          long ldc, double alpha, double beta, long m0, long n0, double* smem) {
  constexpr int NWM = BM / WM, NWN = BN / WN;
  constexpr int NT = NWM * NWN * 32;
  constexpr int MI = WM / 8, NI = WN / 8;
  using Sm = DmmaSmem<BM, BN, BK>;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int wm = warp % NWM, wn = warp / NWM;
  const int fr = lane >> 2, fk = lane & 3;    // fragment row (m or n) and k within an 8x4 block
  const bool vecA = ((uintptr_t)A % 16 == 0) && (lda % 2 == 0);
  const bool vecB = ((uintptr_t)B % 16 == 0) && (ldb % 2 == 0);

  double acc[MI][NI][2];
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < NI; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  const long ktiles = (k + BK - 1) / BK;
  auto issue = [&](long kt) {
    double* sa = smem + (kt % STAGES) * Sm::STAGE;
    double* sb = sa + Sm::A_MAX;
    load_slab<BM, BK, NT, A_MN>(sa, A, m, k, lda, m0, kt * BK, vecA);
    load_slab<BN, BK, NT, B_MN>(sb, B, n, k, ldb, n0, kt * BK, vecB);
  };
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < ktiles) issue(s);
    cp_commit();
  }
  for (long kt = 0; kt < ktiles; ++kt) {
    cp_wait<STAGES - 2>();
    __syncthreads();
    if (kt + STAGES - 1 < ktiles) issue(kt + STAGES - 1);
    cp_commit();
    const double* sa = smem + (kt % STAGES) * Sm::STAGE;
    const double* sb = sa + Sm::A_MAX;
#pragma unroll 2
    for (int k4 = 0; k4 < BK / 4; ++k4) {
      const int kk = 4 * k4 + fk;
      double af[MI], bf[NI];
#pragma unroll
      for (int i = 0; i < MI; ++i) {
        const int r = wm * WM + 8 * i + fr;
        af[i] = A_MN ? sa[kk * Sm::PMN_A + r] : sa[r * Sm::PK + kk];
      }
#pragma unroll
      for (int j = 0; j < NI; ++j) {
        const int c = wn * WN + 8 * j + fr;
        bf[j] = B_MN ? sb[kk * Sm::PMN_B + c] : sb[c * Sm::PK + kk];
      }
#pragma unroll
      for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < NI; ++j) dmma(acc[i][j], af[i], bf[j]);
    }
  }
  cp_wait<0>();
  __syncthreads();   // the next tile's copies reuse the stage buffers

  // epilogue: lane holds C rows m0 + wm*WM + 8i + fr, columns n0 + wn*WN + 8j + 2fk + {0,1}
  const bool read_c = beta != 0.0;
#pragma unroll
  for (int j = 0; j < NI; ++j) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const long gj = n0 + wn * WN + 8 * j + 2 * fk + h;
      if (gj >= n) continue;
      double cv[MI];
#pragma unroll
      for (int i = 0; i < MI; ++i) {
        const long gi = m0 + wm * WM + 8 * i + fr;
        cv[i] = (read_c && gi < m) ? C[gi + gj * ldc] : 0.0;
      }
#pragma unroll
      for (int i = 0; i < MI; ++i) {
        const long gi = m0 + wm * WM + 8 * i + fr;
        if (gi < m) {
          const double tb = read_c ? beta * cv[i] : 0.0;
          C[gi + gj * ldc] = fma(acc[i][j][h], alpha, tb);
        }
      }
    }
  }
}

template <int BM, int BN, int BK, int WM, int WN, int STAGES, int MINB, bool A_MN, bool B_MN>
__global__ void __launch_bounds__((BM / WM) * (BN / WN) * 32, MINB) dmma_gemm_kernel(DmmaArgs args) {
  extern __shared__ __align__(16) double smem[];
  const long tiles_m = (args.m + BM - 1) / BM;
  const long m0 = (blockIdx.x % tiles_m) * BM;
  const long n0 = (blockIdx.x / tiles_m) * BN;
  for (long b = blockIdx.y; b < args.batch; b += gridDim.y)
    dmma_tile<BM, BN, BK, WM, WN, STAGES, A_MN, B_MN>(args.A[b], args.B[b], args.C[b], args.m, args.n, args.k,
                                                       args.lda, args.ldb, args.ldc, args.alpha, args.beta, m0, n0,
                                                       smem);
}

// Grouped form (plain fp64 instances of ssblasGemmGroupedBatchedEx): one CTA per (instance,
// 64 x 64 tile) entry of a tile table whose instances all have this op(A) / op(B) layout.
constexpr int kGBM = 64, kGBK = 16, kGW = 32, kGST = 4;
template <bool A_MN, bool B_MN>
__global__ void __launch_bounds__((kGBM / kGW) * (kGBM / kGW) * 32, 2)
dmma_grouped_kernel(const SimtGInst* __restrict__ inst, const int* __restrict__ tiles, const double* const* A,
                    const double* const* B, double* const* C) {
  extern __shared__ __align__(16) double smem[];
  const int* t = tiles + 3 * (long)blockIdx.x;
  const SimtGInst g = inst[t[0]];
  dmma_tile<kGBM, kGBM, kGBK, kGW, kGW, kGST, A_MN, B_MN>(A[g.idx], B[g.idx], C[g.idx], g.m, g.n, g.k, g.lda, g.ldb,
                                                          g.ldc, g.alpha_d, g.beta_d, (long)t[1] * kGBM,
                                                          (long)t[2] * kGBM, smem);
}

template <int BM, int BN, int BK, int WM, int WN, int STAGES, int MINB, bool A_MN, bool B_MN>
cudaError_t launch_cfg(const DmmaArgs& a, cudaStream_t st) {
  constexpr int NT = (BM / WM) * (BN / WN) * 32;
  constexpr int SMEM = STAGES * DmmaSmem<BM, BN, BK>::STAGE * 8;
  auto kern = dmma_gemm_kernel<BM, BN, BK, WM, WN, STAGES, MINB, A_MN, B_MN>;
  static bool attr[kMaxDevices] = {};
  if (cudaError_t e = smem_attr_once(attr, kern, SMEM)) return e;
  const long tiles = ((a.m + BM - 1) / BM) * ((a.n + BN - 1) / BN);
  if (tiles > 0x7fffffffL) return cudaErrorInvalidValue;
  dim3 grid((unsigned)tiles, (unsigned)(a.batch < 65535 ? a.batch : 65535));
  kern<<<grid, NT, SMEM, st>>>(a);
  return cudaGetLastError();
}

template <int BM, int BN, int BK, int WM, int WN, int STAGES, int MINB>
cudaError_t launch_layout(const DmmaArgs& a, bool a_mn, bool b_mn, cudaStream_t st) {
  if (a_mn && b_mn) return launch_cfg<BM, BN, BK, WM, WN, STAGES, MINB, true, true>(a, st);
  if (a_mn) return launch_cfg<BM, BN, BK, WM, WN, STAGES, MINB, true, false>(a, st);
  if (b_mn) return launch_cfg<BM, BN, BK, WM, WN, STAGES, MINB, false, true>(a, st);
  return launch_cfg<BM, BN, BK, WM, WN, STAGES, MINB, false, false>(a, st);
}

template <bool A_MN, bool B_MN>
cudaError_t launch_grouped_layout(const GroupedSimt& s, int lay, cudaStream_t st) {
  constexpr int SMEM = kGST * DmmaSmem<kGBM, kGBM, kGBK>::STAGE * 8;
  auto kern = dmma_grouped_kernel<A_MN, B_MN>;
  static bool attr[kMaxDevices] = {};
  if (cudaError_t e = smem_attr_once(attr, kern, SMEM)) return e;
  kern<<<(unsigned)s.ndmma[lay], (kGBM / kGW) * (kGBM / kGW) * 32, SMEM, st>>>(
      (const SimtGInst*)s.inst64, (const int*)s.dmma_tiles[lay], (const double* const*)s.A,
      (const double* const*)s.B, (double* const*)s.C);
  note_launch();
  return cudaGetLastError();
}

}  // namespace

// The plain fp64 tiles of a grouped call, one launch per op(A) / op(B) layout present
// (layout index = 2 * (op(A) rows contiguous) + (op(B) columns contiguous)).
cudaError_t launch_dmma_grouped(const GroupedSimt& s, cudaStream_t st) {
  if (!s.ndmma[0] && !s.ndmma[1] && !s.ndmma[2] && !s.ndmma[3]) return cudaSuccess;
  ProfScope prof("dmma_grouped", st);
  cudaError_t e = cudaSuccess;
  for (int lay = 0; lay < 4 && e == cudaSuccess; ++lay) {
    if (!s.ndmma[lay]) continue;
    switch (lay) {
      case 3: e = launch_grouped_layout<true, true>(s, lay, st); break;
      case 2: e = launch_grouped_layout<true, false>(s, lay, st); break;
      case 1: e = launch_grouped_layout<false, true>(s, lay, st); break;
      default: e = launch_grouped_layout<false, false>(s, lay, st); break;
    }
  }
  return e;
}

cudaError_t launch_dmma_f64(const BatchDesc& d, cudaStream_t st) {
  DmmaArgs a;
  a.m = d.m; a.n = d.n; a.k = d.k; a.lda = d.lda; a.ldb = d.ldb; a.ldc = d.ldc; a.batch = d.batch;
  a.A = (const double* const*)d.A;
  a.B = (const double* const*)d.B;
  a.C = (double* const*)d.C;
  a.alpha = d.alpha_d;
  a.beta = d.beta_d;
  const bool a_mn = d.transa == SSBLAS_OP_N;   // op(A) rows (m) contiguous
  const bool b_mn = d.transb == SSBLAS_OP_T;   // op(B) columns (n) contiguous
  // Configurations (ssblasSetKernelConfig(SSBLAS_PATH_DMMA, c)):
  //   0: 64 x 64 tiles, 4 warps of 32 x 32, 16-deep K stages x 4
  //   1: 128 x 128 tiles, 8 warps of 64 x 32, 16-deep K stages x 4
  //   3: 128 x 128 tiles, 16 warps of 32 x 32, 16-deep K stages x 4
  //   4: 128 x 128 tiles, 16 warps of 32 x 32, 32-deep K stages x 3
  // (2 selects the DFMA SIMT kernel, handled by the caller). Default: configuration 4 when there
  // are enough 128 x 128 tiles to fill the GPU (fastest on 32 x 1024^3: 2.40 ms against 2.54 for
  // 3 and 2.60 for 1), else 0.
  const long big_tiles = ((d.m + 127) / 128) * ((d.n + 127) / 128) * d.batch;
  const bool big_default = d.m >= 128 && d.n >= 128 && big_tiles >= 2L * num_sms();
  const int cfg = choose_config(SSBLAS_PATH_DMMA, d.m, d.n, d.k, d.batch, big_default ? 4 : 0);
  ProfScope prof("dmma_gemm", st);
  cudaError_t e;
  switch (cfg) {
    case 1: e = launch_layout<128, 128, 16, 64, 32, 4, 1>(a, a_mn, b_mn, st); break;
    case 3: e = launch_layout<128, 128, 16, 32, 32, 4, 1>(a, a_mn, b_mn, st); break;
    case 4: e = launch_layout<128, 128, 32, 32, 32, 3, 1>(a, a_mn, b_mn, st); break;
    default: e = launch_layout<64, 64, 16, 32, 32, 4, 2>(a, a_mn, b_mn, st); break;
  }
  note_launch();
  return e;
}

}  // namespace ssb
