// Grouped batched GEMM: host-side description shared by api.cpp, grouped.cu and gemm_simt.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "internal.h"

namespace ssb {

struct GroupedInst {
  Row row;
  int transa, transb;
  long m, n, k, lda, ldb, ldc;
  long idx;                  // position in the A/B/C pointer arrays
  double alpha_d, beta_d;
  float alpha_f, beta_f;
  int32_t alpha_i, beta_i;
};

struct GroupedDesc {
  std::vector<GroupedInst> inst;
  const void* const* A;      // device arrays of device pointers
  const void* const* B;
  void* const* C;
};

// plain fp32/fp64 instances of a grouped call (64 x 64 tiles: FFMA / DMMA kernels, or the SIMT
// kernel where a forced configuration asks for it)
struct SimtGInst {
  int transa, transb;
  long m, n, k, lda, ldb, ldc, idx;
  double alpha_d, beta_d;
  float alpha_f, beta_f;
};
struct GroupedSimt {
  void *inst32 = nullptr, *tiles32 = nullptr, *inst64 = nullptr, *tiles64 = nullptr;
  long ntiles32 = 0, ntiles64 = 0;
  // fp64 tiles for the FP64 tensor cores (gemm_dmma.cu), one table per op(A) / op(B) layout
  // (2 * (op(A) rows contiguous) + (op(B) columns contiguous)), longest k first; their instances
  // are in inst64
  void* dmma_tiles[4] = {};
  long ndmma[4] = {};
  // fp32 tiles for the cp.async FFMA kernel (gemm_sgemm.cu), the same way; instances in inst32
  void* sg_tiles[4] = {};
  long nsg[4] = {};
  const void* const* A = nullptr;
  const void* const* B = nullptr;
  void* const* C = nullptr;
  int launches = 0;
  ~GroupedSimt();
};
cudaError_t plan_simt_grouped(const GroupedDesc& g, const std::vector<int>& members, GroupedSimt& out,
                              cudaStream_t st);
cudaError_t launch_simt_grouped(const GroupedSimt& s, cudaStream_t st);
cudaError_t launch_dmma_grouped(const GroupedSimt& s, cudaStream_t st);
cudaError_t launch_sgemm_grouped(const GroupedSimt& s, cudaStream_t st);

// Runs all instances with device-resident operands: one pre-pass and one persistent GEMM launch per
// kind, replayed from a captured CUDA graph when the same call signature repeats.
cudaError_t grouped_run(const GroupedDesc& g, cudaStream_t st);
void grouped_release();

}  // namespace ssb
