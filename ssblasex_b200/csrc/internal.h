// Internal interfaces shared by the host layer (api.cpp) and the kernel files.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ssblasBatch.h"

namespace ssb {

enum Row { ROW_F32 = 0, ROW_F64 = 1, ROW_I8 = 2 };

// One uniform batch: every instance has the same shape; the pointer arrays live in device memory.
struct BatchDesc {
  Row row;
  int transa, transb;      // SSBLAS_OP_N / SSBLAS_OP_T
  long m, n, k;
  long lda, ldb, ldc;
  long batch;
  const void* const* A;    // device array of `batch` device pointers
  const void* const* B;
  void* const* C;
  // When the instances are equally spaced in memory, base + b*stride (bytes) equals A[b]; the
  // tensor-core paths then address the batch through one tensor map. stride 0 = not uniform.
  const void* A0; long strideA;
  const void* B0; long strideB;
  void* C0; long strideC;
  // scalars by value, in the row's scale type
  double alpha_d, beta_d;
  float alpha_f, beta_f;
  int32_t alpha_i, beta_i;
};

// Process-wide knobs (set through the extension entry points)
struct Settings {
  cudaStream_t stream = nullptr;
  bool synchronous = true;
  int math_mode = SSBLAS_MATH_PLAIN;
  int ozaki_slices = 0;        // 0 = automatic
};
Settings& settings();

// Device workspace: a grow-only cached allocation per device and slot.
enum WsSlot { WS_PTRS = 0, WS_PACK_A, WS_PACK_B, WS_EXP, WS_STAGE_A, WS_STAGE_B, WS_STAGE_C, WS_MISC, WS_SPLIT,
               WS_SPLIT_CNT, WS_ROWMAX, WS_NUM };
void* workspace(WsSlot slot, size_t bytes, cudaError_t* err);

// Launch bookkeeping for ssblasGetLastRunInfo and the benchmark's launch count.
void note_launch(int count = 1);
void note_path(int path, int slices = 0);
void note_splits(int splits);

// Device-side error flag (set by kernels whose bounded waits give up).
int* device_error_flag();

// ---- kernel entry points (each returns a CUDA error code; launches on `stream`) ----
cudaError_t launch_simt_gemm(const BatchDesc& d, cudaStream_t stream);
// plain fp32 with a cp.async pipeline (config 3: 64 x 64 tiles, 4: 128 x 128)
cudaError_t launch_sgemm_async(const BatchDesc& d, int config, cudaStream_t stream);
// plain fp64 on the FP64 tensor cores (DMMA)
cudaError_t launch_dmma_f64(const BatchDesc& d, cudaStream_t stream);
// int8 -> int32 on tcgen05; returns cudaErrorNotSupported when the layout is not eligible.
cudaError_t launch_i8_tcgen05(const BatchDesc& d, cudaStream_t stream);
// fp64 via Ozaki int8 slices; slices = per-operand slice count
cudaError_t launch_ozaki_f64(const BatchDesc& d, int slices, cudaStream_t stream);
// the Ozaki GEMM phase alone, on slice planes and exponents already in (caller-provided) memory:
// planes [batch][S][rows][Kp] for op(A) then op(B), exponents [batch][m] then [batch][n]
cudaError_t launch_ozaki_gemm_on(const BatchDesc& d, int slices, const int8_t* planes_a, const int8_t* planes_b,
                                 const int32_t* exps, long Kp, cudaStream_t stream);
// fp32 via three BF16 products
cudaError_t launch_bf16x3_f32(const BatchDesc& d, cudaStream_t stream);

int num_sms();

// Tiled TMA tensor map of `rank` dimensions (dims[0] innermost; strides_bytes[i] is the stride
// of dimension i + 1), box `box`, swizzle 0 / 32 / 64 / 128 bytes, zero fill outside the tensor.
// False if the driver entry point is missing or the encoder rejects the arguments.
bool make_tiled_map(CUtensorMap* map, CUtensorMapDataType dt, int rank, const void* base, const long* dims,
                    const long* strides_bytes, const int* box, int swz_bytes);

// Configuration index of a kernel family for a problem (tune.cpp): forced, tuned, or `fallback`.
int choose_config(int path, long m, long n, long k, long batch, int fallback);

// Optional per-kernel CUDA-event timing (ssblasSetProfiling): records an event pair around each
// launch on its stream; ssblasGetProfile resolves them.
void prof_start(const char* name, cudaStream_t st);
void prof_stop(cudaStream_t st);
struct ProfScope {
  cudaStream_t st;
  ProfScope(const char* name, cudaStream_t s) : st(s) { prof_start(name, s); }
  ~ProfScope() { prof_stop(st); }
};

}  // namespace ssb
