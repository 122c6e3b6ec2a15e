// Internal interfaces shared by the host layer (api.cpp) and the kernel files.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include <nvtx3/nvToolsExt.h>

#include "../../include/ssblasBatch.h"
#include "per_device.h"

namespace ssb {

// Type rows: the reference's three (fp32, fp64, int8 -> int32), plus the fp16 row of the type
// extensions (fp16 inputs, fp16 or fp32 C, fp32 scale and accumulation).
enum Row { ROW_F32 = 0, ROW_F64 = 1, ROW_I8 = 2, ROW_F16 = 3 };

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
  // int8 row: operands of type SSBLAS_R_8U (type extensions); fp16 row: C in fp32 instead of fp16
  bool a_unsigned, b_unsigned;
  bool c_f32;
  // fp32 row with computeType SSBLAS_COMPUTE_32F under SSBLAS_EXT_COMPUTE_TYPE: FP32 arithmetic
  // (no 3xBF16 emulation)
  bool exact_f32;
};

// Process-wide knobs (set through the extension entry points)
struct Settings {
  cudaStream_t stream = nullptr;
  bool synchronous = true;
  int math_mode = SSBLAS_MATH_PLAIN;
  int ozaki_slices = 0;        // 0 = automatic: from ozaki_tolerance
  double ozaki_tolerance = 0;  // 0 = kOzakiDefaultTolerance
  int fault = 0;               // one-shot ssblasFault_t armed by ssblasSetFaultInjection
  int extensions = 0;          // ssblasExtension_t flags (ssblasSetExtensions)
  bool log = false;            // SSBLAS_LOG: one line per call on stderr (path, slices, launches)
};
Settings& settings();

// Host-side lock of the library state (settings, run info, workspaces, per-device tables): every
// entry point that launches work holds it for the whole call.
std::unique_lock<std::mutex> lock_api();
// Clears the run info of ssblasGetLastRunInfo at the start of a call.
void reset_run_info();
// Waits for `st`, reads and clears the device error flag; INTERNAL_ERROR (and the flag's code in
// the run info) when a kernel's bounded wait gave up.
ssblasStatus_t check_device_error(cudaStream_t st);

// ---- Ozaki slice count ----
// A-priori bound of the Ozaki emulation with S int8 slices per operand, per product term, in units
// of |alpha| * 2^(e_i + f_j) (2^e_i, 2^f_j: the powers of two just above the largest magnitude of
// row i of op(A) and of column j of op(B)): (S + 1) * 2^(2 - 8S). It covers rounding op(A) and
// op(B) to 8S - 2 bits below their row (column) exponent and the dropped slice pairs p + q >= S.
double ozaki_term_bound(int slices);
// Default target of the slice choice: 4u (u = 2^-53), the 4*k*u tolerance of an FP64 GEMM spread
// over its k product terms. It gives 7 slices.
constexpr double kOzakiDefaultTolerance = 0x1p-51;
// Slices of the next fp64 Ozaki call: the forced count (ssblasSetOzakiSlices), else the smallest
// count in [3, 8] whose bound meets the tolerance (ssblasSetOzakiTolerance).
int ozaki_slices_for_call();
// The tensor-core paths can run here (sm_100 device, tensor-map encoder present).
bool tcgen05_available();

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
// plain fp32 with TMA staging (gemm_sgemm_tma.cu); cudaErrorNotSupported unless the instances are
// equally spaced with 16-byte-aligned bases, strides and leading dimensions
bool sgemm_tma_fits(const BatchDesc& d);
cudaError_t launch_sgemm_tma(const BatchDesc& d, int variant, cudaStream_t stream);
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
// fp32 via three BF16 products in one kernel for instances of at most 128 x 128 (bf16x3_small.cu)
bool bf16x3_small_fits(const BatchDesc& d);
cudaError_t launch_bf16x3_small(const BatchDesc& d, cudaStream_t stream);
// fp16 inputs (type extension row) on tcgen05 kind::f16, fp32 accumulation
cudaError_t launch_f16_tcgen05(const BatchDesc& d, cudaStream_t stream);

// Ordinal of the current device, or -1 when it cannot be read or lies outside the per-device
// tables (per_device.h).
int current_device();
// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) of `kern` on the current device, once per
// device (`done` is the caller's per-kernel table): the attribute belongs to one device's context.
template <class K>
inline cudaError_t smem_attr_once(bool (&done)[kMaxDevices], K kern, int bytes) {
  return (cudaError_t)once_per_device(
      done, current_device(),
      [&] { return (int)cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes); },
      (int)cudaErrorInvalidDevice);
}

// SM count of the current device.
int num_sms();

// Tiled TMA tensor map of `rank` dimensions (dims[0] innermost; strides_bytes[i] is the stride
// of dimension i + 1), box `box`, swizzle 0 / 32 / 64 / 128 bytes, zero fill outside the tensor.
// False if the driver entry point is missing or the encoder rejects the arguments.
bool make_tiled_map(CUtensorMap* map, CUtensorMapDataType dt, int rank, const void* base, const long* dims,
                    const long* strides_bytes, const int* box, int swz_bytes);

// Configuration index of a kernel family for a problem (tune.cpp): forced, tuned, or `fallback`.
int choose_config(int path, long m, long n, long k, long batch, int fallback);
// the configuration forced by ssblasSetKernelConfig for `path`, -1 if none
int forced_config(int path);

// Optional per-kernel CUDA-event timing (ssblasSetProfiling): records an event pair around each
// launch on its stream; ssblasGetProfile resolves them. Each launch is also an NVTX range of the
// same name (slicing, GEMM, pre-pass phases), nested in the range of the API call, for timeline
// tools; with no tool attached an NVTX call is a test of one function pointer.
void prof_start(const char* name, cudaStream_t st);
void prof_stop(cudaStream_t st);
struct ProfScope {
  cudaStream_t st;
  ProfScope(const char* name, cudaStream_t s) : st(s) {
    nvtxRangePushA(name);
    prof_start(name, s);
  }
  ~ProfScope() {
    prof_stop(st);
    nvtxRangePop();
  }
};
// NVTX range of one API call.
struct ApiRange {
  explicit ApiRange(const char* name) { nvtxRangePushA(name); }
  ~ApiRange() { nvtxRangePop(); }
};

}  // namespace ssb
