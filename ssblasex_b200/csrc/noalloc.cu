// ssblasGemmBatchedExNoAlloc: the FP64 Ozaki-emulated batched GEMM with its scratch memory in a
// fixed, statically sized device array instead of the library's cudaMalloc'd workspace.
//
// Who needs it: callers that cannot let a library allocate device memory -- services that hand
// all of the GPU's memory to their own pool allocator up front, and latency-critical loops in
// which a cudaMalloc/cudaFree (which may synchronise the whole device) is not allowed. Such a
// caller passes its inputs and outputs as usual; the slice planes and exponents the emulation
// needs live in g_noalloc_scratch below.
//
// Costs and rules of the static array:
//   * every GPU on which the library is loaded holds kNoAllocScratchBytes (64 MiB) for this
//     array until the process exits, whether or not the entry point is used;
//   * a problem needs S*(m+n)*Kp*batch + 4*(m+n)*batch bytes (S = Ozaki slices, Kp = k rounded
//     up to 16); larger problems are rejected with SSBLAS_STATUS_INVALID_VALUE and a message on
//     stderr -- nothing is computed and C is untouched;
//   * all calls share the one array per device and it keeps the previous call's contents. Calls
//     whose GPU work overlaps (different streams or host threads without ordering) race on it;
//     the caller must order them. No part of the array has to start at zero: the slicing
//     pre-pass writes every byte and exponent the GEMM phase then reads.
//   * the first call on each device looks the array's device address up (cudaGetSymbolAddress
//     with that device current) and caches it; make that first call before starting any stream
//     capture on the device.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "internal.h"
#include "prepass.h"

namespace ssb {
namespace {

constexpr size_t kNoAllocScratchBytes = 64ull << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (host code cannot use the symbol
// itself: in host code its name is only a stand-in for the device object).
cudaError_t scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return cudaSuccess;
}

bool on_device(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

inline long round_up(long x, long a) { return (x + a - 1) / a * a; }

}  // namespace
}  // namespace ssb

using namespace ssb;

extern "C" ssblasStatus_t ssblasGemmBatchedExNoAlloc(
    ssblasOperation_t transa, ssblasOperation_t transb, SSINT m, SSINT n, SSINT k, const void* alpha,
    const void* const A[], ssblasDataType_t Atype, const SSINT lda, const void* const B[], ssblasDataType_t Btype,
    const SSINT ldb, const void* beta, void* const C[], ssblasDataType_t Ctype, const SSINT ldc,
    const SSINT batchCount, ssblasComputeType_t, ssblasGemmAlgo_t) {
  if (!(Atype == SSBLAS_R_64F && Btype == SSBLAS_R_64F && Ctype == SSBLAS_R_64F)) {
    // only the fp64 row has this variant; the other type rows are valid elsewhere
    const bool valid_row = (Atype == SSBLAS_R_32F && Btype == SSBLAS_R_32F && Ctype == SSBLAS_R_32F) ||
                           (Atype == SSBLAS_R_8I && Btype == SSBLAS_R_8I && Ctype == SSBLAS_R_32I);
    return valid_row ? SSBLAS_STATUS_NOTIMPLEMENTED_ERROR : SSBLAS_STATUS_INVALID_VALUE;
  }
  if ((transa != SSBLAS_OP_N && transa != SSBLAS_OP_T) || (transb != SSBLAS_OP_N && transb != SSBLAS_OP_T))
    return SSBLAS_STATUS_INVALID_VALUE;
  if (m <= 0 || n <= 0 || batchCount <= 0) return SSBLAS_STATUS_INTERNAL_ERROR;
  if (k <= 0) return SSBLAS_STATUS_SUCCESS;
  if (!alpha || !beta || !A || !B || !C) return SSBLAS_STATUS_INVALID_VALUE;
  const long arows = (transa == SSBLAS_OP_N) ? m : k, brows = (transb == SSBLAS_OP_N) ? k : n;
  if (lda < arows || ldb < brows || ldc < m) return SSBLAS_STATUS_INVALID_VALUE;
  if (k > 16384) return SSBLAS_STATUS_INVALID_VALUE;   // int32 exactness bound of the emulation
  // this entry point takes device arrays of device pointers only: staging host data would allocate
  if (!on_device((const void*)A) || !on_device((const void*)B) || !on_device((const void*)C))
    return SSBLAS_STATUS_INVALID_VALUE;

  const int S = settings().ozaki_slices == 0 ? 7 : settings().ozaki_slices;
  const long Kp = round_up(k, 16);
  const size_t bytes_a = (size_t)S * m * Kp * batchCount;
  const size_t bytes_b = (size_t)S * n * Kp * batchCount;
  const size_t bytes_e = sizeof(int32_t) * (size_t)(m + n) * batchCount;
  const size_t off_b = round_up((long)bytes_a, 256), off_e = round_up((long)(off_b + bytes_b), 256);
  const size_t need = off_e + bytes_e;
  if (need > kNoAllocScratchBytes) {
    fprintf(stderr,
            "ssblasGemmBatchedExNoAlloc: this problem needs %zu bytes of scratch; the static maximum is %zu "
            "bytes (use ssblasGemmBatchedEx, or split the batch)\n",
            need, kNoAllocScratchBytes);
    return SSBLAS_STATUS_INVALID_VALUE;
  }

  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  void* scratch = nullptr;
  cudaError_t e = scratch_address(&scratch);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return SSBLAS_STATUS_INTERNAL_ERROR;
  }
  int8_t* pa = (int8_t*)scratch;
  int8_t* pb = (int8_t*)scratch + off_b;
  int32_t* ex = (int32_t*)((uint8_t*)scratch + off_e);

  BatchDesc d{};
  d.row = ROW_F64;
  d.transa = transa; d.transb = transb;
  d.m = m; d.n = n; d.k = k; d.lda = lda; d.ldb = ldb; d.ldc = ldc; d.batch = batchCount;
  d.A = A; d.B = B; d.C = C;
  d.alpha_d = *(const double*)alpha;
  d.beta_d = *(const double*)beta;

  cudaStream_t st = settings().stream;
  const long sa = m * Kp, sb = n * Kp;
  PlaneArgs pa_args{A, m, k, lda, transa == SSBLAS_OP_T, batchCount, pa, Kp, sa, sa * S};
  PlaneArgs pb_args{B, n, k, ldb, transb == SSBLAS_OP_N, batchCount, pb, Kp, sb, sb * S};
  if ((e = launch_ozaki_slice(pa_args, S, ex, st)) != cudaSuccess ||
      (e = launch_ozaki_slice(pb_args, S, ex + m * batchCount, st)) != cudaSuccess ||
      (e = launch_ozaki_gemm_on(d, S, pa, pb, ex, Kp, st)) != cudaSuccess) {
    cudaGetLastError();
    return SSBLAS_STATUS_INTERNAL_ERROR;
  }
  if (!settings().synchronous) return SSBLAS_STATUS_SUCCESS;
  if (cudaStreamSynchronize(st) != cudaSuccess) return SSBLAS_STATUS_INTERNAL_ERROR;
  int* flag = device_error_flag();
  int h = 0;
  if (!flag || cudaMemcpy(&h, flag, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return SSBLAS_STATUS_INTERNAL_ERROR;
  if (h != 0) {
    const int zero = 0;
    cudaMemcpy(flag, &zero, sizeof(int), cudaMemcpyHostToDevice);
    return SSBLAS_STATUS_INTERNAL_ERROR;
  }
  return SSBLAS_STATUS_SUCCESS;
}
