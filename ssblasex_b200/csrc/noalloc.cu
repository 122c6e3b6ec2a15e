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

#include "internal.h"
#include "prepass.h"

namespace ssb {
namespace {

constexpr size_t kNoAllocScratchBytes = 64ull << 20;

static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

void* g_noalloc_ptr[kMaxDevices] = {};   // device address of the array, per device

// Device address of g_noalloc_scratch on the current device (host code cannot use the symbol
// itself: in host code its name is only a stand-in for the device object). Called with the
// library lock held.
cudaError_t scratch_address(void** out) {
  const int dev = current_device();
  if (dev < 0) return cudaErrorInvalidDevice;
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
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

inline size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Layout of the scratch array for one call: S slice planes of op(A), then of op(B) (each region
// 256-byte aligned), then the int32 exponents of both. False when the sizes overflow or the
// layout does not fit the array.
struct ScratchLayout {
  size_t off_b = 0, off_e = 0, need = 0;
};
bool scratch_layout(int S, long m, long n, long Kp, long batch, ScratchLayout* L) {
  // every factor alone must fit before any product is formed
  const size_t cap = kNoAllocScratchBytes;
  if ((size_t)m > cap || (size_t)n > cap || (size_t)Kp > cap || (size_t)batch > cap) return false;
  size_t bytes_a, bytes_b, bytes_e, t;
  if (__builtin_mul_overflow((size_t)S * (size_t)m, (size_t)Kp, &t) || __builtin_mul_overflow(t, (size_t)batch, &bytes_a) ||
      __builtin_mul_overflow((size_t)S * (size_t)n, (size_t)Kp, &t) || __builtin_mul_overflow(t, (size_t)batch, &bytes_b) ||
      __builtin_mul_overflow(sizeof(int32_t) * ((size_t)m + (size_t)n), (size_t)batch, &bytes_e))
    return false;
  if (bytes_a > cap || bytes_b > cap || bytes_e > cap) return false;
  L->off_b = round_up(bytes_a, 256);
  L->off_e = round_up(L->off_b + bytes_b, 256);
  L->need = L->off_e + bytes_e;
  return L->need <= cap;
}

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

  ApiRange range("ssblasGemmBatchedExNoAlloc");
  auto lock = lock_api();
  reset_run_info();
  const int S = ozaki_slices_for_call();
  const long Kp = (k + 15) / 16 * 16;
  ScratchLayout L;
  if (!scratch_layout(S, m, n, Kp, batchCount, &L)) {
    fprintf(stderr,
            "ssblasGemmBatchedExNoAlloc: a %ld x %ld x %ld problem of %ld instances with %d slices needs more "
            "scratch than the static maximum of %zu bytes (use ssblasGemmBatchedEx, or split the batch)\n",
            (long)m, (long)n, (long)k, (long)batchCount, S, kNoAllocScratchBytes);
    return SSBLAS_STATUS_INVALID_VALUE;
  }
  // nothing is launched on a device the tensor-core kernels do not support
  if (!tcgen05_available()) return SSBLAS_STATUS_NOTIMPLEMENTED_ERROR;
  // this entry point takes device arrays of device pointers only: staging host data would allocate
  if (!on_device((const void*)A) || !on_device((const void*)B) || !on_device((const void*)C))
    return SSBLAS_STATUS_INVALID_VALUE;

  void* scratch = nullptr;
  cudaError_t e = scratch_address(&scratch);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return SSBLAS_STATUS_INTERNAL_ERROR;
  }
  int8_t* pa = (int8_t*)scratch;
  int8_t* pb = (int8_t*)scratch + L.off_b;
  int32_t* ex = (int32_t*)((uint8_t*)scratch + L.off_e);

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
  // same device-error reporting as the other entry points (run info records the flag's code)
  return check_device_error(st);
}
