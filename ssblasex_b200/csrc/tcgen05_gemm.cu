// placeholder until the tensor-core kernels land
#include "internal.h"
namespace ssb {
cudaError_t launch_i8_tcgen05(const BatchDesc&, cudaStream_t) { return cudaErrorNotSupported; }
cudaError_t launch_ozaki_f64(const BatchDesc&, int, cudaStream_t) { return cudaErrorNotSupported; }
cudaError_t launch_bf16x3_f32(const BatchDesc&, cudaStream_t) { return cudaErrorNotSupported; }
}
namespace ssb {
ssblasStatus_t grouped_persistent(const ssblasOperation_t*, const ssblasOperation_t*, const SSINT*, const SSINT*, const SSINT*,
    const void* const*, const void* const*, const ssblasDataType_t*, const SSINT*, const void* const*, const ssblasDataType_t*,
    const SSINT*, const void* const*, void* const*, const ssblasDataType_t*, const SSINT*, SSINT, const SSINT*) {
  return SSBLAS_STATUS_NOT_COMPUTED_ERROR;
}
}
