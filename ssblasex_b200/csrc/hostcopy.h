// Host <-> device copies of scattered host instances through pinned staging (hostcopy.cpp).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace ssb {

// Copies `batch` host instances of `bytes` each (src[b], pageable or not) to dst + b * pitch on
// `st`; returns once the host data has been packed (the caller's buffers may then change).
cudaError_t gather_to_device(char* dst, size_t pitch, const void* const* src, long batch, size_t bytes,
                             cudaStream_t st);
// Copies the first row_bytes of each of the `cols` columns (ld_bytes apart) of every instance at
// src + b * pitch on the device to dst[b] (same column layout); returns when the data is in place.
cudaError_t scatter_to_host(void* const* dst, size_t ld_bytes, const char* src, size_t pitch, long batch,
                            size_t row_bytes, long cols, cudaStream_t st);

}  // namespace ssb
