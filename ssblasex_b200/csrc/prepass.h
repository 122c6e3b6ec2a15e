// Operand pre-pass interfaces (prepass.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ssb {

struct PlaneArgs {
  const void* const* X;   // device array of per-instance operand pointers
  long rows;              // rows of the K-major result (m for op(A), n for op(B))
  long K;
  long ld;                // caller's leading dimension
  bool kcontig;           // element (r, k) at X[r*ld + k] (true) or X[r + k*ld] (false)
  long batch;
  void* out;              // planes [batch][P][rows][Kp]
  long Kp;                // padded K (elements) = row pitch of a plane
  long plane_stride;      // bytes between planes = rows * Kp * elem
  long batch_stride;      // bytes between instances = P * plane_stride
  // When the instances are equally spaced (X[b] = X0 + b * xstride bytes), a pre-pass may address
  // the whole batch through one tensor map; X0 = nullptr if not.
  const void* X0 = nullptr;
  long xstride = 0;
};

cudaError_t launch_pack_i8(const PlaneArgs& a, cudaStream_t st);
// both operands of one call in one launch
cudaError_t launch_split_bf16_pair(const PlaneArgs& a, const PlaneArgs& b, cudaStream_t st);
cudaError_t launch_ozaki_slice(const PlaneArgs& a, int slices, int32_t* exps, cudaStream_t st);
// both operands of one call: two launches in all (exponents of both, then digits of both)
cudaError_t launch_ozaki_slice_pair(const PlaneArgs& a, int32_t* exps_a, const PlaneArgs& b, int32_t* exps_b,
                                    int slices, cudaStream_t st);
// the one-pass cluster slicer with a given item shape (the SSBLAS_PATH_OZAKI_SLICER configurations
// 2-6) for one or two operands, k <= 2048
cudaError_t launch_ozaki_cluster(const PlaneArgs& a0, int32_t* e0, const PlaneArgs& a1, int32_t* e1, bool two,
                                 int slices, int shape, cudaStream_t st);
bool cluster_kernel_fits(const PlaneArgs& a);

}  // namespace ssb
