/*
 * ssblasGemmBatchedEx for NVIDIA B200 (sm_100a): public C ABI.
 *
 * The two entry points of the reference library (hirokitokura/ssblasEx, include/ssblasBatch.h:15-57)
 * keep their exact names, argument order, types and status codes, so a caller of the reference
 * relinks against libssblas_b200.so unchanged. Differences in meaning:
 *
 *  - A[], B[], C[] may be (a) host arrays of host pointers, as the reference takes them: the
 *    library stages the matrices through device memory and returns after C is written back;
 *    (b) host arrays of device pointers; or (c) device arrays of device pointers (the cuBLAS
 *    batched convention). The kind is detected from the first pointer of each array; all
 *    pointers of one array must be of the same kind.
 *  - Calls are synchronous by default, as in the reference: the call returns after C is final.
 *    ssblasSetSyncMode(0) makes device-pointer calls asynchronous on the stream set with
 *    ssblasSetStream.
 *  - op C, which the reference rejects on the fp rows and mis-computes on the int8 row, returns
 *    SSBLAS_STATUS_INVALID_VALUE on every row. A leading dimension smaller than the stored row
 *    count, or a NULL alpha/beta/array, also returns SSBLAS_STATUS_INVALID_VALUE (the reference
 *    does not check these). Everything else follows the reference, including:
 *      m, n or batchCount <= 0 -> SSBLAS_STATUS_INTERNAL_ERROR;  k <= 0 -> success, C unchanged;
 *      beta == 0 -> C is not read; int8 arithmetic wraps modulo 2^32;
 *      alpha/beta point to float (fp32 row), double (fp64 row) or int32 (int8 row), in host memory.
 *    ssblasSetExtensions can replace some of these rules (op C, k = 0, more type rows); all of
 *    its flags are off by default.
 *  - If SSBLAS_GEMMBATCHEDEX_DEBUG is set in the environment, every call first prints the
 *    reference's argument dump (reference src/include/Impl/GemmBatchedEx/ssblasGemmBatchedEx.cpp:48-93).
 */
#ifndef SSBLASBATCH
#define SSBLASBATCH

#ifdef __cplusplus
extern "C" {
#endif

#include "ssblasBatch_type.h"

/* Replaces reference include/ssblasBatch.h:15-35 (implementation:
 * src/include/Impl/GemmBatchedEx/ssblasGemmBatchedEx.cpp:173-220). */
ssblasStatus_t ssblasGemmBatchedEx(ssblasOperation_t transa, ssblasOperation_t transb, SSINT m,
                                   SSINT n, SSINT k, const void* alpha, const void* const A[],
                                   ssblasDataType_t Atype, const SSINT lda, const void* const B[],
                                   ssblasDataType_t Btype, const SSINT ldb, const void* beta,
                                   void* const C[], ssblasDataType_t Ctype, const SSINT ldc,
                                   const SSINT batchCount, ssblasComputeType_t computeType,
                                   ssblasGemmAlgo_t algo);

/* Replaces reference include/ssblasBatch.h:37-57. The reference's body is a stub that returns an
 * uninitialised status (ssblasGemmBatchedEx.cpp:222-268); here it is the same computation as
 * ssblasGemmBatchedEx (all integers are already 64-bit). */
ssblasStatus_t ssblasGemmBatchedEx_64(ssblasOperation_t transa, ssblasOperation_t transb,
                                      SSLONG m, SSLONG n, SSLONG k, const void* alpha,
                                      const void* const A[], ssblasDataType_t Atype,
                                      const SSLONG lda, const void* const B[],
                                      ssblasDataType_t Btype, const SSLONG ldb, const void* beta,
                                      void* const C[], ssblasDataType_t Ctype, const SSLONG ldc,
                                      const SSLONG batchCount, ssblasComputeType_t computeType,
                                      ssblasGemmAlgo_t algo);

/* ============================ EXTENSIONS (not in the reference) ============================ */

/* Grouped batched GEMM: group g holds group_size[g] instances sharing transa/transb/m/n/k/
 * alpha/beta/ld/types of index g; the A/B/C pointer arrays list the instances of all groups in
 * order. alpha_array[g]/beta_array[g] point to the group's host scalar of its scale type. The
 * per-group types must form one of the three rows (fp32, fp64, int8->int32); rows may differ
 * between groups, and all instances run in one persistent launch per phase. Pointer arrays
 * follow the same three conventions as ssblasGemmBatchedEx. */
ssblasStatus_t ssblasGemmGroupedBatchedEx(
    const ssblasOperation_t transa_array[], const ssblasOperation_t transb_array[],
    const SSINT m_array[], const SSINT n_array[], const SSINT k_array[],
    const void* const alpha_array[], const void* const A[], const ssblasDataType_t Atype_array[],
    const SSINT lda_array[], const void* const B[], const ssblasDataType_t Btype_array[],
    const SSINT ldb_array[], const void* const beta_array[], void* const C[],
    const ssblasDataType_t Ctype_array[], const SSINT ldc_array[], const SSINT group_count,
    const SSINT group_size[], ssblasComputeType_t computeType, ssblasGemmAlgo_t algo);

/* The CUDA stream (a cudaStream_t passed as void*) used by all following calls of this host
 * thread's process; NULL selects the legacy default stream. */
ssblasStatus_t ssblasSetStream(void* stream);
ssblasStatus_t ssblasGetStream(void** stream);

/* 1 (default): every call returns after its result is final. 0: calls whose pointer arrays and
 * matrices are all in device memory return after enqueueing their work on the stream. */
ssblasStatus_t ssblasSetSyncMode(int synchronous);

/* Bitwise OR of ssblasMathMode_t flags for the fp64 and fp32 rows.
 * In SSBLAS_MATH_FP64_OZAKI mode, a row of op(A) or a column of op(B) that holds an Inf or a NaN
 * makes every C(i, j) it touches a quiet NaN (the plain paths follow IEEE arithmetic). */
ssblasStatus_t ssblasSetMathMode(int mode);
ssblasStatus_t ssblasGetMathMode(int* mode);

/* Slice count of SSBLAS_MATH_FP64_OZAKI mode and its error bound.
 *
 * Each row i of op(A) is scaled by its power of two 2^e_i (the smallest above max_k |op(A)_ik|),
 * rounded to an integer of 8S-2 bits and cut into S signed int8 slices; likewise each column j of
 * op(B) with 2^f_j. The slice pairs p + q < S are multiplied exactly on the int8 tensor cores and
 * recombined in FP64. For finite inputs and a result that neither overflows nor underflows:
 *
 *   |C_computed(i,j) - C_exact(i,j)| <= |alpha| * k * 2^(e_i + f_j) * (S + 1) * 2^(2 - 8S)
 *                                        + (S + 1) * u * (|alpha| * sum_k |op(A)_ik op(B)_kj| + |beta C(i,j)|)
 *
 * with u = 2^-53. The first term covers the rounding of op(A) and op(B) to 8S-2 bits and the
 * dropped pairs p + q >= S; the second the FP64 recombination and the alpha/beta epilogue.
 *
 * ssblasSetOzakiSlices(S), S in 3..8, fixes the count; 0 (the default) chooses the smallest S
 * whose per-term bound (S + 1) * 2^(2 - 8S) is at most the tolerance of ssblasSetOzakiTolerance:
 * by default 4u = 2^-51 (the FP64 tolerance 4*k*u spread over the k product terms), which selects
 * S = 7 for every k. A tolerance of 0 restores the default; a negative tolerance, or one below the
 * 8-slice bound (9 * 2^-62), returns SSBLAS_STATUS_INVALID_VALUE. ssblasGetOzakiSlices returns the
 * count the next call will use; ssblasGetLastRunInfo reports the count a call used.
 * ssblasGemmGroupedBatchedEx always uses 7 slices: its fp64 instances return
 * SSBLAS_STATUS_NOTIMPLEMENTED_ERROR when another count is fixed or the tolerance needs 8. */
ssblasStatus_t ssblasSetOzakiSlices(int slices);
ssblasStatus_t ssblasSetOzakiTolerance(double tolerance);
ssblasStatus_t ssblasGetOzakiSlices(int* slices);

/* Type and semantics extensions (none is in the reference; all are off by default, and with a flag
 * off the call behaves as the reference does). Bitwise OR of:
 *   SSBLAS_EXT_R16F: the row (R_16F, R_16F, R_16F or R_32F): fp16 op(A) and op(B), fp16 or fp32 C,
 *     float alpha/beta, fp32 accumulation on tcgen05 kind::f16 (declared but unimplemented in the
 *     reference: ssblasBatch_type.h, ssblasGemmBatchedExSelector.hpp:105-107).
 *   SSBLAS_EXT_R8U: SSBLAS_R_8U for either int8 operand (C SSBLAS_R_32I, int32 alpha/beta):
 *     unsigned bytes, exact int32 products with wrap-around.
 *   SSBLAS_EXT_OP_C: op C accepted on every row as op T (the conjugate transpose of a real
 *     matrix); the reference rejects it on the fp rows and mis-computes it on the int8 row.
 *   SSBLAS_EXT_K0_BETA: k == 0 computes C <- beta*C (BLAS; beta == 0 writes zeros without reading
 *     C) instead of leaving C untouched, and k < 0 returns SSBLAS_STATUS_INVALID_VALUE.
 *   SSBLAS_EXT_COMPUTE_TYPE: computeType is checked against the row and honoured:
 *     SSBLAS_COMPUTE_32I only with int8 operands; SSBLAS_COMPUTE_32F only on the fp32 and fp16 rows,
 *     where it asks for FP32 arithmetic (the fp32 row then never uses the 3xBF16 emulation); other
 *     combinations return SSBLAS_STATUS_INVALID_VALUE. Without the flag computeType is ignored.
 * The grouped entry point keeps the reference's three rows. Unknown flags return
 * SSBLAS_STATUS_INVALID_VALUE. */
typedef enum {
  SSBLAS_EXT_NONE = 0,
  SSBLAS_EXT_R16F = 1,
  SSBLAS_EXT_R8U = 2,
  SSBLAS_EXT_OP_C = 4,
  SSBLAS_EXT_K0_BETA = 8,
  SSBLAS_EXT_COMPUTE_TYPE = 16
} ssblasExtension_t;
ssblasStatus_t ssblasSetExtensions(int flags);
ssblasStatus_t ssblasGetExtensions(int* flags);

/* Fault injection for tests of the failure paths (no GPU is faulted or hung). The armed fault
 * applies once, to the next point it names, then disarms:
 *   SSBLAS_FAULT_SKIP_COPY: the next tensor-core GEMM launch (int8, Ozaki or 3xBF16 path) skips
 *     one operand copy in its first thread block and gives every bounded wait a short limit; the
 *     waits on that copy run out, the kernel records the error and exits, and the call returns
 *     SSBLAS_STATUS_INTERNAL_ERROR with ssblasRunInfo_t.device_error set. The next call is normal.
 *   SSBLAS_FAULT_ALLOC: the next request for library workspace fails as if the device were out
 *     of memory; the call returns SSBLAS_STATUS_ALLOC_FAILED before launching anything.
 * SSBLAS_FAULT_NONE disarms. Other values return SSBLAS_STATUS_INVALID_VALUE. */
typedef enum {
  SSBLAS_FAULT_NONE = 0,
  SSBLAS_FAULT_SKIP_COPY = 1,
  SSBLAS_FAULT_ALLOC = 2
} ssblasFault_t;
ssblasStatus_t ssblasSetFaultInjection(int fault);

/* Description of the most recent call on this process. */
typedef struct {
  int path;          /* ssblasPath_t of the main GEMM phase */
  int slices;        /* Ozaki slices per operand (0 when not emulated) */
  int kernel_launches;
  int device_error;  /* nonzero if a bounded device-side wait gave up (the call then returned
                        SSBLAS_STATUS_INTERNAL_ERROR) */
  int split_k;       /* K pieces per output tile of a tcgen05 GEMM (1 = not split; 0 on the
                        paths without split-K) */
} ssblasRunInfo_t;

typedef enum {
  SSBLAS_PATH_NONE = 0,
  SSBLAS_PATH_SIMT = 1,            /* register-tiled FFMA / DFMA / integer kernel */
  SSBLAS_PATH_I8_TCGEN05 = 2,      /* int8 -> int32 on tcgen05.mma kind::i8, TMA staging */
  SSBLAS_PATH_OZAKI_TCGEN05 = 3,   /* fp64 via int8 slices on tcgen05.mma kind::i8 */
  SSBLAS_PATH_BF16X3_TCGEN05 = 4,  /* fp32 via three BF16 split products, tcgen05 kind::f16 */
  SSBLAS_PATH_GROUPED = 5,         /* grouped persistent launch; as a ssblasSetKernelConfig key:
                                      0 = all Ozaki instances on 128 x 64 tiles, 1 (default) = tile
                                      shape per size bucket (key 12), 2 = all on 128 x 32 tiles
                                      with a static tile order */
  SSBLAS_PATH_DMMA = 6,            /* plain fp64 on the FP64 tensor cores (mma.sync f64) */
  SSBLAS_PATH_OZAKI_SLICER = 7,    /* not a path: ssblasSetKernelConfig key of the Ozaki slicing
                                      pre-pass. 3: one pass with thread-block clusters of 16 rows
                                      x 512 k per CTA when k <= 2048 (the default for k <= 512);
                                      2: the same with 32 rows x 256 k; 4: 8 rows x 1024 k (the
                                      default for 512 < k <= 2048); 5: 16 rows x
                                      256 k per 256-thread CTA, two CTAs per SM; 6: 4 rows x
                                      256 k per 128-thread CTA; 1: row-maximum pass then digits
                                      per 32 rows x 128 k chunk; 7: row-maximum pass then digits
                                      by persistent CTAs over 16 rows x 512 k slabs (what every
                                      form but 1 does when k > 2048) */
  SSBLAS_PATH_SPLITK_I8 = 8,       /* not a path: ssblasSetKernelConfig keys of the split-K factor */
  SSBLAS_PATH_SPLITK_OZAKI = 9,    /* of the int8 and Ozaki tcgen05 GEMMs. config = number of K
                                      pieces per output tile (1 = none, at most 64), 0 = automatic
                                      (split only when the tiles fill less than half of the SMs).
                                      Each piece's exact int32 sums are added in 64 bits, so the
                                      result does not depend on the factor; the Ozaki GEMM always
                                      splits k > 16384 into pieces of at most 16384. */
  SSBLAS_PATH_OZAKI_PIPELINE = 10  /* not a path: ssblasSetKernelConfig key of the Ozaki slicing /
                                      GEMM pipeline: config = chunks of the batch (1 = none, at most
                                      8), 0 = automatic (none); the slicing of chunk c + 1 runs
                                      beside the GEMM of chunk c. */,
  SSBLAS_PATH_F16_TCGEN05 = 11,     /* fp16 inputs (SSBLAS_EXT_R16F row) on tcgen05.mma kind::f16 */
  SSBLAS_PATH_GROUPED_OZAKI_TILE = 12 /* not a path: ssblasSetKernelConfig / tuning key of the tile
                                      shape of a grouped call's Ozaki instances per size bucket
                                      (batch 1): 0 = 128 x 64 tiles, one accumulator; 1 (default)
                                      = 128 x 32 tiles, two accumulators */
} ssblasPath_t;

ssblasStatus_t ssblasGetLastRunInfo(ssblasRunInfo_t* info);

/* Per-kernel device timing: while enabled, the library records a CUDA event pair around each of
 * its kernel launches on the launching stream. ssblasGetProfile returns, per kernel name, the
 * number of launches and their summed event time since profiling was (re)enabled; it waits for
 * the recorded events. *entries receives the number of kernels (which may exceed max_entries). */
typedef struct {
  char name[48];
  int launches;
  double total_ms;
} ssblasKernelProfile_t;

ssblasStatus_t ssblasSetProfiling(int enable);
ssblasStatus_t ssblasGetProfile(ssblasKernelProfile_t* out, int max_entries, int* entries);

/* Frees the device workspace cached by the library (it is re-created on the next call). */
ssblasStatus_t ssblasReleaseWorkspace(void);

/* Kernel configuration (tile shape / pipeline depth) of one path (an ssblasPath_t value):
 * config >= 0 forces that configuration, -1 returns to automatic choice -- the tuning table
 * written by the autotuner ($SSBLAS_TUNE_FILE, else tune/ssblas_tune.json next to the library),
 * keyed by path and power-of-two size bucket, else the built-in default. Configurations a path
 * does not have fall back to its default. ssblasReloadTuning re-reads the table. */
ssblasStatus_t ssblasSetKernelConfig(int path, int config);
ssblasStatus_t ssblasReloadTuning(void);

/* Allocation-free FP64 batched GEMM (no counterpart in the reference).
 * Same arguments and results as ssblasGemmBatchedEx on the fp64 row in SSBLAS_MATH_FP64_OZAKI
 * mode, for callers that cannot let a library allocate device memory: services whose pool
 * allocator owns all of the GPU's memory, and latency-critical loops in which a cudaMalloc or
 * cudaFree -- which may synchronise the whole device -- is not allowed. It calls no allocating
 * function: the Ozaki slices and exponents go to one fixed 64 MiB device array that every GPU
 * loading the library holds until the process exits.
 *  - A[], B[], C[] must be device arrays of device pointers; other type rows return
 *    SSBLAS_STATUS_NOTIMPLEMENTED_ERROR.
 *  - A problem needs S*(m+n)*Kp*batchCount + 4*(m+n)*batchCount bytes (S = Ozaki slices, as
 *    ssblasGetOzakiSlices reports: 7 by default; Kp = k rounded up to 16); larger problems, or
 *    k > 16384, return SSBLAS_STATUS_INVALID_VALUE (with a message on stderr) and leave C
 *    untouched. On a device the tensor-core kernels do not support it returns
 *    SSBLAS_STATUS_NOTIMPLEMENTED_ERROR without launching anything.
 *  - All calls share the array; calls whose GPU work overlaps race on it and must be ordered by
 *    the caller. Its contents carry over between calls; nothing in it needs to start at zero.
 *  - The first call on a device looks the array's address up for that device; make it before
 *    starting any stream capture on the device. */
ssblasStatus_t ssblasGemmBatchedExNoAlloc(ssblasOperation_t transa, ssblasOperation_t transb, SSINT m,
                                          SSINT n, SSINT k, const void* alpha, const void* const A[],
                                          ssblasDataType_t Atype, const SSINT lda, const void* const B[],
                                          ssblasDataType_t Btype, const SSINT ldb, const void* beta,
                                          void* const C[], ssblasDataType_t Ctype, const SSINT ldc,
                                          const SSINT batchCount, ssblasComputeType_t computeType,
                                          ssblasGemmAlgo_t algo);

#ifdef __cplusplus
}
#endif

#endif
