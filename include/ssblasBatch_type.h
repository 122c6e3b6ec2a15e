/*
 * Types of the ssblasGemmBatchedEx C ABI.
 *
 * The typedefs and enumerators are value-for-value those of the reference library
 * (hirokitokura/ssblasEx, include/ssblasBatch_type.h:5-103), so that code written against the
 * reference compiles and links against this library unchanged. Additions (marked EXTENSION)
 * have no counterpart in the reference.
 */
#ifndef SSBLASBATCH_TYPE
#define SSBLASBATCH_TYPE

#include <stdio.h>

typedef long int SSINT;  /* 64-bit on LP64, as in the reference (ssblasBatch_type.h:5-6) */
typedef long int SSLONG;

typedef enum { SSBLAS_int_32, SSBLAS_int_64 } ssblasIntType_t;

/* reference ssblasBatch_type.h:14-22 */
typedef enum {
  SSBLAS_STATUS_SUCCESS = 0,
  SSBLAS_STATUS_ALLOC_FAILED,
  SSBLAS_STATUS_INVALID_VALUE,
  SSBLAS_STATUS_INTERNAL_ERROR,
  SSBLAS_STATUS_NOTIMPLEMENTED_ERROR,
  SSBLAS_STATUS_NOT_COMPUTED_ERROR
} ssblasStatus_t;

/* Prints the status name; same output as the reference helper (ssblasBatch_type.h:24-47). */
static void ssblasShowError(ssblasStatus_t retval) {
  if (SSBLAS_STATUS_SUCCESS == retval) printf("SSBLAS_STATUS_SUCCESS\n");
  else if (SSBLAS_STATUS_ALLOC_FAILED == retval) printf("SSBLAS_STATUS_ALLOC_FAILED\n");
  else if (SSBLAS_STATUS_INVALID_VALUE == retval) printf("SSBLAS_STATUS_INVALID_VALUE\n");
  else if (SSBLAS_STATUS_INTERNAL_ERROR == retval) printf("SSBLAS_STATUS_INTERNAL_ERROR\n");
  else if (SSBLAS_STATUS_NOTIMPLEMENTED_ERROR == retval) printf("SSBLAS_STATUS_NOTIMPLEMENTED_ERROR\n");
  else if (SSBLAS_STATUS_NOT_COMPUTED_ERROR == retval) printf("SSBLAS_STATUS_NOT_COMPUTED_ERROR\n");
  else printf("SSBLAS_UNKNOWN\n");
}

/* reference ssblasBatch_type.h:50-54 */
typedef enum { SSBLAS_OP_N = 0, SSBLAS_OP_T = 1, SSBLAS_OP_C = 2 } ssblasOperation_t;

typedef signed char SSBLAS_SCHAR;
typedef unsigned char SSBLAS_UCHAR;

/* reference ssblasBatch_type.h:61-68 */
typedef enum {
  SSBLAS_R_8I,
  SSBLAS_R_8U,
  SSBLAS_R_16F,
  SSBLAS_R_32I,
  SSBLAS_R_32F,
  SSBLAS_R_64F
} ssblasDataType_t;

/* reference ssblasBatch_type.h:70-74 */
typedef enum { SSBLAS_COMPUTE_DEFAULT_TYPE, SSBLAS_COMPUTE_32I, SSBLAS_COMPUTE_32F } ssblasComputeType_t;

/* reference ssblasBatch_type.h:77-79 */
typedef enum { SSBLAS_COMPUTE_DEFAULT } ssblasGemmAlgo_t;

typedef struct {
  char x;
  char y;
  char z;
  char w;
} ssblaschar4;

typedef enum { SSBLAS_STATUS_COMPUTED = 0, SSBLAS_STATUS_NOT_COMPUTED } ssblasinternalComputeStatus_t;

/* ---- EXTENSION: arithmetic mode of the fp rows (no counterpart in the reference) ----------
 *  SSBLAS_MATH_PLAIN       fp32 row in FP32 FMA, fp64 row in FP64 FMA (the default).
 *  SSBLAS_MATH_FP64_OZAKI  fp64 row emulated on the int8 tensor cores: each row of op(A) and
 *                          column of op(B) is split into int8 slices under a shared power-of-two
 *                          exponent, slice pairs are multiplied exactly with int32 accumulation,
 *                          and the products are recombined in FP64 (Ozaki scheme).
 *  SSBLAS_MATH_FP32_BF16X3 fp32 row as three BF16 split products (hi*hi + hi*lo + lo*hi) on the
 *                          tensor cores with FP32 accumulation.
 *  The int8 row is always exact. The environment variable SSBLAS_MATH_MODE (PLAIN, OZAKI,
 *  BF16X3, or OZAKI+BF16X3) sets the initial mode. */
typedef enum {
  SSBLAS_MATH_PLAIN = 0,
  SSBLAS_MATH_FP64_OZAKI = 1,
  SSBLAS_MATH_FP32_BF16X3 = 2
} ssblasMathMode_t;

#endif
