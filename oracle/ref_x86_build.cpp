// Translation unit that compiles the UNMODIFIED reference library (hirokitokura/ssblasEx) from
// its own source tree on an x86 host, for use as a CPU parity oracle and CPU baseline.
//
// TEST INFRASTRUCTURE ONLY. Nothing in the shipped library links this file; it is built into
// oracle/_ref/ (git-ignored) by oracle/Makefile and loaded only by tests/, bench.py's CPU
// baseline/reference arm and the smoke check.
//
// The reference selects its x86 emulation of the SVE instruction macros
// (src/include/asm/GENERIC/*) when __ARM_FEATURE_SVE is undefined (src/include/asm/def_asm.h:5-10).
// As shipped, that emulation layer does not compile the int8 row and computes it wrongly.
// Three fixes are applied here, all by re-defining emulation macros between the reference's
// own headers; no reference source file is copied or edited:
//
//  1. ST1B_ZXI is missing from the emulation layer but used by the int8 B packer
//     (src/include/BCopy/Xgemm_ncopy_sve_1.hpp:141-177). Defined below with the semantics of
//     the SVE instruction (src/include/asm/SVE/def_sve_asm_float.h:135-137): a predicated
//     byte store of one 64-byte vector at x1 + imm*VL.
//  2. FMLA_ZSP tests std::is_same_v<DEF_DOUBLE_AB, char> for the int8 dot product
//     (src/include/asm/GENERIC/def_generic_asm_float.h:80), but the int8 row is instantiated
//     with signed char (src/include/Impl/GemmBatchedEx/ssblasGemmBatchedExSelector.hpp:38-39),
//     so the int8 multiply-accumulate compiled to nothing. Re-defined to dispatch on
//     SSBLAS_SCHAR, as the SVE macro does (def_sve_asm_float.h:45-46).
//  3. The emulated ZIP1/ZIP2 (def_generic_asm_float.h:229-257) ignore their second operand,
//     which corrupts vec_col_pack4 (src/include/asm/GENERIC/def_generic_acle.hpp:9-38). The
//     int8 A packer's call (src/include/ACopy/Xgemm_ncopy_sve_v4.hpp:528) is redirected to
//     oracle_vec_col_pack4 below, which produces the char4 interleave that the SVE version
//     (src/include/asm/SVE/def_sve_acle.hpp:74-113) produces: dest[i] = {A[i], A[lda+i],
//     A[2*lda+i], A[3*lda+i]} for the 64 byte lanes i of one vector.
//
// Everything else -- blocking, packing layouts, K-block accumulation order, the beta-scale and
// the alpha epilogue -- is the reference's own code.

#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <type_traits>

#include "asm/def_asm.h"

// ---- fix 1: byte store ------------------------------------------------------------------
#define ST1B_ZXI(zt, pg, x1, imm)                                                   \
  {                                                                               \
    signed char* oracle_src_ = (signed char*)(zt).get();                          \
    int* oracle_pred_ = (int*)(pg).get();                                         \
    signed char* oracle_dst_ = (signed char*)(x1) + (imm) * svcntb();             \
    for (int oracle_i_ = 0; oracle_i_ < svcntb(); ++oracle_i_)                     \
      if (oracle_pred_[oracle_i_] == 1) oracle_dst_[oracle_i_] = oracle_src_[oracle_i_]; \
  }

// ---- fix 2: int8 dot product dispatch -----------------------------------------------------
#undef FMLA_ZSP_base
#define FMLA_ZSP_base(zds3, pg, zs1, zs2)                                                   \
  {                                                                                         \
    if constexpr ((std::is_same_v<DEF_DOUBLE_AB, float> && std::is_same_v<DEF_DOUBLE_C, float>)) \
      genericfmla<DEF_DOUBLE_C>(zds3, pg, zs1, zs2);                                        \
    else if constexpr ((std::is_same_v<DEF_DOUBLE_AB, double> &&                           \
                        std::is_same_v<DEF_DOUBLE_C, double>))                              \
      genericfmla<DEF_DOUBLE_C>(zds3, pg, zs1, zs2);                                        \
    else if constexpr ((std::is_same_v<DEF_DOUBLE_AB, SSBLAS_SCHAR> &&                      \
                        std::is_same_v<DEF_DOUBLE_C, int>))                                 \
      genericfmla_dot<DEF_DOUBLE_AB, DEF_DOUBLE_C>(zds3, pg, zs1, zs2);                     \
  }

// ---- fix 3: char4 interleave of four byte rows --------------------------------------------
namespace ssblasEx {
namespace cpu {
namespace vecdef {
template <typename INDEXINT, typename T_SCALE, typename DEF_DOUBLE_AB, typename DEF_DOUBLE_C>
void oracle_vec_col_pack4(const DEF_DOUBLE_AB* A, const INDEXINT lda, DEF_DOUBLE_C* dest) {
  if constexpr ((sizeof(DEF_DOUBLE_AB) == 1) && (sizeof(DEF_DOUBLE_C) == 4)) {
    const int lanes = svcntb();
    signed char* out = (signed char*)dest;
    for (int i = 0; i < lanes; ++i)
      for (int r = 0; r < 4; ++r) out[4 * i + r] = (signed char)A[(INDEXINT)r * lda + i];
  }
}
}  // namespace vecdef
}  // namespace cpu
}  // namespace ssblasEx
#define vec_col_pack4 oracle_vec_col_pack4

#include "Impl/GemmBatchedEx/ssblasGemmBatchedEx.cpp"
