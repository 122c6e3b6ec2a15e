// Ozaki digit arithmetic shared by the slicing kernels (prepass.cu) and the grouped pre-pass
// (grouped.cu). A value x of a row with exponent e becomes X = rint(x * 2^(8S-2-e)) and its S
// balanced base-256 digits d_0..d_{S-1}: with Y = X + 0x80..80 (128 added to each of the S-1 low
// bytes), d_p = byte_{S-1-p}(Y) with its top bit flipped for p >= 1, d_0 = byte_{S-1}(Y).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ssb {

// Rows (of op(A)) and columns (of op(B)) holding an Inf or a NaN get this exponent and zero
// digits; every C(i, j) they touch becomes a quiet NaN (kOzakiNaN). The row maximum is taken over
// the bit patterns of |x| as unsigned integers, which orders finite values like their magnitudes
// and puts every Inf and NaN above them.
constexpr int kNonFiniteExp = 4096;
constexpr unsigned long long kOzakiNaN = 0x7FF8000000000000ull;
static __device__ __forceinline__ unsigned long long abs_bits(double x) {
  return (unsigned long long)__double_as_longlong(x) & 0x7FFFFFFFFFFFFFFFull;
}
static __device__ __forceinline__ unsigned long long max_u64(unsigned long long a, unsigned long long b) {
  return a > b ? a : b;
}
// A key for the row maximum of N values, ordered like their largest |x| bit pattern as far as
// row_exponent can tell: the high word of |x| (exponent and top 20 fraction bits) fixes frexp's
// exponent whenever it is nonzero, so the key is max(high words) << 32; only when every high
// word is zero (|x| below 2^-1042: zeros and the smallest subnormals) is the key the largest low
// word. Inf and NaN keep a high word >= 0x7FF00000. Two integer operations per value instead of
// the five of a 64-bit compare-and-select; the row maximum of the per-thread keys is then taken
// with max_u64 as for bit patterns.
template <int N>
static __device__ __forceinline__ unsigned long long row_key(const double (&v)[N]) {
  uint32_t mh = 0;
#pragma unroll
  for (int e = 0; e < N; ++e) mh = max(mh, (uint32_t)__double2hiint(v[e]) & 0x7FFFFFFFu);
  if (mh != 0) return (unsigned long long)mh << 32;
  uint32_t ml = 0;
#pragma unroll
  for (int e = 0; e < N; ++e) ml = max(ml, (uint32_t)__double2loint(v[e]));
  return ml;
}

// Running form of row_key for values that arrive one at a time: fold each into the maxima of the
// high words of |x| (mh) and of the low words (ml); key_of(mh, ml) is then the key. The low-word
// maximum runs over every value, which is the right one whenever it is used (all high words zero).
static __device__ __forceinline__ void key_fold(double x, uint32_t& mh, uint32_t& ml) {
  mh = max(mh, (uint32_t)__double2hiint(x) & 0x7FFFFFFFu);
  ml = max(ml, (uint32_t)__double2loint(x));
}
static __device__ __forceinline__ unsigned long long key_of(uint32_t mh, uint32_t ml) {
  return mh != 0 ? (unsigned long long)mh << 32 : (unsigned long long)ml;
}

// e with max|x| < 2^e (0 for an all-zero row), or kNonFiniteExp -- frexp's exponent, read off the
// bit pattern: E - 1022 for a biased exponent E > 0, and for a subnormal f * 2^-1074 (f < 2^52)
// the position of f's leading bit, 64 - clz(f) - 1074.
static __device__ __forceinline__ int row_exponent(unsigned long long maxbits) {
  if (maxbits >= 0x7FF0000000000000ull) return kNonFiniteExp;
  const int E = (int)(maxbits >> 52);
  if (E > 0) return E - 1022;
  return maxbits ? 64 - __clzll((long long)maxbits) - 1074 : 0;
}
// 2^h for -1022 <= h <= 1023, built from its bit pattern
static __device__ __forceinline__ double pow2(int h) {
  return __longlong_as_double((long long)(h + 1023) << 52);
}
// the two power-of-two factors of 2^(8S-2-e) (0 for a non-finite row: its digits are zero):
// s0 = 2^(8S-2-e) and s1 = 1 when that is a normal double (every row whose largest magnitude is
// above 2^-960), else the shift split in halves, which with e in [-1073, 1024] both stay inside
// the normal range. x * s0 * s1 is the exact product x * 2^(8S-2-e) (or that product rounded
// once, when it is below the normal range and so rounds to zero digits) either way, so the
// digits do not depend on the split; with s1 = 1 the second multiplication can be skipped.
static __device__ __forceinline__ void row_scale(int S, int e, double& s0, double& s1) {
  if (e == kNonFiniteExp) {
    s0 = s1 = 0.0;
    return;
  }
  const int sh = 8 * S - 2 - e;
  if (sh >= -1022 && sh <= 1023) {
    s0 = pow2(sh);
    s1 = 1.0;
    return;
  }
  const int h1 = sh / 2;
  s0 = pow2(h1);
  s1 = pow2(sh - h1);
}

// 4 x 4 byte transpose: out[b] holds byte b of w[0..3] (byte j of out[b] = byte b of w[j]).
static __device__ __forceinline__ void byte_transpose4(const uint32_t (&w)[4], uint32_t (&out)[4]) {
  const uint32_t t0 = __byte_perm(w[0], w[1], 0x5140), t1 = __byte_perm(w[0], w[1], 0x7362);
  const uint32_t t2 = __byte_perm(w[2], w[3], 0x5140), t3 = __byte_perm(w[2], w[3], 0x7362);
  out[0] = __byte_perm(t0, t2, 0x5410);
  out[1] = __byte_perm(t0, t2, 0x7632);
  out[2] = __byte_perm(t1, t3, 0x5410);
  out[3] = __byte_perm(t1, t3, 0x7632);
}

// Y = rint(x * s0 * s1) + bias (mod 2^64), s0 * s1 = 2^(8S-2-e), |x * s0 * s1| < 2^62, rounding
// to nearest even -- computed with FP64 additions instead of a double -> int64 conversion (which
// runs on the narrow XU pipe and would bound the slicing passes):
//   v  = x * s0 * s1                 exact (power-of-two scaling)
//   a  = v + 1.5*2^63                a in [2^63, 2^64), ulp 2^11: a = 1.5*2^63 + v1, v1 = v rounded
//                                    to a multiple of 2^11, and the bits of a hold
//                                    bits(1.5*2^63) + v1 / 2^11
//   v2 = v - (a - 1.5*2^63)          exact, |v2| <= 2^10
//   t2 = v2 + 1.5*2^52               the low word of t2 is rint(v2) (|v2| < 2^51)
// rint(v) = v1 + rint(v2) (v1 is an even integer), so
//   Y = (bits(a) << 11) + rint(v2) + bias - (bits(1.5*2^63) << 11)   (mod 2^64).
template <bool ONE = false>
static __device__ __forceinline__ unsigned long long slice_y(double x, double s0, double s1, unsigned long long bias) {
  const double C1 = 0x1.8p63, M = 0x1.8p52;
  const double v = ONE ? __dmul_rn(x, s0) : __dmul_rn(__dmul_rn(x, s0), s1);   // ONE: s1 == 1
  const double a = __dadd_rn(v, C1);
  const double v2 = __dsub_rn(v, __dsub_rn(a, C1));
  const int32_t r2 = (int32_t)__double2loint(__dadd_rn(v2, M));
  return ((unsigned long long)__double_as_longlong(a) << 11) + (unsigned long long)(long long)r2 +
         (bias - 0x4000000000000000ull);
}

// Digit words of 4 consecutive-k values of one row: word p holds digit p of the 4 values (the
// value with the lowest k in the lowest byte). s0 * s1 = 2^(8S-2-e); ONE: s1 == 1 (one
// multiplication per value instead of two; digit_words_rs picks the form for a row).
template <int S, bool ONE = false>
static __device__ __forceinline__ void digit_words(const double (&x)[4], double s0, double s1, uint32_t (&wd)[S]) {
  unsigned long long bias = 0;
#pragma unroll
  for (int j = 0; j < S - 1; ++j) bias |= 0x80ull << (8 * j);
  uint32_t lo[4], hi[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const unsigned long long Y = slice_y<ONE>(x[i], s0, s1, bias);
    lo[i] = (uint32_t)Y;
    hi[i] = (uint32_t)(Y >> 32);
  }
  uint32_t L[4], H[4];
  byte_transpose4(lo, L);
  byte_transpose4(hi, H);
#pragma unroll
  for (int p = 0; p < S; ++p) {
    const int byte = S - 1 - p;
    const uint32_t w = byte < 4 ? L[byte] : H[byte - 4];
    wd[p] = p > 0 ? (w ^ 0x80808080u) : w;
  }
}

template <int S>
static __device__ __forceinline__ void digit_words_rs(const double (&x)[4], double s0, double s1, uint32_t (&wd)[S]) {
  if (s1 == 1.0) digit_words<S, true>(x, s0, s1, wd);
  else digit_words<S, false>(x, s0, s1, wd);
}

}  // namespace ssb
