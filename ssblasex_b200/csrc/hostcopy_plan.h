// Byte arithmetic of the staged host <-> device copies (hostcopy.cpp), kept free of CUDA so that
// it is unit-tested on the CPU.
//
// The device side holds instance b at b * pitch. A staging slot covers a window [c0, c1) of that
// layout; host threads split a window into parts [p0, p1) and copy, for each part, exactly the
// bytes of the instances that fall inside it.
#pragma once

#include <stddef.h>

namespace ssb {

// Gather: instance b occupies [b * pitch, b * pitch + bytes) of the device layout (pitch >= bytes).
// Calls f(b, offset in the instance, offset in the layout, length) for every piece of an instance
// inside [p0, p1).
template <class F>
inline void gather_pieces(size_t p0, size_t p1, size_t pitch, long batch, size_t bytes, F&& f) {
  if (pitch == 0 || p1 <= p0) return;
  for (long b = (long)(p0 / pitch); b < batch && (size_t)b * pitch < p1; ++b) {
    const size_t i0 = (size_t)b * pitch, i1 = i0 + bytes;
    const size_t lo = p0 > i0 ? p0 : i0, hi = p1 < i1 ? p1 : i1;
    if (lo < hi) f(b, lo - i0, lo, hi - lo);
  }
}

// Scatter: column j of instance b starts at b * pitch + j * ld_bytes of the device layout, and
// only its first row_bytes are copied (the caller's ld padding stays untouched); cols columns.
// Calls f(b, offset in the instance, offset in the layout, length) for every piece inside
// [p0, p1).
template <class F>
inline void scatter_pieces(size_t p0, size_t p1, size_t pitch, long batch, size_t ld_bytes, size_t row_bytes,
                           long cols, F&& f) {
  if (pitch == 0 || ld_bytes == 0 || p1 <= p0) return;
  for (long b = (long)(p0 / pitch); b < batch && (size_t)b * pitch < p1; ++b) {
    const size_t ib = (size_t)b * pitch;
    long j = p0 > ib ? (long)((p0 - ib) / ld_bytes) : 0;
    for (; j < cols && ib + (size_t)j * ld_bytes < p1; ++j) {
      const size_t s0 = ib + (size_t)j * ld_bytes, s1 = s0 + row_bytes;
      const size_t lo = p0 > s0 ? p0 : s0, hi = p1 < s1 ? p1 : s1;
      if (lo < hi) f(b, (size_t)j * ld_bytes + (lo - s0), lo, hi - lo);
    }
  }
}

// Part `part` of `parts` equal parts of the window [c0, c1).
inline void window_part(size_t c0, size_t c1, int part, int parts, size_t* p0, size_t* p1) {
  *p0 = c0 + (c1 - c0) * (size_t)part / (size_t)parts;
  *p1 = c0 + (c1 - c0) * (size_t)(part + 1) / (size_t)parts;
}

}  // namespace ssb
