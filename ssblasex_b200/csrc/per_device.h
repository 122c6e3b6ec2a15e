// Per-device tables for a process that drives several GPUs (cudaSetDevice between calls).
//
// Everything the library caches that belongs to one device's context -- kernel attributes,
// streams, events, workspaces, SM counts -- is kept in a table indexed by the device ordinal, so
// a call on device 1 never uses a stream, event or attribute that was set up on device 0. This
// header has no CUDA dependency (the ordinal is passed in), so its logic is unit-tested on the CPU.
#pragma once

namespace ssb {

// Devices a process may use at once; ordinals at or above it are rejected.
constexpr int kMaxDevices = 64;

inline bool valid_device(int dev) { return dev >= 0 && dev < kMaxDevices; }

// Runs init() the first time it is asked for device `dev` and remembers a success (a failure is
// retried on the next call). Returns init()'s code, 0 when already done, or `bad_device` for an
// ordinal outside the table.
template <class F>
inline int once_per_device(bool (&done)[kMaxDevices], int dev, F&& init, int bad_device) {
  if (!valid_device(dev)) return bad_device;
  if (done[dev]) return 0;
  const int e = (int)init();
  if (e == 0) done[dev] = true;
  return e;
}

}  // namespace ssb
