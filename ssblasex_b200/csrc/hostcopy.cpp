// Host <-> device copies of scattered host instances (the reference's callers allocate every
// matrix on its own, in pageable memory: example/main.cpp:58-66) through pinned staging slots.
// A pool of host threads packs the next slot while the copy engine moves the previous one, so the
// transfer runs near the PCIe rate instead of the driver's bounce-buffered pageable copies, one
// instance at a time.
//
// Slots mirror the device layout (instance b at b * pitch): one DMA per slot, whatever the
// instance size. The staging memory and the pool are process-wide; callers hold the API lock.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "hostcopy.h"
#include "hostcopy_plan.h"
#include "internal.h"

namespace ssb {
namespace {

constexpr size_t kSlotBytes = (size_t)16 << 20;
constexpr int kSlots = 3;

// Persistent worker threads; run(n, f) calls f(0..n-1) on the workers and the caller and returns
// when all are done.
class Pool {
 public:
  explicit Pool(int workers) {
    for (int i = 0; i < workers; ++i) std::thread([this] { loop(); }).detach();
    size_ = workers + 1;
  }
  int size() const { return size_; }
  void run(int n, const std::function<void(int)>& f) {
    {
      std::lock_guard<std::mutex> g(mu_);
      job_ = &f;
      n_ = n;
      next_ = 0;
      done_ = 0;
      ++gen_;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> g(mu_);
    done_cv_.wait(g, [this] { return done_ == n_; });
    job_ = nullptr;
  }

 private:
  void work() {
    for (;;) {
      int i;
      const std::function<void(int)>* job;
      {
        std::lock_guard<std::mutex> g(mu_);
        if (!job_ || next_ >= n_) return;
        i = next_++;
        job = job_;
      }
      (*job)(i);
      std::lock_guard<std::mutex> g(mu_);
      if (++done_ == n_) done_cv_.notify_all();
    }
  }
  void loop() {
    long seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return gen_ != seen; });
        seen = gen_;
      }
      work();
    }
  }
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int)>* job_ = nullptr;
  int n_ = 0, next_ = 0, done_ = 0, size_ = 1;
  long gen_ = 0;
};

Pool& pool() {
  static Pool* p = [] {
    const unsigned hw = std::thread::hardware_concurrency();
    const int w = (int)std::min(7u, hw > 1 ? hw - 1 : 1u);
    return new Pool(w);   // never destroyed: the workers are detached
  }();
  return *p;
}

struct Staging {
  char* buf[kSlots] = {};
  cudaEvent_t ev[kSlots] = {};
  bool used[kSlots] = {};
};

// one set per device: the slots' events belong to the device whose stream records them
cudaError_t staging(Staging** out) {
  static Staging per_dev[kMaxDevices];
  const int dev = current_device();
  if (dev < 0) return cudaErrorInvalidDevice;
  Staging& s = per_dev[dev];
  if (!s.buf[0]) {
    for (int i = 0; i < kSlots; ++i) {
      cudaError_t e = cudaHostAlloc((void**)&s.buf[i], kSlotBytes, cudaHostAllocPortable);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.ev[i], cudaEventDisableTiming);
      if (e != cudaSuccess) {
        cudaGetLastError();
        return e;
      }
    }
  }
  *out = &s;
  return cudaSuccess;
}

// waits until the slot's last copy is done (events recorded on the device the copy ran on)
cudaError_t slot_free(Staging& s, int i) {
  if (!s.used[i]) return cudaSuccess;
  s.used[i] = false;
  return cudaEventSynchronize(s.ev[i]);
}

}  // namespace

cudaError_t gather_to_device(char* dst, size_t pitch, const void* const* src, long batch, size_t bytes,
                             cudaStream_t st) {
  Staging* sg = nullptr;
  cudaError_t e = staging(&sg);
  if (e != cudaSuccess) return e;
  Pool& P = pool();
  const size_t total = pitch * (size_t)(batch - 1) + bytes;   // the device span
  int slot = 0;
  for (size_t c0 = 0; c0 < total; c0 += kSlotBytes, slot = (slot + 1) % kSlots) {
    const size_t c1 = std::min(total, c0 + kSlotBytes);
    if ((e = slot_free(*sg, slot)) != cudaSuccess) return e;
    char* buf = sg->buf[slot];
    // the chunk's bytes of every instance overlapping [c0, c1), split over the pool
    const int parts = P.size() * 2;
    P.run(parts, [&](int part) {
      size_t p0, p1;
      window_part(c0, c1, part, parts, &p0, &p1);
      gather_pieces(p0, p1, pitch, batch, bytes, [&](long b, size_t in_inst, size_t at, size_t len) {
        memcpy(buf + (at - c0), (const char*)src[b] + in_inst, len);
      });
    });
    if ((e = cudaMemcpyAsync(dst + c0, buf, c1 - c0, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(sg->ev[slot], st)) != cudaSuccess) return e;
    sg->used[slot] = true;
  }
  return cudaSuccess;
}

cudaError_t scatter_to_host(void* const* dst, size_t ld_bytes, const char* src, size_t pitch, long batch,
                            size_t row_bytes, long cols, cudaStream_t st) {
  Staging* sg = nullptr;
  cudaError_t e = staging(&sg);
  if (e != cudaSuccess) return e;
  Pool& P = pool();
  const size_t total = pitch * (size_t)(batch - 1) + ld_bytes * (size_t)(cols - 1) + row_bytes;
  const long nch = (long)((total + kSlotBytes - 1) / kSlotBytes);
  // copy chunk q into slot q % kSlots (the slot's previous unpacking is done: it ran on this thread)
  auto fetch = [&](long q) -> cudaError_t {
    const int slot = (int)(q % kSlots);
    cudaError_t r = slot_free(*sg, slot);
    if (r != cudaSuccess) return r;
    const size_t c0 = (size_t)q * kSlotBytes, c1 = std::min(total, c0 + kSlotBytes);
    if ((r = cudaMemcpyAsync(sg->buf[slot], src + c0, c1 - c0, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return r;
    if ((r = cudaEventRecord(sg->ev[slot], st)) != cudaSuccess) return r;
    sg->used[slot] = true;
    return cudaSuccess;
  };
  if (nch > 0 && (e = fetch(0)) != cudaSuccess) return e;
  for (long q = 0; q < nch; ++q) {
    if (q + 1 < nch && (e = fetch(q + 1)) != cudaSuccess) return e;   // next chunk in flight
    const int slot = (int)(q % kSlots);
    if ((e = slot_free(*sg, slot)) != cudaSuccess) return e;
    const char* buf = sg->buf[slot];
    const size_t c0 = (size_t)q * kSlotBytes, c1 = std::min(total, c0 + kSlotBytes);
    // the first row_bytes of every column that overlap [c0, c1), split over the pool
    const int parts = P.size() * 2;
    P.run(parts, [&](int part) {
      size_t p0, p1;
      window_part(c0, c1, part, parts, &p0, &p1);
      scatter_pieces(p0, p1, pitch, batch, ld_bytes, row_bytes, cols,
                     [&](long b, size_t in_inst, size_t at, size_t len) {
                       memcpy((char*)dst[b] + in_inst, buf + (at - c0), len);
                     });
    });
  }
  return cudaSuccess;
}

}  // namespace ssb
