// Host layer of the C ABI: argument dump, validation, pointer-kind handling, staging of host
// matrices, dispatch to the device kernels, and the synchronous return.
//
// Follows the reference's entry chain: ssblasGemmBatchedEx -> ssblasGemmEx_main (argument dump
// when SSBLAS_GEMMBATCHEDEX_DEBUG is set, src/include/Impl/GemmBatchedEx/ssblasGemmBatchedEx.cpp:97-172)
// -> type-row selection (ssblasGemmBatchedExSelector.hpp:35-107) -> per-row trans checks
// (ssblasGemmBatchedEx_ALLDATASIZESAME.hpp:45-157) -> launch (src/include/Launcher/launcher.hpp:165-246,
// whose empty-grid check gives INTERNAL_ERROR for m, n or batchCount <= 0).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cstdio>
#include <iostream>
#include <mutex>
#include <string>
#include <vector>

#include "grouped.h"
#include "hostcopy.h"
#include "internal.h"

namespace ssb {

Settings& settings() {
  static Settings s = [] {
    Settings t;
    if (const char* e = getenv("SSBLAS_MATH_MODE")) {
      std::string v(e);
      int mode = 0;
      if (v.find("OZAKI") != std::string::npos) mode |= SSBLAS_MATH_FP64_OZAKI;
      if (v.find("BF16X3") != std::string::npos) mode |= SSBLAS_MATH_FP32_BF16X3;
      t.math_mode = mode;
    }
    // SSBLAS_OZAKI_SLICES: forced slice count (3..8); SSBLAS_OZAKI_TOLERANCE: the bound's target
    // (a positive number, e.g. 1e-15); both as ssblasSetOzakiSlices / ssblasSetOzakiTolerance
    if (const char* e = getenv("SSBLAS_OZAKI_SLICES")) {
      const int v = atoi(e);
      if (v >= 3 && v <= 8) t.ozaki_slices = v;
    }
    if (const char* e = getenv("SSBLAS_OZAKI_TOLERANCE")) {
      const double v = strtod(e, nullptr);
      if (v > 0.0) t.ozaki_tolerance = v;
    }
    t.log = getenv("SSBLAS_LOG") != nullptr;
    return t;
  }();
  return s;
}

// SSBLAS_LOG: the kernel choice of each call, after it returns
static void log_call(const char* entry, ssblasStatus_t st, long m, long n, long k, long batch);

static std::mutex g_mutex;
static ssblasRunInfo_t g_info;

std::unique_lock<std::mutex> lock_api() { return std::unique_lock<std::mutex>(g_mutex); }
void reset_run_info() { g_info = ssblasRunInfo_t{}; }

// ---------------------------------------------------------------- kernel profiling -----------
struct ProfPending {
  const char* name;
  cudaEvent_t a, b;
  int dev;
};
struct ProfTotal {
  std::string name;
  int launches = 0;
  double ms = 0.0;
};
static bool g_prof_on = false;
static std::vector<ProfPending> g_prof_pending;
static std::vector<ProfTotal> g_prof_total;
static std::vector<cudaEvent_t> g_prof_free[kMaxDevices];   // events are created on one device

static cudaEvent_t prof_event(int dev) {
  cudaEvent_t e = nullptr;
  if (dev < 0) return nullptr;
  if (!g_prof_free[dev].empty()) {
    e = g_prof_free[dev].back();
    g_prof_free[dev].pop_back();
  } else if (cudaEventCreate(&e) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return e;
}

void prof_start(const char* name, cudaStream_t st) {
  if (!g_prof_on) return;
  const int dev = current_device();
  ProfPending p{name, prof_event(dev), prof_event(dev), dev};
  if (p.a) cudaEventRecord(p.a, st);
  g_prof_pending.push_back(p);
}

void prof_stop(cudaStream_t st) {
  if (!g_prof_on || g_prof_pending.empty()) return;
  ProfPending& p = g_prof_pending.back();
  if (p.b) cudaEventRecord(p.b, st);
}

static void prof_resolve() {
  for (auto& p : g_prof_pending) {
    float ms = 0.f;
    if (p.a && p.b && cudaEventSynchronize(p.b) == cudaSuccess &&
        cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      ProfTotal* t = nullptr;
      for (auto& q : g_prof_total)
        if (q.name == p.name) t = &q;
      if (!t) {
        g_prof_total.push_back(ProfTotal{p.name});
        t = &g_prof_total.back();
      }
      t->launches += 1;
      t->ms += ms;
    }
    cudaGetLastError();
    if (p.a) g_prof_free[p.dev].push_back(p.a);
    if (p.b) g_prof_free[p.dev].push_back(p.b);
  }
  g_prof_pending.clear();
}

void note_launch(int count) { g_info.kernel_launches += count; }
void note_splits(int splits) { g_info.split_k = splits; }
void note_path(int path, int slices) {
  g_info.path = path;
  g_info.slices = slices;
}

int current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return (dev >= 0 && dev < kMaxDevices) ? dev : -1;
}

int num_sms() {
  static int sms[kMaxDevices] = {};
  const int dev = current_device();
  if (dev < 0) return 148;
  if (!sms[dev]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) {
      cudaGetLastError();
      v = 148;
    }
    sms[dev] = v;
  }
  return sms[dev];
}

// ---------------------------------------------------------------- workspace ------------------
struct DeviceWs {
  void* ptr[WS_NUM] = {};
  size_t size[WS_NUM] = {};
};
static std::vector<DeviceWs> g_ws;

void* workspace(WsSlot slot, size_t bytes, cudaError_t* err) {
  int dev = 0;
  *err = cudaGetDevice(&dev);
  if (*err != cudaSuccess) return nullptr;
  if ((int)g_ws.size() <= dev) g_ws.resize(dev + 1);
  DeviceWs& w = g_ws[dev];
  if (bytes == 0) bytes = 256;
  if (settings().fault == SSBLAS_FAULT_ALLOC) {
    // one-shot test fault: this request fails as if the device were out of memory
    settings().fault = SSBLAS_FAULT_NONE;
    *err = cudaErrorMemoryAllocation;
    return nullptr;
  }
  if (w.size[slot] >= bytes) return w.ptr[slot];
  if (w.ptr[slot]) {
    // the old buffer may still be read by work in flight
    cudaStreamSynchronize(settings().stream);
    cudaFree(w.ptr[slot]);
    w.ptr[slot] = nullptr;
    w.size[slot] = 0;
  }
  size_t grow = bytes + bytes / 4;
  grow = (grow + 4095) & ~(size_t)4095;
  *err = cudaMalloc(&w.ptr[slot], grow);
  if (*err != cudaSuccess) {
    cudaGetLastError();
    w.ptr[slot] = nullptr;
    return nullptr;
  }
  w.size[slot] = grow;
  return w.ptr[slot];
}

static void release_pointer_arrays(int dev);
static void release_workspace() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  cudaDeviceSynchronize();
  release_pointer_arrays(dev);
  if ((int)g_ws.size() <= dev) return;
  for (int s = 0; s < WS_NUM; ++s) {
    if (g_ws[dev].ptr[s]) cudaFree(g_ws[dev].ptr[s]);
    g_ws[dev].ptr[s] = nullptr;
    g_ws[dev].size[s] = 0;
  }
}

__device__ int g_device_error = 0;
int* device_error_flag() {
  int* p = nullptr;
  if (cudaGetSymbolAddress((void**)&p, g_device_error) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

// ---------------------------------------------------------------- debug dump -----------------
// Byte-for-byte the reference's dump (ssblasGemmBatchedEx.cpp:8-93), including its spellings.
static void print_op(ssblasOperation_t t) {
  if (SSBLAS_OP_N == t) printf("SSBLAS_OP_N");
  else if (SSBLAS_OP_T == t) printf("SSBLAS_OP_T");
  else if (SSBLAS_OP_C == t) printf("SSBLAS_OP_C");
  else printf("UNKNOWN");
}
static void print_type(ssblasDataType_t t) {
  if (SSBLAS_R_8I == t) printf("SSBLAS_R_8I");
  else if (SSBLAS_R_8U == t) printf("SSBLAS_R_8U");
  else if (SSBLAS_R_16F == t) printf("SSBLAS_R_16F");
  else if (SSBLAS_R_32I == t) printf("SSBLAS_R_32I");
  else if (SSBLAS_R_32F == t) printf("SSBLAS_R_32F");
  else if (SSBLAS_R_64F == t) printf("SSBLAS_R_64F");
  else printf("UNKNONW");
}
static void print_compute(ssblasComputeType_t c) {
  if (SSBLAS_COMPUTE_DEFAULT_TYPE == c) printf("SSBLAS_COMPUTE_DEFAULT_TYPE");
  else if (SSBLAS_COMPUTE_32I == c) printf("SSBLAS_COMPUTE_32I");
  else if (SSBLAS_COMPUTE_32F == c) printf("SSBLAS_COMPUTE_32F");
  else printf("UNKNONW");
}
static void print_algo(ssblasGemmAlgo_t a) {
  if (SSBLAS_COMPUTE_DEFAULT == a) printf("SSBLAS_COMPUTE_DEFAULT");
  else printf("UNKNONW");
}
static void debug_dump(ssblasOperation_t transa, ssblasOperation_t transb, SSINT m, SSINT n, SSINT k,
                       ssblasDataType_t Atype, SSINT lda, ssblasDataType_t Btype, SSINT ldb,
                       ssblasDataType_t Ctype, SSINT ldc, SSINT batchCount,
                       ssblasComputeType_t computeType, ssblasGemmAlgo_t algo) {
  printf("ssblasGemmBatchedExShowdebug: START\n");
  printf("transa: "); print_op(transa); printf("\n");
  printf("transb: "); print_op(transb); printf("\n");
  std::cout << "M: " << m << std::endl;
  std::cout << "N: " << n << std::endl;
  std::cout << "K: " << k << std::endl;
  std::cout << "alpha: " << "" << std::endl;
  std::cout << "A: " << "" << std::endl;
  printf("Atype: "); print_type(Atype); printf("\n");
  std::cout << "lda: " << lda << std::endl;
  std::cout << "B: " << "" << std::endl;
  printf("Btype: "); print_type(Btype); printf("\n");
  std::cout << "ldb: " << ldb << std::endl;
  std::cout << "beta: " << "" << std::endl;
  std::cout << "C: " << "" << std::endl;
  printf("Ctype: "); print_type(Ctype); printf("\n");
  std::cout << "ldc: " << ldc << std::endl;
  std::cout << "batchCount: " << batchCount << std::endl;
  printf("computeType: "); print_compute(computeType); printf("\n");
  printf("algo: "); print_algo(algo); printf("\n");
  printf("ssblasGemmBatchedExShowdebug: END\n");
  fflush(stdout);
}

// ---------------------------------------------------------------- pointers -------------------
enum PtrKind { PK_HOST = 0, PK_DEVICE = 1 };

static PtrKind kind_of(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return PK_HOST;
  }
  return (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) ? PK_DEVICE : PK_HOST;
}

static size_t elem_size(Row r, bool c_operand) {
  if (r == ROW_F32) return 4;
  if (r == ROW_F64) return 8;
  if (r == ROW_F16) return 2;   // C of the fp16 row may be fp32 instead (BatchDesc::c_f32)
  return c_operand ? 4 : 1;
}

// Uniform byte stride of a host pointer array (0 if not uniform or not increasing).
static long uniform_stride(const void* const* ptrs, long batch) {
  if (batch <= 1) return 0;
  long s = (long)((const char*)ptrs[1] - (const char*)ptrs[0]);
  if (s <= 0) return 0;
  for (long b = 2; b < batch; ++b)
    if ((long)((const char*)ptrs[b] - (const char*)ptrs[b - 1]) != s) return 0;
  return s;
}

// Pinned host scratch for pointer-array uploads: a ring of slots, so an asynchronous call only
// waits for the upload issued kPinSlots calls earlier (not for the previous call's kernels, which
// the previous upload is queued behind).
constexpr int kPinSlots = 8;
struct PinnedSlot {
  void* host = nullptr;
  size_t size = 0;
  cudaEvent_t done = nullptr;
  bool pending = false;
};
// One ring per device: a slot's event belongs to the device whose stream recorded it.
static PinnedSlot g_pins[kMaxDevices][kPinSlots];
static int g_pin_cur[kMaxDevices] = {};

static void* pinned(size_t bytes, cudaError_t* err) {
  *err = cudaSuccess;
  const int dev = current_device();
  if (dev < 0) {
    *err = cudaErrorInvalidDevice;
    return nullptr;
  }
  g_pin_cur[dev] = (g_pin_cur[dev] + 1) % kPinSlots;
  PinnedSlot& s = g_pins[dev][g_pin_cur[dev]];
  if (s.pending) cudaEventSynchronize(s.done);
  s.pending = false;
  if (s.size < bytes) {
    if (s.host) cudaFreeHost(s.host);
    s.host = nullptr;
    s.size = 0;
    size_t sz = (bytes + bytes / 4 + 4095) & ~(size_t)4095;
    *err = cudaMallocHost(&s.host, sz);
    if (*err != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    s.size = sz;
  }
  if (!s.done && (*err = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming)) != cudaSuccess) return nullptr;
  return s.host;
}

// marks the current slot as read by an upload just enqueued on `st`
static void pinned_done(cudaStream_t st) {
  const int dev = current_device();
  if (dev < 0) return;
  PinnedSlot& s = g_pins[dev][g_pin_cur[dev]];
  if (cudaEventRecord(s.done, st) == cudaSuccess) s.pending = true;
}

// Device copies of the pointer arrays of recent calls, per device, keyed by the pointer values.
// A caller that repeats a layout (a loop over steps; the staging slots of host matrices) gets
// the arrays it had before: no host->device copy on the stream and no wait for a pinned slot, so
// the calls of a loop queue up behind one another. Since the key is the values, memory freed and
// allocated again at the same addresses is harmless. An entry is rewritten only after the last
// call that read it has finished (its `used` event), and a call on another stream than the
// entry's last user first waits for that use, so `used` always covers every earlier use.
struct PtrArrays {
  std::vector<const void*> key;   // A[0..batch), B[0..batch), C[0..batch)
  void** dev = nullptr;
  size_t cap = 0;                 // pointers the device buffer holds
  cudaEvent_t used = nullptr;
  cudaStream_t last_stream = nullptr;
  bool in_use = false;
  unsigned long tick = 0;
};
constexpr int kPtrEntries = 4;
static PtrArrays g_ptr_arrays[kMaxDevices][kPtrEntries];
static unsigned long g_ptr_tick = 0;
static PtrArrays* g_ptr_current = nullptr;   // entry of the call in progress

static bool same_key(const PtrArrays& e, const std::vector<void*>& a, const std::vector<void*>& b,
                     const std::vector<void*>& c) {
  const size_t n = a.size();
  if (e.key.size() != 3 * n) return false;
  const void* const* k = e.key.data();
  return memcmp(k, a.data(), n * sizeof(void*)) == 0 && memcmp(k + n, b.data(), n * sizeof(void*)) == 0 &&
         memcmp(k + 2 * n, c.data(), n * sizeof(void*)) == 0;
}

static cudaError_t device_pointer_arrays(const std::vector<void*>& a, const std::vector<void*>& b,
                                         const std::vector<void*>& c, cudaStream_t st, void*** out) {
  const int dev = current_device();
  if (!valid_device(dev)) return cudaErrorInvalidDevice;
  const size_t n = a.size();
  PtrArrays* hit = nullptr;
  PtrArrays* victim = nullptr;
  for (PtrArrays& e : g_ptr_arrays[dev]) {
    if (same_key(e, a, b, c)) {
      hit = &e;
      break;
    }
    if (!victim || e.tick < victim->tick) victim = &e;
  }
  cudaError_t err;
  if (hit) {
    if (hit->in_use && hit->last_stream != st && (err = cudaStreamWaitEvent(st, hit->used, 0)) != cudaSuccess)
      return err;
  } else {
    hit = victim;
    if (hit->in_use) {
      if ((err = cudaEventSynchronize(hit->used)) != cudaSuccess) return err;
      hit->in_use = false;
    }
    hit->key.clear();   // no valid contents until the upload below is queued
    if (!hit->used && (err = cudaEventCreateWithFlags(&hit->used, cudaEventDisableTiming)) != cudaSuccess)
      return err;
    if (hit->cap < 3 * n) {
      if (hit->dev) cudaFree(hit->dev);
      hit->dev = nullptr;
      hit->cap = 0;
      const size_t cap = std::max<size_t>(3 * n, 64);
      if ((err = cudaMalloc((void**)&hit->dev, cap * sizeof(void*))) != cudaSuccess) {
        cudaGetLastError();
        return err;
      }
      hit->cap = cap;
    }
    void* h = pinned(3 * n * sizeof(void*), &err);
    if (!h) return err;
    void** hp = (void**)h;
    memcpy(hp, a.data(), n * sizeof(void*));
    memcpy(hp + n, b.data(), n * sizeof(void*));
    memcpy(hp + 2 * n, c.data(), n * sizeof(void*));
    if ((err = cudaMemcpyAsync(hit->dev, hp, 3 * n * sizeof(void*), cudaMemcpyHostToDevice, st)) != cudaSuccess)
      return err;
    pinned_done(st);
    hit->key.assign((const void* const*)hp, (const void* const*)hp + 3 * n);
  }
  hit->tick = ++g_ptr_tick;
  g_ptr_current = hit;
  *out = hit->dev;
  return cudaSuccess;
}

// after the launches of the call that took its arrays from device_pointer_arrays
static void pointer_arrays_used(cudaStream_t st) {
  PtrArrays* e = g_ptr_current;
  g_ptr_current = nullptr;
  if (!e) return;
  if (cudaEventRecord(e->used, st) == cudaSuccess) {
    e->in_use = true;
    e->last_stream = st;
  } else {
    cudaGetLastError();
    e->key.clear();   // cannot tell when its readers finish: never reused, rewritten after a sync
    cudaStreamSynchronize(st);
  }
}

static void release_pointer_arrays(int dev) {
  if (!valid_device(dev)) return;
  for (PtrArrays& e : g_ptr_arrays[dev]) {
    if (e.dev) cudaFree(e.dev);
    if (e.used) cudaEventDestroy(e.used);
    e = PtrArrays{};
  }
}

static ssblasStatus_t map_err(cudaError_t e) {
  if (e == cudaSuccess) return SSBLAS_STATUS_SUCCESS;
  if (e == cudaErrorMemoryAllocation) return SSBLAS_STATUS_ALLOC_FAILED;
  return SSBLAS_STATUS_INTERNAL_ERROR;
}

// Stages the instances of one host-resident operand into device memory. Returns the device
// pointers in dptr (host vector). copy_in=false allocates without copying.
// Pageable (not page-locked) host memory: copied through the pinned staging of hostcopy.cpp
// rather than by the driver's bounce-buffered copies.
static bool is_pageable(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return at.type == cudaMemoryTypeUnregistered;
}
constexpr size_t kStagedCopyMin = (size_t)4 << 20;   // below this, plain per-instance copies

static cudaError_t stage_operand(WsSlot slot, const void* const* hptr, long batch, size_t inst_bytes,
                                 bool copy_in, cudaStream_t st, std::vector<void*>& dptr,
                                 long* dev_stride) {
  long s = uniform_stride(hptr, batch);
  dptr.resize(batch);
  cudaError_t e;
  const bool staged = copy_in && inst_bytes * (size_t)batch >= kStagedCopyMin && is_pageable(hptr[0]);
  // one copy of the whole span when the instances are equally spaced and densely packed
  if (batch == 1 || (s > 0 && (size_t)s >= inst_bytes && (size_t)s <= 2 * inst_bytes + 4096)) {
    size_t span = (batch == 1) ? inst_bytes : (size_t)s * (batch - 1) + inst_bytes;
    char* d = (char*)workspace(slot, span, &e);
    if (!d) return e;
    if (staged && batch > 1) {
      if ((e = gather_to_device(d, (size_t)s, hptr, batch, inst_bytes, st)) != cudaSuccess) return e;
    } else if (copy_in) {
      e = cudaMemcpyAsync(d, hptr[0], span, cudaMemcpyHostToDevice, st);
      if (e != cudaSuccess) return e;
    }
    for (long b = 0; b < batch; ++b) dptr[b] = d + (size_t)b * (size_t)s;
    *dev_stride = (batch == 1) ? (long)((inst_bytes + 255) & ~(size_t)255) : s;
    return cudaSuccess;
  }
  size_t pitch = (inst_bytes + 255) & ~(size_t)255;
  char* d = (char*)workspace(slot, pitch * batch, &e);
  if (!d) return e;
  if (staged) {
    // scattered pageable instances: packed by host threads into pinned slots, one DMA per slot
    for (long b = 0; b < batch; ++b) dptr[b] = d + pitch * b;
    *dev_stride = (long)pitch;
    return gather_to_device(d, pitch, hptr, batch, inst_bytes, st);
  }
  for (long b = 0; b < batch; ++b) {
    dptr[b] = d + pitch * b;
    if (copy_in) {
      e = cudaMemcpyAsync(dptr[b], hptr[b], inst_bytes, cudaMemcpyHostToDevice, st);
      if (e != cudaSuccess) return e;
    }
  }
  *dev_stride = (long)pitch;
  return cudaSuccess;
}

struct Rowsel {
  Row row;
  bool ok;
  bool a_unsigned = false, b_unsigned = false, c_f32 = false;
};

// The reference's three type rows (ssblasGemmBatchedExSelector.hpp:35-107), plus the rows the
// type extensions enable: R_8U for either int8 operand, and fp16 inputs with fp16 or fp32 C.
static Rowsel select_row(ssblasDataType_t a, ssblasDataType_t b, ssblasDataType_t c, int ext = 0) {
  if (a == SSBLAS_R_8I && b == SSBLAS_R_8I && c == SSBLAS_R_32I) return {ROW_I8, true};
  if (a == SSBLAS_R_64F && b == SSBLAS_R_64F && c == SSBLAS_R_64F) return {ROW_F64, true};
  if (a == SSBLAS_R_32F && b == SSBLAS_R_32F && c == SSBLAS_R_32F) return {ROW_F32, true};
  const auto i8 = [](ssblasDataType_t t) { return t == SSBLAS_R_8I || t == SSBLAS_R_8U; };
  if ((ext & SSBLAS_EXT_R8U) && i8(a) && i8(b) && c == SSBLAS_R_32I)
    return {ROW_I8, true, a == SSBLAS_R_8U, b == SSBLAS_R_8U, false};
  if ((ext & SSBLAS_EXT_R16F) && a == SSBLAS_R_16F && b == SSBLAS_R_16F && (c == SSBLAS_R_16F || c == SSBLAS_R_32F))
    return {ROW_F16, true, false, false, c == SSBLAS_R_32F};
  return {ROW_F32, false};
}

// computeType under SSBLAS_EXT_COMPUTE_TYPE: DEFAULT fits every row, 32I the int8 rows, 32F the
// fp32 and fp16 rows (on the fp32 row it asks for FP32 arithmetic, so the 3xBF16 emulation is not
// used). Without the extension computeType is ignored, as in the reference
// (ssblasGemmBatchedEx_ALLDATASIZESAME.hpp:46-49).
static bool compute_type_fits(ssblasComputeType_t c, Row row) {
  if (c == SSBLAS_COMPUTE_DEFAULT_TYPE) return true;
  if (c == SSBLAS_COMPUTE_32I) return row == ROW_I8;
  if (c == SSBLAS_COMPUTE_32F) return row == ROW_F32 || row == ROW_F16;
  return false;
}

// Runs the row's kernels on device-resident data.
static cudaError_t dispatch(const BatchDesc& d, cudaStream_t st) {
  const int mode = d.exact_f32 ? (settings().math_mode & ~SSBLAS_MATH_FP32_BF16X3) : settings().math_mode;
  if (d.k == 0) {
    // k = 0 under SSBLAS_EXT_K0_BETA: C <- beta * C (no operand is read)
    note_path(SSBLAS_PATH_SIMT);
    return launch_simt_gemm(d, st);
  }
  if (d.row == ROW_F16) {
    cudaError_t e = launch_f16_tcgen05(d, st);
    if (e != cudaErrorNotSupported) {
      if (e == cudaSuccess) note_path(SSBLAS_PATH_F16_TCGEN05);
      return e;
    }
  } else if (d.row == ROW_I8) {
    cudaError_t e = launch_i8_tcgen05(d, st);
    if (e != cudaErrorNotSupported) {
      if (e == cudaSuccess) note_path(SSBLAS_PATH_I8_TCGEN05);
      return e;
    }
  } else if (d.row == ROW_F64 && (mode & SSBLAS_MATH_FP64_OZAKI)) {
    cudaError_t e = launch_ozaki_f64(d, ozaki_slices_for_call(), st);
    if (e != cudaErrorNotSupported) return e;
  } else if (d.row == ROW_F64 && choose_config(SSBLAS_PATH_DMMA, d.m, d.n, d.k, d.batch, 0) != 2) {
    // plain fp64: DMMA tiles (configuration 2 selects the DFMA SIMT kernel instead)
    note_path(SSBLAS_PATH_DMMA);
    return launch_dmma_f64(d, st);
  } else if (d.row == ROW_F32 && (mode & SSBLAS_MATH_FP32_BF16X3)) {
    cudaError_t e = launch_bf16x3_f32(d, st);
    if (e != cudaErrorNotSupported) {
      if (e == cudaSuccess) note_path(SSBLAS_PATH_BF16X3_TCGEN05);
      return e;
    }
  }
  note_path(SSBLAS_PATH_SIMT);
  return launch_simt_gemm(d, st);
}

ssblasStatus_t check_device_error(cudaStream_t st) {
  int* flag = device_error_flag();
  if (!flag) return SSBLAS_STATUS_INTERNAL_ERROR;
  int h = 0;
  if (cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return SSBLAS_STATUS_INTERNAL_ERROR;
  if (h != 0) {
    g_info.device_error = h;
    int zero = 0;
    cudaMemcpyAsync(flag, &zero, sizeof(int), cudaMemcpyHostToDevice, st);
    cudaStreamSynchronize(st);
    return SSBLAS_STATUS_INTERNAL_ERROR;
  }
  return SSBLAS_STATUS_SUCCESS;
}

static ssblasStatus_t map_err(cudaError_t e);
static void* pinned(size_t bytes, cudaError_t* err);

// Grouped call with device-resident matrices: validation of every group (the batched call's
// rules), pointer arrays made device-resident, then grouped_run (grouped.cu). Returns
// SSBLAS_STATUS_NOT_COMPUTED_ERROR when the matrices are in host memory, which the caller then
// stages group by group.
static ssblasStatus_t grouped_device(
    const ssblasOperation_t transa_array[], const ssblasOperation_t transb_array[],
    const SSINT m_array[], const SSINT n_array[], const SSINT k_array[],
    const void* const alpha_array[], const void* const A[], const ssblasDataType_t Atype_array[],
    const SSINT lda_array[], const void* const B[], const ssblasDataType_t Btype_array[],
    const SSINT ldb_array[], const void* const beta_array[], void* const C[],
    const ssblasDataType_t Ctype_array[], const SSINT ldc_array[], SSINT group_count,
    const SSINT group_size[]) {
  GroupedDesc g;
  long total = 0;
  for (SSINT gi = 0; gi < group_count; ++gi) {
    Rowsel rs = select_row(Atype_array[gi], Btype_array[gi], Ctype_array[gi]);
    if (!rs.ok) return SSBLAS_STATUS_INVALID_VALUE;
    const int ta = transa_array[gi], tb = transb_array[gi];
    if ((ta != SSBLAS_OP_N && ta != SSBLAS_OP_T) || (tb != SSBLAS_OP_N && tb != SSBLAS_OP_T))
      return SSBLAS_STATUS_INVALID_VALUE;
    const long m = m_array[gi], n = n_array[gi], k = k_array[gi];
    if (m <= 0 || n <= 0 || group_size[gi] <= 0) return SSBLAS_STATUS_INTERNAL_ERROR;
    if (!alpha_array[gi] || !beta_array[gi]) return SSBLAS_STATUS_INVALID_VALUE;
    const long arows = (ta == SSBLAS_OP_N) ? m : k, brows = (tb == SSBLAS_OP_N) ? k : n;
    if (k > 0 && (lda_array[gi] < arows || ldb_array[gi] < brows)) return SSBLAS_STATUS_INVALID_VALUE;
    if (ldc_array[gi] < m) return SSBLAS_STATUS_INVALID_VALUE;
    GroupedInst in{};
    in.row = rs.row; in.transa = ta; in.transb = tb;
    in.m = m; in.n = n; in.k = k; in.lda = lda_array[gi]; in.ldb = ldb_array[gi]; in.ldc = ldc_array[gi];
    if (rs.row == ROW_F32) { in.alpha_f = *(const float*)alpha_array[gi]; in.beta_f = *(const float*)beta_array[gi]; }
    else if (rs.row == ROW_F64) { in.alpha_d = *(const double*)alpha_array[gi]; in.beta_d = *(const double*)beta_array[gi]; }
    else { in.alpha_i = *(const int32_t*)alpha_array[gi]; in.beta_i = *(const int32_t*)beta_array[gi]; }
    for (SSINT j = 0; j < group_size[gi]; ++j) {
      in.idx = total++;
      g.inst.push_back(in);
    }
  }
  std::lock_guard<std::mutex> lock(g_mutex);
  g_info = ssblasRunInfo_t{};
  if (settings().math_mode & SSBLAS_MATH_FP64_OZAKI) {
    // the grouped kernels are built for 7 slices: a fixed other count, or a tolerance that needs
    // 8, cannot be honoured (a looser tolerance is met by 7 slices as well)
    bool any_f64 = false;
    for (const GroupedInst& in : g.inst) any_f64 |= in.row == ROW_F64;
    const int S = ozaki_slices_for_call();
    if (any_f64 && (settings().ozaki_slices != 0 ? S != 7 : S > 7)) return SSBLAS_STATUS_NOTIMPLEMENTED_ERROR;
  }
  cudaStream_t st = settings().stream;
  cudaError_t e;
  const bool dev_arrays = kind_of((const void*)A) == PK_DEVICE;
  if (dev_arrays) {
    if (kind_of((const void*)B) != PK_DEVICE || kind_of((const void*)C) != PK_DEVICE)
      return SSBLAS_STATUS_INVALID_VALUE;
    g.A = A; g.B = B; g.C = C;
  } else {
    if (kind_of((const void*)B) == PK_DEVICE || kind_of((const void*)C) == PK_DEVICE)
      return SSBLAS_STATUS_INVALID_VALUE;
    if (kind_of(A[0]) != PK_DEVICE) return SSBLAS_STATUS_NOT_COMPUTED_ERROR;
    if (kind_of(B[0]) != PK_DEVICE || kind_of(C[0]) != PK_DEVICE) return SSBLAS_STATUS_INVALID_VALUE;
    void* h = pinned(3 * sizeof(void*) * total, &e);
    if (!h) return map_err(e);
    void** hp = (void**)h;
    memcpy(hp, A, sizeof(void*) * total);
    memcpy(hp + total, B, sizeof(void*) * total);
    memcpy(hp + 2 * total, C, sizeof(void*) * total);
    void** dp = (void**)workspace(WS_PTRS, 3 * sizeof(void*) * total, &e);
    if (!dp) return map_err(e);
    if ((e = cudaMemcpyAsync(dp, hp, 3 * sizeof(void*) * total, cudaMemcpyHostToDevice, st))) return map_err(e);
    pinned_done(st);
    g.A = (const void* const*)dp;
    g.B = (const void* const*)(dp + total);
    g.C = (void* const*)(dp + 2 * total);
  }
  if ((e = grouped_run(g, st)) != cudaSuccess) return map_err(e);
  if (settings().synchronous) {
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_err(e);
    return check_device_error(st);
  }
  return SSBLAS_STATUS_SUCCESS;
}

// Host matrices in equally spaced instances (the usual layout of a reference caller): the batch
// is split into chunks whose host->device copies, kernels and device->host copies run on three
// streams, so the copies of one chunk overlap the computation and the copies of the others and
// both PCIe directions are busy at once. Returns SSBLAS_STATUS_NOT_COMPUTED_ERROR when the layout
// does not qualify, or when the operands are pageable and large (the caller then stages the whole
// batch at once, through pinned slots: 32 x 1024^3 FP64 from one pageable array took 70 ms through
// this pipeline's pageable copies and 22 ms staged).
static ssblasStatus_t run_host_pipelined(BatchDesc d, const void* const A[], const void* const B[],
                                         void* const C[], size_t a_bytes, size_t b_bytes, size_t c_bytes,
                                         size_t ec, cudaStream_t st) {
  const long batch = d.batch;
  const long sa = uniform_stride(A, batch), sb = uniform_stride(B, batch);
  const long sc = uniform_stride((const void* const*)C, batch);
  auto dense = [](long s, size_t bytes) { return s > 0 && (size_t)s >= bytes && (size_t)s <= 2 * bytes + 4096; };
  if (!dense(sa, a_bytes) || !dense(sb, b_bytes) || !dense(sc, c_bytes)) return SSBLAS_STATUS_NOT_COMPUTED_ERROR;
  // pageable operands: the driver bounces every chunk through its own staging on this thread;
  // the pinned staging of hostcopy.cpp packs them with several threads instead
  if (a_bytes * (size_t)batch >= kStagedCopyMin && (is_pageable(A[0]) || is_pageable(B[0])))
    return SSBLAS_STATUS_NOT_COMPUTED_ERROR;

  constexpr int NCH = 16;  // chunks: copies of chunk c+1 overlap the GEMM of chunk c and the copy-back of c-1
  struct PipeStreams {
    cudaStream_t s_in = nullptr, s_out = nullptr;
    cudaEvent_t ev_start = nullptr, ev_in[NCH] = {}, ev_cp[NCH] = {};
  };
  static PipeStreams per_dev[kMaxDevices];   // streams and events belong to one device
  const int dev = current_device();
  if (dev < 0) return SSBLAS_STATUS_INTERNAL_ERROR;
  cudaStream_t& s_in = per_dev[dev].s_in;
  cudaStream_t& s_out = per_dev[dev].s_out;
  cudaEvent_t& ev_start = per_dev[dev].ev_start;
  cudaEvent_t* ev_in = per_dev[dev].ev_in;
  cudaEvent_t* ev_cp = per_dev[dev].ev_cp;
  cudaError_t e;
  if (!s_in) {
    if ((e = cudaStreamCreateWithFlags(&s_in, cudaStreamNonBlocking)) ||
        (e = cudaStreamCreateWithFlags(&s_out, cudaStreamNonBlocking)) ||
        (e = cudaEventCreateWithFlags(&ev_start, cudaEventDisableTiming)))
      return map_err(e);
    for (int c = 0; c < NCH; ++c)
      if ((e = cudaEventCreateWithFlags(&ev_in[c], cudaEventDisableTiming)) ||
          (e = cudaEventCreateWithFlags(&ev_cp[c], cudaEventDisableTiming)))
        return map_err(e);
  }
  const bool read_c = d.beta_d != 0.0 || d.beta_f != 0.0f || d.beta_i != 0;
  char* dA = (char*)workspace(WS_STAGE_A, (size_t)sa * (batch - 1) + a_bytes, &e);
  if (!dA) return map_err(e);
  char* dB = (char*)workspace(WS_STAGE_B, (size_t)sb * (batch - 1) + b_bytes, &e);
  if (!dB) return map_err(e);
  char* dC = (char*)workspace(WS_STAGE_C, (size_t)sc * (batch - 1) + c_bytes, &e);
  if (!dC) return map_err(e);
  void** dp = (void**)workspace(WS_PTRS, 3 * sizeof(void*) * batch, &e);
  if (!dp) return map_err(e);
  void** hp = (void**)pinned(3 * sizeof(void*) * batch, &e);
  if (!hp) return map_err(e);
  for (long b = 0; b < batch; ++b) {
    hp[b] = dA + (size_t)b * sa;
    hp[batch + b] = dB + (size_t)b * sb;
    hp[2 * batch + b] = dC + (size_t)b * sc;
  }
  if ((e = cudaMemcpyAsync(dp, hp, 3 * sizeof(void*) * batch, cudaMemcpyHostToDevice, st))) return map_err(e);
  pinned_done(st);
  // the staging buffers may still be in use by earlier work on the library stream
  if ((e = cudaEventRecord(ev_start, st)) || (e = cudaStreamWaitEvent(s_in, ev_start, 0))) return map_err(e);
  d.strideA = sa; d.strideB = sb; d.strideC = sc;
  const long per = (batch + NCH - 1) / NCH;
  const size_t row_bytes = (size_t)d.m * ec, pitch = (size_t)d.ldc * ec;
  for (int c = 0; c < NCH; ++c) {
    const long b0 = c * per, b1 = b0 + per < batch ? b0 + per : batch;
    if (b0 >= b1) break;
    const long nb = b1 - b0;
    if ((e = cudaMemcpyAsync(dA + (size_t)b0 * sa, A[b0], (size_t)sa * (nb - 1) + a_bytes, cudaMemcpyHostToDevice, s_in)) ||
        (e = cudaMemcpyAsync(dB + (size_t)b0 * sb, B[b0], (size_t)sb * (nb - 1) + b_bytes, cudaMemcpyHostToDevice, s_in)))
      return map_err(e);
    if (read_c &&
        (e = cudaMemcpyAsync(dC + (size_t)b0 * sc, C[b0], (size_t)sc * (nb - 1) + c_bytes, cudaMemcpyHostToDevice, s_in)))
      return map_err(e);
    if ((e = cudaEventRecord(ev_in[c], s_in)) || (e = cudaStreamWaitEvent(st, ev_in[c], 0))) return map_err(e);
    BatchDesc sub = d;
    sub.batch = nb;
    sub.A = (const void* const*)(dp + b0);
    sub.B = (const void* const*)(dp + batch + b0);
    sub.C = (void* const*)(dp + 2 * batch + b0);
    sub.A0 = dA + (size_t)b0 * sa; sub.B0 = dB + (size_t)b0 * sb; sub.C0 = dC + (size_t)b0 * sc;
    if (nb == 1) sub.strideA = sub.strideB = sub.strideC = 0;
    if ((e = dispatch(sub, st)) != cudaSuccess) return map_err(e);
    if ((e = cudaEventRecord(ev_cp[c], st)) || (e = cudaStreamWaitEvent(s_out, ev_cp[c], 0))) return map_err(e);
    // only the m x n part of each C goes back (the caller's ld padding stays untouched)
    if ((size_t)sc == pitch * d.n) {
      e = cudaMemcpy2DAsync(C[b0], pitch, dC + (size_t)b0 * sc, pitch, row_bytes, (size_t)d.n * nb,
                            cudaMemcpyDeviceToHost, s_out);
    } else {
      for (long b = b0; b < b1 && e == cudaSuccess; ++b)
        e = cudaMemcpy2DAsync(C[b], pitch, dC + (size_t)b * sc, pitch, row_bytes, d.n, cudaMemcpyDeviceToHost, s_out);
    }
    if (e != cudaSuccess) return map_err(e);
  }
  if ((e = cudaStreamSynchronize(s_out)) || (e = cudaStreamSynchronize(st))) return map_err(e);
  return check_device_error(st);
}

static ssblasStatus_t gemm_batched(ssblasOperation_t transa, ssblasOperation_t transb, SSINT m,
                                   SSINT n, SSINT k, const void* alpha, const void* const A[],
                                   ssblasDataType_t Atype, SSINT lda, const void* const B[],
                                   ssblasDataType_t Btype, SSINT ldb, const void* beta,
                                   void* const C[], ssblasDataType_t Ctype, SSINT ldc,
                                   SSINT batchCount, ssblasComputeType_t computeType,
                                   ssblasGemmAlgo_t algo) {
  if (getenv("SSBLAS_GEMMBATCHEDEX_DEBUG") != nullptr)
    debug_dump(transa, transb, m, n, k, Atype, lda, Btype, ldb, Ctype, ldc, batchCount, computeType, algo);
  ApiRange range("ssblasGemmBatchedEx");

  const int ext = settings().extensions;
  Rowsel rs = select_row(Atype, Btype, Ctype, ext);
  if (!rs.ok) return SSBLAS_STATUS_INVALID_VALUE;
  // op C: rejected (the reference rejects it on the fp rows and mis-computes it on the int8 row);
  // under SSBLAS_EXT_OP_C it is op T, the conjugate transpose of a real matrix
  if ((ext & SSBLAS_EXT_OP_C) && transa == SSBLAS_OP_C) transa = SSBLAS_OP_T;
  if ((ext & SSBLAS_EXT_OP_C) && transb == SSBLAS_OP_C) transb = SSBLAS_OP_T;
  if ((transa != SSBLAS_OP_N && transa != SSBLAS_OP_T) || (transb != SSBLAS_OP_N && transb != SSBLAS_OP_T))
    return SSBLAS_STATUS_INVALID_VALUE;
  if ((ext & SSBLAS_EXT_COMPUTE_TYPE) && !compute_type_fits(computeType, rs.row)) return SSBLAS_STATUS_INVALID_VALUE;
  if (m <= 0 || n <= 0 || batchCount <= 0) return SSBLAS_STATUS_INTERNAL_ERROR;
  const bool k0_beta = (ext & SSBLAS_EXT_K0_BETA) != 0;
  if (k < 0 && k0_beta) return SSBLAS_STATUS_INVALID_VALUE;
  if (k <= 0 && !k0_beta) return SSBLAS_STATUS_SUCCESS;  // the reference leaves C untouched
  if (!alpha || !beta || !A || !B || !C) return SSBLAS_STATUS_INVALID_VALUE;
  const long arows = (transa == SSBLAS_OP_N) ? m : k, acols = (transa == SSBLAS_OP_N) ? k : m;
  const long brows = (transb == SSBLAS_OP_N) ? k : n, bcols = (transb == SSBLAS_OP_N) ? n : k;
  if (ldc < m) return SSBLAS_STATUS_INVALID_VALUE;
  if (k > 0 && (lda < arows || ldb < brows)) return SSBLAS_STATUS_INVALID_VALUE;

  std::lock_guard<std::mutex> lock(g_mutex);
  g_info = ssblasRunInfo_t{};
  cudaStream_t st = settings().stream;
  cudaError_t e;

  BatchDesc d{};
  d.row = rs.row;
  d.transa = transa; d.transb = transb;
  d.m = m; d.n = n; d.k = k; d.lda = lda; d.ldb = ldb; d.ldc = ldc; d.batch = batchCount;
  d.a_unsigned = rs.a_unsigned; d.b_unsigned = rs.b_unsigned; d.c_f32 = rs.c_f32;
  d.exact_f32 = (ext & SSBLAS_EXT_COMPUTE_TYPE) && computeType == SSBLAS_COMPUTE_32F;
  if (rs.row == ROW_F32 || rs.row == ROW_F16) {
    d.alpha_f = *(const float*)alpha; d.beta_f = *(const float*)beta;
  } else if (rs.row == ROW_F64) {
    d.alpha_d = *(const double*)alpha; d.beta_d = *(const double*)beta;
  } else {
    d.alpha_i = *(const int32_t*)alpha; d.beta_i = *(const int32_t*)beta;
  }

  const size_t ea = elem_size(rs.row, false), ec = rs.c_f32 ? 4 : elem_size(rs.row, true);
  // with k = 0 (SSBLAS_EXT_K0_BETA) no operand is read: nothing of A or B is staged
  const size_t a_bytes = k > 0 ? (size_t)(lda * (acols - 1) + arows) * ea : 0;
  const size_t b_bytes = k > 0 ? (size_t)(ldb * (bcols - 1) + brows) * ea : 0;
  const size_t c_bytes = (size_t)(ldc * (n - 1) + m) * ec;

  const PtrKind arr_kind = kind_of((const void*)A);
  if (arr_kind == PK_HOST && (kind_of((const void*)B) != PK_HOST || kind_of((const void*)C) != PK_HOST))
    return SSBLAS_STATUS_INVALID_VALUE;
  const bool sync = settings().synchronous;

  std::vector<const void*> ha, hb;
  std::vector<void*> hc, staged_c;
  bool host_matrices = false;
  if (arr_kind == PK_DEVICE) {
    if (kind_of((const void*)B) != PK_DEVICE || kind_of((const void*)C) != PK_DEVICE)
      return SSBLAS_STATUS_INVALID_VALUE;
    d.A = (const void* const*)A; d.B = (const void* const*)B; d.C = (void* const*)C;
    if (sync) {  // read the pointers back to find uniform strides for the tensor-map paths
      void* h = pinned(3 * sizeof(void*) * batchCount, &e);
      if (!h) return map_err(e);
      void** hp = (void**)h;
      if ((e = cudaMemcpyAsync(hp, A, sizeof(void*) * batchCount, cudaMemcpyDeviceToHost, st)) ||
          (e = cudaMemcpyAsync(hp + batchCount, B, sizeof(void*) * batchCount, cudaMemcpyDeviceToHost, st)) ||
          (e = cudaMemcpyAsync(hp + 2 * batchCount, C, sizeof(void*) * batchCount, cudaMemcpyDeviceToHost, st)) ||
          (e = cudaStreamSynchronize(st)))
        return map_err(e);
      d.A0 = hp[0]; d.strideA = uniform_stride((const void* const*)hp, batchCount);
      d.B0 = hp[batchCount]; d.strideB = uniform_stride((const void* const*)(hp + batchCount), batchCount);
      d.C0 = hp[2 * batchCount]; d.strideC = uniform_stride((const void* const*)(hp + 2 * batchCount), batchCount);
    }
  } else {
    const PtrKind mk = kind_of(A[0]);
    if (kind_of(B[0]) != mk || kind_of(C[0]) != mk) return SSBLAS_STATUS_INVALID_VALUE;
    std::vector<void*> da, db, dc;
    if (mk == PK_DEVICE) {
      da.assign((void* const*)A, (void* const*)A + batchCount);
      db.assign((void* const*)B, (void* const*)B + batchCount);
      dc.assign(C, C + batchCount);
      d.strideA = uniform_stride(A, batchCount);
      d.strideB = uniform_stride(B, batchCount);
      d.strideC = uniform_stride((const void* const*)C, batchCount);
    } else {
      // host matrices, as the reference takes them: stage through device memory
      host_matrices = true;
      if (batchCount >= 8) {
        const ssblasStatus_t ps = run_host_pipelined(d, A, B, C, a_bytes, b_bytes, c_bytes, ec, st);
        if (ps != SSBLAS_STATUS_NOT_COMPUTED_ERROR) return ps;
      }
      if ((e = stage_operand(WS_STAGE_A, A, batchCount, a_bytes, true, st, da, &d.strideA)) ||
          (e = stage_operand(WS_STAGE_B, B, batchCount, b_bytes, true, st, db, &d.strideB)) ||
          (e = stage_operand(WS_STAGE_C, (const void* const*)C, batchCount, c_bytes,
                             d.beta_d != 0.0 || d.beta_f != 0.0f || d.beta_i != 0, st, dc, &d.strideC)))
        return map_err(e);
      if (batchCount == 1) { d.strideA = d.strideB = d.strideC = 0; }
    }
    d.A0 = da[0]; d.B0 = db[0]; d.C0 = dc[0];
    // the three pointer arrays on the device (uploaded unless a recent call had the same)
    void** dp = nullptr;
    if ((e = device_pointer_arrays(da, db, dc, st, &dp)) != cudaSuccess) return map_err(e);
    d.A = (const void* const*)dp;
    d.B = (const void* const*)(dp + batchCount);
    d.C = (void* const*)(dp + 2 * batchCount);
    if (host_matrices) {
      hc.assign(C, C + batchCount);
      staged_c = dc;
    }
  }

  e = dispatch(d, st);
  pointer_arrays_used(st);
  if (e != cudaSuccess) return map_err(e);

  if (host_matrices) {
    // copy back only the m x n part of each C (the ld padding of the caller stays untouched)
    long hs = uniform_stride((const void* const*)C, batchCount);
    const long dstride = batchCount > 1 ? (long)((char*)staged_c[1] - (char*)staged_c[0]) : 0;
    if (batchCount > 1 && (size_t)(ldc * n * ec) * batchCount >= kStagedCopyMin && is_pageable(hc[0]) &&
        uniform_stride((const void* const*)staged_c.data(), batchCount) == dstride) {
      // pageable destinations: through the pinned staging, unpacked by host threads
      e = scatter_to_host(hc.data(), (size_t)(ldc * ec), (const char*)staged_c[0], (size_t)dstride, batchCount,
                          (size_t)(m * ec), n, st);
    } else if (batchCount > 1 && hs == (long)(ldc * n * ec) && (char*)staged_c[1] - (char*)staged_c[0] == hs) {
      e = cudaMemcpy2DAsync(hc[0], ldc * ec, staged_c[0], ldc * ec, m * ec, (size_t)n * batchCount,
                            cudaMemcpyDeviceToHost, st);
    } else {
      for (long b = 0; b < batchCount && e == cudaSuccess; ++b)
        e = cudaMemcpy2DAsync(hc[b], ldc * ec, staged_c[b], ldc * ec, m * ec, n,
                              cudaMemcpyDeviceToHost, st);
    }
    if (e != cudaSuccess) return map_err(e);
  }
  if (sync || host_matrices) {
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_err(e);
    return check_device_error(st);
  }
  return SSBLAS_STATUS_SUCCESS;
}

static void log_call(const char* entry, ssblasStatus_t st, long m, long n, long k, long batch) {
  static const char* const names[] = {"none", "simt", "i8_tcgen05", "ozaki_tcgen05", "bf16x3_tcgen05", "grouped",
                                      "dmma", "", "", "", "", "f16_tcgen05"};
  const int p = g_info.path;
  fprintf(stderr, "ssblas: %s m=%ld n=%ld k=%ld batch=%ld status=%d path=%s slices=%d launches=%d split_k=%d%s\n",
          entry, m, n, k, batch, (int)st, (p >= 0 && p < 12 && names[p][0]) ? names[p] : "?", g_info.slices,
          g_info.kernel_launches, g_info.split_k, g_info.device_error ? " device_error" : "");
}

}  // namespace ssb

using namespace ssb;

extern "C" {

ssblasStatus_t ssblasGemmBatchedEx(ssblasOperation_t transa, ssblasOperation_t transb, SSINT m,
                                   SSINT n, SSINT k, const void* alpha, const void* const A[],
                                   ssblasDataType_t Atype, const SSINT lda, const void* const B[],
                                   ssblasDataType_t Btype, const SSINT ldb, const void* beta,
                                   void* const C[], ssblasDataType_t Ctype, const SSINT ldc,
                                   const SSINT batchCount, ssblasComputeType_t computeType,
                                   ssblasGemmAlgo_t algo) {
  const ssblasStatus_t st = gemm_batched(transa, transb, m, n, k, alpha, A, Atype, lda, B, Btype, ldb, beta,
                                          C, Ctype, ldc, batchCount, computeType, algo);
  if (ssb::settings().log) ssb::log_call("ssblasGemmBatchedEx", st, m, n, k, batchCount);
  return st;
}

ssblasStatus_t ssblasGemmBatchedEx_64(ssblasOperation_t transa, ssblasOperation_t transb,
                                      SSLONG m, SSLONG n, SSLONG k, const void* alpha,
                                      const void* const A[], ssblasDataType_t Atype,
                                      const SSLONG lda, const void* const B[],
                                      ssblasDataType_t Btype, const SSLONG ldb, const void* beta,
                                      void* const C[], ssblasDataType_t Ctype, const SSLONG ldc,
                                      const SSLONG batchCount, ssblasComputeType_t computeType,
                                      ssblasGemmAlgo_t algo) {
  const ssblasStatus_t st = gemm_batched(transa, transb, m, n, k, alpha, A, Atype, lda, B, Btype, ldb, beta,
                                          C, Ctype, ldc, batchCount, computeType, algo);
  if (ssb::settings().log) ssb::log_call("ssblasGemmBatchedEx_64", st, m, n, k, batchCount);
  return st;
}

// Grouped batched GEMM. Validation follows the batched call for each group; groups run in order
// on the library stream. (The persistent single-launch scheduler replaces this loop when all
// groups are device-resident; see grouped.cu.)
ssblasStatus_t ssblasGemmGroupedBatchedEx(
    const ssblasOperation_t transa_array[], const ssblasOperation_t transb_array[],
    const SSINT m_array[], const SSINT n_array[], const SSINT k_array[],
    const void* const alpha_array[], const void* const A[], const ssblasDataType_t Atype_array[],
    const SSINT lda_array[], const void* const B[], const ssblasDataType_t Btype_array[],
    const SSINT ldb_array[], const void* const beta_array[], void* const C[],
    const ssblasDataType_t Ctype_array[], const SSINT ldc_array[], const SSINT group_count,
    const SSINT group_size[], ssblasComputeType_t computeType, ssblasGemmAlgo_t algo) {
  ApiRange range("ssblasGemmGroupedBatchedEx");
  if (group_count <= 0) return SSBLAS_STATUS_INTERNAL_ERROR;
  if (!transa_array || !transb_array || !m_array || !n_array || !k_array || !alpha_array || !A ||
      !Atype_array || !lda_array || !B || !Btype_array || !ldb_array || !beta_array || !C ||
      !Ctype_array || !ldc_array || !group_size)
    return SSBLAS_STATUS_INVALID_VALUE;
  ssblasStatus_t st = grouped_device(transa_array, transb_array, m_array, n_array, k_array,
                                     alpha_array, A, Atype_array, lda_array, B, Btype_array,
                                     ldb_array, beta_array, C, Ctype_array, ldc_array, group_count,
                                     group_size);
  if (st != SSBLAS_STATUS_NOT_COMPUTED_ERROR) return st;
  // host matrices (the reference's convention): each group through the batched path
  long off = 0;
  for (SSINT g = 0; g < group_count; ++g) {
    if (group_size[g] <= 0) return SSBLAS_STATUS_INTERNAL_ERROR;
    st = gemm_batched(transa_array[g], transb_array[g], m_array[g], n_array[g], k_array[g],
                      alpha_array[g], A + off, Atype_array[g], lda_array[g], B + off,
                      Btype_array[g], ldb_array[g], beta_array[g], C + off, Ctype_array[g],
                      ldc_array[g], group_size[g], computeType, algo);
    if (st != SSBLAS_STATUS_SUCCESS) return st;
    off += group_size[g];
  }
  return SSBLAS_STATUS_SUCCESS;
}

ssblasStatus_t ssblasSetStream(void* stream) {
  std::lock_guard<std::mutex> lock(g_mutex);
  settings().stream = (cudaStream_t)stream;
  return SSBLAS_STATUS_SUCCESS;
}

ssblasStatus_t ssblasGetStream(void** stream) {
  if (!stream) return SSBLAS_STATUS_INVALID_VALUE;
  *stream = (void*)settings().stream;
  return SSBLAS_STATUS_SUCCESS;
}

ssblasStatus_t ssblasSetSyncMode(int synchronous) {
  std::lock_guard<std::mutex> lock(g_mutex);
  settings().synchronous = synchronous != 0;
  return SSBLAS_STATUS_SUCCESS;
}

ssblasStatus_t ssblasSetMathMode(int mode) {
  if (mode & ~(SSBLAS_MATH_FP64_OZAKI | SSBLAS_MATH_FP32_BF16X3)) return SSBLAS_STATUS_INVALID_VALUE;
  std::lock_guard<std::mutex> lock(g_mutex);
  settings().math_mode = mode;
  return SSBLAS_STATUS_SUCCESS;
}

ssblasStatus_t ssblasGetMathMode(int* mode) {
  if (!mode) return SSBLAS_STATUS_INVALID_VALUE;
  *mode = settings().math_mode;
  return SSBLAS_STATUS_SUCCESS;
}

ssblasStatus_t ssblasSetOzakiSlices(int slices) {
  if (slices != 0 && (slices < 3 || slices > 8)) return SSBLAS_STATUS_INVALID_VALUE;
  std::lock_guard<std::mutex> lock(g_mutex);
  settings().ozaki_slices = slices;
  return SSBLAS_STATUS_SUCCESS;
}

ssblasStatus_t ssblasSetOzakiTolerance(double tolerance) {
  // NaN and negative targets are refused; a target below the 8-slice bound cannot be met
  if (!(tolerance >= 0.0) || (tolerance > 0.0 && tolerance < ozaki_term_bound(8)))
    return SSBLAS_STATUS_INVALID_VALUE;
  std::lock_guard<std::mutex> lock(g_mutex);
  settings().ozaki_tolerance = tolerance;
  return SSBLAS_STATUS_SUCCESS;
}

ssblasStatus_t ssblasGetOzakiSlices(int* slices) {
  if (!slices) return SSBLAS_STATUS_INVALID_VALUE;
  std::lock_guard<std::mutex> lock(g_mutex);
  *slices = ozaki_slices_for_call();
  return SSBLAS_STATUS_SUCCESS;
}

ssblasStatus_t ssblasSetExtensions(int flags) {
  if (flags & ~(SSBLAS_EXT_R16F | SSBLAS_EXT_R8U | SSBLAS_EXT_OP_C | SSBLAS_EXT_K0_BETA | SSBLAS_EXT_COMPUTE_TYPE))
    return SSBLAS_STATUS_INVALID_VALUE;
  std::lock_guard<std::mutex> lock(g_mutex);
  settings().extensions = flags;
  return SSBLAS_STATUS_SUCCESS;
}

ssblasStatus_t ssblasGetExtensions(int* flags) {
  if (!flags) return SSBLAS_STATUS_INVALID_VALUE;
  *flags = settings().extensions;
  return SSBLAS_STATUS_SUCCESS;
}

ssblasStatus_t ssblasSetFaultInjection(int fault) {
  if (fault != SSBLAS_FAULT_NONE && fault != SSBLAS_FAULT_SKIP_COPY && fault != SSBLAS_FAULT_ALLOC)
    return SSBLAS_STATUS_INVALID_VALUE;
  std::lock_guard<std::mutex> lock(g_mutex);
  settings().fault = fault;
  return SSBLAS_STATUS_SUCCESS;
}

ssblasStatus_t ssblasGetLastRunInfo(ssblasRunInfo_t* info) {
  if (!info) return SSBLAS_STATUS_INVALID_VALUE;
  *info = g_info;
  return SSBLAS_STATUS_SUCCESS;
}

ssblasStatus_t ssblasSetProfiling(int enable) {
  std::lock_guard<std::mutex> lock(g_mutex);
  prof_resolve();
  g_prof_total.clear();
  g_prof_on = enable != 0;
  return SSBLAS_STATUS_SUCCESS;
}

ssblasStatus_t ssblasGetProfile(ssblasKernelProfile_t* out, int max_entries, int* entries) {
  if (!entries || (max_entries > 0 && !out)) return SSBLAS_STATUS_INVALID_VALUE;
  std::lock_guard<std::mutex> lock(g_mutex);
  prof_resolve();
  int n = 0;
  for (auto& t : g_prof_total) {
    if (n < max_entries) {
      snprintf(out[n].name, sizeof(out[n].name), "%s", t.name.c_str());
      out[n].launches = t.launches;
      out[n].total_ms = t.ms;
    }
    ++n;
  }
  *entries = n;
  return SSBLAS_STATUS_SUCCESS;
}

ssblasStatus_t ssblasReleaseWorkspace(void) {
  std::lock_guard<std::mutex> lock(g_mutex);
  release_workspace();
  grouped_release();
  return SSBLAS_STATUS_SUCCESS;
}

}  // extern "C"
