// Hand-written PTX wrappers for sm_100a: mbarriers (with bounded waits), TMA tensor loads,
// tcgen05 tensor-memory allocation, MMA, commit and loads, and the UMMA shared-memory and
// instruction descriptors.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace ssb {
namespace ptx {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ------------------------------------------------------------------------------ mbarrier ----
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, P;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Non-blocking probe of a barrier phase (no suspension of the thread).
__device__ __forceinline__ bool mbar_test_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, P;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Every wait in the library's kernels is bounded. When a wait gives up, the kernel records
// `code` in the device error flag and the caller abandons its loop; the host turns a set flag
// into SSBLAS_STATUS_INTERNAL_ERROR. `limit` is the number of try_wait rounds (kWaitLimit unless
// a launch asks for a shorter one, as the fault-injection test does).
constexpr uint32_t kWaitLimit = 1u << 22;
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int* err, int code,
                                          uint32_t limit = kWaitLimit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  if (err) atomicExch(err, code);
  return false;
}

// Bounded wait by polling (test_wait): for waits on short tensor-core work that many threads share,
// where a suspended try_wait may resume later than the phase completes. The limit counts polls.
constexpr uint32_t kPollLimit = 1u << 26;
__device__ __forceinline__ bool mbar_poll(uint32_t bar, uint32_t parity, int* err, int code) {
  for (uint32_t i = 0; i < kPollLimit; ++i)
    if (mbar_test_wait(bar, parity)) return true;
  if (err) atomicExch(err, code);
  return false;
}

// ------------------------------------------------------------------------------ TMA ---------
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int c0,
                                            int c1, int c2, int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
      : "memory");
}
// Plain (untiled) bulk copy global -> shared; addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(bar)
               : "memory");
}
// Bulk tensor store shared -> global (3-D map), in this thread's bulk async group; writes outside
// the tensor are dropped. commit closes the group; wait_read waits until the stores' shared-memory
// reads are done (the buffer may be written again), wait_all until they are complete.
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, uint32_t src, int c0, int c1, int c2) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(src), "r"(c0), "r"(c1), "r"(c2)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// L2 prefetch of one tile of a 4-D tensor map (no shared memory written, nothing to wait for).
__device__ __forceinline__ void tma_prefetch_l2_4d(const CUtensorMap* map, int c0, int c1, int c2, int c3) {
  asm volatile("cp.async.bulk.prefetch.tensor.4d.L2.global.tile [%0, {%1, %2, %3, %4}];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(c0), "r"(c1), "r"(c2), "r"(c3)
               : "memory");
}
__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// Programmatic dependent launch. A kernel launched with programmatic stream serialization may
// start while the kernel before it in the stream is still running: grid_dep_wait() blocks until
// that kernel has completed and its writes are visible (returns at once for a kernel launched
// the ordinary way), so everything before it must touch no global memory that the previous kernel
// writes or reads. grid_dep_launch() lets the next kernel's CTAs be scheduled onto SMs this grid
// frees; it changes nothing for a next kernel launched the ordinary way.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// ------------------------------------------------------------------------------ tcgen05 -----
__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, int8 x int8 -> int32
__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// The same with the tensor core's A collector buffer: COLLECT = 1 reads A from shared memory and
// keeps it in the collector (.collector::a::fill), 2 takes A from the collector and releases it
// (.collector::a::lastuse; the descriptor names the same A tile as the fill before it), 0 = plain.
template <int COLLECT>
__device__ __forceinline__ void mma_i8_collect(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                               uint32_t accumulate) {
  if constexpr (COLLECT == 1) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8.collector::a::fill [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  } else if constexpr (COLLECT == 2) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8.collector::a::lastuse [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  } else {
    mma_i8(d_tmem, adesc, bdesc, idesc, accumulate);
  }
}
// D[tmem] (+)= A[smem] * B[smem]^T, 16-bit floating inputs -> fp32
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// Arrives on `bar` once all previously issued tcgen05 operations of this thread complete.
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

// 32 lanes x 32 bits, 16 consecutive columns: thread t of the warp gets lane (base + t).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
      "%13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ------------------------------------------------------------------------------ descriptors -
// Shared-memory matrix descriptor for a K-major operand tile whose rows are exactly one swizzle
// span wide (swz_bytes = 32, 64 or 128) and stored back to back: 8-row groups are 8*swz_bytes
// apart (stride byte offset); the leading byte offset is unused for this layout. The tile must
// start on a 1024-byte boundary; advancing along K inside the span adds the byte offset to the
// start address.
__device__ __forceinline__ uint64_t smem_desc_kmajor(uint32_t saddr, int swz_bytes) {
  const uint64_t layout = (swz_bytes == 128) ? 2 : (swz_bytes == 64) ? 4 : 6;
  const uint64_t sbo = (uint64_t)(8 * swz_bytes) >> 4;
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFF) >> 4);  // start address, bits 0-13
  d |= (uint64_t)1 << 16;                    // leading byte offset (unused), bits 16-29
  d |= sbo << 32;                            // stride byte offset, bits 32-45
  d |= (uint64_t)1 << 46;                    // descriptor version for sm_100, bits 46-47
  d |= layout << 61;                         // swizzle mode, bits 61-63
  return d;
}

// Shared-memory matrix descriptor for an MN-major operand tile in the 128-byte swizzled layout:
// the tile is stored as blocks of 128 bytes of M (or N) by the stage's K rows, each K row one
// 128-byte line (8-row groups 1024 bytes apart: stride byte offset), consecutive 128-byte M blocks
// `mn_block_bytes` apart (leading byte offset). The start address must sit on a 1024-byte boundary;
// advancing along K by 8 rows adds 1024 bytes.
__device__ __forceinline__ uint64_t smem_desc_mnmajor(uint32_t saddr, uint32_t mn_block_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFF) >> 4);                // start address, bits 0-13
  d |= (uint64_t)((mn_block_bytes >> 4) & 0x3FFF) << 16;  // leading byte offset: next M block
  d |= (uint64_t)(1024 >> 4) << 32;                       // stride byte offset: next 8 K rows
  d |= (uint64_t)1 << 46;                                 // descriptor version for sm_100
  d |= (uint64_t)2 << 61;                                 // 128-byte swizzle
  return d;
}

// Instruction descriptor (kind::i8 / kind::f16, dense).
//   c_format bits 4-5 (1 = f32, 2 = s32); a_format bits 7-9, b_format bits 10-12
//   (i8: 0 = unsigned, 1 = signed; f16 kind: 0 = f16, 1 = bf16); bits 15/16: A/B MN-major (else
//   K-major); N >> 3 at bits 17-22; M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N, bool a_signed, bool b_signed, bool a_mn = false,
                                                bool b_mn = false) {
  return (2u << 4) | ((a_signed ? 1u : 0u) << 7) | ((b_signed ? 1u : 0u) << 10) | ((a_mn ? 1u : 0u) << 15) |
         ((b_mn ? 1u : 0u) << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn = false, bool b_mn = false) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
// fp16 inputs, fp32 accumulation (kind::f16 with a_format = b_format = f16)
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N, bool a_mn = false, bool b_mn = false) {
  return (1u << 4) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

}  // namespace ptx
}  // namespace ssb
