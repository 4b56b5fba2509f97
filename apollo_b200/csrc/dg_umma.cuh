// tcgen05 (5th-generation tensor core) helpers for sm_100a: shared-memory
// matrix descriptors, the instruction descriptor for kind::tf32, MMA issue,
// commit to an mbarrier, TMEM allocation and loads, and bounded waits.
//
// Operand layout used throughout: K-major, no swizzle ("interleave").  A
// matrix of R rows (multiple of 8) and K columns (multiple of 4 fp32) is
// stored as 8-row x 16-byte core matrices; element (r, k) sits at byte
//   (r / 8) * SBO + (k / 4) * LBO + (r % 8) * 16 + (k % 4) * 4
// with LBO = 128 (core matrices adjacent along K) and SBO = K * 32 (one
// 8-row group after another).  One kind::tf32 MMA consumes K = 8 (two core
// matrices along K); the k-th step starts 2 * k * LBO bytes further.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace apollo {
namespace umma {

constexpr uint32_t kLBO = 128;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__host__ __device__ constexpr uint32_t kmajor_offset(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K * 32) + (k >> 2) * kLBO + (r & 7) * 16 + (k & 3) * 4);
}
// The same layout with an explicit 8-row group stride (SBO); a stride of
// K * 32 + 16 staggers the groups across the shared-memory banks.
__host__ __device__ constexpr uint32_t kmajor_offset_sbo(int r, int k, int sbo) {
  return (uint32_t)((r >> 3) * sbo + (k >> 2) * kLBO + (r & 7) * 16 + (k & 3) * 4);
}

// Shared-memory matrix descriptor (sm_100: version 1, no swizzle).
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // version
  // base offset 0, lbo mode 0, layout type 0 (no swizzle)
  return d;
}

// Instruction descriptor: D fp32, A and B tf32, both K-major, shape M x N.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4)            // D format F32
         | (2u << 7)          // A format TF32
         | (2u << 10)         // B format TF32
         | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[desc] * B[desc]^T, issued by one thread.
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

// Arrive on an mbarrier once all MMAs issued so far by this thread complete.
__device__ __forceinline__ void commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

// One poll of an mbarrier phase.  The thread may be suspended until the phase
// completes or kSuspendNs nanoseconds pass, so a waiting warp issues one poll
// per interval instead of spinning on the scheduler its working warps share.
constexpr uint32_t kSuspendNs = 500;
__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity), "r"(kSuspendNs)
      : "memory");
  return ok != 0;
}

// One poll without a suspend hint (returns at once).
__device__ __forceinline__ bool mbar_test_wait(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded spin on an mbarrier phase for a single waiting warp whose wait is
// short (the tensor core finishing a few MMAs): polls without suspending, so
// the warp sees the phase complete at once; gives up after `limit` polls
// (about 2^27 cycles at the default) and returns false.
__device__ __forceinline__ bool mbar_spin_bounded(uint32_t mbar, uint32_t parity, uint32_t limit = (1u << 22)) {
  for (uint32_t i = 0; i < limit; ++i) {
    if (mbar_test_wait(mbar, parity)) return true;
    if (i > 64) __nanosleep(32);
  }
  return false;
}

// Bounded wait on an mbarrier phase: gives up after `limit` polls (each poll
// suspends for at most kSuspendNs: about 2 s in all) and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mbar, uint32_t parity, uint32_t limit = (1u << 22)) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(mbar, parity)) return true;
  return false;
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// TMEM allocation by one full warp; the base address is written to smem.
__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive fp32 columns of this thread's TMEM lane (warp w reads lanes
// 32 (w % 4) .. + 31; taddr carries the lane in bits 31..16).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 4 and 8 consecutive fp32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, float (&v)[4]) {
  uint32_t r[4];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 4; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// Round to tf32 (nearest, ties away): the value keeps 10 mantissa bits.
__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// The same rounding on the bit pattern with two integer operations: adding
// half a tf32 unit to the magnitude and clearing the 13 dropped bits rounds to
// nearest with ties away from zero (a carry into the exponent is the correct
// result).  Finite inputs give the value cvt.rna gives; a NaN may come out as
// an infinity, which the float64 epilogue's finiteness check still reports.
__device__ __forceinline__ float round_tf32(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

// One-dimensional bulk copy global -> this CTA's shared memory, completing
// on an mbarrier (both addresses 16-byte aligned, size a multiple of 16).
__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}

// One-dimensional bulk copy of this CTA's shared memory to global memory
// (both addresses 16-byte aligned, size a multiple of 16), tracked as a bulk
// group of the issuing thread.
__device__ __forceinline__ void bulk_s2g(void* dst, uint32_t src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the issuing thread's bulk groups have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// ... and their writes are complete
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

}  // namespace umma
}  // namespace apollo
