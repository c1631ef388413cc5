// Blackwell (sm_100a) tensor-core building blocks: fifth-generation MMA
// (tcgen05.mma kind::tf32) issued by one thread with operands in shared
// memory and accumulators in Tensor Memory (TMEM), completion through an
// mbarrier, results read back with tcgen05.ld.
//
// Shared-memory operands use the no-swizzle K-major layout: 8-row x 16-byte
// core matrices (8 rows x 4 TF32 values, rows 16 bytes apart), the two core
// matrices of one K = 8 step LBO bytes apart, consecutive 8-row groups SBO
// bytes apart.  The matrix descriptor holds start, LBO and SBO in 16-byte
// units, version 1, layout type 0 (no swizzle).  The instruction descriptor
// of kind::tf32: D format F32 (bits 4-5 = 1), A and B format TF32 (bits 7-9
// and 10-12 = 2), optional negation of A (bit 13), both operands K-major,
// N >> 3 in bits 17-22, M >> 4 in bits 24-28.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace negf {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---------------------------------------------------------------- TMEM --
// Allocates `ncols` TMEM columns (a power of two >= 32) for the CTA; one full
// warp calls it.  The address lands in *slot (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes made visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ------------------------------------------------------------ mbarrier --
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// Waits for the phase with the given parity to complete, polling with the
// non-blocking test_wait; gives up after `limit_ns` nanoseconds of wall time
// and returns false (the caller reports the failure).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
  const uint32_t a = smem_u32(bar);
  const uint64_t t0 = globaltimer_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (globaltimer_ns() - t0 > limit_ns) return false;
    __nanosleep(20);
  }
}
// The mbarrier receives one arrival when every tcgen05.mma issued so far by
// this thread has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// --------------------------------------------------------- descriptors --
__device__ __forceinline__ uint64_t smem_desc(const void* start, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  const uint64_t addr = (smem_u32(start) >> 4) & 0x3FFFu;
  const uint64_t lbo = (lbo_bytes >> 4) & 0x3FFFu;
  const uint64_t sbo = (sbo_bytes >> 4) & 0x3FFFu;
  return addr | (lbo << 16) | (sbo << 32) | (uint64_t(1) << 46);  // version 1, no swizzle
}
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N, bool negate_a) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((negate_a ? 1u : 0u) << 13) | (uint32_t(N >> 3) << 17) |
         (uint32_t(M >> 4) << 24);
}

// D[tmem] (+)= A B for one M x N x 8 step (kind::tf32); `accumulate` false
// overwrites D.  Issued by a single thread.
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         bool accumulate) {
  const uint32_t acc = accumulate ? 1u : 0u;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      :
      : "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(acc)
      : "memory");
}

// 8 consecutive 32-bit TMEM columns of this thread's lane (warp w reads
// lanes 32 (w % 4) .. 32 (w % 4) + 31; taddr carries that lane base).
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace umma
}  // namespace negf
