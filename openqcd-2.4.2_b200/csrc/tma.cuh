// Bulk asynchronous copies global -> shared memory (cp.async.bulk, the
// untiled TMA path of sm_90+/sm_100) completed through an mbarrier, for
// kernels that stream contiguous field planes through shared memory.  No
// cluster multicast: every CTA copies into its own shared memory from this
// GPU's global memory.  Waits are bounded: a wait that gives up records an
// error in *err for the host to check.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace qcd {

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

// Per-thread asynchronous copies global -> shared memory (cp.async, 16 or
// 8 bytes), zero-filled when ok is false (nothing is read from src then; src
// must still be a valid address).  Completion per thread: commit_group after
// a set of copies, wait_group<N> until at most N committed sets are pending;
// a thread then reads its own copies.
__device__ __forceinline__ void cp_async16(void *dst, const void *src, bool ok) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(ok ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src, bool ok) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(ok ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// make the initialised barriers visible to the async (bulk copy) proxy
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// dst (shared) <- src (global), bytes a multiple of 16, both 16-byte aligned
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// L2 policy for data read once (evict first), for the cache-hint form below
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

// bulk_g2s with an L2 cache-eviction policy
__device__ __forceinline__ void bulk_g2s_hint(void *dst, const void *src, unsigned bytes, uint64_t *bar,
                                              uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// wait for phase `parity` of the barrier; false (and *err set) if it does
// not complete within the iteration limit
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, int *err) {
  for (int it = 0; it < (1 << 22); it++)
    if (mbar_try_wait(bar, parity)) return true;
  atomicOr(err, 1);
  return false;
}

// the same with the error recorded by a plain store (for a flag in mapped
// host memory, where device atomics are not guaranteed), and an explicit
// iteration limit
__device__ __forceinline__ bool mbar_wait_st_lim(uint64_t *bar, unsigned parity, int *err, int limit) {
  for (int it = 0; it < limit; it++)
    if (mbar_try_wait(bar, parity)) return true;
  *(volatile int *)err = 1;
  return false;
}
__device__ __forceinline__ bool mbar_wait_st(uint64_t *bar, unsigned parity, int *err) {
  return mbar_wait_st_lim(bar, parity, err, 1 << 22);
}

}  // namespace qcd
