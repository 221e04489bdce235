// mpm_bulk.cuh -- shared-memory staging of a block's particle slices with the
// Blackwell bulk-copy engine (cp.async.bulk without a tensor map: every
// particle field is a contiguous array, so a block's slice of a field is one
// contiguous segment) and mbarrier completion.
//
// Rules kept by every caller: source and destination 16-byte aligned, sizes
// multiples of 16 bytes (particle arrays are padded to whole blocks), no
// multicast.  Waits are bounded: a wait that runs out reports failure and the
// kernel sets ERR_TIMEOUT instead of spinning forever.
#pragma once

#include <cstdint>

namespace mpm_b200 {
namespace bulk {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

// make the initialised barriers visible to the bulk-copy (async) proxy
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// arrive once and announce the bytes the barrier's phase will receive
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// global -> shared copy of `bytes`, completing on `bar`
__device__ __forceinline__ void load(void* dst_smem, const void* src, unsigned bytes,
                                     uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst_smem)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait for the phase with the given parity (each try_wait suspends
// the thread for a hardware-limited time).  False: the copies did not arrive.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int tries = 1 << 20) {
  for (int i = 0; i < tries; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Test hook of the wait-timeout path: after phase 0 of `bar` has completed,
// wait a few tries for phase 1, which no thread or copy ever completes, so
// the wait runs out exactly as a lost copy would make it.  Every copy of
// phase 0 has landed by then; the caller's final drain waits for the rest.
__device__ __forceinline__ bool mbar_wait_never(uint64_t* bar) { return mbar_wait(bar, 1, 16); }

// order this thread's generic-proxy shared-memory writes before later
// bulk-copy reads of them
__device__ __forceinline__ void fence_shared_to_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// shared -> global copy of `bytes` (bulk-group completion)
__device__ __forceinline__ void store(void* dst, const void* src_smem, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
               "r"(smem_addr(src_smem)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void store_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// wait until every committed store has completed (writes visible)
__device__ __forceinline__ void store_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// wait until every committed store has read its shared-memory source: enough
// before a block exits (its shared memory may then be reused), since the
// writes complete before the kernel does
__device__ __forceinline__ void store_wait_read() {
#ifdef MPM_BULK_STORE_FULL_WAIT
  store_wait_all();
#else
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
#endif
}

}  // namespace bulk
}  // namespace mpm_b200
