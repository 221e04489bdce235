// mpm_grid.cuh -- a barrier across the blocks of a cooperative launch.
//
// The persistent step kernel runs the passes of several steps in one launch;
// between two passes every block waits for every other.  A cooperative launch
// makes all blocks co-resident, so the wait ends once each block arrives; the
// wait is still bounded (an iteration limit, then ERR_TIMEOUT and the kernel
// leaves), so that no fault of the kernel can keep the GPU busy for good.
#pragma once

#include <cstdint>

#include "mpm_state.cuh"

namespace mpm_b200 {
namespace {

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Global-memory writes of the generic proxy (plain stores of other blocks,
// made visible by the barrier) ordered before this thread's later bulk-copy
// reads, and the bulk-copy writes it waited for before its later plain reads.
__device__ __forceinline__ void fence_global_async() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

constexpr unsigned GRID_BARRIER_SPINS = 1u << 24;  // x 100 ns sleeps: about 2 s

// word[0] counts the blocks that arrived, word[1] is the generation; both are
// zero before the launch.  gen is thread 0's copy of the generation it waits
// to leave.  Returns false in every thread of the block when this block's wait
// ran out or another block raised ERR_TIMEOUT: the caller then returns.
__device__ __forceinline__ bool grid_barrier(const DevState& s, unsigned* word, unsigned nblocks,
                                             unsigned& gen, int& go) {
  __syncthreads();
  if (threadIdx.x == 0) {
    bool ok = true;
    __threadfence();  // this block's writes before its arrival
    if (atomicAdd(&word[0], 1u) == nblocks - 1) {
      atomicExch(&word[0], 0u);
      __threadfence();
      atomicAdd(&word[1], 1u);
    } else {
      unsigned spins = 0;
      while (ld_acquire_gpu(&word[1]) == gen) {
        if (++spins > GRID_BARRIER_SPINS) {
          ok = false;
          break;
        }
        __nanosleep(100);
      }
    }
    __threadfence();
    fence_global_async();
    ++gen;
    if (!ok) atomicOr(s.err, ERR_TIMEOUT);
    go = ok && !(ld_acquire_gpu(s.err) & ERR_TIMEOUT);
  }
  __syncthreads();
  return go != 0;
}

}  // namespace
}  // namespace mpm_b200
