// Bounded grid-wide barrier among the CTAs of one cooperative launch (co-resident by construction).
// Each CTA's thread 0 releases its writes (__threadfence), arrives on a monotone counter and spins with acquire
// loads until the counter reaches `target`.  The spin is bounded: past limit_ns of global time it stores `code`
// in *status and gives up, and a CTA that sees another CTA's code gives up too, so a missing arrival ends every
// waiting CTA with an error instead of a hang.  Returns false in every thread of a CTA that gave up.
#pragma once
#include "ptx.cuh"

namespace db200 {

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ bool grid_barrier(unsigned* count, unsigned target, int* status, int code,
                                             unsigned long long limit_ns, bool arrive = true) {
  __syncthreads();
  int ok = 1;
  if (threadIdx.x == 0) {
    __threadfence();
    if (arrive) atomicAdd(count, 1u);
    const uint64_t t0 = global_timer_ns();
    while (ld_acquire_u32(count) < target) {
      if (*reinterpret_cast<volatile int*>(status)) {
        ok = 0;
        break;
      }
      if (global_timer_ns() - t0 > limit_ns) {
        atomicCAS(status, 0, code);
        ok = 0;
        break;
      }
    }
    __threadfence();
  }
  return __syncthreads_and(ok) != 0;
}

}  // namespace db200
