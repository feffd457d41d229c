// Round-synchronous sweeps in one cooperative launch (forward and adjoint solves): the
// grid barrier between rounds and the warp-aggregated append to a round's worklist.
#pragma once

#include "kernels.cuh"

namespace eik {

constexpr int SOLVE_THREADS = 256;  // threads per CTA of the round kernels

__device__ __forceinline__ unsigned long long ld_volatile(const unsigned long long* p) {
  return *(volatile const unsigned long long*)p;
}

__device__ __forceinline__ long long gtimer_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid-wide barrier of the cooperative solve launch (all CTAs co-resident). The wait is
// bounded by the global timer; a CTA that gives up raises the abort flag, which releases
// the others. Returns false when the solve is aborted.
__device__ __forceinline__ bool grid_barrier(const SolveArgs& a) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    volatile unsigned int* gen = a.rs.bar + 1;
    const unsigned int g0 = *gen;
    const unsigned int arrived = atomicAdd(a.rs.bar, 1u);
    bool ok = true;
    if (arrived == gridDim.x - 1) {
      atomicExch(a.rs.bar, 0u);
      __threadfence();
      atomicAdd(a.rs.bar + 1, 1u);
    } else {
      const long long t0 = gtimer_ns();
      while (*gen == g0) {
        if (*(volatile int*)a.abort_flag) {
          ok = false;
          break;
        }
        if (gtimer_ns() - t0 > a.timeout_ns) {
          atomicOr(a.err, ERRB_QUEUE_TIMEOUT);
          atomicExch(a.abort_flag, 1);
          ok = false;
          break;
        }
        __nanosleep(40);
      }
    }
    __threadfence();
    s_ok = ok && !*(volatile int*)a.abort_flag;
  }
  __syncthreads();
  return s_ok != 0;
}

// Appends val for every lane of the warp with have set to the worklist of round r, one
// atomic per warp. All 32 lanes must call it.
__device__ __forceinline__ void warp_append(const SolveArgs& a, int r, bool have, unsigned int val) {
  const unsigned m = __ballot_sync(0xffffffffu, have);
  if (!m) return;
  const int lane = threadIdx.x & 31;
  unsigned int base = 0;
  if (lane == 0) base = atomicAdd(a.rs.cnt + (r % 3), (unsigned int)__popc(m));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (have) a.rs.list[r & 1][base + __popc(m & ((1u << lane) - 1u))] = (unsigned long long)val << 32;
}

}  // namespace eik
