// Tile queue shared by the forward and adjoint solves: a bucketed priority queue of
// tile ids (bounded multi-producer/multi-consumer rings, Vyukov's sequence scheme) and the
// per-tile state machine that keeps a tile out of two CTAs at once. Every wait is bounded
// by the global timer and reports through the error word.
#pragma once

#include "kernels.cuh"

namespace eik {

// ---------------------------------------------------------------------- queue --
__device__ __forceinline__ unsigned long long ld_volatile(const unsigned long long* p) {
  return *(volatile const unsigned long long*)p;
}

__device__ __forceinline__ long long gtimer_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Push into bucket b; the caller guarantees at most (mask+1) items are ever in one bucket.
__device__ __forceinline__ bool q_push(const SolveArgs& a, int b, unsigned long long item) {
  const unsigned long long cap = a.q.mask + 1;
  unsigned long long* seq = a.q.seq + (unsigned long long)b * cap;
  unsigned long long* items = a.q.items + (unsigned long long)b * cap;
  const unsigned long long pos = atomicAdd(a.q.tail + b, 1ull);
  const unsigned long long slot = pos & a.q.mask;
  const long long t0 = gtimer_ns();
  while (ld_volatile(seq + slot) != pos) {
    if (gtimer_ns() - t0 > a.timeout_ns) {
      atomicOr(a.err, ERRB_QUEUE_TIMEOUT);
      atomicExch(a.abort_flag, 1);
      return false;
    }
    __nanosleep(64);
  }
  items[slot] = item;
  __threadfence();
  atomicExch(seq + slot, pos + 1);
  return true;
}

// Warp-cooperative pop of up to QCLAIM items from the lowest non-empty bucket with one CAS
// (called by all lanes of one warp; results valid in every lane). Returns the count (0 when
// every bucket looks empty).
constexpr int QCLAIM = 4;
__device__ __forceinline__ int q_pop_warp(const SolveArgs& a, unsigned long long* items_out) {
  const int lane = threadIdx.x & 31;
  const unsigned long long cap = a.q.mask + 1;
  for (int attempt = 0; attempt < 4096; attempt++) {
    const int b0 = lane, b1 = lane + 32;
    const unsigned long long h0 = ld_volatile(a.q.head + b0), t0v = ld_volatile(a.q.tail + b0);
    const unsigned long long h1 = ld_volatile(a.q.head + b1), t1v = ld_volatile(a.q.tail + b1);
    const unsigned m0 = __ballot_sync(0xffffffffu, h0 < t0v), m1 = __ballot_sync(0xffffffffu, h1 < t1v);
    if (!m0 && !m1) return 0;
    const int b = m0 ? __ffs(m0) - 1 : 32 + __ffs(m1) - 1;
    int got = 0;
    if (lane == 0) {
      const unsigned long long h = ld_volatile(a.q.head + b), t = ld_volatile(a.q.tail + b);
      if (h < t) {
        const unsigned long long k = (t - h) < (unsigned long long)QCLAIM ? (t - h) : (unsigned long long)QCLAIM;
        if (atomicCAS(a.q.head + b, h, h + k) == h) {
          unsigned long long* seq = a.q.seq + (unsigned long long)b * cap;
          for (unsigned long long j = 0; j < k; j++) {
            const unsigned long long pos = h + j, slot = pos & a.q.mask;
            const long long tt0 = gtimer_ns();
            bool ok = true;
            while (ld_volatile(seq + slot) != pos + 1) {
              if (gtimer_ns() - tt0 > a.timeout_ns) {
                atomicOr(a.err, ERRB_QUEUE_TIMEOUT);
                atomicExch(a.abort_flag, 1);
                ok = false;
                break;
              }
              __nanosleep(32);
            }
            if (!ok) break;
            items_out[got++] = ld_volatile(a.q.items + (unsigned long long)b * cap + slot);
            __threadfence();
            atomicExch(seq + slot, pos + cap);
          }
        }
      }
    }
    got = __shfl_sync(0xffffffffu, got, 0);
    if (got) {
      for (int j = 0; j < QCLAIM; j++) items_out[j] = __shfl_sync(0xffffffffu, items_out[j], 0);
      return got;
    }
    if (*(volatile int*)a.abort_flag) return 0;
    if (lane == 0) __nanosleep(20 + (threadIdx.x * 7 + attempt * 13) % 200);
    __syncwarp();
  }
  return 0;
}

// Bucket of a trigger time; a nearly full bucket spills into the next one (ordering degrades
// gracefully instead of a producer waiting on a full ring).
__device__ __forceinline__ int bucket_of(const SolveArgs& a, const CoarseProblem& P, double prio) {
  const double x = prio * P.tinv;
  int b = (!(x < (double)(QBUCKETS - 1))) ? QBUCKETS - 1 : (x > 0.0 ? (int)x : 0);
  const unsigned long long lim = (a.q.mask + 1) - 4096;
  while (b < QBUCKETS - 1 && ld_volatile(a.q.tail + b) - ld_volatile(a.q.head + b) >= lim) b++;
  return b;
}

// Tile states: 0 idle, 1 queued, 2 being processed, 3 being processed and changed again
// by a neighbour meanwhile (re-queued by its processor when it finishes). A tile is never
// processed by two CTAs at once, so a write-back can never overwrite newer values.
constexpr int TS_IDLE = 0, TS_QUEUED = 1, TS_BUSY = 2, TS_BUSY_DIRTY = 3;

__device__ __forceinline__ unsigned long long tile_item(int prob, long long tile) {
  return ((unsigned long long)prob << 40) | (unsigned long long)tile;
}

// Marks faces of a tile dirty with trigger time prio and queues it unless it is queued
// already or its current processor will re-queue it.
__device__ __forceinline__ void enqueue_tile(const SolveArgs& a, int prob, long long tile, uint32_t faces, double prio) {
  const long long gt = a.probs[prob].tbase + tile;
  atomicOr(a.tile_faces + gt, faces);
  atomicMin(a.tile_prio + gt, (unsigned long long)__double_as_longlong(prio));
  int s = *(volatile int*)(a.tile_flag + gt);
  for (int it = 0; it < 64; it++) {
    if (s == TS_IDLE) {
      const int o = atomicCAS(a.tile_flag + gt, TS_IDLE, TS_QUEUED);
      if (o == TS_IDLE) {
        atomicAdd(a.pending, 1);
        const double pr = __longlong_as_double((long long)ld_volatile(a.tile_prio + gt));
        q_push(a, bucket_of(a, a.probs[prob], pr), tile_item(prob, tile));
        return;
      }
      s = o;
    } else if (s == TS_BUSY) {
      const int o = atomicCAS(a.tile_flag + gt, TS_BUSY, TS_BUSY_DIRTY);
      if (o == TS_BUSY) return;
      s = o;
    } else {
      return;  // already queued, or its processor will re-queue it
    }
  }
  atomicOr(a.err, ERRB_QUEUE_TIMEOUT);
  atomicExch(a.abort_flag, 1);
}

// Called by the processor of a tile when it is done with it.
__device__ __forceinline__ void finish_tile(const SolveArgs& a, int prob, long long tile) {
  const long long gt = a.probs[prob].tbase + tile;
  const int o = atomicCAS(a.tile_flag + gt, TS_BUSY, TS_IDLE);
  if (o == TS_BUSY) {
    atomicSub(a.pending, 1);
    return;
  }
  // TS_BUSY_DIRTY: stays counted in pending, goes back to the queue
  atomicExch(a.tile_flag + gt, TS_QUEUED);
  const double pr = __longlong_as_double((long long)ld_volatile(a.tile_prio + gt));
  q_push(a, bucket_of(a, a.probs[prob], pr), tile_item(prob, tile));
}


// ------------------------------------------------------------------ tile shapes --
template <int ND> struct TileCfg;
template <> struct TileCfg<3> {
  static constexpr int TX = 4, TY = 4, TZ = 4, H = 2;
  static constexpr int HX = TX + 2 * H, HY = TY + 2 * H, HZ = TZ + 2 * H;
};
template <> struct TileCfg<2> {
  static constexpr int TX = 8, TY = 8, TZ = 1, H = 2;
  static constexpr int HX = TX + 2 * H, HY = TY + 2 * H, HZ = 1;
};
constexpr int SOLVE_THREADS = 256;  // 8 warps, one tile per warp
constexpr int SOLVE_WARPS = SOLVE_THREADS / 32;

}  // namespace eik
