// Coarse-grid forward solve: the reference's heap-ordered FMM main loop
// (ttFMM_core!, src/EikSolv/eikmainfwd.jl:427-823) restated as the fixed point of the
// order rule of stencil.cuh and solved by a node-level worklist iteration.
//
// One cooperative persistent launch serves many problems (the sources of a call, or the
// refined windows around them). It runs in rounds separated by a grid barrier. In round r
// the warps take the round's worklist 32 entries at a time; a node whose potential is at
// most the problem's threshold is evaluated, and when its value or key changes the nodes
// whose stencil reads it are listed for round r+1; a node still above the threshold is
// listed again with its pending front. The threshold follows the front (smallest pending
// front + a round width of about one node's traveltime), so the rounds sweep the grid in
// traveltime order. Every wait is bounded (global timer), the number of rounds is bounded;
// both report through an error word instead of trapping.
#include "kernels.cuh"
#include "node.cuh"
#include "rounds.cuh"

namespace eik {


// Worklist entry: node id (problem * N + node) in the high word, a lower bound of the
// node's pending front (float, rounded down) in the low word.
__device__ __forceinline__ unsigned long long list_entry(unsigned int gid, double front) {
  const float f = front < EIK_INF ? __double2float_rd(front) : __int_as_float(0x7f800000);
  return ((unsigned long long)gid << 32) | (unsigned long long)__float_as_uint(f);
}

// Lists node gid for round r, once per round.
__device__ __forceinline__ void list_node(const SolveArgs& a, int r, unsigned int gid, double front) {
  if (atomicExch(a.rs.stamp + gid, r) != r) {
    const unsigned int i = atomicAdd(a.rs.cnt + (r % 3), 1u);
    a.rs.list[r & 1][i] = list_entry(gid, front);
  }
}

// ----------------------------------------------------------------------- init --
__global__ void coarse_init_kernel(const CoarseProblem* probs, int nprob, long long N) {
  const long long tot = N * nprob;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot;
       q += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(q / N);
    const long long l = q - (long long)p * N;
    probs[p].t[l] = EIK_INF;
    probs[p].code[l] = CODE_NONE;
  }
}

__global__ void rounds_init_kernel(SolveArgs a) {
  const long long tot = (long long)a.rs.stride * a.nprob;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot;
       q += (long long)gridDim.x * blockDim.x) {
    a.rs.stamp[q] = -1;
    a.rs.dirty[q] = 1;
  }
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < 3LL * a.nprob;
       q += (long long)gridDim.x * blockDim.x)
    a.rs.nextmin[q] = (unsigned long long)__double_as_longlong(EIK_INF);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < 2LL * a.nprob;
       q += (long long)gridDim.x * blockDim.x)
    a.rs.thr[q] = -EIK_INF;
  if (blockIdx.x == 0 && threadIdx.x < 3) {
    a.rs.cnt[threadIdx.x] = 0;
    a.rs.grab[threadIdx.x] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.rs.bar[0] = 0;
    a.rs.bar[1] = 0;
    *a.rs.rounds = 0;
    for (int k = 0; k < 7; k++) a.rs.visits[k] = 0;
    *a.activations = 0;
    *a.node_evals = 0;
    *a.abort_flag = 0;
  }
}

// Seeds: fixed traveltimes of the source points (coarse source box, coarse-coincident
// accepted fine nodes, or the source box of a refined window); the nodes within two steps
// of a seed start round 0, whose threshold is based on the smallest seed traveltime.
template <int ND>
__global__ void seed_kernel(SolveArgs a, const int32_t* seed_lin, const double* seed_tt, const SrcOut* out,
                            int fine_corners, int seedcap) {
  const int s = blockIdx.x;
  const CoarseProblem& P = a.probs[s];
  const int ns = fine_corners ? out[s].nsrcf : out[s].nseeds;
  for (int q = threadIdx.x; q < ns; q += blockDim.x) {
    const long long l = seed_lin[(size_t)s * seedcap + q];
    P.t[l] = seed_tt[(size_t)s * seedcap + q];
    P.code[l] = (uint8_t)(CODE_NONE | CODE_SRC_BIT);
    P.kL[l] = -EIK_INF;
    P.kd[l] = 0;
  }
  __syncthreads();
  __threadfence();
  for (int q = threadIdx.x; q < ns; q += blockDim.x) {
    const long long l = seed_lin[(size_t)s * seedcap + q];
    const int i = (int)(l % P.g.n[0]);
    const int j = (int)((l / P.g.n[0]) % P.g.n[1]);
    const int k = (int)(l / ((long long)P.g.n[0] * P.g.n[1]));
    const int c[3] = {i, j, k};
    const double tt = seed_tt[(size_t)s * seedcap + q];
    if (tt < EIK_INF) atomicMin(a.rs.nextmin + s, (unsigned long long)__double_as_longlong(tt));
    const unsigned long long gbase = (unsigned long long)s * a.rs.stride;
    for (int ax = 0; ax < ND; ax++)
      for (int d = -2; d <= 2; d++) {
        if (d == 0) continue;
        int p[3] = {c[0], c[1], c[2]};
        p[ax] += d;
        if (p[ax] < 0 || p[ax] >= P.g.n[ax]) continue;
        list_node(a, 0, (unsigned int)(gbase + lin3(P.g, p[0], p[1], p[2])), tt);
      }
  }
}

#ifdef EIK_PHASE
// tuning builds only: clock cycles per phase summed over warps (lane 0); 9..11: cycles of
// the entry loads of a queue fill, and the counts of fill and evaluation steps
__device__ unsigned long long eik_phase[12];
extern "C" int eik_phase_read(unsigned long long* out) {
  return (int)cudaMemcpyFromSymbol(out, eik_phase, sizeof(unsigned long long) * 12);
}
#define PH_T(v) const long long v = clock64()
#define PH_ADD(k, t0) if ((threadIdx.x & 31) == 0) atomicAdd(&eik_phase[k], (unsigned long long)(clock64() - (t0)))
#define PH_CNT(k) if ((threadIdx.x & 31) == 0) atomicAdd(&eik_phase[k], 1ull)
#else
#define PH_T(v)
#define PH_ADD(k, t0)
#define PH_CNT(k)
#endif
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ void atomic_min_pos(unsigned long long* p, double v) {
  // traveltimes and potentials are >= 0: their bit patterns order as the values
  if (v < EIK_INF && v < __longlong_as_double((long long)ld_volatile(p)))
    atomicMin(p, (unsigned long long)__double_as_longlong(v));
}

// Forward coarse solve in rounds (one cooperative launch for all problems). Round r takes
// the listed nodes; problem p only evaluates nodes whose potential (smallest neighbouring
// traveltime) is at most T_p(r) = (smallest pending front of p after round r-1) + delta_p,
// delta_p being about one node's traveltime at the largest velocity. The rounds thus
// follow the front like a Dijkstra sweep with buckets one node wide. A node whose value or
// key changed lists the nodes whose stencil reads it for the next round; a node below the
// front is listed again. The result is the same fixed point as any other evaluation order.
//
// QUEUE selects how a warp works through its entries: true settles the visits whose front
// still stands at once and queues the others in shared memory, evaluating them 32 at a time
// (the lanes of a warp then run the long evaluation path together, and the later
// evaluation sees more final neighbours); false evaluates each lane's entry in place. The
// queue pays on large rounds; on small ones a warp left holding queued entries at the end
// of a round keeps the others waiting at the barrier.
//
// MB is the number of resident CTAs per SM the register budget is sized for (4: 64
// registers a thread, 3: 80, 2: 128); the launch's ctas_per_sm selects it. Fewer resident
// warps with fewer spills pay on large launches, where every SM has work each round.
template <int ND, bool QUEUE, int MB>
__global__ void __launch_bounds__(SOLVE_THREADS, MB) coarse_rounds_kernel(SolveArgs a) {
  const int lane = threadIdx.x & 31;
  __shared__ unsigned long long wq[SOLVE_THREADS / 32][QUEUE ? 64 : 1];  // per-warp queue of entries to evaluate
  __shared__ unsigned long long wv[SOLVE_THREADS / 32][8];  // per-warp visit counts by outcome
  const unsigned long long N = a.rs.stride;  // node id = problem * stride + node
  const unsigned N32 = (unsigned)N;            // node ids are 32-bit: so is the stride
  unsigned long long* wvis = wv[threadIdx.x >> 5];
  clear_visits(wvis, lane);
#ifdef EIK_PHASE
  VisitCount vk[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // lane cycles at 7..10: gates, node path, rule, relist filter
#else
  VisitCount* vk = nullptr;
#endif
  int r = 0;
  for (; r < a.rs.max_rounds; r++) {
    const int b3 = r % 3, nb3 = (r + 1) % 3;
    const unsigned int n = *(volatile unsigned int*)(a.rs.cnt + b3);
    if (n == 0) break;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(a.activations, (unsigned long long)n);  // list entries
    const unsigned long long* L = a.rs.list[r & 1];
    unsigned long long* Lnext = a.rs.list[(r + 1) & 1];
    const unsigned long long* nm = a.rs.nextmin + (size_t)b3 * a.nprob;
    unsigned long long* nmn = a.rs.nextmin + (size_t)nb3 * a.nprob;
    const double* thr_prev = a.rs.thr + (size_t)((r + 1) & 1) * a.nprob;  // thresholds of round r-1
    double* thr_cur = a.rs.thr + (size_t)(r & 1) * a.nprob;
    if (blockIdx.x == 0)
      for (int p = threadIdx.x; p < a.nprob; p += blockDim.x)
        thr_cur[p] = fmax(__ldcg(thr_prev + p), __longlong_as_double((long long)ld_volatile(nm + p)) + a.probs[p].delta);
    if constexpr (QUEUE) {
      // Visits whose front still stands (nothing they read has changed) are settled when
      // taken; the others wait in a per-warp queue in shared memory and are evaluated 32 at a
      // time, so that a warp's lanes run the long evaluation path together.
      unsigned long long* q = wq[threadIdx.x >> 5];
      int qn = 0;  // queued entries (warp-uniform)
      bool more = true;
      while (more || qn > 0) {
        unsigned dirs = visit_code(VISIT_NONE);
        double front = EIK_INF;
        int prob = 0;
        long long l = 0;
        if (more && qn < 32) {
          PH_T(tg);
          unsigned int base = 0;
          if (lane == 0) base = atomicAdd(a.rs.grab + b3, 32u);
          base = __shfl_sync(0xffffffffu, base, 0);
          PH_ADD(0, tg);
          if (base >= n) {
            more = false;
            continue;
          }
          PH_T(tl);
          PH_CNT(10);
          const unsigned int idx = base + lane;
          bool queue = false;
          unsigned long long e = 0;
          if (idx < n) {
            e = __ldcg(L + idx);
            const unsigned int gid = (unsigned int)(e >> 32);
            const double ef = (double)__uint_as_float((unsigned int)e);
            prob = (int)(gid / N32);
            l = (long long)(gid - (unsigned long long)prob * N);
            // threshold inputs and the dirty flag in one batch
            const double tp = __ldcg(thr_prev + prob);
            const unsigned long long nmv = ld_volatile(nm + prob);
            const double del = a.probs[prob].delta;
            const uint8_t dq = __ldcg(a.rs.dirty + gid);
            const double T = fmax(tp, __longlong_as_double((long long)nmv) + del);
            if (ef > T && ef < EIK_INF && !dq) {
              front = ef;
              dirs = (1u << DIR_SELF) | visit_code(VISIT_STANDS);
            } else {
              queue = true;
            }
          }
          const unsigned qm = __ballot_sync(0xffffffffu, queue);
          if (queue) q[qn + __popc(qm & ((1u << lane) - 1u))] = e;
          qn += __popc(qm);
          __syncwarp();
          PH_ADD(9, tl);
        } else {
          PH_T(tp);
          PH_CNT(11);
          const int k = qn < 32 ? qn : 32;
          if (lane < k) {
            const unsigned long long e = q[qn - k + lane];
            const unsigned int gid = (unsigned int)(e >> 32);
            prob = (int)(gid / N32);
            l = (long long)(gid - (unsigned long long)prob * N);
            const CoarseProblem& P = a.probs[prob];
            const double T = fmax(__ldcg(thr_prev + prob), __longlong_as_double((long long)ld_volatile(nm + prob)) + P.delta);
            const unsigned long long gb = (unsigned long long)prob * N;
            dirs = (ND == 3) ? process_node<3>(GlobalNodes{a, P, gb}, P, l, T, r, &front, vk)
                             : process_node<2>(GlobalNodes{a, P, gb}, P, l, T, r, &front, vk);
          }
          qn -= k;
          __syncwarp();
          PH_ADD(1, tp);
        }
        count_visits(wvis, dirs, lane);
        PH_T(ts);
        // list the next round's nodes once each (per-node round stamps)
        const CoarseProblem& P = a.probs[prob];
        const unsigned long long gbase = (unsigned long long)prob * N;
        unsigned keep = 0;
        for (int k = 0; k <= DIR_SELF; k++) {
          if (!((dirs >> k) & 1u)) continue;
          const long long nl = dir_lin(P.g, l, k);
          if (atomicExch(a.rs.stamp + gbase + nl, r + 1) != r + 1) keep |= 1u << k;
        }
        __syncwarp();
        PH_ADD(2, ts);
        PH_T(ta);
        // warp-aggregated append: one atomic per 32 nodes
        const int cntl = __popc(keep);
        int incl = cntl;
  #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        unsigned int wbase = 0;
        if (lane == 0 && total) wbase = atomicAdd(a.rs.cnt + nb3, (unsigned int)total);
        wbase = __shfl_sync(0xffffffffu, wbase, 0) + (unsigned int)(incl - cntl);
        for (int k = 0; k <= DIR_SELF; k++) {
          if (!((keep >> k) & 1u)) continue;
          const long long nl = dir_lin(P.g, l, k);
          Lnext[wbase++] = list_entry((unsigned int)(gbase + nl), front);
        }
        {
          // one update per problem and warp: the lanes of a problem agree on their smallest front
          const double fv = keep ? front : EIK_INF;
          const unsigned grp = __match_any_sync(0xffffffffu, prob);
          double gmin = fv;
          for (unsigned m = grp; m; m &= m - 1) {
            const int src = __ffs(m) - 1;
            gmin = fmin(gmin, __shfl_sync(grp, fv, src));
          }
          if (lane == __ffs(grp) - 1) atomic_min_pos(nmn + prob, gmin);
        }
        __syncwarp();
        PH_ADD(3, ta);
      }
    } else {
      // every lane evaluates its own entry in place
      for (;;) {
        PH_T(tg);
        unsigned int base = 0;
        if (lane == 0) base = atomicAdd(a.rs.grab + b3, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        PH_ADD(0, tg);
        if (base >= n) break;
        PH_T(tp);
        const unsigned int idx = base + lane;
        unsigned dirs = visit_code(VISIT_NONE);
        double front = EIK_INF;
        int prob = 0;
        long long l = 0;
        if (idx < n) {
          const unsigned long long e = __ldcg(L + idx);
          const unsigned int gid = (unsigned int)(e >> 32);
          const double ef = (double)__uint_as_float((unsigned int)e);
          prob = (int)(gid / N32);
          l = (long long)(gid - (unsigned long long)prob * N);
          const CoarseProblem& P = a.probs[prob];
          // window of one round width above the smallest pending front, never moving back
          // (its inputs and the dirty flag in one batch)
          const double tp = __ldcg(thr_prev + prob);
          const unsigned long long nmv = ld_volatile(nm + prob);
          const double del = P.delta;
          const uint8_t dq = __ldcg(a.rs.dirty + gid);
          const double T = fmax(tp, __longlong_as_double((long long)nmv) + del);
          const unsigned long long gb = (unsigned long long)prob * N;
          if (ef > T && ef < EIK_INF && !dq) {
            // still waiting and nothing it reads has changed: its front stands
            front = ef;
            dirs = (1u << DIR_SELF) | visit_code(VISIT_STANDS);
          } else {
            dirs = (ND == 3) ? process_node<3>(GlobalNodes{a, P, gb}, P, l, T, r, &front, vk)
                             : process_node<2>(GlobalNodes{a, P, gb}, P, l, T, r, &front, vk);
          }
        }
        __syncwarp();
        PH_ADD(1, tp);
        count_visits(wvis, dirs, lane);
        PH_T(ts);
        // list the next round's nodes once each (per-node round stamps)
        const CoarseProblem& P = a.probs[prob];
        const unsigned long long gbase = (unsigned long long)prob * N;
        unsigned keep = 0;
        for (int k = 0; k <= DIR_SELF; k++) {
          if (!((dirs >> k) & 1u)) continue;
          const long long nl = dir_lin(P.g, l, k);
          if (atomicExch(a.rs.stamp + gbase + nl, r + 1) != r + 1) keep |= 1u << k;
        }
        __syncwarp();
        PH_ADD(2, ts);
        PH_T(ta);
        // warp-aggregated append: one atomic per 32 nodes
        const int cntl = __popc(keep);
        int incl = cntl;
  #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        unsigned int wbase = 0;
        if (lane == 0 && total) wbase = atomicAdd(a.rs.cnt + nb3, (unsigned int)total);
        wbase = __shfl_sync(0xffffffffu, wbase, 0) + (unsigned int)(incl - cntl);
        for (int k = 0; k <= DIR_SELF; k++) {
          if (!((keep >> k) & 1u)) continue;
          const long long nl = dir_lin(P.g, l, k);
          Lnext[wbase++] = list_entry((unsigned int)(gbase + nl), front);
        }
        {
          // one update per problem and warp: the lanes of a problem agree on their smallest front
          const double fv = keep ? front : EIK_INF;
          const unsigned grp = __match_any_sync(0xffffffffu, prob);
          double gmin = fv;
          for (unsigned m = grp; m; m &= m - 1) {
            const int src = __ffs(m) - 1;
            gmin = fmin(gmin, __shfl_sync(grp, fv, src));
          }
          if (lane == __ffs(grp) - 1) atomic_min_pos(nmn + prob, gmin);
        }
        __syncwarp();
        PH_ADD(3, ta);
      }
    }
    // buffers of round r+2 (last used in round r-1)
    if (blockIdx.x == 0) {
      const int c3 = (r + 2) % 3;
      if (threadIdx.x == 0) {
        a.rs.cnt[c3] = 0;
        a.rs.grab[c3] = 0;
      }
      for (int p = threadIdx.x; p < a.nprob; p += blockDim.x)
        a.rs.nextmin[(size_t)c3 * a.nprob + p] = (unsigned long long)__double_as_longlong(EIK_INF);
    }
    PH_T(tb);
    if (!grid_barrier(a)) break;
    PH_ADD(4, tb);
  }
  flush_visits(wvis, a.rs.visits, a.node_evals, lane);
#ifdef EIK_PHASE
  for (int k = 7; k < 11; k++) atomicAdd(&eik_phase[k - 2], vk[k]);  // per lane
#endif
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *a.rs.rounds = r;
    if (r >= a.rs.max_rounds) {
      atomicOr(a.err, ERRB_NOT_CONVERGED);
      atomicExch(a.abort_flag, 1);
    }
  }
}

// ------------------------------------------------------------------ picks --
// bilinear_interp / trilinear_interp value mode (eikforward2D.jl:17-87,
// eikforward3D.jl:17-140), corner (i+1,j,k+1) weighted xd*(1-yd)*(1-zd) as the reference.
__global__ void picks_kernel(GridDesc g, const double* t, long long N, int nsrc, const long long* recoff,
                             const double* rec, double* picks) {
  const long long ntot = recoff[nsrc];
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < ntot;
       r += (long long)gridDim.x * blockDim.x) {
    int s = 0;
    while (recoff[s + 1] <= r) s++;
    const double* tt = t + (size_t)s * N;
    const double* p = rec + r * g.nd;
    if (g.nd == 2) {
      const double xh = (p[0] - g.co[0]) / g.spac[0];
      const double yh = (p[1] - g.co[1]) / g.spac[1];
      long long i = (long long)floor(xh + 1), j = (long long)floor(yh + 1);
      if (i == g.n[0]) i -= 1;
      else if (i > g.n[0]) i -= 2;
      if (j == g.n[1]) j -= 1;
      else if (j > g.n[1]) j -= 2;
      const double xd = xh - (double)(i - 1), yd = yh - (double)(j - 1);
      const long long a = lin3(g, (int)i - 1, (int)j - 1, 0);
      const double f00 = tt[a], f10 = tt[a + 1], f01 = tt[a + g.n[0]], f11 = tt[a + g.n[0] + 1];
      picks[r] = f00 * (1.0 - xd) * (1.0 - yd) + f10 * (1.0 - yd) * xd + f01 * (1.0 - xd) * yd + f11 * xd * yd;
    } else {
      const double dx = g.spac[0], dy = g.spac[1], dz = g.spac[2];
      const double xh = (p[0] - g.co[0]) / dx, yh = (p[1] - g.co[1]) / dy, zh = (p[2] - g.co[2]) / dz;
      const double x = p[0] - g.co[0], y = p[1] - g.co[1], z = p[2] - g.co[2];
      long long i = (long long)floor(xh + 1), j = (long long)floor(yh + 1), k = (long long)floor(zh + 1);
      if (i == g.n[0]) i -= 1;
      else if (i > g.n[0]) i -= 2;
      if (j == g.n[1]) j -= 1;
      else if (j > g.n[1]) j -= 2;
      if (k == g.n[2]) k -= 1;
      else if (k > g.n[2]) k -= 2;
      const double x0 = (double)(i - 1) * dx, y0 = (double)(j - 1) * dy, z0 = (double)(k - 1) * dz;
      const double x1 = (double)i * dx, y1 = (double)j * dy, z1 = (double)k * dz;
      const double xd = (x - x0) / (x1 - x0), yd = (y - y0) / (y1 - y0), zd = (z - z0) / (z1 - z0);
      auto T = [&](int a, int b, int c) { return tt[lin3(g, (int)i - 1 + a, (int)j - 1 + b, (int)k - 1 + c)]; };
      picks[r] = T(0, 0, 0) * (1 - xd) * (1 - yd) * (1 - zd) + T(1, 0, 0) * xd * (1 - yd) * (1 - zd) +
                 T(0, 1, 0) * (1 - xd) * yd * (1 - zd) + T(0, 0, 1) * (1 - xd) * (1 - yd) * zd +
                 T(1, 1, 0) * xd * yd * (1 - zd) + T(0, 1, 1) * (1 - xd) * yd * zd +
                 T(1, 0, 1) * xd * (1 - yd) * (1 - zd) + T(1, 1, 1) * xd * yd * zd;
    }
  }
}

// ------------------------------------------------------------------ launchers --
void launch_coarse_init(const CoarseProblem* hprobs, const CoarseProblem* dprobs, int nprob,
                        const ForwardBatch& fb, const SolveArgs& sa, cudaStream_t st) {
  (void)hprobs;
  // every problem's first stride nodes: its grid, and the padding up to the call's largest grid
  coarse_init_kernel<<<1184, 256, 0, st>>>(dprobs, nprob, (long long)sa.rs.stride);
  rounds_init_kernel<<<296, 256, 0, st>>>(sa);
  launch_rounds_seed(sa, fb.seed_lin, fb.seed_tt, fb.out, false, fb.seedcap, st);
}

void launch_rounds_init(const SolveArgs& sa, cudaStream_t st) { rounds_init_kernel<<<296, 256, 0, st>>>(sa); }

void launch_rounds_seed(const SolveArgs& sa, const int32_t* seed_lin, const double* seed_tt, const SrcOut* out,
                        bool fine_corners, int seedcap, cudaStream_t st) {
  if (sa.nd == 3) seed_kernel<3><<<sa.nprob, 128, 0, st>>>(sa, seed_lin, seed_tt, out, fine_corners ? 1 : 0, seedcap);
  else seed_kernel<2><<<sa.nprob, 128, 0, st>>>(sa, seed_lin, seed_tt, out, fine_corners ? 1 : 0, seedcap);
}

template <int ND, bool QUEUE, int MB>
static cudaError_t launch_solve_mb(const SolveArgs& sa, int nsm, int ctas_per_sm, cudaStream_t st) {
  const size_t sm = 0;
  int per = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, coarse_rounds_kernel<ND, QUEUE, MB>, SOLVE_THREADS, sm);
  if (ctas_per_sm > 0 && ctas_per_sm < per) per = ctas_per_sm;
  per = per < 1 ? 1 : per;
  SolveArgs args = sa;
  void* kargs[] = {&args};
  // cooperative: every CTA is resident, so the grid barrier between rounds cannot deadlock
  return cudaLaunchCooperativeKernel((const void*)coarse_rounds_kernel<ND, QUEUE, MB>, dim3(nsm * per),
                                     dim3(SOLVE_THREADS), kargs, sm, st);
}

template <int ND, bool QUEUE>
static cudaError_t launch_solve_nd(const SolveArgs& sa, int nsm, int ctas_per_sm, cudaStream_t st) {
  // 2 and 3 resident CTAs per SM take the register budget of that residency; else 4
  if (ctas_per_sm == 2) return launch_solve_mb<ND, QUEUE, 2>(sa, nsm, ctas_per_sm, st);
  if (ctas_per_sm == 3) return launch_solve_mb<ND, QUEUE, 3>(sa, nsm, ctas_per_sm, st);
  return launch_solve_mb<ND, QUEUE, 4>(sa, nsm, ctas_per_sm, st);
}

cudaError_t launch_coarse_solve(const SolveArgs& sa, int nsm, int ctas_per_sm, int queue, cudaStream_t st) {
  // automatic choice: the queue from 2^27 node-sources per launch (256^3 x 8 sources) up
  const bool q = queue > 0 || (queue < 0 && (unsigned long long)sa.nprob * sa.rs.stride >= (1ull << 27));
  if (sa.nd == 3)
    return q ? launch_solve_nd<3, true>(sa, nsm, ctas_per_sm, st) : launch_solve_nd<3, false>(sa, nsm, ctas_per_sm, st);
  return q ? launch_solve_nd<2, true>(sa, nsm, ctas_per_sm, st) : launch_solve_nd<2, false>(sa, nsm, ctas_per_sm, st);
}

void launch_picks(const GridDesc& g, const double* t, long long N, int nsrc, const long long* recoff,
                  const double* rec, double* picks, cudaStream_t st) {
  picks_kernel<<<64, 128, 0, st>>>(g, t, N, nsrc, recoff, rec, picks);
}

}  // namespace eik
