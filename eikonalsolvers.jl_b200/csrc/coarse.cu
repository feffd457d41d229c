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
// tuning builds only: clock cycles per phase summed over warps (lane 0)
__device__ unsigned long long eik_phase[9];
extern "C" int eik_phase_read(unsigned long long* out) {
  return (int)cudaMemcpyFromSymbol(out, eik_phase, sizeof(unsigned long long) * 9);
}
#define PH_T(v) const long long v = clock64()
#define PH_ADD(k, t0) if ((threadIdx.x & 31) == 0) atomicAdd(&eik_phase[k], (unsigned long long)(clock64() - (t0)))
#define PL_T(v) const long long v = clock64()
#define PL_ADD(k, t0) vk[k] += (unsigned long long)(clock64() - (t0))
#else
#define PH_T(v)
#define PH_ADD(k, t0)
#define PL_T(v)
#define PL_ADD(k, t0)
#endif
// ------------------------------------------------------------------ node solve --
// Key of node l of problem P: (L, d) of a special node, (t, 0) otherwise.
__device__ __forceinline__ void node_key(const CoarseProblem& P, long long l, double t, uint8_t cb, double* L, int* d) {
  if (cb & CODE_SRC_BIT) {
    *L = __ldcg(P.kL + l);
    *d = __ldcg(P.kd + l);
  } else {
    *L = t;
    *d = 0;
  }
}

// Neighbour directions of a node: k = 4*axis + {0: -2, 1: -1, 2: +1, 3: +2}; bit 12 = itself.
constexpr int DIR_SELF = 12;
__device__ __forceinline__ int dir_off(int k) { return (k & 3) < 2 ? (k & 3) - 2 : (k & 3) - 1; }

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

// One listed node: gate, evaluate, write back. Returns the directions of the nodes to list
// for the next round (bit DIR_SELF: this node again) and, in *front, the traveltime that
// bounds their next evaluation from below.
//
// The visit is a chain of dependent L2 round trips, which sets the length of a round when
// fronts are small. Each stage therefore issues all of its loads before it uses any: the
// node's own state, its immediate neighbours, their codes with the distance-2 nodes, and
// the relist filter's reads per axis. Reordering these reads does not change what they
// can observe (see the notes at each stage).
template <int ND>
__device__ unsigned process_node(const SolveArgs& a, const CoarseProblem& P, unsigned long long gbase, long long l,
                                 double T, int r, double* front, unsigned long long* evals,
                                 unsigned long long* vk) {
  PL_T(tq0);
  const GridDesc& g = P.g;
  const int c[3] = {(int)(l % g.n[0]), (int)((l / g.n[0]) % g.n[1]), (int)(l / ((long long)g.n[0] * g.n[1]))};
  // The node's own state in one batch. Only this visit writes its t, code and key during
  // the round (a node is listed once per round), so their order of reading is free.
  const uint8_t dirty0 = __ldcg(a.rs.dirty + gbase + l);
  const double tv = __ldcg(a.rs.tent + gbase + l);
  const uint8_t cb = __ldcg(P.code + l);
  const double told = __ldcg(P.t + l);
  // last evaluated value, still valid while nothing the node reads has changed
  if (!dirty0 && tv > T && tv < EIK_INF) {
    *front = tv;
    vk[0]++;
    return 1u << DIR_SELF;
  }
  double Lold;
  int dold;
  node_key(P, l, told, cb, &Lold, &dold);
  if ((cb & CODE_SRC_BIT) && Lold == -EIK_INF) {  // source points are fixed
    vk[1]++;
    return 0;
  }
  // from here the node reads its neighbours' current values: a change after this point
  // marks it dirty again (writers store the value, fence, then the flag)
  a.rs.dirty[gbase + l] = 0;
  __threadfence();
  // immediate neighbours (one batch with the slowness): potential = smallest traveltime
  double t1[ND][2];
  long long l1[ND][2];
#pragma unroll
  for (int ax = 0; ax < ND; ax++)
#pragma unroll
    for (int s = 0; s < 2; s++) {
      const int sh = s == 0 ? 1 : -1;
      l1[ax][s] = -1;
      if (c[ax] + sh < 0 || c[ax] + sh >= g.n[ax]) continue;
      int p[3] = {c[0], c[1], c[2]};
      p[ax] += sh;
      l1[ax][s] = lin3(g, p[0], p[1], p[2]);
    }
#pragma unroll
  for (int ax = 0; ax < ND; ax++)
#pragma unroll
    for (int s = 0; s < 2; s++) t1[ax][s] = l1[ax][s] >= 0 ? __ldcg(P.t + l1[ax][s]) : EIK_INF;
  const double slow = __ldg(P.slow + l);
  double pot = EIK_INF;
#pragma unroll
  for (int ax = 0; ax < ND; ax++)
#pragma unroll
    for (int s = 0; s < 2; s++) pot = fmin(pot, t1[ax][s]);
  if (!(pot < EIK_INF)) {  // nothing reached around it yet
    a.rs.tent[gbase + l] = EIK_INF;
    vk[2]++;
    return 0;
  }
  PL_ADD(7, tq0);
  PL_T(tq1);
  Nbhd nb;
  nb_clear(nb);
  node_dh(g, c[0], nb.dh);
  nb.slow = slow;
  nb.c1u = P.c1u;
  nb.c2u = P.c2u;
  // Lower bound of the node's value: every term of the local update is at least pot and
  // the quadratic adds at least (2/3) h s / sqrt(ND) (2nd-order coefficients 9/(4h^2)).
  // Until the round threshold reaches it the node cannot be final: no evaluation yet.
  double hmin = nb.dh[0];
#pragma unroll
  for (int ax = 1; ax < ND; ax++) hmin = fmin(hmin, nb.dh[ax]);
  const double lb = pot + 0.999 * (2.0 / 3.0) * hmin * nb.slow * (ND == 3 ? 0.5773502691896258 : 0.7071067811865476);
  if (lb > T) {
    a.rs.tent[gbase + l] = lb;  // stands, like an evaluated value, while the node stays clean
    *front = lb;
    vk[3]++;
    return 1u << DIR_SELF;
  }
  // Codes of the immediate neighbours and the distance-2 nodes with their codes, one batch.
  // A neighbour's key is read after its traveltime here as in any order: the key changes
  // only together with the traveltime, in the neighbour's own visit.
  uint8_t cd1[ND][2], cd2[ND][2];
  double t2[ND][2];
  long long l2[ND][2];
#pragma unroll
  for (int ax = 0; ax < ND; ax++)
#pragma unroll
    for (int s = 0; s < 2; s++) {
      const int sh = s == 0 ? 1 : -1;
      l2[ax][s] = -1;
      if (l1[ax][s] < 0) continue;
      int p[3] = {c[0], c[1], c[2]};
      p[ax] += sh;
      bool ok = true;  // isonbord on the first neighbour, in every coordinate (eikutils.jl:129-162)
#pragma unroll
      for (int dd = 0; dd < ND; dd++)
        if (p[dd] < 1 || p[dd] > g.n[dd] - 2) ok = false;
      if (ok) {
        p[ax] += sh;
        l2[ax][s] = lin3(g, p[0], p[1], p[2]);
      }
    }
#pragma unroll
  for (int ax = 0; ax < ND; ax++)
#pragma unroll
    for (int s = 0; s < 2; s++) {
      cd1[ax][s] = l1[ax][s] >= 0 ? __ldcg(P.code + l1[ax][s]) : (uint8_t)0;
      t2[ax][s] = l2[ax][s] >= 0 ? __ldcg(P.t + l2[ax][s]) : EIK_INF;
      cd2[ax][s] = l2[ax][s] >= 0 ? __ldcg(P.code + l2[ax][s]) : (uint8_t)0;
    }
#pragma unroll
  for (int ax = 0; ax < ND; ax++)
#pragma unroll
    for (int s = 0; s < 2; s++) {
      if (l1[ax][s] < 0) continue;
      double L;
      int d;
      node_key(P, l1[ax][s], t1[ax][s], cd1[ax][s], &L, &d);
      nb_put1(nb, ax, s, t1[ax][s], L, d);
      if (l2[ax][s] >= 0) {
        node_key(P, l2[ax][s], t2[ax][s], cd2[ax][s], &L, &d);
        nb_put2(nb, ax, s, t2[ax][s], L, d);
      }
    }
  int8_t cd[3] = {0, 0, 0};
  Key nk;
  bool neg = false;
  PL_T(tq2);
  const double nv = prefix_rule<ND>(nb, cd, &nk, &neg);
  PL_ADD(9, tq2);
  (*evals)++;
  const uint8_t nc = pack_codes(cd, ND);
  const bool same_t = (nv == told) || (isinf(nv) && isinf(told));
  const bool tkchange = !(same_t && key_eq(nk, Key{Lold, dold, told}));
  const bool special = !(nk.L == nv && nk.d == 0);
  const uint8_t ncb = (uint8_t)(nc | (special ? CODE_SRC_BIT : 0));
  a.rs.tent[gbase + l] = nv;
  if (!tkchange) {
    if (ncb != cb) P.code[l] = ncb;
    vk[5]++;
    return 0;
  }
  if (nv > T) {  // not final yet: keep the old value and come back when the front is there
    *front = nv;
    vk[4]++;
    return 1u << DIR_SELF;
  }
  P.t[l] = nv;
  P.code[l] = ncb;
  if (special) {
    P.kL[l] = nk.L;
    P.kd[l] = (uint8_t)nk.d;
  }
  __threadfence();
  PL_T(tq3);
  // The nodes whose stencil reads this one (+-1, +-2 along each axis) are evaluated again,
  // except those whose stored key is at most both the old and the new key of this node:
  // the order rule of such a node never accepts this one, nor is its termination test
  // affected, so its value cannot change. A node listed for the current round may be
  // under evaluation right now and is always listed again. The node two steps away reads
  // this one only through the node in between, which must be reached first; when it is,
  // its own change lists that node.
  //
  // Reads per axis in one batch, all after the fence above: the in-between node's
  // traveltime (the +-1 node's, read fresh), and the stamp, traveltime and code of each
  // candidate. A candidate whose stamp is below r is in no list of this round, so nothing
  // writes its traveltime, code or key while this round runs: reading them before or after
  // the stamp observes the same values.
  const Key kold = Key{Lold, dold, told};
  unsigned dirs = 0;
#pragma unroll
  for (int ax = 0; ax < ND; ax++) {
    long long lj[4];
    double tj[4];
    uint8_t cj[4];
    int32_t sj[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int off = dir_off(j);
      lj[j] = -1;
      if (c[ax] + off < 0 || c[ax] + off >= g.n[ax]) continue;
      int p[3] = {c[0], c[1], c[2]};
      p[ax] += off;
      lj[j] = lin3(g, p[0], p[1], p[2]);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      tj[j] = lj[j] >= 0 ? __ldcg(P.t + lj[j]) : EIK_INF;
      cj[j] = lj[j] >= 0 ? __ldcg(P.code + lj[j]) : (uint8_t)0;
      sj[j] = lj[j] >= 0 ? *(volatile const int32_t*)(a.rs.stamp + gbase + lj[j]) : 0;
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      if (lj[j] < 0) continue;
      // j = 0 (-2) reads this node through j = 1 (-1), j = 3 (+2) through j = 2 (+1)
      if (j == 0 && !(tj[1] < EIK_INF)) continue;
      if (j == 3 && !(tj[2] < EIK_INF)) continue;
      if (sj[j] < r) {
        double Lj;
        int dj;
        node_key(P, lj[j], tj[j], cj[j], &Lj, &dj);
        const Key kj = Key{Lj, dj, tj[j]};
        if (key_le(kj, kold) && key_le(kj, nk)) continue;
      }
      a.rs.dirty[gbase + lj[j]] = 1;
      dirs |= 1u << (4 * ax + j);
    }
  }
  *front = nv + P.incmin;  // no node reading this one can get a smaller value from it
  PL_ADD(10, tq3);
  PL_ADD(8, tq1);
  vk[6]++;
  return dirs;
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
  const unsigned long long N = a.rs.stride;  // node id = problem * stride + node
  unsigned long long evals = 0;
#ifdef EIK_PHASE
  unsigned long long vk[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // + lane cycles: gates, node path, rule, relist filter
#else
  unsigned long long vk[7] = {0, 0, 0, 0, 0, 0, 0};  // visit outcomes, see eik_stats.fwd_visits
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
        unsigned dirs = 0;
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
          const unsigned int idx = base + lane;
          bool queue = false;
          unsigned long long e = 0;
          if (idx < n) {
            e = __ldcg(L + idx);
            const unsigned int gid = (unsigned int)(e >> 32);
            const double ef = (double)__uint_as_float((unsigned int)e);
            prob = (int)(gid / N);
            l = (long long)(gid - (unsigned long long)prob * N);
            // threshold inputs and the dirty flag in one batch
            const double tp = __ldcg(thr_prev + prob);
            const unsigned long long nmv = ld_volatile(nm + prob);
            const double del = a.probs[prob].delta;
            const uint8_t dq = __ldcg(a.rs.dirty + gid);
            const double T = fmax(tp, __longlong_as_double((long long)nmv) + del);
            if (ef > T && ef < EIK_INF && !dq) {
              front = ef;
              dirs = 1u << DIR_SELF;
              vk[0]++;
            } else {
              queue = true;
            }
          }
          const unsigned qm = __ballot_sync(0xffffffffu, queue);
          if (queue) q[qn + __popc(qm & ((1u << lane) - 1u))] = e;
          qn += __popc(qm);
          __syncwarp();
        } else {
          PH_T(tp);
          const int k = qn < 32 ? qn : 32;
          if (lane < k) {
            const unsigned long long e = q[qn - k + lane];
            const unsigned int gid = (unsigned int)(e >> 32);
            prob = (int)(gid / N);
            l = (long long)(gid - (unsigned long long)prob * N);
            const CoarseProblem& P = a.probs[prob];
            const double T = fmax(__ldcg(thr_prev + prob), __longlong_as_double((long long)ld_volatile(nm + prob)) + P.delta);
            const unsigned long long gb = (unsigned long long)prob * N;
            dirs = (ND == 3) ? process_node<3>(a, P, gb, l, T, r, &front, &evals, vk)
                             : process_node<2>(a, P, gb, l, T, r, &front, &evals, vk);
          }
          qn -= k;
          __syncwarp();
          PH_ADD(1, tp);
        }
        PH_T(ts);
        // list the next round's nodes once each (per-node round stamps)
        const CoarseProblem& P = a.probs[prob];
        const int c[3] = {(int)(l % P.g.n[0]), (int)((l / P.g.n[0]) % P.g.n[1]),
                          (int)(l / ((long long)P.g.n[0] * P.g.n[1]))};
        const unsigned long long gbase = (unsigned long long)prob * N;
        unsigned keep = 0;
        for (int k = 0; k <= DIR_SELF; k++) {
          if (!((dirs >> k) & 1u)) continue;
          long long nl = l;
          if (k != DIR_SELF) {
            int p[3] = {c[0], c[1], c[2]};
            p[k >> 2] += dir_off(k);
            nl = lin3(P.g, p[0], p[1], p[2]);
          }
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
          long long nl = l;
          if (k != DIR_SELF) {
            int p[3] = {c[0], c[1], c[2]};
            p[k >> 2] += dir_off(k);
            nl = lin3(P.g, p[0], p[1], p[2]);
          }
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
        unsigned dirs = 0;
        double front = EIK_INF;
        int prob = 0;
        long long l = 0;
        if (idx < n) {
          const unsigned long long e = __ldcg(L + idx);
          const unsigned int gid = (unsigned int)(e >> 32);
          const double ef = (double)__uint_as_float((unsigned int)e);
          prob = (int)(gid / N);
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
            dirs = 1u << DIR_SELF;
            vk[0]++;
          } else {
            dirs = (ND == 3) ? process_node<3>(a, P, gb, l, T, r, &front, &evals, vk)
                             : process_node<2>(a, P, gb, l, T, r, &front, &evals, vk);
          }
        }
        __syncwarp();
        PH_ADD(1, tp);
        PH_T(ts);
        // list the next round's nodes once each (per-node round stamps)
        const CoarseProblem& P = a.probs[prob];
        const int c[3] = {(int)(l % P.g.n[0]), (int)((l / P.g.n[0]) % P.g.n[1]),
                          (int)(l / ((long long)P.g.n[0] * P.g.n[1]))};
        const unsigned long long gbase = (unsigned long long)prob * N;
        unsigned keep = 0;
        for (int k = 0; k <= DIR_SELF; k++) {
          if (!((dirs >> k) & 1u)) continue;
          long long nl = l;
          if (k != DIR_SELF) {
            int p[3] = {c[0], c[1], c[2]};
            p[k >> 2] += dir_off(k);
            nl = lin3(P.g, p[0], p[1], p[2]);
          }
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
          long long nl = l;
          if (k != DIR_SELF) {
            int p[3] = {c[0], c[1], c[2]};
            p[k >> 2] += dir_off(k);
            nl = lin3(P.g, p[0], p[1], p[2]);
          }
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
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) evals += __shfl_xor_sync(0xffffffffu, evals, o);
  if (lane == 0 && evals) atomicAdd(a.node_evals, evals);
#ifdef EIK_PHASE
  for (int k = 7; k < 11; k++) atomicAdd(&eik_phase[k - 2], vk[k]);  // per lane
#endif
#pragma unroll
  for (int k = 0; k < 7; k++) {
    unsigned long long v = vk[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0 && v) atomicAdd(a.rs.visits + k, v);
  }
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
