// One node visit of the forward round solver (coarse.cu, cluster.cu): the FMM order rule
// of stencil.cuh evaluated on a node of one problem, with the gates, the write-back and the
// relisting filter around it. The state it reads and writes is reached through an accessor
// (M), so that the same visit runs on state in global memory and on state in a cluster's
// distributed shared memory.
#pragma once

#include "kernels.cuh"

namespace eik {

#ifdef EIK_PHASE
// tuning builds sum the clock cycles of the visit's stages per lane (vk[7..10])
#define PL_T(v) const long long v = clock64()
#define PL_ADD(k, t0) vk[k] += (unsigned long long)(clock64() - (t0))
#else
#define PL_T(v)
#define PL_ADD(k, t0)
#endif
typedef unsigned long long VisitCount;  // the per-lane cycle sums (vk) of tuning builds

// Visit outcomes, in the order of eik_stats.fwd_visits. process_node returns the outcome in
// bits VISIT_SHIFT.. of its result, above the direction bits; VISIT_NONE marks a lane that
// visited nothing in a step.
constexpr int VISIT_SHIFT = 16;
enum : unsigned {
  VISIT_STANDS = 0,  // value cached above the front, nothing it reads changed
  VISIT_SOURCE,      // source point (fixed)
  VISIT_UNREACHED,   // no neighbour reached yet
  VISIT_BOUND,       // lower bound above the front
  VISIT_WAIT,        // evaluated, above the front
  VISIT_SAME,        // evaluated, value and key unchanged
  VISIT_CHANGED,     // evaluated and accepted
  VISIT_NONE
};
__device__ __forceinline__ unsigned visit_code(unsigned v) { return v << VISIT_SHIFT; }

// Adds one step's visit outcomes of a (converged) warp to the warp's counters in shared
// memory, w[0..6]: three ballots split the lanes by outcome. Counting in shared memory keeps
// seven per-lane counters out of the registers of the visit.
__device__ __forceinline__ void count_visits(unsigned long long* w, unsigned res, int lane) {
  const unsigned oc = (res >> VISIT_SHIFT) & 7u;
  const unsigned b0 = __ballot_sync(0xffffffffu, oc & 1u), b1 = __ballot_sync(0xffffffffu, oc & 2u),
                 b2 = __ballot_sync(0xffffffffu, oc & 4u);
  if (lane < 7) {
    const unsigned mk = ((lane & 1) ? b0 : ~b0) & ((lane & 2) ? b1 : ~b1) & ((lane & 4) ? b2 : ~b2);
    w[lane] += (unsigned long long)__popc(mk);
  }
}
__device__ __forceinline__ void clear_visits(unsigned long long* w, int lane) {
  if (lane < 8) w[lane] = 0;
  __syncwarp();
}
// Adds a warp's counters to the solve's: visits by outcome, and the evaluations of the order
// rule (the outcomes that follow one: wait, same, changed).
__device__ __forceinline__ void flush_visits(const unsigned long long* w, unsigned long long* visits,
                                             unsigned long long* evals, int lane) {
  __syncwarp();
  if (lane < 7 && w[lane]) atomicAdd(visits + lane, w[lane]);
  if (lane == 0) {
    const unsigned long long ev = w[VISIT_WAIT] + w[VISIT_SAME] + w[VISIT_CHANGED];
    if (ev) atomicAdd(evals, ev);
  }
}

// ------------------------------------------------------------------ node solve --
// Key of node l of problem P: (L, d) of a special node, (t, 0) otherwise. A special key counts
// only beside a reached traveltime. Every special node has one (a source point's or an
// accepted value), so this changes nothing a consistent read sees; but a visit's loads of a
// neighbour changed in the same round are unordered, and one that sees the new code beside
// the old, unreached traveltime must not take a key level that belongs to neither (it made
// NaN traveltimes and a wrong fixed point in a host emulation of such reads).
__device__ __forceinline__ void node_key(const CoarseProblem& P, long long l, double t, uint8_t cb, double* L, int* d) {
  if ((cb & CODE_SRC_BIT) && t < EIK_INF) {
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
// Linear index of the node in direction k (or DIR_SELF) of node l, which the direction must
// keep in the grid: the grid is column-major (lin3), so a step along an axis adds that axis's
// stride. Arithmetic only: an array indexed by the loop's axis would live in local memory.
// Grid coordinates of node l. A problem has fewer than 2^32 nodes (a launch numbers its
// node-sources in 32 bits), so 32-bit division is exact and far cheaper than 64-bit.
__device__ __forceinline__ void node_coords(const GridDesc& g, long long l, int* c) {
  const unsigned ul = (unsigned)l, n0 = (unsigned)g.n[0], n1 = (unsigned)g.n[1];
  const unsigned q = ul / n0;
  c[0] = (int)(ul - q * n0);
  c[1] = (int)(q % n1);
  c[2] = (int)(q / n1);
}
__device__ __forceinline__ long long dir_lin(const GridDesc& g, long long l, int k) {
  if (k == DIR_SELF) return l;
  const int ax = k >> 2;
  const long long st = ax == 0 ? 1LL : (ax == 1 ? (long long)g.n[0] : (long long)g.n[0] * g.n[1]);
  return l + dir_off(k) * st;
}

// The round-solver state of problem P in global memory: node l at l (problem arrays) and at
// gb + l (round-solver arrays, numbered over the problems of a launch).
struct GlobalNodes {
  const SolveArgs& a;
  const CoarseProblem& P;
  unsigned long long gb;
  __device__ __forceinline__ uint8_t dirty(long long l) const { return __ldcg(a.rs.dirty + gb + l); }
  __device__ __forceinline__ void set_dirty(long long l, uint8_t v) const { a.rs.dirty[gb + l] = v; }
  __device__ __forceinline__ double tent(long long l) const { return __ldcg(a.rs.tent + gb + l); }
  __device__ __forceinline__ void set_tent(long long l, double v) const { a.rs.tent[gb + l] = v; }
  __device__ __forceinline__ uint8_t code(long long l) const { return __ldcg(P.code + l); }
  __device__ __forceinline__ void set_code(long long l, uint8_t v) const { P.code[l] = v; }
  __device__ __forceinline__ double t(long long l) const { return __ldcg(P.t + l); }
  __device__ __forceinline__ void set_t(long long l, double v) const { P.t[l] = v; }
  __device__ __forceinline__ int32_t stamp(long long l) const {
    return *(volatile const int32_t*)(a.rs.stamp + gb + l);
  }
  __device__ __forceinline__ void fence() const { __threadfence(); }
};

// The order rule on a neighbourhood with special keys (source points, non-causal
// acceptances), from the full keys of the immediate and distance-2 neighbours. Kept out of
// line because it is rare; its inputs and outputs go by value, so that no array of the visit
// has its address taken (which would keep it in local memory on every visit).
struct RuleIn {
  long long l1[3][2], l2[3][2];  // neighbour indices, < 0 where there is no such node
  double t1[3][2], t2[3][2];
  uint8_t cd1[3][2], cd2[3][2];
  double dh[3];
  double slow;
};
struct RuleOut {
  double v;
  Key key;
  int8_t cd[3];
  bool neg;
};
template <int ND>
__device__ __noinline__ RuleOut rule_full(const CoarseProblem& P, const RuleIn in) {
  Nbhd nb;
  nb_clear(nb);
  for (int ax = 0; ax < 3; ax++) nb.dh[ax] = in.dh[ax];
  nb.slow = in.slow;
  nb.c1u = P.c1u;
  nb.c2u = P.c2u;
  for (int ax = 0; ax < ND; ax++)
    for (int s = 0; s < 2; s++) {
      if (in.l1[ax][s] < 0) continue;
      double L;
      int d;
      node_key(P, in.l1[ax][s], in.t1[ax][s], in.cd1[ax][s], &L, &d);
      nb_put1(nb, ax, s, in.t1[ax][s], L, d);
      if (in.l2[ax][s] >= 0) {
        node_key(P, in.l2[ax][s], in.t2[ax][s], in.cd2[ax][s], &L, &d);
        nb_put2(nb, ax, s, in.t2[ax][s], L, d);
      }
    }
  RuleOut o;
  o.neg = false;
  o.v = prefix_rule<ND>(nb, o.cd, &o.key, &o.neg);
  return o;
}

// One listed node: gate, evaluate, write back. Returns the directions of the nodes to list
// for the next round (bit DIR_SELF: this node again) with the visit's outcome
// (visit_code) above them and, in *front, the traveltime that
// bounds their next evaluation from below. M holds the problem's round-solver state (the
// node's traveltime, code, cached front, dirty flag and round stamp): global memory
// (GlobalNodes) or the distributed shared memory of a thread-block cluster; key levels and
// depths of special nodes and the slowness stay in global memory.
//
// The visit is a chain of dependent L2 round trips, which sets the length of a round when
// fronts are small. Each stage therefore issues all of its loads before it uses any: the
// node's own state, its immediate neighbours, their codes with the distance-2 nodes, and
// the relist filter's reads per axis. Reordering these reads does not change what they
// can observe (see the notes at each stage).
template <int ND, class M>
__device__ __forceinline__ unsigned process_node(const M& m, const CoarseProblem& P, long long l, double T, int r,
                                                 double* front, VisitCount* vk) {
  PL_T(tq0);
  const GridDesc& g = P.g;
  int c[3];
  node_coords(g, l, c);
  // The node's own state in one batch. Only this visit writes its t, code and key during
  // the round (a node is listed once per round), so their order of reading is free.
  const uint8_t dirty0 = m.dirty(l);
  const double tv = m.tent(l);
  const uint8_t cb = m.code(l);
  const double told = m.t(l);
  // last evaluated value, still valid while nothing the node reads has changed
  if (!dirty0 && tv > T && tv < EIK_INF) {
    *front = tv;
    return (1u << DIR_SELF) | visit_code(VISIT_STANDS);
  }
  double Lold;
  int dold;
  node_key(P, l, told, cb, &Lold, &dold);
  if ((cb & CODE_SRC_BIT) && Lold == -EIK_INF) {  // source points are fixed
    return visit_code(VISIT_SOURCE);
  }
  // from here the node reads its neighbours' current values: a change after this point
  // marks it dirty again (writers store the value, fence, then the flag)
  m.set_dirty(l, 0);
  m.fence();
  // immediate neighbours (one batch with the slowness): potential = smallest traveltime.
  // Indices are 32-bit (a problem has fewer than 2^32 nodes) with a presence bit per
  // neighbour (bit slot(ax, s)): half the registers of 64-bit indices with -1 for "none".
  const unsigned ul = (unsigned)l;
  const unsigned st1 = (unsigned)g.n[0], st2 = (unsigned)g.n[0] * (unsigned)g.n[1];
  double t1[ND][2];
  unsigned l1[ND][2];
  unsigned in1 = 0u;
#pragma unroll
  for (int ax = 0; ax < ND; ax++)
#pragma unroll
    for (int s = 0; s < 2; s++) {
      const int sh = s == 0 ? 1 : -1;
      const unsigned st = ax == 0 ? 1u : (ax == 1 ? st1 : st2);
      l1[ax][s] = s == 0 ? ul + st : ul - st;
      if (c[ax] + sh >= 0 && c[ax] + sh < g.n[ax]) in1 |= 1u << slot(ax, s);
    }
#pragma unroll
  for (int ax = 0; ax < ND; ax++)
#pragma unroll
    for (int s = 0; s < 2; s++) t1[ax][s] = ((in1 >> slot(ax, s)) & 1u) ? m.t(l1[ax][s]) : EIK_INF;
  const double slow = __ldg(P.slow + l);
  double pot = EIK_INF;
#pragma unroll
  for (int ax = 0; ax < ND; ax++)
#pragma unroll
    for (int s = 0; s < 2; s++) pot = fmin(pot, t1[ax][s]);
  if (!(pot < EIK_INF)) {  // nothing reached around it yet
    m.set_tent(l, EIK_INF);
    return visit_code(VISIT_UNREACHED);
  }
  PL_ADD(7, tq0);
  PL_T(tq1);
  double dh[3];
  node_dh(g, c[0], dh);
  // Lower bound of the node's value: every term of the local update is at least pot and
  // the quadratic adds at least (2/3) h s / sqrt(ND) (2nd-order coefficients 9/(4h^2)).
  // Until the round threshold reaches it the node cannot be final: no evaluation yet.
  double hmin = dh[0];
#pragma unroll
  for (int ax = 1; ax < ND; ax++) hmin = fmin(hmin, dh[ax]);
  const double lb = pot + 0.999 * (2.0 / 3.0) * hmin * slow * (ND == 3 ? 0.5773502691896258 : 0.7071067811865476);
  if (lb > T) {
    m.set_tent(l, lb);  // stands, like an evaluated value, while the node stays clean
    *front = lb;
    return (1u << DIR_SELF) | visit_code(VISIT_BOUND);
  }
  // Codes of the immediate neighbours and the distance-2 nodes with their codes, one batch.
  // A neighbour's key is read after its traveltime here as in any order: the key changes
  // only together with the traveltime, in the neighbour's own visit.
  uint8_t cd1[ND][2], cd2[ND][2];
  double t2[ND][2];
  unsigned l2[ND][2];
  unsigned ok2 = 0u;
  // isonbord on the first neighbour, in every coordinate (eikutils.jl:129-162): the other
  // coordinates are the node's own, the one along ax is one step out
#pragma unroll
  for (int ax = 0; ax < ND; ax++) {
    bool side = true;
#pragma unroll
    for (int dd = 0; dd < ND; dd++)
      if (dd != ax) side = side && c[dd] >= 1 && c[dd] <= g.n[dd] - 2;
#pragma unroll
    for (int s = 0; s < 2; s++) {
      const int sh = s == 0 ? 1 : -1;
      const unsigned st = ax == 0 ? 1u : (ax == 1 ? st1 : st2);
      l2[ax][s] = s == 0 ? l1[ax][s] + st : l1[ax][s] - st;
      if (side && c[ax] + sh >= 1 && c[ax] + sh <= g.n[ax] - 2) ok2 |= 1u << slot(ax, s);
    }
  }
#pragma unroll
  for (int ax = 0; ax < ND; ax++)
#pragma unroll
    for (int s = 0; s < 2; s++) {
      const bool h1 = (in1 >> slot(ax, s)) & 1u, h2 = (ok2 >> slot(ax, s)) & 1u;
      cd1[ax][s] = h1 ? m.code(l1[ax][s]) : (uint8_t)0;
      t2[ax][s] = h2 ? m.t(l2[ax][s]) : EIK_INF;
      cd2[ax][s] = h2 ? m.code(l2[ax][s]) : (uint8_t)0;
    }
  // Without a special key among them (the common case) every key is the traveltime: the
  // rule runs on traveltimes alone (prefix_rule_plain), else on the full keys (rule_full).
  bool plain = true;
#pragma unroll
  for (int ax = 0; ax < ND; ax++)
#pragma unroll
    for (int s = 0; s < 2; s++)
      if ((cd1[ax][s] | cd2[ax][s]) & CODE_SRC_BIT) plain = false;
  int8_t cd[3] = {0, 0, 0};
  Key nk;
  bool neg = false;
  PL_T(tq2);
  double nv;
  if (plain) {
    NbhdT nb;
    nb.in1 = in1;
    nb.ok2 = ok2;  // within in1: a distance-2 node lies beyond an immediate one
#pragma unroll
    for (int ax = 0; ax < 3; ax++)
#pragma unroll
      for (int s = 0; s < 2; s++) {
        nb.t1[ax][s] = ax < ND ? t1[ax < ND ? ax : 0][s] : EIK_INF;  // EIK_INF where absent
        nb.t2[ax][s] = ax < ND ? t2[ax < ND ? ax : 0][s] : EIK_INF;
      }
#pragma unroll
    for (int ax = 0; ax < 3; ax++) nb.dh[ax] = dh[ax];
    nb.slow = slow;
    nb.c1u = P.c1u;
    nb.c2u = P.c2u;
    nv = prefix_rule_plain<ND>(nb, cd, &nk, &neg);
  } else {
    RuleIn in;
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
#pragma unroll
      for (int s = 0; s < 2; s++) {
        const bool use = ax < ND;
        const bool h1 = use && ((in1 >> slot(ax, s)) & 1u), h2 = use && ((ok2 >> slot(ax, s)) & 1u);
        in.l1[ax][s] = h1 ? (long long)l1[ax < ND ? ax : 0][s] : -1;
        in.l2[ax][s] = h2 ? (long long)l2[ax < ND ? ax : 0][s] : -1;
        in.t1[ax][s] = use ? t1[ax < ND ? ax : 0][s] : EIK_INF;
        in.t2[ax][s] = use ? t2[ax < ND ? ax : 0][s] : EIK_INF;
        in.cd1[ax][s] = use ? cd1[ax < ND ? ax : 0][s] : (uint8_t)0;
        in.cd2[ax][s] = use ? cd2[ax < ND ? ax : 0][s] : (uint8_t)0;
      }
      in.dh[ax] = dh[ax];
    }
    in.slow = slow;
    const RuleOut o = rule_full<ND>(P, in);
    nv = o.v;
    nk = o.key;
    neg = o.neg;
#pragma unroll
    for (int a = 0; a < 3; a++) cd[a] = o.cd[a];
  }
  PL_ADD(9, tq2);
  const uint8_t nc = pack_codes(cd, ND);
  const bool same_t = (nv == told) || (isinf(nv) && isinf(told));
  const bool tkchange = !(same_t && key_eq(nk, Key{Lold, dold, told}));
  const bool special = !(nk.L == nv && nk.d == 0);
  const uint8_t ncb = (uint8_t)(nc | (special ? CODE_SRC_BIT : 0));
  m.set_tent(l, nv);
  if (!tkchange) {
    if (ncb != cb) m.set_code(l, ncb);
    return visit_code(VISIT_SAME);
  }
  if (nv > T) {  // not final yet: keep the old value and come back when the front is there
    *front = nv;
    return (1u << DIR_SELF) | visit_code(VISIT_WAIT);
  }
  m.set_t(l, nv);
  m.set_code(l, ncb);
  if (special) {
    P.kL[l] = nk.L;
    P.kd[l] = (uint8_t)nk.d;
  }
  m.fence();
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
    const unsigned st = ax == 0 ? 1u : (ax == 1 ? st1 : st2);
    unsigned lj[4];
    unsigned hj = 0u;  // bit j: the node exists
    double tj[4];
    uint8_t cj[4];
    int32_t sj[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int off = dir_off(j);
      lj[j] = off < 0 ? ul - (unsigned)(-off) * st : ul + (unsigned)off * st;
      if (c[ax] + off >= 0 && c[ax] + off < g.n[ax]) hj |= 1u << j;
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const bool h = (hj >> j) & 1u;
      tj[j] = h ? m.t(lj[j]) : EIK_INF;
      cj[j] = h ? m.code(lj[j]) : (uint8_t)0;
      sj[j] = h ? m.stamp(lj[j]) : 0;
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      if (!((hj >> j) & 1u)) continue;
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
      m.set_dirty(lj[j], 1);
      dirs |= 1u << (4 * ax + j);
    }
  }
  *front = nv + P.incmin;  // no node reading this one can get a smaller value from it
  PL_ADD(10, tq3);
  PL_ADD(8, tq1);
  return dirs | visit_code(VISIT_CHANGED);
}

}  // namespace eik
