// Host emulation of the forward round solver's schedule (test harness, not product code).
//
// Restates, one visit at a time, what coarse_rounds_kernel does to a Cartesian grid: worklist
// rounds under the threshold T(r) = max(T(r-1), smallest pending front + delta), the node
// visit of node.cuh (cached front, lower-bound gate, the order rule of stencil.cuh on
// traveltimes alone or on full keys, write-back, relist filter) and the per-round stamps.
// The order rule itself is the product's (stencil.cuh, compiled for the host). Visits within
// a round run in list order (mode 0), in a seeded random order (mode 1), or in a random order
// with waiting nodes parked by front instead of listed again every round (mode 2: a node
// whose front still stands is taken out of the lists and comes back in the first round whose
// threshold reaches its front, unless a neighbour's change lists it earlier; modes 3-6: the
// same with the parked nodes in buckets of 1, 1/4, 1/16 or 1/64 round width by front, a bucket
// coming back whole once the threshold reaches its smallest front). Mode 7 runs each round's
// visits as concurrent visits may interleave at the extreme: all reads at the round's start,
// then all writes, then all relist filters, each in a random order. Mode 8 runs them one
// after the other in a random order, each read of a neighbour written earlier in the round
// returning, at random, its value of the round's start or its current one (a traveltime and
// the code beside it may disagree, as unordered loads of concurrent visits may; modes 9-11 tie
// some of a neighbour's fields to one moment, see Solver::agree); such a read
// places the visit before that neighbour's change, so the neighbour's relist filter leaves the
// visited node's dirty flag set.
//
// Usage: round_schedule_harness in.bin out.bin
//   in:  int32 nd, n0, n1, n2; double h, gate; int32 mode; uint64 seed; int64 nseed;
//        N doubles slowness (1/v, as the product computes it); nseed int64 node indices;
//        nseed doubles traveltimes of the fixed source points.
//   out: N doubles traveltime; int64 rounds, list entries, rule evaluations, visits by
//        outcome (7: stands, source, unreached, bound, wait, same, changed), parked nodes
//        taken back, nodes whose rule would still change their value or key at the end,
//        special nodes (code bit 7) left with an unreached traveltime.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <map>
#include <queue>
#include <tuple>
#include <random>
#include <vector>

#include "stencil.cuh"

using namespace eik;

namespace {

struct Solver {
  int nd;
  int n[3];
  double h;
  long long N;
  std::vector<double> slow, t, tent, kL;
  std::vector<uint8_t> code, kd, dirty;
  std::vector<int> stamp;
  double delta, incmin, c1u, c2u;
  long long evals = 0, visits[7] = {0, 0, 0, 0, 0, 0, 0};
  // mode 8: a neighbour written earlier in the round is read at its value of the round's
  // start or at its current one, each read on its own (old_* hold the start values)
  bool stale = false;
  int round = -1;
  std::vector<int> wround;
  std::vector<double> old_t, old_kL;
  std::vector<uint8_t> old_code, old_kd;
  mutable std::mt19937_64 coin{12345};
  mutable bool saw_stale = false;
  // how the reads of one neighbour within a visit agree (modes 8-11): 0 each read on its own;
  // 1 traveltime, code and key level from the same moment; 2 code and key level together,
  // the traveltime on its own; 3 traveltime and code together, the key level on its own
  int agree = 0;
  mutable std::vector<std::pair<long long, unsigned>> picks;  // this visit's choices per node
  bool old_of(long long x, int field) const {  // field 0: t, 1: code, 2: key level
    if (!(stale && wround[x] == round)) return false;
    const int group = agree == 0 ? field : (agree == 1 ? 0 : (agree == 2 ? (field == 0 ? 0 : 1) : (field == 2 ? 1 : 0)));
    unsigned have = 0, bits = 0;
    for (auto& pr : picks)
      if (pr.first == x) {
        have = pr.second & 3u;
        bits = pr.second >> 2;
      }
    bool o;
    if (agree != 0 && ((have >> group) & 1u)) {
      o = (bits >> group) & 1u;
    } else {
      o = coin() & 1u;
      bool found = false;
      for (auto& pr : picks)
        if (pr.first == x) {
          pr.second |= (1u << group) | ((o ? 1u : 0u) << (2 + group));
          found = true;
        }
      if (!found) picks.push_back({x, (1u << group) | ((o ? 1u : 0u) << (2 + group))});
    }
    saw_stale = saw_stale || o;
    return o;
  }
  double rt(long long x) const { return old_of(x, 0) ? old_t[x] : t[x]; }
  uint8_t rc(long long x) const { return old_of(x, 1) ? old_code[x] : code[x]; }
  void rkey(long long x, double tv, uint8_t cb, double* L, int* d) const {
    if ((cb & CODE_SRC_BIT) && tv < EIK_INF) {
      const bool o = old_of(x, 2);
      *L = o ? old_kL[x] : kL[x];
      *d = o ? old_kd[x] : kd[x];
    } else {
      *L = tv;
      *d = 0;
    }
  }

  long long lin(const int* c) const { return c[0] + (long long)n[0] * (c[1] + (long long)n[1] * c[2]); }
  void coords(long long l, int* c) const {
    c[0] = (int)(l % n[0]);
    c[1] = (int)((l / n[0]) % n[1]);
    c[2] = (int)(l / ((long long)n[0] * n[1]));
  }
  // node_key of node.cuh: a special key counts only beside a reached traveltime
  void key(long long l, double tv, uint8_t cb, double* L, int* d) const {
    if ((cb & CODE_SRC_BIT) && tv < EIK_INF) {
      *L = kL[l];
      *d = kd[l];
    } else {
      *L = tv;
      *d = 0;
    }
  }
};

// Float of the list entry: the front rounded down (the kernel's __double2float_rd).
double entry_front(double f) {
  if (!(f < EIK_INF)) return EIK_INF;
  float g = (float)f;
  if ((double)g > f) g = std::nextafterf(g, -INFINITY);
  return (double)g;
}

enum { V_STANDS, V_SOURCE, V_UNREACHED, V_BOUND, V_WAIT, V_SAME, V_CHANGED };

// What a visit decides from what it reads (node.cuh, process_node): its outcome, the
// direction bit of the node itself for the waiting outcomes, the front, and the writes to its
// own node. evaluate() only reads; commit() writes; relist() is the filter that follows an
// accepted change, reading the state as it is then.
struct Visit {
  int outcome = 0;
  unsigned dirs = 0;
  double front = EIK_INF;
  bool clear_dirty = false;  // the visit reads its neighbours: its dirty flag is cleared first
  bool set_tent = false;
  double tent = EIK_INF;
  bool set_code = false;
  uint8_t code = 0;
  bool changed = false;  // value or key accepted: t, code and key are written, then the filter
  double nv = EIK_INF;
  Key nk{}, kold{};
  bool special = false;
};

template <int ND>
Visit evaluate(const Solver& S, long long l, double T) {
  Visit v;
  int c[3];
  S.coords(l, c);
  const uint8_t dirty0 = S.dirty[l];
  const double tv = S.tent[l];
  const uint8_t cb = S.code[l];
  const double told = S.t[l];
  if (!dirty0 && tv > T && tv < EIK_INF) {
    v.front = tv;
    v.outcome = V_STANDS;
    v.dirs = 1u << 12;
    return v;
  }
  double Lold;
  int dold;
  S.key(l, told, cb, &Lold, &dold);
  if ((cb & CODE_SRC_BIT) && Lold == -EIK_INF) {
    v.outcome = V_SOURCE;
    return v;
  }
  v.clear_dirty = true;
  long long l1[3][2], l2[3][2];
  double t1[3][2], t2[3][2];
  uint8_t cd1[3][2], cd2[3][2];
  double pot = EIK_INF;
  for (int ax = 0; ax < ND; ax++)
    for (int s = 0; s < 2; s++) {
      const int sh = s == 0 ? 1 : -1;
      int p[3] = {c[0], c[1], c[2]};
      p[ax] += sh;
      l1[ax][s] = (p[ax] < 0 || p[ax] >= S.n[ax]) ? -1 : S.lin(p);
      t1[ax][s] = l1[ax][s] >= 0 ? S.rt(l1[ax][s]) : EIK_INF;
      pot = std::fmin(pot, t1[ax][s]);
    }
  if (!(pot < EIK_INF)) {
    v.set_tent = true;
    v.tent = EIK_INF;
    v.outcome = V_UNREACHED;
    return v;
  }
  const double slow = S.slow[l];
  const double hmin = S.h;
  const double lb = pot + 0.999 * (2.0 / 3.0) * hmin * slow * (ND == 3 ? 0.5773502691896258 : 0.7071067811865476);
  if (lb > T) {
    v.set_tent = true;
    v.tent = lb;
    v.front = lb;
    v.outcome = V_BOUND;
    v.dirs = 1u << 12;
    return v;
  }
  bool plain = true;
  for (int ax = 0; ax < ND; ax++)
    for (int s = 0; s < 2; s++) {
      const int sh = s == 0 ? 1 : -1;
      l2[ax][s] = -1;
      cd1[ax][s] = cd2[ax][s] = 0;
      t2[ax][s] = EIK_INF;
      if (l1[ax][s] < 0) continue;
      cd1[ax][s] = S.rc(l1[ax][s]);
      int p[3] = {c[0], c[1], c[2]};
      p[ax] += sh;
      bool ok = true;  // isonbord on the first neighbour
      for (int dd = 0; dd < ND; dd++)
        if (p[dd] < 1 || p[dd] > S.n[dd] - 2) ok = false;
      if (ok) {
        p[ax] += sh;
        l2[ax][s] = S.lin(p);
        t2[ax][s] = S.rt(l2[ax][s]);
        cd2[ax][s] = S.rc(l2[ax][s]);
      }
      if ((cd1[ax][s] | cd2[ax][s]) & CODE_SRC_BIT) plain = false;
    }
  int8_t cd[3] = {0, 0, 0};
  Key nk;
  bool neg = false;
  double nv;
  if (plain) {
    NbhdT nb;
    nb.in1 = nb.ok2 = 0u;
    for (int ax = 0; ax < 3; ax++)
      for (int s = 0; s < 2; s++) {
        nb.t1[ax][s] = EIK_INF;
        nb.t2[ax][s] = EIK_INF;
      }
    for (int ax = 0; ax < ND; ax++)
      for (int s = 0; s < 2; s++) {
        if (l1[ax][s] < 0) continue;
        nb.t1[ax][s] = t1[ax][s];
        nb.in1 |= 1u << slot(ax, s);
        if (l2[ax][s] >= 0) {
          nb.t2[ax][s] = t2[ax][s];
          nb.ok2 |= 1u << slot(ax, s);
        }
      }
    for (int ax = 0; ax < 3; ax++) nb.dh[ax] = S.h;
    nb.slow = slow;
    nb.c1u = S.c1u;
    nb.c2u = S.c2u;
    nv = prefix_rule_plain<ND>(nb, cd, &nk, &neg);
  } else {
    Nbhd nb;
    nb_clear(nb);
    for (int ax = 0; ax < 3; ax++) nb.dh[ax] = S.h;
    nb.slow = slow;
    nb.c1u = S.c1u;
    nb.c2u = S.c2u;
    for (int ax = 0; ax < ND; ax++)
      for (int s = 0; s < 2; s++) {
        if (l1[ax][s] < 0) continue;
        double L;
        int d;
        S.rkey(l1[ax][s], t1[ax][s], cd1[ax][s], &L, &d);
        nb_put1(nb, ax, s, t1[ax][s], L, d);
        if (l2[ax][s] >= 0) {
          S.rkey(l2[ax][s], t2[ax][s], cd2[ax][s], &L, &d);
          nb_put2(nb, ax, s, t2[ax][s], L, d);
        }
      }
    nv = prefix_rule<ND>(nb, cd, &nk, &neg);
  }
  const uint8_t nc = pack_codes(cd, ND);
  const bool same_t = (nv == told) || (std::isinf(nv) && std::isinf(told));
  const bool tkchange = !(same_t && key_eq(nk, Key{Lold, dold, told}));
  const bool special = !(nk.L == nv && nk.d == 0);
  const uint8_t ncb = (uint8_t)(nc | (special ? CODE_SRC_BIT : 0));
  v.set_tent = true;
  v.tent = nv;
  if (!tkchange) {
    v.set_code = ncb != cb;
    v.code = ncb;
    v.outcome = V_SAME;
    return v;
  }
  if (nv > T) {
    v.front = nv;
    v.outcome = V_WAIT;
    v.dirs = 1u << 12;
    return v;
  }
  v.changed = true;
  v.set_code = true;
  v.code = ncb;
  v.nv = nv;
  v.nk = nk;
  v.kold = Key{Lold, dold, told};
  v.special = special;
  v.front = nv + S.incmin;
  v.outcome = V_CHANGED;
  return v;
}

void commit(Solver& S, long long l, const Visit& v) {
  if (S.stale && S.wround[l] != S.round && v.changed) {
    S.wround[l] = S.round;  // first write of the round: keep the start values
    S.old_t[l] = S.t[l];
    S.old_code[l] = S.code[l];
    S.old_kL[l] = S.kL[l];
    S.old_kd[l] = S.kd[l];
  }
  if (v.set_tent) S.tent[l] = v.tent;
  if (v.set_code) S.code[l] = v.code;
  if (v.changed) {
    S.t[l] = v.nv;
    if (v.special) {
      S.kL[l] = v.nk.L;
      S.kd[l] = (uint8_t)v.nk.d;
    }
  }
}

// The relist filter after an accepted change of node l in round r: the nodes whose stencil
// reads l, except those whose key is at most both the old and the new key of l and that are
// in no list of this round or the next.
template <int ND>
unsigned relist(Solver& S, long long l, const Visit& v, int r) {
  int c[3];
  S.coords(l, c);
  unsigned dirs = 0;
  for (int ax = 0; ax < ND; ax++) {
    long long lj[4];
    double tj[4];
    for (int j = 0; j < 4; j++) {
      const int off = j < 2 ? j - 2 : j - 1;
      int p[3] = {c[0], c[1], c[2]};
      p[ax] += off;
      lj[j] = (p[ax] < 0 || p[ax] >= S.n[ax]) ? -1 : S.lin(p);
      tj[j] = lj[j] >= 0 ? S.t[lj[j]] : EIK_INF;
    }
    for (int j = 0; j < 4; j++) {
      if (lj[j] < 0) continue;
      if (j == 0 && !(tj[1] < EIK_INF)) continue;
      if (j == 3 && !(tj[2] < EIK_INF)) continue;
      if (S.stamp[lj[j]] < r) {
        double Lj;
        int dj;
        S.key(lj[j], tj[j], S.code[lj[j]], &Lj, &dj);
        const Key kj = Key{Lj, dj, tj[j]};
        if (key_le(kj, v.kold) && key_le(kj, v.nk)) continue;
      }
      S.dirty[lj[j]] = 1;
      dirs |= 1u << (4 * ax + j);
    }
  }
  return dirs;
}

long long dir_node(const Solver& S, long long l, int k) {
  if (k == 12) return l;
  const int ax = k >> 2, j = k & 3;
  const int off = j < 2 ? j - 2 : j - 1;
  const long long st = ax == 0 ? 1 : (ax == 1 ? S.n[0] : (long long)S.n[0] * S.n[1]);
  return l + off * st;
}

struct Entry {
  long long l;
  double f;  // front as stored in the list (rounded down to float)
};

template <int ND>
void solve(Solver& S, const std::vector<long long>& seeds, const std::vector<double>& seedtt, int mode,
           unsigned long long seed, long long* rounds_out, long long* entries_out, long long* unparked_out) {
  std::mt19937_64 rng(seed);
  if (mode >= 8 && mode <= 11) {
    S.stale = true;
    S.agree = mode - 8;
    S.coin.seed(seed ^ 0x9e3779b97f4a7c15ull);
    S.wround.assign(S.N, -1);
    S.old_t.assign(S.N, EIK_INF);
    S.old_kL.assign(S.N, -EIK_INF);
    S.old_code.assign(S.N, CODE_NONE);
    S.old_kd.assign(S.N, 0);
  }
  std::vector<Entry> cur, next;
  double nm_next = EIK_INF, thr = -EIK_INF;
  auto list = [&](int r, long long l, double f, std::vector<Entry>& L) {
    if (S.stamp[l] != r) {
      S.stamp[l] = r;
      L.push_back(Entry{l, entry_front(f)});
      return true;
    }
    return false;
  };
  for (size_t q = 0; q < seeds.size(); q++) {
    const long long l = seeds[q];
    S.t[l] = seedtt[q];
    S.code[l] = (uint8_t)(CODE_NONE | CODE_SRC_BIT);
    S.kL[l] = -EIK_INF;
    S.kd[l] = 0;
  }
  double nm = EIK_INF;
  for (size_t q = 0; q < seeds.size(); q++) {
    const long long l = seeds[q];
    int c[3];
    S.coords(l, c);
    if (seedtt[q] < EIK_INF) nm = std::fmin(nm, seedtt[q]);
    for (int ax = 0; ax < ND; ax++)
      for (int d = -2; d <= 2; d++) {
        if (d == 0) continue;
        int p[3] = {c[0], c[1], c[2]};
        p[ax] += d;
        if (p[ax] < 0 || p[ax] >= S.n[ax]) continue;
        list(0, S.lin(p), seedtt[q], cur);
      }
  }
  std::vector<int> parked_at(S.N, -1);
  // parked nodes (mode 2): (front, node, round parked), smallest front first; an entry is
  // live while the node is still parked from that round (a listing by a neighbour, or a
  // later parking, supersedes it)
  typedef std::tuple<double, long long, int> Parked;
  std::priority_queue<Parked, std::vector<Parked>, std::greater<Parked>> park;
  auto live = [&](const Parked& p) { return parked_at[std::get<1>(p)] == std::get<2>(p); };
  // modes 3-6: parked nodes in buckets by front (1, 1/4, 1/16, 1/64 of the round width),
  // each with its smallest front; a bucket comes back whole once the threshold reaches its
  // smallest front (the form a device queue in memory would take)
  std::map<long long, std::vector<Parked>> buckets;
  std::map<long long, double> bucket_min;
  long long entries = 0, unparked = 0;
  int r = 0;
  for (;; r++) {
    // parked nodes whose front the threshold of this round can reach come back
    double pmin = EIK_INF;
    while (!park.empty() && !live(park.top())) park.pop();
    if (!park.empty()) pmin = std::get<0>(park.top());
    while (!bucket_min.empty()) {  // buckets left with superseded entries only
      const long long b = bucket_min.begin()->first;
      bool any = false;
      for (const Parked& p : buckets[b]) any = any || live(p);
      if (any) break;
      buckets.erase(b);
      bucket_min.erase(b);
    }
    if (!bucket_min.empty()) pmin = bucket_min.begin()->second;
    const double T = std::fmax(thr, std::fmin(nm, pmin) + S.delta);
    while (!park.empty() && std::get<0>(park.top()) <= T) {
      const Parked p = park.top();
      park.pop();
      if (!live(p)) continue;
      parked_at[std::get<1>(p)] = -1;
      if (list(r, std::get<1>(p), std::get<0>(p), cur)) unparked++;
    }
    while (!bucket_min.empty() && bucket_min.begin()->second <= T) {
      const long long b = bucket_min.begin()->first;
      for (const Parked& p : buckets[b]) {
        if (!live(p)) continue;
        parked_at[std::get<1>(p)] = -1;
        if (list(r, std::get<1>(p), std::get<0>(p), cur)) unparked++;
      }
      buckets.erase(b);
      bucket_min.erase(b);
    }
    if (cur.empty()) break;
    if (r >= (1 << 20)) break;  // not settling: reported as 2^20 rounds
    thr = T;
    S.round = r;
    entries += (long long)cur.size();
    if (mode >= 1) std::shuffle(cur.begin(), cur.end(), rng);
    next.clear();
    nm_next = EIK_INF;
    // the visits of the round: one after the other (modes 0-6), or all reads first, then all
    // writes, then all filters, each in a random order (mode 7: the extreme interleaving of
    // concurrent visits, every visit seeing the state of the round's start)
    std::vector<Visit> vs(cur.size());
    auto take = [&](size_t i) {
      const Entry& e = cur[i];
      if (e.f > T && e.f < EIK_INF && !S.dirty[e.l]) {
        vs[i] = Visit();
        vs[i].front = e.f;
        vs[i].dirs = 1u << 12;
        vs[i].outcome = V_STANDS;
      } else {
        vs[i] = evaluate<ND>(S, e.l, T);
      }
    };
    if (mode != 7) {
      for (size_t i = 0; i < cur.size(); i++) {
        S.saw_stale = false;
        S.picks.clear();
        take(i);
        const long long l = cur[i].l;
        if (vs[i].clear_dirty) S.dirty[l] = 0;
        // a read of a neighbour's value from before its change this round means that, in
        // real time, the read preceded that change, whose relist filter then ran after this
        // visit had cleared its flag: the flag that filter set stands
        if (S.saw_stale) S.dirty[l] = 1;
        commit(S, l, vs[i]);
        if (vs[i].changed) vs[i].dirs |= relist<ND>(S, l, vs[i], r);
      }
    } else {
      for (size_t i = 0; i < cur.size(); i++) take(i);
      for (size_t i = 0; i < cur.size(); i++)
        if (vs[i].clear_dirty) S.dirty[cur[i].l] = 0;
      std::vector<size_t> ord(cur.size());
      for (size_t i = 0; i < ord.size(); i++) ord[i] = i;
      std::shuffle(ord.begin(), ord.end(), rng);
      for (size_t i : ord) commit(S, cur[i].l, vs[i]);
      std::shuffle(ord.begin(), ord.end(), rng);
      for (size_t i : ord)
        if (vs[i].changed) vs[i].dirs |= relist<ND>(S, cur[i].l, vs[i], r);
    }
    for (size_t i = 0; i < cur.size(); i++) {
      const Entry& e = cur[i];
      const unsigned dirs = vs[i].dirs;
      const double front = vs[i].front;
      const int oc = vs[i].outcome;
      if (oc >= V_WAIT) S.evals++;
      S.visits[oc]++;
      bool kept = false;
      for (int k = 0; k <= 12; k++) {
        if (!((dirs >> k) & 1u)) continue;
        const long long nl = dir_node(S, e.l, k);
        if (mode >= 2 && mode <= 6 && k == 12 && (oc == V_STANDS || oc == V_BOUND || oc == V_WAIT) &&
            !S.dirty[nl] && S.stamp[nl] != r + 1) {
          parked_at[nl] = r;  // waiting above the front: parked instead of listed again
          const double pf = entry_front(front);
          if (mode == 2) {
            park.push(Parked{pf, nl, r});
          } else {
            const double bw = S.delta / (mode == 3 ? 1.0 : (double)(1 << (2 * (mode - 3))));
            const long long b = (long long)std::floor(pf / bw);
            buckets[b].push_back(Parked{pf, nl, r});
            auto it = bucket_min.find(b);
            if (it == bucket_min.end() || pf < it->second) bucket_min[b] = pf;
          }
          continue;
        }
        if (list(r + 1, nl, front, next)) {
          kept = true;
          parked_at[nl] = -1;
        }
      }
      if (kept) nm_next = std::fmin(nm_next, front);
    }
    std::swap(cur, next);
    nm = nm_next;
  }
  *rounds_out = r;
  *entries_out = entries;
  *unparked_out = unparked;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]);
    return 2;
  }
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 3;
  int32_t hdr[4];
  double hg[2];
  int32_t mode;
  uint64_t seed;
  int64_t nseed;
  if (std::fread(hdr, 4, 4, f) != 4 || std::fread(hg, 8, 2, f) != 2 || std::fread(&mode, 4, 1, f) != 1 ||
      std::fread(&seed, 8, 1, f) != 1 || std::fread(&nseed, 8, 1, f) != 1)
    return 4;
  Solver S;
  S.nd = hdr[0];
  S.n[0] = hdr[1];
  S.n[1] = hdr[2];
  S.n[2] = hdr[3];
  S.h = hg[0];
  S.N = (long long)S.n[0] * S.n[1] * S.n[2];
  S.slow.resize(S.N);
  std::vector<long long> seeds(nseed);
  std::vector<double> seedtt(nseed);
  if (std::fread(S.slow.data(), 8, S.N, f) != (size_t)S.N || std::fread(seeds.data(), 8, nseed, f) != (size_t)nseed ||
      std::fread(seedtt.data(), 8, nseed, f) != (size_t)nseed)
    return 5;
  std::fclose(f);
  S.t.assign(S.N, EIK_INF);
  S.tent.assign(S.N, EIK_INF);
  S.kL.assign(S.N, -EIK_INF);  // never read unless written: any value will do, this one is the worst
  S.code.assign(S.N, CODE_NONE);
  S.kd.assign(S.N, 0);
  S.dirty.assign(S.N, 1);
  S.stamp.assign(S.N, -1);
  double smin = EIK_INF;
  for (double s : S.slow) smin = std::fmin(smin, s);
  const double hmin = S.h;
  S.delta = hg[1] * hmin * smin;
  S.incmin = 0.999 * (2.0 / 3.0) * hmin * smin / std::sqrt((double)S.nd);
  S.c1u = 1.0 / (S.h * S.h);
  S.c2u = 9.0 / (4.0 * (S.h * S.h));
  long long rounds = 0, entries = 0, unparked = 0;
  if (S.nd == 3)
    solve<3>(S, seeds, seedtt, mode, seed, &rounds, &entries, &unparked);
  else
    solve<2>(S, seeds, seedtt, mode, seed, &rounds, &entries, &unparked);
  // nodes whose order rule, evaluated on the final state with no threshold, would still change
  // their value or key (0 for a fixed point)
  S.stale = false;
  long long unsettled = 0, special_unreached = 0;
  for (long long l = 0; l < S.N; l++) {
    if ((S.code[l] & CODE_SRC_BIT) && !(S.t[l] < EIK_INF)) special_unreached++;
    S.dirty[l] = 1;
    const Visit v = S.nd == 3 ? evaluate<3>(S, l, EIK_INF) : evaluate<2>(S, l, EIK_INF);
    if (v.changed) unsettled++;
  }
  FILE* o = std::fopen(argv[2], "wb");
  if (!o) return 6;
  std::fwrite(S.t.data(), 8, S.N, o);
  const int64_t st[13] = {rounds,      entries,     S.evals,     S.visits[0], S.visits[1],
                          S.visits[2], S.visits[3], S.visits[4], S.visits[5], S.visits[6],
                          unparked,    unsettled,   special_unreached};
  std::fwrite(st, 8, 13, o);
  std::fclose(o);
  return 0;
}
