// Local 2nd-order upwind update of EikonalSolvers.jl (calcttpt_2ndord!,
// src/EikSolv/eikforward2D.jl:98-433 and src/EikSolv/eikforward3D.jl:151-532) and the
// order rule that turns it into a fixed-point problem solvable in parallel.
//
// The reference evaluates the update inside a heap-ordered fast-marching loop
// (ttFMM_core!, src/EikSolv/eikmainfwd.jl:427-823): a node is recomputed each time one
// of its 2*nd immediate neighbours is accepted, using only accepted nodes, and keeps the
// value of its last recomputation. This header restates that final value as a function
// of the neighbourhood alone ("prefix rule"):
//
//   sort the immediate neighbours by acceptance key (source points first, then
//   traveltime); for each group g of equal keys K_g, evaluate the update with
//   accepted(x) := key(x) <= K_g; the first group whose result v_g does not exceed the
//   key of the next group is the one after which the node is accepted itself, so v_g is
//   its traveltime and the derivative codes of that evaluation are its codes.
//
// Iterating the rule on every node from t = +inf to a fixed point reproduces the FMM
// traveltimes bit for bit: keys (below) place the rare non-causal acceptances of the
// reference (an overwritten band value below the current front) right after the node
// that triggered them, as the heap does.
//
// The arithmetic is the reference's, operation by operation (x^2 as x*x, left-to-right
// sums, no FMA contraction: translation units including this header are compiled with
// --fmad=false / -ffp-contract=off).
#pragma once

#include <cstdint>
#include <math.h>

#if defined(__CUDACC__)
#define EIK_HD __host__ __device__ __forceinline__
#else
#define EIK_HD inline
#endif

namespace eik {

#ifndef EIK_INF
#define EIK_INF (__builtin_huge_val())
#endif

// Acceptance key: the position at which the heap-ordered FMM accepts a node, as a
// lexicographic triple (L, d, t). A node accepted in the batch of its own traveltime t has
// key (t, 0, t). A node whose last recomputation, triggered by the acceptance of a node of
// key (L, d, .), produced a value v <= L is accepted right after that trigger although v is
// below the current front (the reference overwrites band values, BinHeaps.jl:394-430, and
// takes no causality check, eikforward2D.jl:425-430): its key is (L, d+1, v). Source points
// are accepted together before anything else: L = -inf (their t does not order them).
#ifndef EIK_MAX_DEPTH
#define EIK_MAX_DEPTH 4
#endif
struct Key {
  double L;
  int d;
  double t;
};
EIK_HD bool key_le(const Key& a, const Key& b) {
  if (a.L != b.L) return a.L < b.L;
  if (a.d != b.d) return a.d < b.d;
  if (a.L == -EIK_INF) return true;
  return a.t <= b.t;
}
EIK_HD bool key_eq(const Key& a, const Key& b) {
  return a.L == b.L && a.d == b.d && (a.L == -EIK_INF || a.t == b.t);
}
EIK_HD Key key_normal(double t) { return Key{t, 0, t}; }
EIK_HD Key key_source() { return Key{-EIK_INF, 0, -EIK_INF}; }
EIK_HD Key key_unreached() { return Key{EIK_INF, 0, EIK_INF}; }
EIK_HD bool key_reached(const Key& k) { return k.L < EIK_INF; }

// Neighbourhood of one node as seen by the update, index [axis][side]: side 0 is the +1
// neighbour (l=1 in the reference), side 1 the -1 neighbour (l=2). Compact so that the
// whole record lives in registers: key levels as doubles, depths and flags as bit fields.
struct Nbhd {
  double t1[3][2];   // traveltime at distance 1 (+inf if not reached / outside)
  double t2[3][2];   // traveltime at distance 2
  double L1[3][2];   // key level at distance 1 (t for ordinary nodes, -inf for sources)
  double L2[3][2];   // key level at distance 2
  uint32_t d1, d2;   // key depths, 4 bits per slot (2*axis+side)
  uint32_t in1;      // bit slot: distance-1 node inside the grid (!isonb1)
  uint32_t ok2;      // bit slot: 2nd order allowed on that side (!isonb2 of the distance-1 node)
  double dh[3];      // node spacing per axis
  double slow;       // 1/vel at the node (computed as 1.0/vel, as the reference)
  double c1u, c2u;   // 1/h^2 and 9/(4h^2) when every axis has spacing h (else 0: per axis)
};
EIK_HD int slot(int a, int l) { return 2 * a + l; }
EIK_HD Key nb_key1(const Nbhd& nb, int a, int l) {
  return Key{nb.L1[a][l], (int)((nb.d1 >> (4 * slot(a, l))) & 15u), nb.t1[a][l]};
}
EIK_HD Key nb_key2(const Nbhd& nb, int a, int l) {
  return Key{nb.L2[a][l], (int)((nb.d2 >> (4 * slot(a, l))) & 15u), nb.t2[a][l]};
}
EIK_HD bool nb_in1(const Nbhd& nb, int a, int l) { return (nb.in1 >> slot(a, l)) & 1u; }
EIK_HD bool nb_ok2(const Nbhd& nb, int a, int l) { return (nb.ok2 >> slot(a, l)) & 1u; }
EIK_HD void nb_clear(Nbhd& nb) {
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int l = 0; l < 2; l++) {
      nb.t1[a][l] = EIK_INF;
      nb.t2[a][l] = EIK_INF;
      nb.L1[a][l] = EIK_INF;
      nb.L2[a][l] = EIK_INF;
    }
  nb.d1 = nb.d2 = nb.in1 = nb.ok2 = 0u;
  nb.c1u = nb.c2u = 0.0;
}

// Fill one slot: distance-1 node inside the grid (t, key level L, depth d).
EIK_HD void nb_put1(Nbhd& nb, int a, int l, double t, double L, int d) {
  nb.t1[a][l] = t;
  nb.L1[a][l] = L;
  nb.d1 |= (uint32_t)d << (4 * slot(a, l));
  nb.in1 |= 1u << slot(a, l);
}
// Distance-2 node on a side where 2nd order is allowed.
EIK_HD void nb_put2(Nbhd& nb, int a, int l, double t, double L, int d) {
  nb.t2[a][l] = t;
  nb.L2[a][l] = L;
  nb.d2 |= (uint32_t)d << (4 * slot(a, l));
  nb.ok2 |= 1u << slot(a, l);
}

// Acceptance by a group key T: the neighbour is in the grid (distance 1) or 2nd order is
// allowed on that side (distance 2), and its key is at most T.
EIK_HD bool acc1(const Nbhd& nb, int a, int l, const Key& T) { return nb_in1(nb, a, l) && key_le(nb_key1(nb, a, l), T); }
EIK_HD bool acc2(const Nbhd& nb, int a, int l, const Key& T) { return nb_ok2(nb, a, l) && key_le(nb_key2(nb, a, l), T); }

// Neighbourhood in which no node (distance 1 or 2) has a special key: every key is
// (t, 0, t), so a key is its traveltime and acceptance by the group key (tg, 0, tg) is
// t <= tg (key_le of two such keys; tg is a reached neighbour's finite traveltime).
struct NbhdT {
  double t1[3][2];
  double t2[3][2];
  uint32_t in1, ok2;  // as in Nbhd
  double dh[3];
  double slow;
  double c1u, c2u;
};
EIK_HD bool acc1(const NbhdT& nb, int a, int l, double tg) { return ((nb.in1 >> slot(a, l)) & 1u) && nb.t1[a][l] <= tg; }
EIK_HD bool acc2(const NbhdT& nb, int a, int l, double tg) { return ((nb.ok2 >> slot(a, l)) & 1u) && nb.t2[a][l] <= tg; }

// calcttpt_2ndord! with accepted(x) := key(x) <= T. codes receive the reference's
// derivative codes (codeD): -side for 1st order, -2*side for 2nd order, 0 unused. NB is a
// neighbourhood (Nbhd with group keys, NbhdT with group traveltimes).
template <int ND, class NB, class TK>
EIK_HD double update_at_g(const NB& nb, const TK& T, int8_t* codes, bool* negdisc) {
  double alpha = 0.0, beta = 0.0, gamma = -(nb.slow * nb.slow);
#pragma unroll
  for (int a = 0; a < ND; a++) codes[a] = 0;
#pragma unroll
  for (int a = 0; a < ND; a++) {
    bool use1 = false, use2 = false;
    double cv1 = EIK_INF, cv2 = EIK_INF;
#pragma unroll
    for (int l = 0; l < 2; l++) {
      const int sh = l == 0 ? 1 : -1;
      if (acc1(nb, a, l, T)) {
        const double tv1 = nb.t1[a][l];
        if (tv1 < cv1) {
          cv1 = tv1;
          use1 = true;
          codes[a] = (int8_t)(-sh);
          if (acc2(nb, a, l, T)) {
            const double tv2 = nb.t2[a][l];
            if (tv2 <= cv1) {
              cv2 = tv2;
              use2 = true;
              codes[a] = (int8_t)(-2 * sh);
            } else {
              cv2 = EIK_INF;
              use2 = false;
              codes[a] = (int8_t)(-sh);
            }
          }
        }
      }
    }
    const double dh = nb.dh[a];
    if (use2 && use1) {
      const double tmpa2 = (1.0 / 3.0) * (4.0 * cv1 - cv2);
      const double ca = nb.c2u > 0.0 ? nb.c2u : 9.0 / (4.0 * (dh * dh));
      alpha += ca;
      beta += (-2.0 * ca) * tmpa2;
      gamma += ca * (tmpa2 * tmpa2);
    } else if (use1) {
      const double ca = nb.c1u > 0.0 ? nb.c1u : 1.0 / (dh * dh);
      alpha += ca;
      beta += (-2.0 * ca) * cv1;
      gamma += ca * (cv1 * cv1);
    }
  }
  double sqarg = beta * beta - (4.0 * alpha) * gamma;
  if (sqarg < 0.0) {  // 1st order on every axis (eikforward2D.jl:265-337)
    alpha = 0.0;
    beta = 0.0;
    gamma = -(nb.slow * nb.slow);
#pragma unroll
    for (int a = 0; a < ND; a++) {
      codes[a] = 0;
      bool use1 = false;
      double cv1 = EIK_INF;
#pragma unroll
      for (int l = 0; l < 2; l++) {
        const int sh = l == 0 ? 1 : -1;
        if (acc1(nb, a, l, T)) {
          const double tv1 = nb.t1[a][l];
          if (tv1 < cv1) {
            cv1 = tv1;
            use1 = true;
            codes[a] = (int8_t)(-sh);
          }
        }
      }
      if (use1) {
        const double dh = nb.dh[a];
        const double ca = nb.c1u > 0.0 ? nb.c1u : 1.0 / (dh * dh);
        alpha += ca;
        beta += (-2.0 * ca) * cv1;
        gamma += ca * (cv1 * cv1);
      }
    }
    sqarg = beta * beta - (4.0 * alpha) * gamma;
  }
  if (sqarg < 0.0) {  // one-dimensional update (eikforward2D.jl:340-411)
    if (negdisc) *negdisc = true;
    double cv[3] = {EIK_INF, EIK_INF, EIK_INF};
    int8_t cd[3] = {0, 0, 0};
#pragma unroll
    for (int a = 0; a < ND; a++) {
#pragma unroll
      for (int l = 0; l < 2; l++) {
        const int sh = l == 0 ? 1 : -1;
        if (acc1(nb, a, l, T)) {
          const double tv1 = nb.t1[a][l];
          if (tv1 < cv[a]) {
            cv[a] = tv1;
            cd[a] = (int8_t)(-sh);
          }
        }
      }
    }
    int id = 0;
    double best = cv[0];
#pragma unroll
    for (int a = 1; a < ND; a++)
      if (cv[a] < best) {
        best = cv[a];
        id = a;
      }
    double dhid = nb.dh[0];
#pragma unroll
    for (int a = 1; a < ND; a++)
      if (a == id) dhid = nb.dh[a];
#pragma unroll
    for (int a = 0; a < ND; a++) codes[a] = (a == id) ? cd[a] : (int8_t)0;
    return (dhid * nb.slow) + best;
  }
  // The reference takes the larger of (-beta +- sqrt)/(2 alpha). alpha > 0 (at least one
  // neighbour is used) and sqrt >= 0, and rounded addition and division by a positive number
  // are monotone, so the '+' root is never below the '-' root: it is the larger one.
  const double tmpsq = sqrt(sqarg);
  return (-beta + tmpsq) / (2.0 * alpha);
}

template <int ND>
EIK_HD double update_at(const Nbhd& nb, const Key& T, int8_t* codes, bool* negdisc) {
  return update_at_g<ND>(nb, T, codes, negdisc);
}

// Smallest key of a reached in-grid immediate neighbour, strictly above lo if strict.
template <int ND>
EIK_HD void next_key_above(const Nbhd& nb, const Key& lo, bool strict, Key* out, bool* found) {
  *found = false;
#pragma unroll
  for (int a = 0; a < ND; a++)
#pragma unroll
    for (int l = 0; l < 2; l++) {
      const Key k = nb_key1(nb, a, l);
      if (!nb_in1(nb, a, l) || !key_reached(k)) continue;
      if (strict && key_le(k, lo)) continue;
      if (!*found || !key_le(*out, k)) {
        *out = k;
        *found = true;
      }
    }
}

// Prefix rule: returns the node's traveltime (+inf if no neighbour is reached yet),
// writes its derivative codes and its own acceptance key. The groups of equal keys are
// visited in increasing order by repeatedly taking the smallest neighbour key above the
// previous one (no arrays: everything stays in registers on the GPU).
template <int ND>
EIK_HD double prefix_rule(const Nbhd& nb, int8_t* codes, Key* key_out, bool* negdisc) {
#pragma unroll
  for (int a = 0; a < ND; a++) codes[a] = 0;
  Key kg;
  bool have;
  next_key_above<ND>(nb, key_unreached(), false, &kg, &have);
  double vprev = EIK_INF;
  Key kprev = key_unreached();
  int8_t cprev[3] = {0, 0, 0};
  bool first = true;
#pragma unroll 1
  for (int g = 0; g < 2 * ND && have; g++) {
    int8_t cg[3];
    const double v = update_at<ND>(nb, kg, cg, negdisc);
    if (!(v > kg.L) && kg.d >= EIK_MAX_DEPTH && !first) {
      // A cascade of non-causal acceptances deeper than the heap ever produces: the
      // group is ordered after this node (transient of the iteration, not an FMM state).
#pragma unroll
      for (int a = 0; a < ND; a++) codes[a] = cprev[a];
      *key_out = kprev;
      return vprev;
    }
    const Key mine = (v > kg.L) ? key_normal(v) : Key{kg.L, kg.d + 1, v};
#pragma unroll
    for (int a = 0; a < ND; a++) codes[a] = cg[a];
    Key kn;
    bool hn;
    next_key_above<ND>(nb, kg, true, &kn, &hn);
    if (!hn || key_le(mine, kn)) {
      *key_out = mine;
      return v;
    }
    vprev = v;
    kprev = mine;
#pragma unroll
    for (int a = 0; a < ND; a++) cprev[a] = cg[a];
    kg = kn;
    first = false;
  }
  *key_out = key_unreached();
  return EIK_INF;
}

// prefix_rule on a neighbourhood without special keys (NbhdT): the groups are the distinct
// traveltimes of the reached immediate neighbours in increasing order. A group never has a
// depth, so the depth limit of prefix_rule never applies, and its own key is (v, 0, v) when
// the value lies above the group, else (tg, 1, v), accepted right after the group. Same
// value, codes and key as prefix_rule on the same neighbourhood written as an Nbhd.
template <int ND>
EIK_HD double prefix_rule_plain(const NbhdT& nb, int8_t* codes, Key* key_out, bool* negdisc) {
#pragma unroll
  for (int a = 0; a < ND; a++) codes[a] = 0;
  double tg = EIK_INF;
#pragma unroll
  for (int a = 0; a < ND; a++)
#pragma unroll
    for (int l = 0; l < 2; l++)
      if (((nb.in1 >> slot(a, l)) & 1u) && nb.t1[a][l] < tg) tg = nb.t1[a][l];
  if (!(tg < EIK_INF)) {
    *key_out = key_unreached();
    return EIK_INF;
  }
#pragma unroll 1
  for (int g = 0; g < 2 * ND; g++) {
    int8_t cg[3];
    const double v = update_at_g<ND>(nb, tg, cg, negdisc);
#pragma unroll
    for (int a = 0; a < ND; a++) codes[a] = cg[a];
    double tn = EIK_INF;
#pragma unroll
    for (int a = 0; a < ND; a++)
#pragma unroll
      for (int l = 0; l < 2; l++) {
        const double t = nb.t1[a][l];
        if (((nb.in1 >> slot(a, l)) & 1u) && t > tg && t < tn) tn = t;
      }
    const bool above = v > tg;
    if (!(tn < EIK_INF) || !above || v <= tn) {
      *key_out = above ? key_normal(v) : Key{tg, 1, v};
      return v;
    }
    tg = tn;
  }
  *key_out = key_unreached();
  return EIK_INF;
}

// Packed derivative codes: one byte per node, (c0+2) + 5*(c1+2) + 25*(c2+2) in the low
// 7 bits; bit 7 marks a source point (traveltime fixed by the initialisation).
EIK_HD uint8_t pack_codes(const int8_t* c, int nd) {
  int v = (c[0] + 2) + 5 * (c[1] + 2);
  if (nd == 3) v += 25 * (c[2] + 2);
  else v += 25 * 2;
  return (uint8_t)v;
}
EIK_HD void unpack_codes(uint8_t p, int8_t* c) {
  int v = p & 0x7f;
  c[0] = (int8_t)(v % 5 - 2);
  c[1] = (int8_t)((v / 5) % 5 - 2);
  c[2] = (int8_t)((v / 25) % 5 - 2);
}
constexpr uint8_t CODE_SRC_BIT = 0x80;
constexpr uint8_t CODE_NONE = 2 + 5 * 2 + 25 * 2;  // all three codes zero

}  // namespace eik
