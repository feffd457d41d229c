// Discrete adjoint of the forward path and gradient assembly
// (calcgradsomesrc / calcgrads_singlesrc! / solveadjointeq / computestuff_finegrid! /
// calc_duh_dva_finegrid! / calc_dus_dsr* / smoothgradaroundsrc!,
// src/EikSolv/eikmaingrad.jl:174-741, 1140-1273, src/EikSolv/utils.jl:121-338).
//
// The reference assembles the derivative matrices in FMM order and back-substitutes the
// upper-triangular system Jᵀλ = -P_Bᵀr with a sparse solver. Here the same system is solved
// where it lives: row i of J couples node i with the <= 2*nd*2 nodes whose stencil codes
// point at it, so λ_i = (b_i - Σ_r J[r,i] λ_r) / J[i,i] is computed by a tile dataflow the
// moment every downstream λ_r is final (one evaluation per node, no sparse matrices).
// The refined-grid chain rule (the reference's dense N_h x N_acc products) is collapsed by
// linearity into one fine-grid adjoint solve with right-hand side -H_Bᵀz per source.
#include <cstring>
#include <vector>

#include "../../include/eikcuda.h"
#include "node.cuh"
#include "rounds.cuh"
#include "runtime.hpp"

namespace eik {

// λ of a node not computed yet. A NaN payload that arithmetic never produces, so that the
// value and its "final" state travel in one 64-bit word: a reader on another SM sees
// either the sentinel or the final value, never a final flag with a stale value.
constexpr unsigned long long LAM_PENDING_BITS = 0x7ff40000000bad00ull;
__device__ __forceinline__ bool lam_pending(double v) {
  return (unsigned long long)__double_as_longlong(v) == LAM_PENDING_BITS;
}

struct AdjProblem {
  double* lam;   // N: adjoint variable (then the per-source gradient field)
  double* gdt;   // ND x N: 2*(D_a t) of every node's own stencil
  double* rhs;   // N
};

struct AdjArgs {
  SolveArgs sa;
  const AdjProblem* ap;
};

// Stencil coefficients of the derivative matrices (setcoeffderiv!, eikmaingrad.jl:1042-1090;
// createsparsederivativematrices!, eikmainfwd.jl:832-882): point p of a code of magnitude
// abscode, signcod = -sign(code), spacing h of that axis at the node.
__device__ __forceinline__ double dcoeff(int abscode, int p, double h) {
  if (abscode == 1) return p == 0 ? -1.0 / h : 1.0 / h;
  return p == 0 ? -3.0 / (2.0 * h) : (p == 1 ? 4.0 / (2.0 * h) : -1.0 / (2.0 * h));
}

__device__ __forceinline__ bool is_source(const CoarseProblem& P, long long l) {
  return (P.code[l] & CODE_SRC_BIT) && P.kL[l] == -EIK_INF;
}

// ------------------------------------------------------------ per-node preparation --
// Also counts, for every node, the nodes whose stencil reads it (its dependants in Jᵀλ = b)
// and lists the nodes without any for round 0 of the solve.
__global__ void adj_prep_kernel(const CoarseProblem* probs, const AdjProblem* ap, int nprob, long long N,
                                SolveArgs sa) {
  const long long tot = N * nprob;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(q / N);
    const long long l = q - (long long)s * N;
    const CoarseProblem& P = probs[s];
    const AdjProblem& A = ap[s];
    const GridDesc& g = P.g;
    const bool src = is_source(P, l);
    A.lam[l] = src ? 0.0 : __longlong_as_double((long long)LAM_PENDING_BITS);
    A.rhs[l] = 0.0;
    const int i = (int)(l % g.n[0]), j = (int)((l / g.n[0]) % g.n[1]), k = (int)(l / ((long long)g.n[0] * g.n[1]));
    int8_t cd[3];
    unpack_codes(P.code[l], cd);
    double dh[3];
    node_dh(g, i, dh);
    for (int a = 0; a < g.nd; a++) {
      double v = 0.0;
      if (!src && cd[a] != 0) {
        const int ac = cd[a] < 0 ? -cd[a] : cd[a];
        const int sg = cd[a] > 0 ? -1 : 1;
        double tmp1 = 0.0;
        for (int p = ac; p >= 0; p--) {  // the reference sums in ascending FMM column order
          int c[3] = {i, j, k};
          c[a] += sg * p;
          tmp1 += ((double)sg * dcoeff(ac, p, dh[a])) * P.t[lin3(g, c[0], c[1], c[2])];
        }
        v = 2.0 * tmp1;
      }
      A.gdt[(long long)a * N + l] = v;
    }
    int ndep = 0;
    for (int ax = 0; ax < g.nd; ax++)
      for (int dl = -2; dl <= 2; dl++) {
        if (dl == 0) continue;
        int pr[3] = {i, j, k};
        pr[ax] += dl;
        if (pr[ax] < 0 || pr[ax] >= g.n[ax]) continue;
        int8_t cr[3];
        unpack_codes(P.code[lin3(g, pr[0], pr[1], pr[2])], cr);
        const int cc = cr[ax];
        if (cc == 0) continue;
        const int ac = cc < 0 ? -cc : cc;
        const int p = -dl * (cc > 0 ? -1 : 1);
        if (p >= 1 && p <= ac) ndep++;
      }
    sa.rs.stamp[q] = ndep;
    if (ndep == 0 && !src) {
      const unsigned int at = atomicAdd(sa.rs.cnt, 1u);
      sa.rs.list[0][at] = (unsigned long long)q << 32;
    }
  }
}

// J[r, i] for node r = i + delta*e_a if r's stencil contains i, else 0 (and *is_down=false).
__device__ __forceinline__ double jcoef(const GridDesc& g, const uint8_t* code, const double* gdt, long long N,
                                        int a, int delta, long long lr, int ir, bool* is_down) {
  *is_down = false;
  int8_t cd[3];
  unpack_codes(code[lr], cd);
  const int c = cd[a];
  if (c == 0) return 0.0;
  const int ac = c < 0 ? -c : c;
  const int sg = c > 0 ? -1 : 1;
  const int p = -delta * sg;  // r + sg*p*e_a == i
  if (p < 1 || p > ac) return 0.0;
  *is_down = true;
  double dh[3];
  node_dh(g, ir, dh);
  return gdt[(long long)a * N + lr] * ((double)sg * dcoeff(ac, p, dh[a]));
}

__device__ __forceinline__ double jdiag(const GridDesc& g, const uint8_t* code, const double* gdt, long long N,
                                        long long l, int i) {
  int8_t cd[3];
  unpack_codes(code[l], cd);
  double dh[3];
  node_dh(g, i, dh);
  double s = 0.0;
  bool first = true;
  for (int a = 0; a < g.nd; a++) {
    if (cd[a] == 0) continue;
    const int ac = cd[a] < 0 ? -cd[a] : cd[a];
    const int sg = cd[a] > 0 ? -1 : 1;
    const double v = gdt[(long long)a * N + l] * ((double)sg * dcoeff(ac, 0, dh[a]));
    s = first ? v : s + v;
    first = false;
  }
  return s;
}

// --------------------------------------------------------- receivers: misfit, rhs --
struct RecvArgs {
  GridDesc g;
  int nsrc;
  const CoarseProblem* probs;
  const AdjProblem* ap;
  const long long* recoff;
  const double* rec;
  const double* pickobs;
  const double* stdobs;
  const ForwardBatch* fb;
  double* misfit;   // nsrc
  double* dpsi;     // nsrc x seedcap: ∂ψ/∂u_s per source point
};

__device__ int interp_corners(const GridDesc& g, const double* p, double* coeff, long long* node) {
  if (g.nd == 2) {
    const double xh = (p[0] - g.co[0]) / g.spac[0], yh = (p[1] - g.co[1]) / g.spac[1];
    long long i = (long long)floor(xh + 1), j = (long long)floor(yh + 1);
    if (i == g.n[0]) i -= 1;
    else if (i > g.n[0]) i -= 2;
    if (j == g.n[1]) j -= 1;
    else if (j > g.n[1]) j -= 2;
    const double xd = xh - (double)(i - 1), yd = yh - (double)(j - 1);
    coeff[0] = (1.0 - xd) * (1.0 - yd);
    coeff[1] = (1.0 - yd) * xd;
    coeff[2] = (1.0 - xd) * yd;
    coeff[3] = xd * yd;
    const int o[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};
    for (int c = 0; c < 4; c++) node[c] = lin3(g, (int)i - 1 + o[c][0], (int)j - 1 + o[c][1], 0);
    return 4;
  }
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
  coeff[0] = (1 - xd) * (1 - yd) * (1 - zd);
  coeff[1] = xd * (1 - yd) * (1 - zd);
  coeff[2] = (1 - xd) * yd * (1 - zd);
  coeff[3] = (1 - xd) * (1 - yd) * zd;
  coeff[4] = xd * yd * (1 - zd);
  coeff[5] = (1 - xd) * yd * zd;
  coeff[6] = xd * (1 - yd) * (1 - zd);  // eikforward3D.jl:102
  coeff[7] = xd * yd * zd;
  const int o[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0}, {0, 1, 1}, {1, 0, 1}, {1, 1, 1}};
  for (int c = 0; c < 8; c++) node[c] = lin3(g, (int)i - 1 + o[c][0], (int)j - 1 + o[c][1], (int)k - 1 + o[c][2]);
  return 8;
}

__device__ int seed_index(const ForwardBatch& fb, int s, long long node) {
  const int ns = fb.out[s].nseeds;
  const int32_t* sl = fb.seed_lin + (size_t)s * fb.seedcap;
  for (int k = 0; k < ns; k++)
    if (sl[k] == node) return k;
  return -1;
}

// One thread per source, receivers in order (deterministic sums).
__global__ void adj_recv_kernel(RecvArgs ra) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ra.nsrc) return;
  const GridDesc& g = ra.g;
  const CoarseProblem& P = ra.probs[s];
  const AdjProblem& A = ra.ap[s];
  const ForwardBatch& fb = *ra.fb;
  double* dpsi = ra.dpsi + (size_t)s * fb.seedcap;
  for (int k = 0; k < fb.out[s].nseeds; k++) dpsi[k] = 0.0;
  double misf = 0.0;
  for (long long r = ra.recoff[s]; r < ra.recoff[s + 1]; r++) {
    double coeff[8];
    long long node[8];
    const int nc = interp_corners(g, ra.rec + r * g.nd, coeff, node);
    double pick = 0.0;
    for (int c = 0; c < nc; c++) pick += coeff[c] * P.t[node[c]];
    const double pd = pick - ra.pickobs[r];
    const double sd2 = ra.stdobs[r] * ra.stdobs[r];
    misf += (pd * pd) / sd2;
    const double fact = pd / sd2;
    for (int c = 0; c < nc; c++) {
      if (is_source(P, node[c])) {
        const int k = seed_index(fb, s, node[c]);
        if (k >= 0) dpsi[k] += coeff[c] * fact;
      } else {
        A.rhs[node[c]] += (-coeff[c]) * fact;
      }
    }
  }
  ra.misfit[s] = misf;
}

// ------------------------------------------------------------- adjoint solve --
// Jᵀλ = b in topological order of the stencil graph (Kahn): round r takes the nodes whose
// dependants are all final, computes
//   λ_i = (b_i − Σ_{r reads i} J[r,i] λ_r) / J[i,i]
// pulling the dependants' λ in a fixed order (deterministic), then releases the nodes its
// own stencil reads; a node whose dependant count drops to zero is listed for the next
// round. Every node is computed exactly once, after everything it depends on.
__global__ void adj_rounds_init_kernel(SolveArgs a) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int k = 0; k < 3; k++) {
    a.rs.cnt[k] = 0;
    a.rs.grab[k] = 0;
  }
  a.rs.bar[0] = 0;
  a.rs.bar[1] = 0;
  *a.rs.rounds = 0;
  *a.abort_flag = 0;
}

// The node's solve is a chain of dependent L2 round trips; its loads go out in batches: the
// codes of the node and of the 4*ND nodes that may read it (with the right-hand side), then
// per axis the coefficient and λ of the dependants on that axis. The terms are subtracted
// in the same fixed order as they would be one by one (axis, then offset -2, -1, +1, +2).
// Everything read here was written before this node was listed (the forward's codes and
// coefficients, and the dependants' λ, each released only after its store and a fence).
template <int ND>
__device__ void adj_node(const AdjArgs& aa, int prob, long long l, unsigned long long gb, unsigned int* rel) {
  const SolveArgs& a = aa.sa;
  const CoarseProblem& P = a.probs[prob];
  const AdjProblem& A = aa.ap[prob];
  const GridDesc& g = P.g;
  const long long N = npts(g);
  int c[3];
  node_coords(g, l, c);
  long long nl[ND][4];
  uint8_t ncode[ND][4];
#pragma unroll
  for (int ax = 0; ax < ND; ax++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int dl = j < 2 ? j - 2 : j - 1;
      nl[ax][j] = -1;
      if (c[ax] + dl < 0 || c[ax] + dl >= g.n[ax]) continue;
      int pr[3] = {c[0], c[1], c[2]};
      pr[ax] += dl;
      nl[ax][j] = lin3(g, pr[0], pr[1], pr[2]);
    }
  const uint8_t cb = P.code[l];
  const double rhs = A.rhs[l];
#pragma unroll
  for (int ax = 0; ax < ND; ax++)
#pragma unroll
    for (int j = 0; j < 4; j++) ncode[ax][j] = nl[ax][j] >= 0 ? P.code[nl[ax][j]] : (uint8_t)CODE_NONE;
  int8_t cm[3];
  unpack_codes(cb, cm);
  if ((cb & CODE_SRC_BIT) && P.kL[l] == -EIK_INF) return;  // source points: no unknown
  double sum = rhs;
  double dh[3];
  double gself[ND];
#pragma unroll
  for (int ax = 0; ax < ND; ax++) gself[ax] = A.gdt[(long long)ax * N + l];
#pragma unroll
  for (int ax = 0; ax < ND; ax++) {
    double gv[4], lv[4];
    int pp[4], acc4[4], sg4[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int dl = j < 2 ? j - 2 : j - 1;
      pp[j] = 0;
      if (nl[ax][j] < 0) continue;
      int8_t cd[3];
      unpack_codes(ncode[ax][j], cd);
      const int cc = cd[ax];
      if (cc == 0) continue;
      const int ac = cc < 0 ? -cc : cc;
      const int sg = cc > 0 ? -1 : 1;
      const int p = -dl * sg;
      if (p < 1 || p > ac) continue;
      pp[j] = p;
      acc4[j] = ac;
      sg4[j] = sg;
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      gv[j] = pp[j] ? A.gdt[(long long)ax * N + nl[ax][j]] : 0.0;
      lv[j] = pp[j] ? __ldcg(A.lam + nl[ax][j]) : 0.0;
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      if (!pp[j]) continue;
      const int dl = j < 2 ? j - 2 : j - 1;
      node_dh(g, c[0] + (ax == 0 ? dl : 0), dh);
      const double J = gv[j] * ((double)sg4[j] * dcoeff(acc4[j], pp[j], dh[ax]));
      sum -= J * lv[j];
    }
  }
  node_dh(g, c[0], dh);
  double dg = 0.0;
  bool first = true;
#pragma unroll
  for (int ax = 0; ax < ND; ax++) {
    if (cm[ax] == 0) continue;
    const int ac = cm[ax] < 0 ? -cm[ax] : cm[ax];
    const int sg = cm[ax] > 0 ? -1 : 1;
    const double v = gself[ax] * ((double)sg * dcoeff(ac, 0, dh[ax]));
    dg = first ? v : dg + v;
    first = false;
  }
  A.lam[l] = sum / dg;
  __threadfence();
  // release the nodes this node's stencil reads
#pragma unroll
  for (int ax = 0; ax < ND; ax++) {
    const int ac = cm[ax] < 0 ? -cm[ax] : cm[ax];
    const int sg = cm[ax] > 0 ? -1 : 1;
    for (int p = 1; p <= ac; p++) {
      int q[3] = {c[0], c[1], c[2]};
      q[ax] += sg * p;
      const long long lu = lin3(g, q[0], q[1], q[2]);
      if (atomicSub(a.rs.stamp + gb + lu, 1) == 1) rel[2 * ax + p - 1] = (unsigned int)(gb + lu);
    }
  }
}

template <int ND>
__global__ void __launch_bounds__(SOLVE_THREADS) adj_rounds_kernel(AdjArgs aa) {
  const SolveArgs& a = aa.sa;
  const int lane = threadIdx.x & 31;
  const unsigned long long N = (unsigned long long)npts(a.probs[0].g);
  int r = 0;
  for (; r < a.rs.max_rounds; r++) {
    const int b3 = r % 3;
    const unsigned int n = *(volatile unsigned int*)(a.rs.cnt + b3);
    if (n == 0) break;
    const unsigned long long* L = a.rs.list[r & 1];
    for (;;) {
      unsigned int base = 0;
      if (lane == 0) base = atomicAdd(a.rs.grab + b3, 32u);
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= n) break;
      const unsigned int idx = base + lane;
      unsigned int rel[6] = {~0u, ~0u, ~0u, ~0u, ~0u, ~0u};
      if (idx < n) {
        const unsigned int gid = (unsigned int)(__ldcg(L + idx) >> 32);
        const int prob = (int)(gid / N);
        const unsigned long long gb = (unsigned long long)prob * N;
        adj_node<ND>(aa, prob, (long long)(gid - gb), gb, rel);
      }
#pragma unroll
      for (int k = 0; k < 2 * ND; k++) warp_append(a, r + 1, rel[k] != ~0u, rel[k]);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      const int c3 = (r + 2) % 3;
      a.rs.cnt[c3] = 0;
      a.rs.grab[c3] = 0;
    }
    if (!grid_barrier(a)) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *a.rs.rounds = r;
    if (r >= a.rs.max_rounds) {
      atomicOr(a.err, ERRB_ADJ_NOT_CONVERGED);
      atomicExch(a.abort_flag, 1);
    }
  }
}

__global__ void adj_check_kernel(const AdjProblem* ap, int nprob, long long N, uint32_t* err) {
  const long long tot = N * nprob;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(q / N);
    const double v = ap[s].lam[q - (long long)s * N];
    if (lam_pending(v)) atomicOr(err, ERRB_ADJ_NOT_CONVERGED);
    else if (!(fabs(v) <= 1.7976931348623157e308)) atomicOr(err, ERRB_SINGULAR);
  }
}

// ------------------------------------------------------ source-region contributions --
struct SrcTermArgs {
  GridDesc g;
  int nsrc;
  int refine;
  int whichgrad;
  const int32_t* gstart;  // per source of the whole call: first source of its group (own gradient buffer)
  int s0;               // index, in the whole call, of this chunk's first source
  int nsrc_total;       // sources of the whole call (groups are those of the whole call)
  const double* prevbuf;  // N: the group buffer before this chunk (its previous source's final field), or null
  const CoarseProblem* probs;
  const AdjProblem* ap;
  const ForwardBatch* fb;
  const double* vel;
  const double* coordsrc;
  const double* dpsi;   // nsrc x seedcap: ∂ψ/∂u_s
  double* ysrc;         // nsrc x seedcap: ∂ψ/∂u_p ∂u_p/∂u_s
  double* gsrcnode;     // nsrc x seedcap: T2Va + T1Va at the source points
  double* gradsrc;      // nsrc x nd
  double* fine_lam;     // nsrc x nfmax
  double* fine_gdt;     // nsrc x nd x nfmax
  uint32_t* warn;
};

// partderivttsrcpos (eikmaingrad.jl:1235-1273)
__device__ void partderiv(int nd, const double* xyzpt, const double* inpsrc, double vel, double hgrid,
                          double* der, uint32_t* warn) {
  const double shift = 1e-6 * hgrid;
  double src[3];
  for (int d = 0; d < nd; d++) {
    double r = fmod(inpsrc[d], hgrid);  // Base.mod: result takes the sign of the divisor
    if (r == 0.0) r = copysign(0.0, hgrid);
    else if ((r > 0) != (hgrid > 0)) r += hgrid;
    if (r <= 2.220446049250313e-16) {
      src[d] = inpsrc[d] + shift;
      *warn |= WARN_SRCPOS_ALIGNED_SHIFT;
    } else {
      src[d] = inpsrc[d];
    }
  }
  double ss = 0.0;
  for (int d = 0; d < nd; d++) {
    const double t = xyzpt[d] - src[d];
    ss = (d == 0) ? t * t : ss + t * t;
  }
  const double denom = vel * sqrt(ss);
  if (denom == 0.0) {
    *warn |= WARN_SRC_ON_NODE_DERIV;
    for (int d = 0; d < nd; d++) der[d] = 0.0;
    return;
  }
  for (int d = 0; d < nd; d++) der[d] = -(xyzpt[d] - src[d]) / denom;
}

// y_k = Σ_r J[r, k] λ_r over the nodes whose stencil contains source point k.
__global__ void adj_ysrc_kernel(SrcTermArgs sa) {
  const int s = blockIdx.x;
  const ForwardBatch& fb = *sa.fb;
  const CoarseProblem& P = sa.probs[s];
  const AdjProblem& A = sa.ap[s];
  const GridDesc& g = sa.g;
  const long long N = npts(g);
  for (int k = threadIdx.x; k < fb.out[s].nseeds; k += blockDim.x) {
    const long long l = fb.seed_lin[(size_t)s * fb.seedcap + k];
    const int c[3] = {(int)(l % g.n[0]), (int)((l / g.n[0]) % g.n[1]), (int)(l / ((long long)g.n[0] * g.n[1]))};
    double y = 0.0;
    for (int ax = 0; ax < g.nd; ax++)
      for (int dl = -2; dl <= 2; dl++) {
        if (dl == 0) continue;
        int pr[3] = {c[0], c[1], c[2]};
        pr[ax] += dl;
        if (pr[ax] < 0 || pr[ax] >= g.n[ax]) continue;
        const long long lr = lin3(g, pr[0], pr[1], pr[2]);
        if (is_source(P, lr)) continue;
        bool down;
        const double J = jcoef(g, P.code, A.gdt, N, ax, dl, lr, pr[0], &down);
        if (down) y += J * A.lam[lr];
      }
    sa.ysrc[(size_t)s * fb.seedcap + k] = y;
  }
}

// Refined-grid geometry of a source, rebuilt from its window (as in the start-up stage).
__device__ void fine_grid_of(const GridDesc& g, const FineInfo& fi, GridDesc* gf) {
  *gf = g;
  for (int d = 0; d < 3; d++) gf->n[d] = fi.nf[d];
  for (int d = 0; d < g.nd; d++) {
    gf->spac[d] = g.spac[d] / (double)fi.ds;
    gf->co[d] = jr_value(g.ax[d], fi.ijk1[d] + 1);
    gf->ax[d] = make_jrange(gf->co[d], gf->spac[d]);
  }
}

// Coarse node nearest to a fine node along one axis (eikmainfwd.jl:1035-1051), window-local.
__device__ __forceinline__ int fine_nn_axis(const FineInfo& fi, int f) {
  const int di = f / fi.ds;
  const int ri = f + 1 - di * fi.ds;
  return ((double)ri >= (double)fi.ds / 2.0 + 1.0) ? di + 1 : di;
}

__device__ __forceinline__ long long fine_nn_coarse(const GridDesc& g, const FineInfo& fi, long long lf,
                                                    const GridDesc& gf) {
  const int f[3] = {(int)(lf % gf.n[0]), (int)((lf / gf.n[0]) % gf.n[1]), (int)(lf / ((long long)gf.n[0] * gf.n[1]))};
  int c[3] = {0, 0, 0};
  for (int d = 0; d < g.nd; d++) c[d] = fi.ijk1[d] + fine_nn_axis(fi, f[d]);
  return lin3(g, c[0], c[1], c[2]);
}

// 2*(D_a t)_r of a fine node from its stored code and the fine traveltimes.
__device__ double fine_gdt_of(const GridDesc& gf, const double* tt, const uint8_t* code, long long lr, int a) {
  int8_t cd[3];
  unpack_codes(code[lr], cd);
  if (cd[a] == 0) return 0.0;
  const int ac = cd[a] < 0 ? -cd[a] : cd[a];
  const int sg = cd[a] > 0 ? -1 : 1;
  const int c[3] = {(int)(lr % gf.n[0]), (int)((lr / gf.n[0]) % gf.n[1]), (int)(lr / ((long long)gf.n[0] * gf.n[1]))};
  double dh[3];
  node_dh(gf, c[0], dh);
  double tmp1 = 0.0;
  for (int p = ac; p >= 0; p--) {
    int q[3] = {c[0], c[1], c[2]};
    q[a] += sg * p;
    tmp1 += ((double)sg * dcoeff(ac, p, dh[a])) * tt[lin3(gf, q[0], q[1], q[2])];
  }
  return 2.0 * tmp1;
}

// Fine node states during the adjoint: 2 accepted, 3 accepted with a final λ.
constexpr uint8_t FST_FINAL = 3;

// Σ_r Jf[r, l] λf_r over the accepted fine nodes whose stencil contains l; *ready is
// false while one of them has no final λ yet.
__device__ double fine_downsum(const GridDesc& gf, const uint8_t* st, const uint8_t* code, const double* fgdt,
                               long long nfmax, const double* lamf, long long l, bool* ready) {
  const int c[3] = {(int)(l % gf.n[0]), (int)((l / gf.n[0]) % gf.n[1]), (int)(l / ((long long)gf.n[0] * gf.n[1]))};
  double sum = 0.0;
  *ready = true;
  for (int ax = 0; ax < gf.nd; ax++)
    for (int dl = -2; dl <= 2; dl++) {
      if (dl == 0) continue;
      int pr[3] = {c[0], c[1], c[2]};
      pr[ax] += dl;
      if (pr[ax] < 0 || pr[ax] >= gf.n[ax]) continue;
      const long long lr = lin3(gf, pr[0], pr[1], pr[2]);
      const uint8_t sr = st[lr];
      if (sr < 2) continue;
      int8_t cd[3];
      unpack_codes(code[lr], cd);
      const int cc = cd[ax];
      if (cc == 0) continue;
      const int ac = cc < 0 ? -cc : cc;
      const int sg = cc > 0 ? -1 : 1;
      const int p = -dl * sg;
      if (p < 1 || p > ac) continue;
      if (sr != FST_FINAL) {
        *ready = false;
        return 0.0;
      }
      double dh[3];
      node_dh(gf, pr[0], dh);
      const double J = fgdt[(long long)ax * nfmax + lr] * ((double)sg * dcoeff(ac, p, dh[ax]));
      sum += J * lamf[lr];
    }
  return sum;
}

__device__ double fine_diag(const GridDesc& gf, const uint8_t* code, const double* fgdt, long long nfmax, long long l) {
  int8_t cm[3];
  unpack_codes(code[l], cm);
  double dh[3];
  node_dh(gf, (int)(l % gf.n[0]), dh);
  double dg = 0.0;
  bool first = true;
  for (int ax = 0; ax < gf.nd; ax++) {
    if (cm[ax] == 0) continue;
    const int ac = cm[ax] < 0 ? -cm[ax] : cm[ax];
    const int sg = cm[ax] > 0 ? -1 : 1;
    const double v = fgdt[(long long)ax * nfmax + l] * ((double)sg * dcoeff(ac, 0, dh[ax]));
    dg = first ? v : dg + v;
    first = false;
  }
  return dg;
}

// Source-region terms T2Va + T1Va (eikmaingrad.jl:428-479) and the source-location
// gradient (eikmaingrad.jl:362-399); one warp per source.
// With refinement the reference solves the fine adjoint for one right-hand side per coarse
// source point and contracts the results with z = ∂ψ∂up_∂up∂us + ∂ψ_∂u_s
// (computestuff_finegrid!, calc_duh_dva_finegrid!, eikmaingrad.jl:540-741). By linearity
// the same numbers come from ONE fine adjoint solve with right-hand side -z on the
// coarse-coincident fine nodes, done here in reverse fine FMM order, 32 positions at a time.
__global__ void __launch_bounds__(32) adj_srcterm_kernel(SrcTermArgs sa) {
  const int s = blockIdx.x;
  const int lane = threadIdx.x;
  const ForwardBatch& fb = *sa.fb;
  const SrcOut& o = fb.out[s];
  const GridDesc& g = sa.g;
  const double* y = sa.ysrc + (size_t)s * fb.seedcap;
  const double* dpsi = sa.dpsi + (size_t)s * fb.seedcap;
  double* gnode = sa.gsrcnode + (size_t)s * fb.seedcap;
  const double* src = sa.coordsrc + (size_t)s * g.nd;
  uint32_t warn = 0;
  const bool wantvel = sa.whichgrad == 1 || sa.whichgrad == 3;
  const bool wantsrc = sa.whichgrad == 2 || sa.whichgrad == 3;
  if (!sa.refine) {
    for (int k = lane; k < o.nseeds; k += 32) {
      const double dd = (-o.distcorn[k]) * (1.0 / (o.velcorn[k] * o.velcorn[k]));
      gnode[k] = dd * y[k] + dd * dpsi[k];
    }
    if (wantsrc && lane == 0) {
      double gs[3] = {0.0, 0.0, 0.0}, gs2[3] = {0.0, 0.0, 0.0};
      for (int k = 0; k < o.nseeds; k++) {
        double xyz[3], der[3];
        for (int d = 0; d < g.nd; d++) xyz[d] = jr_value(g.ax[d], o.corn[k][d] + 1);
        partderiv(g.nd, xyz, src, o.velcorn[k], g.spac[0], der, &warn);
        for (int d = 0; d < g.nd; d++) {
          gs[d] += der[d] * y[k];
          gs2[d] += der[d] * dpsi[k];
        }
      }
      for (int d = 0; d < g.nd; d++) sa.gradsrc[(size_t)s * g.nd + d] = gs[d] + gs2[d];
    }
    if (warn) atomicOr(sa.warn, warn);
    return;
  }
  __shared__ double qcorn[8];
  GridDesc gf;
  fine_grid_of(g, o.fine, &gf);
  const long long nfmax = fb.nfmax;
  const double* tt = fb.fine_tt + (size_t)s * nfmax;
  uint8_t* st = fb.fine_status + (size_t)s * nfmax;
  const uint8_t* code = fb.fine_code + (size_t)s * nfmax;
  const int32_t* order = fb.fine_order + (size_t)s * nfmax;
  const uint8_t* onh = fb.fine_onh + (size_t)s * nfmax;
  int32_t* hk = fb.fine_idx + (size_t)s * nfmax;  // fine node -> coarse source point index
  double* lamf = sa.fine_lam + (size_t)s * nfmax;
  double* fgdt = sa.fine_gdt + (size_t)s * g.nd * nfmax;
  const int nacc = o.nacc, nsf = o.nsrcf;
  // rows of the fine system and the coarse-point numbering (FMM order of the h points)
  int run = 0;
  for (int b = 0; b < nacc; b += 32) {
    const int p = b + lane;
    long long l = 0;
    bool h = false;
    if (p < nacc) {
      l = order[p];
      lamf[l] = 0.0;
      for (int a = 0; a < g.nd; a++) fgdt[(long long)a * nfmax + l] = (p >= nsf) ? fine_gdt_of(gf, tt, code, l, a) : 0.0;
      h = onh[l] != 0;
    }
    const unsigned m = __ballot_sync(0xffffffffu, h);
    if (p < nacc) hk[l] = h ? run + __popc(m & ((1u << lane) - 1u)) : -1;
    run += __popc(m);
  }
  __syncwarp();
  // reverse sweep: the largest unfinished position of a window is always ready
  for (int b = nacc - 1; b >= nsf; b -= 32) {
    const int p = b - lane;
    const long long l = (p >= nsf) ? order[p] : -1;
    bool done = p < nsf;
    for (int round = 0; round <= 32; round++) {
      double nv = 0.0;
      bool go = false;
      if (!done) {
        bool ready;
        const double sum = fine_downsum(gf, st, code, fgdt, nfmax, lamf, l, &ready);
        if (ready) {
          const int k = hk[l];
          const double rhs = (k >= 0) ? -(y[k] + dpsi[k]) : 0.0;
          nv = (rhs - sum) / fine_diag(gf, code, fgdt, nfmax, l);
          go = true;
        }
      }
      __syncwarp();
      if (go) {
        lamf[l] = nv;
        st[l] = FST_FINAL;
        done = true;
      }
      __syncwarp();
      if (__all_sync(0xffffffffu, done)) break;
    }
  }
  // per source-box corner: (∂g/∂τ_s)ᵀ λf + H_Aᵀ z
  if (lane < nsf) {
    const long long l = order[lane];
    bool ready;
    const double sum = fine_downsum(gf, st, code, fgdt, nfmax, lamf, l, &ready);
    const int k = hk[l];
    qcorn[lane] = sum + ((k >= 0) ? (y[k] + dpsi[k]) : 0.0);
  }
  __syncwarp();
  if (wantvel) {
    // duh_dwq contracted with z, then summed onto the nearest coarse node of each accepted
    // fine node (dwq_dva, eikmaingrad.jl:716-738): here in place in lamf
    for (int p = lane; p < nacc; p += 32) {
      const long long l = order[p];
      if (p < nsf) {
        const double dd = (-o.distcorn[p]) * (1.0 / (o.velcorn[p] * o.velcorn[p]));
        lamf[l] = dd * qcorn[p];
      } else {
        const double v = sa.vel[fine_nn_coarse(g, o.fine, l, gf)];
        lamf[l] = 2.0 * lamf[l] / (v * v * v);
      }
    }
    __syncwarp();
    for (int k = lane; k < o.nseeds; k += 32) {
      const long long cl = fb.seed_lin[(size_t)s * fb.seedcap + k];
      const int c[3] = {(int)(cl % g.n[0]), (int)((cl / g.n[0]) % g.n[1]), (int)(cl / ((long long)g.n[0] * g.n[1]))};
      int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
      for (int d = 0; d < g.nd; d++) {
        const int cc = c[d] - o.fine.ijk1[d];
        lo[d] = max(0, (cc - 1) * o.fine.ds);
        hi[d] = min(gf.n[d] - 1, (cc + 1) * o.fine.ds);
      }
      double acc = 0.0;
      for (int fz = lo[2]; fz <= hi[2]; fz++) {
        if (g.nd == 3 && fine_nn_axis(o.fine, fz) != c[2] - o.fine.ijk1[2]) continue;
        for (int fy = lo[1]; fy <= hi[1]; fy++) {
          if (fine_nn_axis(o.fine, fy) != c[1] - o.fine.ijk1[1]) continue;
          for (int fx = lo[0]; fx <= hi[0]; fx++) {
            if (fine_nn_axis(o.fine, fx) != c[0] - o.fine.ijk1[0]) continue;
            const long long lf = lin3(gf, fx, fy, fz);
            if (st[lf] >= 2) acc += lamf[lf];
          }
        }
      }
      gnode[k] = acc;
    }
  }
  if (wantsrc && lane == 0) {
    double gsv[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < nsf; k++) {
      double xyz[3], der[3];
      for (int d = 0; d < g.nd; d++) xyz[d] = jr_value(gf.ax[d], o.corn[k][d] + 1);
      partderiv(g.nd, xyz, src, o.velcorn[k], gf.spac[0], der, &warn);
      for (int d = 0; d < g.nd; d++) gsv[d] += der[d] * qcorn[k];
    }
    for (int d = 0; d < g.nd; d++) sa.gradsrc[(size_t)s * g.nd + d] = gsv[d];
  }
  if (warn) atomicOr(sa.warn, warn);
}

// ------------------------------------------------------------- gradient assembly --
// Per-source field G_s: 2λ/v³ off the source points (eikmaingrad.jl:417-423).
__global__ void adj_field_kernel(SrcTermArgs sa, long long N) {
  const long long tot = N * sa.nsrc;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(q / N);
    const long long l = q - (long long)s * N;
    const AdjProblem& A = sa.ap[s];
    if (is_source(sa.probs[s], l)) continue;
    const double v = sa.vel[l];
    A.lam[l] = 2.0 * A.lam[l] / (v * v * v);
  }
}

// smoothgradaroundsrc! factor of the source at src for node (i,j,k) (utils.jl:121-338),
// with the reference's k-range built from the x index for off-grid 3D sources.
__device__ double smooth_factor(const GridDesc& g, const double* src, int R, int i, int j, int k) {
  if (R == 0) return 1.0;
  int corn[8][3];
  const int nc = findenclosingbox(g, src, corn);
  int imin, imax, jmin, jmax, kmin = 0, kmax = 0;
  if (nc == 1) {
    imin = corn[0][0] - R;
    imax = corn[0][0] + R;
    jmin = corn[0][1] - R;
    jmax = corn[0][1] + R;
    if (g.nd == 3) {
      kmin = corn[0][2] - R;
      kmax = corn[0][2] + R;
    }
  } else {
    imin = corn[0][0] - R;
    imax = corn[1][0] + R;
    jmin = corn[0][1] - R;
    jmax = corn[2][1] + R;
    if (g.nd == 3) {
      kmin = corn[0][0] - R;
      kmax = corn[3][0] + R;
    }
  }
  if (i < imin || i > imax || j < jmin || j > jmax) return 1.0;
  if (g.nd == 3 && (k < kmin || k > kmax)) return 1.0;
  const double rmax = (double)R * g.spac[0];
  double xs[3] = {0, 0, 0}, xc[3] = {0, 0, 0};
  if (is_cart(g)) {
    for (int d = 0; d < g.nd; d++) xs[d] = src[d];
    xc[0] = jr_value(g.ax[0], i + 1);
    xc[1] = jr_value(g.ax[1], j + 1);
    if (g.nd == 3) xc[2] = jr_value(g.ax[2], k + 1);
  } else if (g.nd == 2) {
    double sn, cs;
    sincosd(src[1], &sn, &cs);
    xs[0] = src[0] * cs;
    xs[1] = src[0] * sn;
    const double r = jr_value(g.ax[0], i + 1), th = jr_value(g.ax[1], j + 1);
    sincosd(th, &sn, &cs);
    xc[0] = r * cs;
    xc[1] = r * sn;
  } else {
    double st, ct, sp, cp;
    sincosd(src[1], &st, &ct);
    sincosd(src[2], &sp, &cp);
    xs[0] = src[0] * st * cp;
    xs[1] = src[0] * st * sp;
    xs[2] = src[0] * ct;
    const double r = jr_value(g.ax[0], i + 1), th = jr_value(g.ax[1], j + 1), ph = jr_value(g.ax[2], k + 1);
    sincosd(th, &st, &ct);
    sincosd(ph, &sp, &cp);
    xc[0] = r * st * cp;
    xc[1] = r * st * sp;
    xc[2] = r * ct;
  }
  double r;
  if (g.nd == 2) {
    const double a = xc[0] - xs[0], b = xs[1] - xc[1];
    r = sqrt(a * a + b * b);
  } else {
    const double a = xc[0] - xs[0], b = xs[1] - xc[1], e = xs[2] - xc[2];
    r = sqrt((a * a + b * b) + e * e);
  }
  return (r <= rmax) ? r / rmax : 1.0;
}

// The reference keeps one gradient buffer per source group and assigns only off the
// current source's points (eikmaingrad.jl:182, 417-479), so a source point starts from
// the previous source's smoothed value there. The carried value is a short recurrence over
// the run of earlier sources sharing the point; one thread per (source, point).
//
// A call split into chunks of sources runs this per chunk with the sources numbered within
// the chunk: a group that began in an earlier chunk starts here from the buffer as the
// previous chunk left it (prevbuf: its last source's final field), which is the value the
// recurrence over the earlier sources produces.
__global__ void adj_carry_kernel(SrcTermArgs sa, int R, double* carry) {
  const int s = blockIdx.x;
  const ForwardBatch& fb = *sa.fb;
  const GridDesc& g = sa.g;
  const int gs = sa.gstart[sa.s0 + s] - sa.s0;  // < 0: began in an earlier chunk
  const int lo = gs > 0 ? gs : 0;
  for (int k = threadIdx.x; k < fb.out[s].nseeds; k += blockDim.x) {
    const long long l = fb.seed_lin[(size_t)s * fb.seedcap + k];
    const int i = (int)(l % g.n[0]), j = (int)((l / g.n[0]) % g.n[1]), kz = (int)(l / ((long long)g.n[0] * g.n[1]));
    int m = s - 1;
    while (m >= lo && seed_index(fb, m, l) >= 0) m--;
    double c = 0.0;
    if (m >= lo) c = smooth_factor(g, sa.coordsrc + (size_t)m * g.nd, R, i, j, kz) * sa.ap[m].lam[l];
    else if (gs < 0 && sa.prevbuf) c = sa.prevbuf[l];
    for (int q = m + 1; q < s; q++) {
      const int kq = seed_index(fb, q, l);
      c = smooth_factor(g, sa.coordsrc + (size_t)q * g.nd, R, i, j, kz) * (c + sa.gsrcnode[(size_t)q * fb.seedcap + kq]);
    }
    carry[(size_t)s * fb.seedcap + k] = c;
  }
}

__global__ void adj_srcnodes_kernel(SrcTermArgs sa, const double* carry) {
  const int s = blockIdx.x;
  const ForwardBatch& fb = *sa.fb;
  for (int k = threadIdx.x; k < fb.out[s].nseeds; k += blockDim.x) {
    const long long l = fb.seed_lin[(size_t)s * fb.seedcap + k];
    sa.ap[s].lam[l] = carry[(size_t)s * fb.seedcap + k] + sa.gsrcnode[(size_t)s * fb.seedcap + k];
  }
}

__global__ void adj_smooth_kernel(SrcTermArgs sa, int R) {
  const int s = blockIdx.x;
  const GridDesc& g = sa.g;
  const double* src = sa.coordsrc + (size_t)s * g.nd;
  int corn[8][3];
  const int nc = findenclosingbox(g, src, corn);
  int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  for (int d = 0; d < g.nd; d++) {
    int mn = corn[0][d], mx = corn[0][d];
    for (int c = 1; c < nc; c++) {
      mn = min(mn, corn[c][d]);
      mx = max(mx, corn[c][d]);
    }
    lo[d] = max(0, mn - R);
    hi[d] = min(g.n[d] - 1, mx + R);
  }
  if (g.nd == 3 && nc > 1) {  // k-range from the x index (utils.jl:257-258)
    lo[2] = max(0, corn[0][0] - R);
    hi[2] = min(g.n[2] - 1, corn[3][0] + R);
  }
  const int nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
  if (nx <= 0 || ny <= 0 || nz <= 0) return;
  for (int q = threadIdx.x; q < nx * ny * nz; q += blockDim.x) {
    const int i = lo[0] + q % nx, j = lo[1] + (q / nx) % ny, k = lo[2] + q / (nx * ny);
    const double f = smooth_factor(g, src, R, i, j, k);
    if (f != 1.0) sa.ap[s].lam[lin3(g, i, j, k)] *= f;
  }
}

// Running state of the ordered sums over a call's sources, carried from chunk to chunk:
// the sum of the finished groups, the current group's partial sum, whether a group has
// finished yet, and the first source of the current group.
struct SumState {
  double* acc;  // N (or 1 for the misfit), null for a call in one chunk
  double* tot;
  int first_group;
  int gcur;
  int final_chunk;
};

// Σ over sources in the reference's order: within a group in source order, then the
// group sums in group order (eikmaingrad.jl:137-150). Sources s0 .. s0+nsrc-1 of a call;
// gstart gives each source's group, the last chunk writes the total. With per-group
// outputs (one chunk) each group's sum goes to out + (its ordinal) * N instead, as a call of
// that group alone computes it.
__global__ void adj_sum_kernel(const AdjProblem* ap, int nsrc, int s0, const int32_t* gstart, int per_group,
                               long long N, SumState ss, double* out) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < N; l += (long long)gridDim.x * blockDim.x) {
    double tot = ss.tot ? ss.tot[l] : 0.0, acc = ss.acc ? ss.acc[l] : 0.0;
    int gcur = ss.gcur, gord = 0;
    bool first_group = ss.first_group != 0;
    for (int s = 0; s < nsrc; s++) {
      const int gs = gstart[s0 + s];
      if (s0 + s > 0 && gs != gcur) {
        if (per_group) out[(size_t)gord * N + l] = acc;
        else tot = first_group ? acc : tot + acc;
        first_group = false;
        acc = 0.0;
        gcur = gs;
        gord++;
      }
      acc = acc + ap[s].lam[l];
    }
    if (ss.final_chunk) {
      if (per_group) out[(size_t)gord * N + l] = acc;
      else out[l] = first_group ? acc : tot + acc;
    } else {
      ss.acc[l] = acc;
      ss.tot[l] = tot;
    }
  }
}

// The group state after sources s0 .. s0+nsrc-1 (the same steps as the sums, on the host).
void sum_state_advance(SumState* ss, int nsrc, int s0, const int32_t* gstart);

template <int ND>
static cudaError_t launch_adj_solve(const AdjArgs& aa, int nsm, cudaStream_t st) {
  int per = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, adj_rounds_kernel<ND>, SOLVE_THREADS, 0);
  per = per < 1 ? 1 : per;
  AdjArgs args = aa;
  void* kargs[] = {&args};
  // cooperative: every CTA is resident, so the grid barrier between rounds cannot deadlock
  return cudaLaunchCooperativeKernel((const void*)adj_rounds_kernel<ND>, dim3(nsm * per), dim3(SOLVE_THREADS),
                                     kargs, 0, st);
}

}  // namespace eik

using namespace eik;



// Per-source misfits summed as the reference does: 0.5*m per source within a group, then
// over the groups (eikmaingrad.jl:137-150, 241); chunked like adj_sum_kernel, per group
// like it with per_group.
__global__ void adj_misfit_kernel(const double* misf, int nsrc, int s0, const int32_t* gstart, int per_group,
                                  SumState ss, double* out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double tot = ss.tot ? ss.tot[0] : 0.0, acc = ss.acc ? ss.acc[0] : 0.0;
  int gcur = ss.gcur, gord = 0;
  bool first_group = ss.first_group != 0;
  for (int s = 0; s < nsrc; s++) {
    const int gs = gstart[s0 + s];
    if (s0 + s > 0 && gs != gcur) {
      if (per_group) out[gord] = acc;
      else tot = first_group ? acc : tot + acc;
      first_group = false;
      acc = 0.0;
      gcur = gs;
      gord++;
    }
    acc += 0.5 * misf[s];
  }
  if (ss.final_chunk) {
    if (per_group) out[gord] = acc;
    else *out = first_group ? acc : tot + acc;
  } else {
    ss.acc[0] = acc;
    ss.tot[0] = tot;
  }
}

namespace eik {
// Source groups (distribsrcs, eikutils.jl:171-190): first source of the group of s when
// nsrc sources are split into nw groups.
int host_group_start(int nsrc, int nw, int s) {
  if (nw <= 1) return 0;
  if (nsrc < nw) return s;
  const int dis = nsrc / nw, resto = nsrc % nw;
  int start = 0;
  for (int gi = 0; gi < nw; gi++) {
    const int sz = dis + (gi < resto ? 1 : 0);
    if (s < start + sz) return start;
    start += sz;
  }
  return start;
}

void sum_state_advance(SumState* ss, int nsrc, int s0, const int32_t* gstart) {
  for (int s = 0; s < nsrc; s++) {
    const int gs = gstart[s0 + s];
    if (s0 + s > 0 && gs != ss->gcur) {
      ss->first_group = 0;
      ss->gcur = gs;
    }
  }
}

void gradient_footprint(const Model& m, const eik_extra& ep, long long nrec, int32_t whichgrad,
                        size_t* per_source, size_t* fixed) {
  // the named buffers of forward_device, gradient_core and eik_gradient, per source and fixed
  const int nd = m.g.nd;
  const unsigned long long N = (unsigned long long)m.N;
  const bool refine = ep.refinearoundsrc != 0;
  unsigned long long win = 1, nfmax = 1;
  for (int d = 0; d < nd; d++) {
    win *= 2ull * ep.noderadius + 2;
    nfmax *= (2ull * ep.noderadius + 1) * ep.downscalefactor + 1;
  }
  const unsigned long long seedcap = refine ? std::max<unsigned long long>(win, 8) : 8;
  const unsigned long long nf = refine ? nfmax : 1;
  unsigned long long per = sizeof(SrcOut) + seedcap * (4 + 8) + N * (8 + 1 + 8 + 1) + sizeof(CoarseProblem) +
                           std::max<unsigned long long>(N, nf) * (4 + 8 + 1 + 8 + 8) + 5 * 8;
  if (refine) per += nf * (8 + 1 + 1 + 4 + 4 + 1) + sizeof(CoarseProblem) + 8 * (4 + 8) + nf * (8 + 8 + 1) + 1;
  per += N * (8 + 8ull * nd + 8) + 8 + seedcap * 4 * 8 + nd * 8 + (refine ? nf * (8 + 8ull * nd) : 16) +
         sizeof(AdjProblem);
  per += 3ull * nd * 8 + 8 + 4;  // coordinates, receiver offsets, source-location gradient, group start
  const bool smoothing = (whichgrad == 1 || whichgrad == 3) && ep.smoothgradkern > 0;
  unsigned long long fix = N * 8 + (smoothing ? N * 8 : 0) + (unsigned long long)std::max<long long>(nrec, 1) *
                                                                 (8ull * nd + 16) + 8192;
  if (smoothing) {
    unsigned long long k = 1;
    for (int d = 0; d < nd; d++) k *= (unsigned long long)ep.smoothgradkern;
    fix += 8 * k;
  }
  *per_source = (size_t)per;
  *fixed = (size_t)fix;
}

// Sources per chunk of a gradient call under the context's budget (nsrc when one call fits).
static long long gradient_chunk(eik_ctx* ctx, const Model& m, const eik_extra& ep, long long nsrc, long long nrec,
                                int32_t whichgrad) {
  size_t per = 0, fix = 0;
  gradient_footprint(m, ep, nrec, whichgrad, &per, &fix);
  const size_t budget = ctx->scratch.budget;
  if (fix + per * (size_t)nsrc <= budget) return nsrc;
  const size_t state = 3 * sizeof(double) * (size_t)m.N + 64;  // carried from chunk to chunk
  if (budget < fix + state + per) return 0;
  long long c = (long long)((budget - fix - state) / per);
  // node-sources of one launch are numbered in 32 bits
  unsigned long long nf = 1;
  for (int d = 0; d < m.g.nd; d++) nf *= (2ull * ep.noderadius + 1) * ep.downscalefactor + 1;
  const unsigned long long span = std::max<unsigned long long>((unsigned long long)m.N, ep.refinearoundsrc ? nf : 1);
  c = std::min<long long>(c, (long long)(((1ull << 32) - 1) / span));
  return std::max<long long>(1, std::min(c, nsrc));
}

int validate_gradient(eik_ctx* ctx, const Model& m, int64_t nsrc, int32_t whichgrad, const eik_extra& ep) {
  if (whichgrad < 1 || whichgrad > 3)
    return fail(ctx, EIK_ERR_ASSERT, "Symbol 'whichgrad' not in (:gradvel, :gradsrcloc, :gradvelandsrcloc)");
  int rc = check_extra(ctx, &ep);
  if (rc) return rc;
  if (nsrc <= 0) return fail(ctx, EIK_ERR_ASSERT, "nsrc >= 1");
  if ((whichgrad == 2 || whichgrad == 3) && !is_cart(m.g))
    return fail(ctx, EIK_ERR_ERROR, "type %s has no field hgrid", m.g.nd == 2 ? "Grid2DSphere" : "Grid3DSphere");
  for (int a = 0; a < m.g.nd; a++)
    if (m.g.n[a] < 3) return fail(ctx, EIK_ERR_ERROR, "BoundsError: grid axis %d has fewer than 3 nodes", a);
  return EIK_OK;
}

// Forward + adjoint + assembly for nsrc sources whose inputs are on the device.
// Outputs (each nullable): d_gradvel N values, d_gradsrc nsrc x nd, d_misfit 1 value.
// Returns after the stream has drained and the device error word has been checked.
int gradient_core(eik_ctx* ctx, const Model& m, int64_t nsrc, const double* d_cs, const long long* d_off,
                         const double* d_rec, const double* d_po, const double* d_so, int32_t whichgrad,
                         const eik_extra& ep, double* d_gradvel, double* d_gradsrc, double* d_misfit,
                         eik_stats* stats, GradTail* tail_out, GradChunk* chunk, const GroupSpec* groups) {
  int rc = EIK_OK;
  cudaStream_t st = ctx->stream;
  Scratch& S = ctx->scratch;
  const int nd = m.g.nd;
  const long long N = m.N;
  if (groups && chunk) return fail(ctx, EIK_ERR_ASSERT, "per-group outputs are computed in one pipeline");
  // :sharedmem splits the sources into groups with separate gradient buffers; explicit
  // groups (one per request of a merged call) each get their own outputs
  const int ngroups = (ep.parallelkind == 1 && ep.nthreads > 1) ? ep.nthreads : 1;
  const int nsrc_total = chunk ? chunk->nsrc_total : (int)nsrc;
  std::vector<int32_t> hgs((size_t)nsrc_total);
  if (groups) {
    for (int64_t gi = 0; gi < groups->ngroups; gi++)
      for (int64_t q = groups->off[gi]; q < groups->off[gi + 1]; q++) hgs[(size_t)q] = (int32_t)groups->off[gi];
  } else {
    for (int q = 0; q < nsrc_total; q++) hgs[(size_t)q] = host_group_start(nsrc_total, ngroups, q);
  }
  const int per_group = groups ? 1 : 0;
  const long long nout = groups ? groups->ngroups : 1;  // gradient fields and misfits written
  const bool wantvel = whichgrad == 1 || whichgrad == 3;
  ForwardState fw;
  rc = forward_device(ctx, m, nsrc, d_cs, ep, &fw, stats);
  if (rc) return rc;
#define GET(var, type, name, count)                                                  \
  var = (type*)S.get(name, sizeof(type) * (size_t)(count), &rc);                     \
  if (!var) return rc == EIK_ERR_OUT_OF_BUDGET                                       \
                     ? fail(ctx, rc, "scratch '%s' exceeds the HBM budget", name)    \
                     : fail(ctx, rc, "cudaMalloc of scratch '%s' failed", name);
  double *lam, *gdt, *rhs, *misf, *dpsi, *ysrc, *gnode, *gsrc, *flam, *fgdt, *carry, *gsum, *gw;
  AdjProblem* dap;
  ForwardBatch* dfb;
  uint32_t* dwarn;
  GET(lam, double, "adj_lam", nsrc * N);
  GET(gdt, double, "adj_gdt", nsrc * N * nd);
  GET(rhs, double, "adj_rhs", nsrc * N);
  GET(misf, double, "adj_misf", nsrc);
  GET(dpsi, double, "adj_dpsi", nsrc * fw.fb.seedcap);
  GET(ysrc, double, "adj_ysrc", nsrc * fw.fb.seedcap);
  GET(gnode, double, "adj_gnode", nsrc * fw.fb.seedcap);
  GET(carry, double, "adj_carry", nsrc * fw.fb.seedcap);
  GET(gsrc, double, "adj_gsrc", nsrc * nd);
  GET(flam, double, "adj_fine_lam", ep.refinearoundsrc ? nsrc * fw.fb.nfmax : 1);
  GET(fgdt, double, "adj_fine_gdt", ep.refinearoundsrc ? nsrc * nd * fw.fb.nfmax : 1);
  // smoothgradkern > 0: the group sum goes to a scratch field, the smoothing writes the output
  const bool smoothing = wantvel && d_gradvel && ep.smoothgradkern > 0;
  const long long nker = smoothing ? (nd == 3 ? (long long)ep.smoothgradkern * ep.smoothgradkern * ep.smoothgradkern
                                              : (long long)ep.smoothgradkern * ep.smoothgradkern)
                                   : 1;
  GET(gsum, double, "adj_gradsum", smoothing ? nout * N : 1);
  GET(gw, double, "adj_smooth_w", nker);
  int32_t* dgs;
  GET(dgs, int32_t, "adj_gstart", nsrc_total);
  GET(dap, AdjProblem, "adj_probs", nsrc);
  GET(dfb, ForwardBatch, "adj_fb", 1);
  GET(dwarn, uint32_t, "adj_warn", 1);
#undef GET
  std::vector<AdjProblem> hap(nsrc);
  for (int64_t s = 0; s < nsrc; s++) {
    hap[s].lam = lam + s * N;
    hap[s].gdt = gdt + s * N * nd;
    hap[s].rhs = rhs + s * N;
  }
  const void* hap_src = stage_host(ctx, hap.data(), sizeof(AdjProblem) * nsrc);
  const void* fb_src = stage_host(ctx, &fw.fb, sizeof(ForwardBatch));
  const void* gs_src = stage_host(ctx, hgs.data(), sizeof(int32_t) * hgs.size());
  if (!hap_src || !fb_src || !gs_src) return fail(ctx, EIK_ERR_CUDA, "cudaMallocHost of a plan's staging copy failed");
  CUDA_OK(ctx, cudaMemcpyAsync(dgs, gs_src, sizeof(int32_t) * hgs.size(), cudaMemcpyHostToDevice, st));
  CUDA_OK(ctx, cudaMemcpyAsync(dap, hap_src, sizeof(AdjProblem) * nsrc, cudaMemcpyHostToDevice, st));
  CUDA_OK(ctx, cudaMemcpyAsync(dfb, fb_src, sizeof(ForwardBatch), cudaMemcpyHostToDevice, st));
  CUDA_OK(ctx, cudaMemsetAsync(dwarn, 0, sizeof(uint32_t), st));
  CUDA_OK(ctx, cudaMemsetAsync(gsrc, 0, sizeof(double) * nsrc * nd, st));
  const CoarseProblem* dprobs = fw.sa.probs;
  // the adjoint sweep reuses the forward's worklists; counts live in its round stamps
  AdjArgs aa;
  aa.sa = fw.sa;
  aa.ap = dap;
  aa.sa.rs.max_rounds = ctx->max_rounds > 0 ? ctx->max_rounds : (1 << 26);
  aa.sa.rs.rounds = fw.sa.rs.rounds + 1;  // the forward's count stays readable
  adj_rounds_init_kernel<<<1, 1, 0, st>>>(aa.sa);
  adj_prep_kernel<<<2 * ctx->nsm * 8, 256, 0, st>>>(dprobs, dap, (int)nsrc, N, aa.sa);
  RecvArgs ra;
  ra.g = m.g;
  ra.nsrc = (int)nsrc;
  ra.probs = dprobs;
  ra.ap = dap;
  ra.recoff = d_off;
  ra.rec = d_rec;
  ra.pickobs = d_po;
  ra.stdobs = d_so;
  ra.fb = dfb;
  ra.misfit = misf;
  ra.dpsi = dpsi;
  adj_recv_kernel<<<(int)((nsrc + 63) / 64), 64, 0, st>>>(ra);
  if (!ctx->capturing) cudaEventRecord(ctx->evk[4], st);
  CUDA_OK(ctx, nd == 3 ? launch_adj_solve<3>(aa, fw.sms, st) : launch_adj_solve<2>(aa, fw.sms, st));
  if (!ctx->capturing) cudaEventRecord(ctx->evk[5], st);
  adj_check_kernel<<<ctx->nsm * 8, 256, 0, st>>>(dap, (int)nsrc, N, fw.fb.err);
  CUDA_OK(ctx, cudaGetLastError());
  SrcTermArgs ta;
  ta.g = m.g;
  ta.nsrc = (int)nsrc;
  ta.refine = ep.refinearoundsrc;
  ta.whichgrad = whichgrad;
  ta.gstart = dgs;
  ta.s0 = chunk ? chunk->s0 : 0;
  ta.nsrc_total = nsrc_total;
  ta.prevbuf = (chunk && chunk->prev_valid) ? chunk->prevbuf : nullptr;
  ta.probs = dprobs;
  ta.ap = dap;
  ta.fb = dfb;
  ta.vel = m.vel;
  ta.coordsrc = d_cs;
  ta.dpsi = dpsi;
  ta.ysrc = ysrc;
  ta.gsrcnode = gnode;
  ta.gradsrc = gsrc;
  ta.fine_lam = flam;
  ta.fine_gdt = fgdt;
  ta.warn = dwarn;
  adj_ysrc_kernel<<<(int)nsrc, 128, 0, st>>>(ta);
  adj_srcterm_kernel<<<(int)nsrc, 32, 0, st>>>(ta);
  if (wantvel) {
    adj_field_kernel<<<ctx->nsm * 8, 256, 0, st>>>(ta, N);
    adj_carry_kernel<<<(int)nsrc, 64, 0, st>>>(ta, ep.radiussmoothgradsrc, carry);
    adj_srcnodes_kernel<<<(int)nsrc, 128, 0, st>>>(ta, carry);
    if (ep.radiussmoothgradsrc > 0) adj_smooth_kernel<<<(int)nsrc, 256, 0, st>>>(ta, ep.radiussmoothgradsrc);
    SumState ss;
    ss.acc = chunk ? chunk->acc : nullptr;
    ss.tot = chunk ? chunk->tot : nullptr;
    ss.first_group = chunk ? chunk->first_group : 1;
    ss.gcur = chunk ? chunk->gcur : 0;
    ss.final_chunk = chunk ? (chunk->final_chunk ? 1 : 0) : 1;
    if (d_gradvel)
      adj_sum_kernel<<<ctx->nsm * 8, 256, 0, st>>>(dap, (int)nsrc, ta.s0, dgs, per_group, N, ss,
                                                   smoothing ? gsum : d_gradvel);
    if (chunk && !chunk->final_chunk) {
      // the group buffer as this chunk leaves it: its last source's final field
      CUDA_OK(ctx, cudaMemcpyAsync(chunk->prevbuf, lam + (nsrc - 1) * N, sizeof(double) * N, cudaMemcpyDeviceToDevice,
                                   st));
    }
    if (smoothing && ss.final_chunk) {
      // weights from pageable memory: the copy has left the vector when cudaMemcpyAsync returns
      const std::vector<double> w = gaussian_weights((int)ep.smoothgradkern, nd);
      const void* w_src = stage_host(ctx, w.data(), sizeof(double) * w.size());
      if (!w_src) return fail(ctx, EIK_ERR_CUDA, "cudaMallocHost of a plan's staging copy failed");
      CUDA_OK(ctx, cudaMemcpyAsync(gw, w_src, sizeof(double) * w.size(), cudaMemcpyHostToDevice, st));
      for (long long q = 0; q < nout; q++)
        CUDA_OK(ctx, launch_smoothgrad(m.g, (int)ep.smoothgradkern, gw, gsum + q * N, d_gradvel + q * N, st));
    }
  }
  if (d_misfit) {
    SumState ms;
    ms.acc = chunk ? chunk->macc : nullptr;
    ms.tot = chunk ? chunk->mtot : nullptr;
    ms.first_group = chunk ? chunk->first_group : 1;
    ms.gcur = chunk ? chunk->gcur : 0;
    ms.final_chunk = chunk ? (chunk->final_chunk ? 1 : 0) : 1;
    adj_misfit_kernel<<<1, 1, 0, st>>>(misf, (int)nsrc, ta.s0, dgs, per_group, ms, d_misfit);
  }
  if (chunk) {
    SumState adv;
    adv.first_group = chunk->first_group;
    adv.gcur = chunk->gcur;
    sum_state_advance(&adv, (int)nsrc, chunk->s0, hgs.data());
    chunk->first_group = adv.first_group;
    chunk->gcur = adv.gcur;
    chunk->prev_valid = true;
  }
  if (d_gradsrc && whichgrad != 1)
    CUDA_OK(ctx, cudaMemcpyAsync(d_gradsrc, gsrc, sizeof(double) * nsrc * nd, cudaMemcpyDeviceToDevice, st));
  CUDA_OK(ctx, cudaGetLastError());
  GradTail tail;
  tail.fw = fw;
  tail.dwarn = dwarn;
  tail.arounds = aa.sa.rs.rounds;
  tail.launches = 7 + (d_misfit ? 1 : 0) +
                  (wantvel ? 3 + (ep.radiussmoothgradsrc > 0 ? 1 : 0) + (d_gradvel ? 1 : 0) : 0) +
                  (smoothing ? (int)nout : 0);
  if (tail_out) *tail_out = tail;
  if (ctx->capturing) return EIK_OK;  // read back after each replay of the captured graph
  rc = gradient_tail_stats(ctx, tail, stats);
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->evk[4], ctx->evk[5]);
    stats->adj_ms = ms;
  }
  return rc;
}

}  // namespace eik

namespace eik {

int gradient_tail_stats(eik_ctx* ctx, GradTail& tail, eik_stats* stats) {
  uint32_t hw = 0;
  int32_t arounds = 0;
  CUDA_OK(ctx, cudaMemcpyAsync(&hw, tail.dwarn, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_OK(ctx, cudaMemcpyAsync(&arounds, tail.arounds, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
  const int rc = collect_forward_stats(ctx, &tail.fw, stats);
  if (stats) {
    stats->warn_mask |= hw;
    stats->adj_rounds = (uint64_t)arounds;
    stats->launches += tail.launches;
  }
  return rc;
}

// A gradient call whose sources do not fit the budget in one pipeline: chunks of `chunk`
// sources in order, each a full forward + adjoint pipeline, with the group buffer and the
// ordered sums handed from chunk to chunk, so that the result is the one-call result bit
// for bit (the reference's per-group buffer, eikmaingrad.jl:182-190, 242-246, and its
// group sums, :137-150). The caller releases the scratch of earlier calls before it
// allocates this call's inputs. Inputs and outputs are device pointers (gradvel N, gradsrc
// nsrc x nd, misfit 1, each nullable).
int gradient_chunked(eik_ctx* ctx, const Model& m, int64_t nsrc, long long chunk, const double* d_cs,
                     const int64_t* rec_off, const double* d_rec, const double* d_po, const double* d_so,
                     int32_t whichgrad, const eik_extra& ep, double* d_gradvel, double* d_gradsrc, double* d_misfit,
                     eik_stats* stats) {
  cudaStream_t st = ctx->stream;
  int rc = EIK_OK;
  const long long N = m.N;
  const int nd = m.g.nd;
  double* state = (double*)ctx->scratch.get("chunk_state", sizeof(double) * (3 * (size_t)N + 4), &rc);
  long long* d_off = (long long*)ctx->scratch.get("chunk_off", sizeof(long long) * (size_t)(chunk + 1), &rc);
  if (!state || !d_off) return fail(ctx, rc ? rc : EIK_ERR_CUDA, "chunk state exceeds the HBM budget");
  CUDA_OK(ctx, cudaMemsetAsync(state, 0, sizeof(double) * (3 * (size_t)N + 4), st));
  GradChunk gc;
  gc.nsrc_total = (int)nsrc;
  gc.acc = state;
  gc.tot = state + N;
  gc.prevbuf = state + 2 * N;
  gc.macc = state + 3 * N;
  gc.mtot = state + 3 * N + 1;
  eik_stats acc_stats;
  std::memset(&acc_stats, 0, sizeof acc_stats);
  std::vector<long long> off((size_t)chunk + 1);
  for (long long c0 = 0; c0 < nsrc; c0 += chunk) {
    const long long nloc = std::min(chunk, (long long)nsrc - c0);
    gc.s0 = (int)c0;
    gc.final_chunk = c0 + nloc >= nsrc;
    for (long long s = 0; s <= nloc; s++) off[(size_t)s] = rec_off[c0 + s] - rec_off[c0];
    CUDA_OK(ctx, cudaMemcpyAsync(d_off, off.data(), sizeof(long long) * (size_t)(nloc + 1), cudaMemcpyHostToDevice, st));
    const long long r0 = rec_off[c0];
    eik_stats cs;
    std::memset(&cs, 0, sizeof cs);
    rc = gradient_core(ctx, m, nloc, d_cs + c0 * nd, d_off, d_rec + r0 * nd, d_po + r0, d_so + r0, whichgrad, ep,
                       d_gradvel, d_gradsrc ? d_gradsrc + c0 * nd : nullptr, d_misfit, &cs, nullptr, &gc);
    if (rc) return rc;  // gradient_core drained the stream: `off` may be rewritten
    acc_stats.warn_mask |= cs.warn_mask;
    acc_stats.err_mask |= cs.err_mask;
    acc_stats.tile_activations += cs.tile_activations;
    acc_stats.node_evals += cs.node_evals;
    acc_stats.fine_ms += cs.fine_ms;
    acc_stats.solve_ms += cs.solve_ms;
    acc_stats.adj_ms += cs.adj_ms;
    acc_stats.adj_rounds = std::max(acc_stats.adj_rounds, cs.adj_rounds);
    acc_stats.launches += cs.launches + 1;
    acc_stats.fwd_rounds = std::max(acc_stats.fwd_rounds, cs.fwd_rounds);
    acc_stats.fine_replays += cs.fine_replays;
    for (int k = 0; k < 7; k++) acc_stats.fwd_visits[k] += cs.fwd_visits[k];
    acc_stats.chunks += 1;
  }
  if (stats) {
    const double dms = stats->device_ms;
    *stats = acc_stats;
    stats->device_ms = dms;
  }
  return EIK_OK;
}

}  // namespace eik

extern "C" int eik_gradient_bytes(eik_ctx* ctx, eik_model_id model, int64_t nsrc, int64_t nrec, const eik_extra* ep_in,
                                  int32_t whichgrad, uint64_t* bytes) {
  if (!ctx || !bytes) return fail(ctx, EIK_ERR_ASSERT, "NULL argument");
  std::lock_guard<std::mutex> lk(ctx->mu);
  auto it = ctx->models.find(model);
  if (it == ctx->models.end()) return fail(ctx, EIK_ERR_ASSERT, "unknown model id %lld", (long long)model);
  eik_extra ep;
  if (ep_in) ep = *ep_in;
  else eik_extra_defaults(&ep);
  if (nsrc < 0 || nrec < 0) return fail(ctx, EIK_ERR_ASSERT, "nsrc >= 0, nrec >= 0");
  size_t per = 0, fix = 0;
  gradient_footprint(it->second, ep, nrec, whichgrad, &per, &fix);
  *bytes = (uint64_t)(fix + per * (size_t)nsrc);
  return EIK_OK;
}

extern "C" int eik_gradient(eik_ctx* ctx, eik_model_id model, int64_t nsrc, const double* coordsrc,
                            const int64_t* rec_off, const double* rec, const double* pickobs,
                            const double* stdobs, int32_t whichgrad, const eik_extra* ep_in, double* gradvel,
                            double* gradsrc, double* misfit, eik_stats* stats) {
  if (!ctx) return fail(ctx, EIK_ERR_ASSERT, "NULL context");
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->scratch.begin_call();
  NvtxRange nvtx_call("eik_gradient");
  auto it = ctx->models.find(model);
  if (it == ctx->models.end()) return fail(ctx, EIK_ERR_ASSERT, "unknown model id %lld", (long long)model);
  const Model& m = it->second;
  eik_extra ep;
  if (ep_in) ep = *ep_in;
  else eik_extra_defaults(&ep);
  if (stats) std::memset(stats, 0, sizeof *stats);
  int rc = validate_gradient(ctx, m, nsrc, whichgrad, ep);
  if (rc) return rc;
  if (!coordsrc || !rec_off || !rec || !pickobs || !stdobs) return fail(ctx, EIK_ERR_ASSERT, "NULL argument");
  rc = check_positions(ctx, m.g, nsrc, coordsrc, rec_off, rec);
  if (rc) return rc;
  CUDA_OK(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  Scratch& S = ctx->scratch;
  const int nd = m.g.nd;
  const long long N = m.N, nrec = rec_off[nsrc];
#define GET(var, type, name, count)                                                  \
  var = (type*)S.get(name, sizeof(type) * (size_t)(count), &rc);                     \
  if (!var) return rc == EIK_ERR_OUT_OF_BUDGET                                       \
                     ? fail(ctx, rc, "scratch '%s' exceeds the HBM budget", name)    \
                     : fail(ctx, rc, "cudaMalloc of scratch '%s' failed", name);
  double *d_cs, *d_rec, *d_po, *d_so, *d_gv, *d_gs, *d_m;
  long long* d_off = nullptr;
  const long long chunk = gradient_chunk(ctx, m, ep, nsrc, nrec, whichgrad);
  if (chunk < 1) return fail(ctx, EIK_ERR_OUT_OF_BUDGET, "one source does not fit the HBM budget");
  if (chunk < nsrc) {
    // split: the inputs and outputs are allocated after the release of earlier scratch
    CUDA_OK(ctx, cudaStreamSynchronize(st));
    S.release_all();
  }
  GET(d_cs, double, "in_cs", nsrc * nd);
  GET(d_rec, double, "in_rec", std::max<long long>(nrec, 1) * nd);
  GET(d_po, double, "in_pickobs", std::max<long long>(nrec, 1));
  GET(d_so, double, "in_stdobs", std::max<long long>(nrec, 1));
  GET(d_gv, double, "out_gradvel", N);
  GET(d_gs, double, "out_gradsrc", nsrc * nd);
  GET(d_m, double, "out_misfit", 1);
  if (chunk >= nsrc) {
    GET(d_off, long long, "in_off", nsrc + 1);
  }
#undef GET
  cudaEventRecord(ctx->ev0, st);
  CUDA_OK(ctx, cudaMemcpyAsync(d_cs, coordsrc, sizeof(double) * nsrc * nd, cudaMemcpyHostToDevice, st));
  if (d_off) CUDA_OK(ctx, cudaMemcpyAsync(d_off, rec_off, sizeof(long long) * (nsrc + 1), cudaMemcpyHostToDevice, st));
  if (nrec) {
    CUDA_OK(ctx, cudaMemcpyAsync(d_rec, rec, sizeof(double) * nrec * nd, cudaMemcpyHostToDevice, st));
    CUDA_OK(ctx, cudaMemcpyAsync(d_po, pickobs, sizeof(double) * nrec, cudaMemcpyHostToDevice, st));
    CUDA_OK(ctx, cudaMemcpyAsync(d_so, stdobs, sizeof(double) * nrec, cudaMemcpyHostToDevice, st));
  }
  const bool wantvel = whichgrad == 1 || whichgrad == 3, wantsrc = whichgrad != 1;
  if (chunk < nsrc)
    rc = gradient_chunked(ctx, m, nsrc, chunk, d_cs, rec_off, d_rec, d_po, d_so, whichgrad, ep,
                          wantvel ? d_gv : nullptr, wantsrc ? d_gs : nullptr, d_m, stats);
  else
    rc = run_with_retry(ctx, stats, [&]() {
      return gradient_core(ctx, m, nsrc, d_cs, d_off, d_rec, d_po, d_so, whichgrad, ep, wantvel ? d_gv : nullptr,
                           wantsrc ? d_gs : nullptr, d_m, stats, nullptr);
    });
  if (rc) return rc;
  double hm = 0.0;
  CUDA_OK(ctx, cudaMemcpyAsync(&hm, d_m, sizeof(double), cudaMemcpyDeviceToHost, st));
  if (gradvel && wantvel) CUDA_OK(ctx, cudaMemcpyAsync(gradvel, d_gv, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  if (gradsrc && wantsrc)
    CUDA_OK(ctx, cudaMemcpyAsync(gradsrc, d_gs, sizeof(double) * nsrc * nd, cudaMemcpyDeviceToHost, st));
  cudaEventRecord(ctx->ev1, st);
  CUDA_OK(ctx, cudaStreamSynchronize(st));
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    stats->device_ms = ms;
  }
  if (misfit) *misfit = hm;
  return EIK_OK;
}

extern "C" int eik_gradient_groups(eik_ctx* ctx, eik_model_id model, int64_t ngroups, const int64_t* group_off,
                                   const double* coordsrc, const int64_t* rec_off, const double* rec,
                                   const double* pickobs, const double* stdobs, int32_t whichgrad,
                                   const eik_extra* ep_in, double* gradvel, double* gradsrc, double* misfit,
                                   eik_stats* stats) {
  if (!ctx) return fail(ctx, EIK_ERR_ASSERT, "NULL context");
  if (ngroups < 1 || !group_off) return fail(ctx, EIK_ERR_ASSERT, "ngroups >= 1 and NULL argument");
  if (group_off[0] != 0) return fail(ctx, EIK_ERR_ASSERT, "group_off[0] must be 0");
  for (int64_t gi = 0; gi < ngroups; gi++)
    if (group_off[gi + 1] <= group_off[gi]) return fail(ctx, EIK_ERR_ASSERT, "every group has at least one source");
  const int64_t nsrc = group_off[ngroups];
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->scratch.begin_call();
  NvtxRange nvtx_call("eik_gradient_groups");
  auto it = ctx->models.find(model);
  if (it == ctx->models.end()) return fail(ctx, EIK_ERR_ASSERT, "unknown model id %lld", (long long)model);
  const Model& m = it->second;
  eik_extra ep;
  if (ep_in) ep = *ep_in;
  else eik_extra_defaults(&ep);
  if (stats) std::memset(stats, 0, sizeof *stats);
  int rc = validate_gradient(ctx, m, nsrc, whichgrad, ep);
  if (rc) return rc;
  if (!coordsrc || !rec_off || !rec || !pickobs || !stdobs) return fail(ctx, EIK_ERR_ASSERT, "NULL argument");
  rc = check_positions(ctx, m.g, nsrc, coordsrc, rec_off, rec);
  if (rc) return rc;
  const long long N = m.N, nrec = rec_off[nsrc];
  if (gradient_chunk(ctx, m, ep, nsrc, nrec, whichgrad) < nsrc)
    return fail(ctx, EIK_ERR_OUT_OF_BUDGET, "a call with per-group outputs runs in one pipeline: it exceeds the HBM "
                                            "budget");
  CUDA_OK(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  Scratch& S = ctx->scratch;
  const int nd = m.g.nd;
#define GET(var, type, name, count)                                                  \
  var = (type*)S.get(name, sizeof(type) * (size_t)(count), &rc);                     \
  if (!var) return rc == EIK_ERR_OUT_OF_BUDGET                                       \
                     ? fail(ctx, rc, "scratch '%s' exceeds the HBM budget", name)    \
                     : fail(ctx, rc, "cudaMalloc of scratch '%s' failed", name);
  double *d_cs, *d_rec, *d_po, *d_so, *d_gv, *d_gs, *d_m;
  long long* d_off;
  GET(d_cs, double, "in_cs", nsrc * nd);
  GET(d_rec, double, "in_rec", std::max<long long>(nrec, 1) * nd);
  GET(d_po, double, "in_pickobs", std::max<long long>(nrec, 1));
  GET(d_so, double, "in_stdobs", std::max<long long>(nrec, 1));
  GET(d_gv, double, "out_gradvel", ngroups * N);
  GET(d_gs, double, "out_gradsrc", nsrc * nd);
  GET(d_m, double, "out_misfit", ngroups);
  GET(d_off, long long, "in_off", nsrc + 1);
#undef GET
  cudaEventRecord(ctx->ev0, st);
  CUDA_OK(ctx, cudaMemcpyAsync(d_cs, coordsrc, sizeof(double) * nsrc * nd, cudaMemcpyHostToDevice, st));
  CUDA_OK(ctx, cudaMemcpyAsync(d_off, rec_off, sizeof(long long) * (nsrc + 1), cudaMemcpyHostToDevice, st));
  if (nrec) {
    CUDA_OK(ctx, cudaMemcpyAsync(d_rec, rec, sizeof(double) * nrec * nd, cudaMemcpyHostToDevice, st));
    CUDA_OK(ctx, cudaMemcpyAsync(d_po, pickobs, sizeof(double) * nrec, cudaMemcpyHostToDevice, st));
    CUDA_OK(ctx, cudaMemcpyAsync(d_so, stdobs, sizeof(double) * nrec, cudaMemcpyHostToDevice, st));
  }
  const bool wantvel = whichgrad == 1 || whichgrad == 3, wantsrc = whichgrad != 1;
  const GroupSpec gsp{ngroups, group_off};
  rc = run_with_retry(ctx, stats, [&]() {
    return gradient_core(ctx, m, nsrc, d_cs, d_off, d_rec, d_po, d_so, whichgrad, ep, wantvel ? d_gv : nullptr,
                         wantsrc ? d_gs : nullptr, d_m, stats, nullptr, nullptr, &gsp);
  });
  if (rc) return rc;
  if (misfit) CUDA_OK(ctx, cudaMemcpyAsync(misfit, d_m, sizeof(double) * ngroups, cudaMemcpyDeviceToHost, st));
  if (gradvel && wantvel)
    CUDA_OK(ctx, cudaMemcpyAsync(gradvel, d_gv, sizeof(double) * ngroups * N, cudaMemcpyDeviceToHost, st));
  if (gradsrc && wantsrc)
    CUDA_OK(ctx, cudaMemcpyAsync(gradsrc, d_gs, sizeof(double) * nsrc * nd, cudaMemcpyDeviceToHost, st));
  cudaEventRecord(ctx->ev1, st);
  CUDA_OK(ctx, cudaStreamSynchronize(st));
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    stats->device_ms = ms;
  }
  return EIK_OK;
}

extern "C" int eik_gradient_device(eik_ctx* ctx, eik_model_id model, int64_t nsrc, const double* coordsrc_dev,
                                   const int64_t* rec_off, const double* rec_dev, const double* pickobs_dev,
                                   const double* stdobs_dev, int32_t whichgrad, const eik_extra* ep_in,
                                   double* gradvel_dev, double* gradsrc_dev, double* misfit_dev,
                                   eik_stats* stats) {
  if (!ctx) return fail(ctx, EIK_ERR_ASSERT, "NULL context");
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->scratch.begin_call();
  NvtxRange nvtx_call("eik_gradient_device");
  auto it = ctx->models.find(model);
  if (it == ctx->models.end()) return fail(ctx, EIK_ERR_ASSERT, "unknown model id %lld", (long long)model);
  const Model& m = it->second;
  eik_extra ep;
  if (ep_in) ep = *ep_in;
  else eik_extra_defaults(&ep);
  if (stats) std::memset(stats, 0, sizeof *stats);
  int rc = validate_gradient(ctx, m, nsrc, whichgrad, ep);
  if (rc) return rc;
  if (!coordsrc_dev || !rec_off || !rec_dev || !pickobs_dev || !stdobs_dev)
    return fail(ctx, EIK_ERR_ASSERT, "NULL argument");
  CUDA_OK(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const int nd = m.g.nd;
  const long long nrec = rec_off[nsrc];
  // positions are checked on the host, as the reference does before any solve
  std::vector<double> hcs((size_t)nsrc * nd), hrec((size_t)std::max<long long>(nrec, 1) * nd);
  cudaEventRecord(ctx->ev0, st);
  CUDA_OK(ctx, cudaMemcpyAsync(hcs.data(), coordsrc_dev, sizeof(double) * nsrc * nd, cudaMemcpyDeviceToHost, st));
  if (nrec) CUDA_OK(ctx, cudaMemcpyAsync(hrec.data(), rec_dev, sizeof(double) * nrec * nd, cudaMemcpyDeviceToHost, st));
  CUDA_OK(ctx, cudaStreamSynchronize(st));
  rc = check_positions(ctx, m.g, nsrc, hcs.data(), rec_off, hrec.data());
  if (rc) return rc;
  const long long chunk = gradient_chunk(ctx, m, ep, nsrc, nrec, whichgrad);
  if (chunk < 1) return fail(ctx, EIK_ERR_OUT_OF_BUDGET, "one source does not fit the HBM budget");
  if (chunk < nsrc) {
    // split: the scratch of earlier calls is released (the inputs are the caller's memory)
    CUDA_OK(ctx, cudaStreamSynchronize(st));
    ctx->scratch.release_all();
    rc = gradient_chunked(ctx, m, nsrc, chunk, coordsrc_dev, rec_off, rec_dev, pickobs_dev, stdobs_dev, whichgrad,
                          ep, (whichgrad != 2) ? gradvel_dev : nullptr, (whichgrad != 1) ? gradsrc_dev : nullptr,
                          misfit_dev, stats);
  } else {
    long long* d_off = (long long*)ctx->scratch.get("in_off", sizeof(long long) * (nsrc + 1), &rc);
    if (!d_off) return fail(ctx, rc, "scratch allocation failed");
    CUDA_OK(ctx, cudaMemcpyAsync(d_off, rec_off, sizeof(long long) * (nsrc + 1), cudaMemcpyHostToDevice, st));
    rc = run_with_retry(ctx, stats, [&]() {
      return gradient_core(ctx, m, nsrc, coordsrc_dev, d_off, rec_dev, pickobs_dev, stdobs_dev, whichgrad, ep,
                           (whichgrad != 2) ? gradvel_dev : nullptr, (whichgrad != 1) ? gradsrc_dev : nullptr,
                           misfit_dev, stats, nullptr);
    });
  }
  if (rc) return rc;
  cudaEventRecord(ctx->ev1, st);
  CUDA_OK(ctx, cudaStreamSynchronize(st));
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    stats->device_ms = ms;
  }
  return EIK_OK;
}
