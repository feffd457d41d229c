// Refined-grid start-up around each source (runrefinementaroundsrc!/createfinegrid/
// sourceboxloctt!/ttFMM_core!, src/EikSolv/eikmainfwd.jl:330-405, 950-1104, 1195-1322,
// 427-823) and the non-refined source box, on the GPU.
//
// The refined grid stops at the first accepted node on a non-border edge of the window;
// which node that is among exact ties is decided by the reference's binary heap
// (src/BinHeap/BinHeaps.jl), so this stage replays the heap exactly: one warp per source,
// the 2*nd stencil updates of every popped batch evaluated in parallel across lanes, heap
// inserts/updates applied by lane 0 in the reference's order. The fine grid is at most
// ((2*noderadius+2)*downscalefactor+1)^nd nodes (46,656 at the defaults in 3D).
#include "kernels.cuh"

namespace eik {

// BinHeapMin (BinHeaps.jl:313-485) over shared memory; positions are 1-based.
struct SmemHeap {
  double* nodes;   // [cap+1]
  int32_t* hand;   // [cap+1] fine node index + 1
  int32_t* idx;    // global [nf] position of a handle (0 = absent)
  int Nh, cap;
  __device__ void swap(int p, int q) {
    const double tn = nodes[p];
    const int32_t th = hand[p];
    nodes[p] = nodes[q];
    nodes[q] = tn;
    hand[p] = hand[q];
    hand[q] = th;
    idx[hand[p] - 1] = p;
    idx[hand[q] - 1] = q;
  }
  __device__ void heapify(int i) {
    for (;;) {
      const int l = 2 * i, r = 2 * i + 1;
      int sm = (l <= Nh && nodes[l] < nodes[i]) ? l : i;
      if (r <= Nh && nodes[r] < nodes[sm]) sm = r;
      if (sm == i) return;
      swap(i, sm);
      i = sm;
    }
  }
  __device__ bool insert(double v, int32_t h) {
    if (Nh + 1 > cap) return false;
    Nh++;
    nodes[Nh] = v;
    hand[Nh] = h;
    idx[h - 1] = Nh;
    int i = Nh;
    while (i > 1 && nodes[i / 2] > nodes[i]) {
      swap(i, i / 2);
      i /= 2;
    }
    return true;
  }
  __device__ void update(double v, int32_t h) {
    int i = idx[h - 1];
    if (i < 1 || i > Nh) return;  // not in the heap (only after a capacity overflow)
    nodes[i] = v;
    while (i > 1 && nodes[i / 2] > nodes[i]) {
      swap(i, i / 2);
      i /= 2;
    }
    if (i < Nh) heapify(i);
  }
  __device__ void pop(int32_t* h, double* v) {
    *h = hand[1];
    *v = nodes[1];
    nodes[1] = nodes[Nh];
    hand[1] = hand[Nh];
    idx[hand[Nh] - 1] = 1;
    nodes[Nh] = 0.0;
    hand[Nh] = 0;
    idx[*h - 1] = 0;
    Nh--;
    heapify(1);
  }
};

// Neighbourhood of fine node (i,j,k) for the reference's stencil: accepted <=> status==2.
__device__ __forceinline__ double fine_update(const GridDesc& gf, const double* tt, const uint8_t* st,
                                              double slow, int i, int j, int k, int8_t* codes,
                                              bool* neg) {
  Nbhd nb;
  nb_clear(nb);
  const int c[3] = {i, j, k};
  node_dh(gf, i, nb.dh);
  nb.slow = slow;
  for (int a = 0; a < gf.nd; a++)
    for (int l = 0; l < 2; l++) {
      const int sh = l == 0 ? 1 : -1;
      int p[3] = {c[0], c[1], c[2]};
      p[a] += sh;
      if (p[a] < 0 || p[a] >= gf.n[a]) continue;
      const long long pl = lin3(gf, p[0], p[1], p[2]);
      if (st[pl] == 2) nb_put1(nb, a, l, tt[pl], -EIK_INF, 0);
      else nb_put1(nb, a, l, EIK_INF, EIK_INF, 0);
      bool ok = true;
      for (int d = 0; d < gf.nd; d++)
        if (p[d] < 1 || p[d] > gf.n[d] - 2) ok = false;
      if (ok) {
        int q[3] = {p[0], p[1], p[2]};
        q[a] += sh;
        const long long ql = lin3(gf, q[0], q[1], q[2]);
        if (st[ql] == 2) nb_put2(nb, a, l, tt[ql], -EIK_INF, 0);
        else nb_put2(nb, a, l, EIK_INF, EIK_INF, 0);
      }
    }
  const Key T = key_normal(0.0);
  return gf.nd == 3 ? update_at<3>(nb, T, codes, neg) : update_at<2>(nb, T, codes, neg);
}

// Fine node -> coarse node used for its velocity (nearest neighbour, eikmainfwd.jl:1035-1051).
__device__ __forceinline__ long long fine_to_coarse(const GridDesc& g, const FineInfo& fi, int i, int j,
                                                    int k) {
  const int f[3] = {i, j, k};
  int c[3] = {0, 0, 0};
  const int ds = fi.ds;
  for (int d = 0; d < g.nd; d++) {
    const int di = f[d] / ds;
    const int ri = f[d] + 1 - di * ds;
    c[d] = fi.ijk1[d] + (((double)ri >= (double)ds / 2.0 + 1.0) ? di + 1 : di);
  }
  return lin3(g, c[0], c[1], c[2]);
}

// Source box on grid gg with velocity accessor; writes corner nodes/times/distances.
// sourceboxloctt! (eikmainfwd.jl:1195-1322): the halfway shift only changes a warning.
template <class VelFn>
__device__ int source_box(const GridDesc& gg, const double* src, VelFn velat, int (*corn)[3],
                          double* tcorn, double* dcorn, double* vcorn, uint32_t* warn) {
  const int nc = findenclosingbox(gg, src, corn);
  for (int l = 0; l < nc; l++) {
    double xyz[3];
    for (int d = 0; d < gg.nd; d++) xyz[d] = jr_value(gg.ax[d], corn[l][d] + 1);
    const double dc = distance2points(gg, xyz, src);
    const double v = velat(corn[l][0], corn[l][1], corn[l][2]);
    dcorn[l] = dc;
    vcorn[l] = v;
    tcorn[l] = dc / v;
  }
  if (nc > 1) {
    bool any = false;
    for (int d = 0; d < gg.nd; d++) {
      const double r = fmod(src[d] - gg.co[d], gg.spac[d]);
      const double h2 = gg.spac[d] / 2.0;
      const bool half = (r == h2) || (isfinite(r) && fabs(r - h2) <= 1.4901161193847656e-8 * fmax(fabs(r), fabs(h2)));
      any = any || half;
    }
    if (any) *warn |= WARN_SRC_HALFWAY_SHIFT;
  }
  return nc;
}

// ------------------------------------------------------------ non-refined source box --
__global__ void srcbox_kernel(ForwardBatch fb) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= fb.nsrc) return;
  const GridDesc& g = fb.g;
  const double* src = fb.coordsrc + (size_t)s * g.nd;
  int corn[8][3];
  double tc[8], dc[8], vc[8];
  uint32_t warn = 0;
  const double* vel = fb.vel;
  auto velat = [&](int i, int j, int k) { return vel[lin3(g, i, j, k)]; };
  const int nc = source_box(g, src, velat, corn, tc, dc, vc, &warn);
  SrcOut& o = fb.out[s];
  o.nseeds = nc;
  o.nsrcf = nc;
  o.warn |= warn;
  for (int l = 0; l < nc; l++) {
    fb.seed_lin[(size_t)s * fb.seedcap + l] = (int32_t)lin3(g, corn[l][0], corn[l][1], corn[l][2]);
    fb.seed_tt[(size_t)s * fb.seedcap + l] = tc[l];
    o.distcorn[l] = dc[l];
    o.velcorn[l] = vc[l];
    for (int d = 0; d < 3; d++) o.corn[l][d] = corn[l][d];
  }
}

// Refined window around a source (createfinegrid, eikmainfwd.jl:964-1009): the enclosing
// box on the coarse grid +- noderadius nodes, clipped at the model's borders, refined by
// downscalefactor. Returns the number of fine nodes.
__device__ long long fine_window(const ForwardBatch& fb, const double* src, FineInfo* fi, GridDesc* gf) {
  const GridDesc& g = fb.g;
  int corn[8][3];
  const int nc = findenclosingbox(g, src, corn);
  fi->ds = fb.ds;
  long long nfine = 1;
  for (int d = 0; d < 3; d++) {
    fi->ijk1[d] = 0;
    fi->nf[d] = 1;
    fi->outmin[d] = 0;
    fi->outmax[d] = 0;
  }
  for (int d = 0; d < g.nd; d++) {
    int mn = corn[0][d], mx = corn[0][d];
    for (int l = 1; l < nc; l++) {
      mn = min(mn, corn[l][d]);
      mx = max(mx, corn[l][d]);
    }
    const int v1 = mn - fb.noderadius, v2 = mx + fb.noderadius;
    fi->outmin[d] = v1 < 0;
    fi->outmax[d] = v2 > g.n[d] - 1;
    fi->ijk1[d] = fi->outmin[d] ? 0 : v1;
    const int i2 = fi->outmax[d] ? g.n[d] - 1 : v2;
    fi->nf[d] = (i2 - fi->ijk1[d]) * fb.ds + 1;
    nfine *= fi->nf[d];
  }
  *gf = g;
  for (int d = 0; d < 3; d++) gf->n[d] = fi->nf[d];
  for (int d = 0; d < g.nd; d++) {
    gf->spac[d] = g.spac[d] / (double)fb.ds;
    gf->co[d] = jr_value(g.ax[d], fi->ijk1[d] + 1);
    gf->ax[d] = make_jrange(gf->co[d], gf->spac[d]);
  }
  return nfine;
}

// ---------------------------------------------------------------- refined start-up --
constexpr int FINE_THREADS = 32;
constexpr int MAXPOP = 128;

__global__ void __launch_bounds__(FINE_THREADS) fine_fmm_kernel(ForwardBatch fb, const uint8_t* only) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int s = blockIdx.x;
  if (only && !only[s]) return;  // replay of the flagged sources only
  const int lane = threadIdx.x;
  const GridDesc& g = fb.g;
  SrcOut& o = fb.out[s];
  __shared__ FineInfo fi;
  __shared__ GridDesc gf;
  __shared__ int sh_err, sh_stop, sh_npop, sh_nseed;
  __shared__ int32_t popped[MAXPOP];
  __shared__ double evv[MAXPOP * 6];
  __shared__ uint8_t evc[MAXPOP * 6];
  __shared__ uint8_t evneg[MAXPOP * 6];
  const double* src = fb.coordsrc + (size_t)s * g.nd;

  if (lane == 0) {
    sh_err = 0;
    sh_stop = 0;
    const long long nfine = fine_window(fb, src, &fi, &gf);
    if (nfine > fb.nfmax) sh_err = ERRB_HEAP_OVERFLOW;
    o.fine = fi;
  }
  __syncthreads();
  if (sh_err) {
    if (lane == 0) atomicOr(fb.err, (uint32_t)sh_err);
    return;
  }
  const long long nf = npts(gf);
  double* tt = fb.fine_tt + (size_t)s * fb.nfmax;
  uint8_t* st = fb.fine_status + (size_t)s * fb.nfmax;
  uint8_t* code = fb.fine_code + (size_t)s * fb.nfmax;
  int32_t* idxh = fb.fine_idx + (size_t)s * fb.nfmax;
  int32_t* order = fb.fine_order + (size_t)s * fb.nfmax;
  uint8_t* onh = fb.fine_onh + (size_t)s * fb.nfmax;
  for (long long l = lane; l < nf; l += FINE_THREADS) {
    tt[l] = EIK_INF;
    st[l] = 0;
    code[l] = CODE_NONE;
    idxh[l] = 0;
    onh[l] = 0;
  }
  __syncwarp();
  __syncthreads();

  SmemHeap H;
  H.cap = fb.heapcap;
  H.nodes = reinterpret_cast<double*>(smem_raw);
  H.hand = reinterpret_cast<int32_t*>(smem_raw + sizeof(double) * (H.cap + 1));
  H.idx = idxh;
  H.Nh = 0;
  const double* slow = fb.slow;
  const double* vel = fb.vel;
  auto velat_f = [&](int i, int j, int k) { return vel[fine_to_coarse(g, fi, i, j, k)]; };
  auto coarse_of = [&](int i, int j, int k, long long* cl) {
    if (i % fi.ds || j % fi.ds || k % fi.ds) return false;
    *cl = lin3(g, fi.ijk1[0] + i / fi.ds, fi.ijk1[1] + j / fi.ds, fi.ijk1[2] + k / fi.ds);
    return true;
  };
  const int nd = g.nd;
  const int nneigh = 2 * nd;
  // neighbour order of ttFMM_core! (eikmainfwd.jl:484-496)
  const int NB2[4][3] = {{1, 0, 0}, {0, 1, 0}, {-1, 0, 0}, {0, -1, 0}};
  const int NB3[6][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {-1, 0, 0}, {0, -1, 0}, {0, 0, -1}};
  int32_t* seed_lin = fb.seed_lin + (size_t)s * fb.seedcap;
  double* seed_tt = fb.seed_tt + (size_t)s * fb.seedcap;
  int naccinit = 0;
  int nacc = 0;
  uint32_t warn = 0;

  if (lane == 0) {
    // fine source box
    int corn[8][3];
    double tc[8], dc[8], vc[8];
    naccinit = source_box(gf, src, velat_f, corn, tc, dc, vc, &warn);
    o.nsrcf = naccinit;
    sh_nseed = 0;
    for (int l = 0; l < naccinit; l++) {
      const long long ll = lin3(gf, corn[l][0], corn[l][1], corn[l][2]);
      st[ll] = 2;
      tt[ll] = tc[l];
      order[l] = (int32_t)ll;
      o.distcorn[l] = dc[l];
      o.velcorn[l] = vc[l];
      for (int d = 0; d < 3; d++) o.corn[l][d] = corn[l][d];
    }
    for (int l = 0; l < naccinit; l++) {
      long long cl;
      if (coarse_of(corn[l][0], corn[l][1], corn[l][2], &cl)) {
        seed_lin[sh_nseed] = (int32_t)cl;
        seed_tt[sh_nseed] = tt[lin3(gf, corn[l][0], corn[l][1], corn[l][2])];
        sh_nseed++;
        onh[lin3(gf, corn[l][0], corn[l][1], corn[l][2])] = 1;
      }
    }
    nacc = naccinit;
    // initial narrow band (eikmainfwd.jl:590-621)
    for (int l = 0; l < naccinit; l++)
      for (int ne = 0; ne < nneigh; ne++) {
        int c[3] = {corn[l][0], corn[l][1], corn[l][2]};
        for (int d = 0; d < nd; d++) c[d] += (nd == 2 ? NB2[ne][d] : NB3[ne][d]);
        bool inb = true;
        for (int d = 0; d < nd; d++)
          if (c[d] < 0 || c[d] >= gf.n[d]) inb = false;
        if (!inb) continue;
        const long long cl = lin3(gf, c[0], c[1], c[2]);
        if (st[cl] == 0) {
          int8_t cd[3];
          bool neg = false;
          const double v = fine_update(gf, tt, st, slow[fine_to_coarse(g, fi, c[0], c[1], c[2])], c[0],
                                       c[1], c[2], cd, &neg);
          if (neg) warn |= WARN_NEG_DISCRIMINANT;
          if (!H.insert(v, (int32_t)(cl + 1))) sh_err |= ERRB_HEAP_OVERFLOW;
          st[cl] = 1;
          code[cl] = pack_codes(cd, nd);
        }
      }
  }
  __syncwarp();

  bool firstwarning = true;
  const long long maxiter = nf;
  for (long long iter = 0; iter < maxiter; iter++) {
    // ---- lane 0: pop all equal minima (eikmainfwd.jl:642-762)
    if (lane == 0) {
      sh_npop = 0;
      if (H.Nh < 1 || sh_err) {
        sh_stop = 1;
      } else {
        bool same = true;
        while (same) {
          if (H.Nh < 1) break;
          int32_t h;
          double v;
          H.pop(&h, &v);
          same = (H.nodes[1] == v);
          const long long al = h - 1;
          st[al] = 2;
          tt[al] = v;
          order[nacc++] = (int32_t)al;
          const int ai = (int)(al % gf.n[0]);
          const int aj = (int)((al / gf.n[0]) % gf.n[1]);
          const int ak = (int)(al / ((long long)gf.n[0] * gf.n[1]));
          long long cl;
          if (coarse_of(ai, aj, ak, &cl)) {
            if (sh_nseed >= fb.seedcap) {
              sh_err |= ERRB_SEED_OVERFLOW;
            } else {
              seed_lin[sh_nseed] = (int32_t)cl;
              seed_tt[sh_nseed] = v;
              sh_nseed++;
            }
            onh[al] = 1;
          }
          const int a3[3] = {ai, aj, ak};
          bool onedge = false;
          for (int d = 0; d < nd; d++) {
            if (a3[d] == 0 && !fi.outmin[d]) onedge = true;
            if (a3[d] == gf.n[d] - 1 && !fi.outmax[d]) onedge = true;
          }
          if (onedge) {
            if (sh_nseed < 1) {
              if (firstwarning) {
                warn |= WARN_BORDER_BEFORE_COARSE;
                firstwarning = false;
              }
              continue;
            }
            sh_stop = 2;
            break;
          }
          if (sh_npop >= MAXPOP) {
            sh_err |= ERRB_BATCH_OVERFLOW;
            break;
          }
          popped[sh_npop++] = (int32_t)al;
        }
      }
    }
    __syncwarp();
    if (sh_stop || sh_err) break;
    // ---- all lanes: stencil updates of the popped nodes' neighbours (read-only phase)
    const int nev = sh_npop * nneigh;
    for (int e = lane; e < nev; e += FINE_THREADS) {
      const long long al = popped[e / nneigh];
      const int ne = e % nneigh;
      int c[3] = {(int)(al % gf.n[0]), (int)((al / gf.n[0]) % gf.n[1]), (int)(al / ((long long)gf.n[0] * gf.n[1]))};
      for (int d = 0; d < nd; d++) c[d] += (nd == 2 ? NB2[ne][d] : NB3[ne][d]);
      bool inb = true;
      for (int d = 0; d < nd; d++)
        if (c[d] < 0 || c[d] >= gf.n[d]) inb = false;
      evc[e] = 0xff;
      if (!inb) continue;
      const long long cl = lin3(gf, c[0], c[1], c[2]);
      if (st[cl] == 2) continue;
      int8_t cd[3];
      bool neg = false;
      evv[e] = fine_update(gf, tt, st, slow[fine_to_coarse(g, fi, c[0], c[1], c[2])], c[0], c[1], c[2], cd,
                           &neg);
      evc[e] = pack_codes(cd, nd);
      evneg[e] = neg;
    }
    __syncwarp();
    // ---- lane 0: heap inserts/updates in the reference's order (eikmainfwd.jl:768-813)
    if (lane == 0) {
      for (int e = 0; e < nev; e++) {
        if (sh_err) break;
        if (evc[e] == 0xff) continue;
        const long long al = popped[e / nneigh];
        const int ne = e % nneigh;
        int c[3] = {(int)(al % gf.n[0]), (int)((al / gf.n[0]) % gf.n[1]), (int)(al / ((long long)gf.n[0] * gf.n[1]))};
        for (int d = 0; d < nd; d++) c[d] += (nd == 2 ? NB2[ne][d] : NB3[ne][d]);
        const long long cl = lin3(gf, c[0], c[1], c[2]);
        if (evneg[e]) warn |= WARN_NEG_DISCRIMINANT;
        if (st[cl] == 0) {
          if (!H.insert(evv[e], (int32_t)(cl + 1))) sh_err |= ERRB_HEAP_OVERFLOW;
          st[cl] = 1;
          code[cl] = evc[e];
        } else if (st[cl] == 1) {
          H.update(evv[e], (int32_t)(cl + 1));
          code[cl] = evc[e];
        }
      }
    }
    __syncwarp();
  }
  if (lane == 0) {
    if (sh_stop != 2) warn |= WARN_FINE_NO_TRIGGER;
    o.nseeds = sh_nseed;
    o.nacc = nacc;
    o.warn |= warn;
    if (sh_err) atomicOr(fb.err, (uint32_t)sh_err);
  }
}

// ------------------------------------------------ refined start-up as a fixed point --
// The refined window is solved by the round solver like any coarse grid (its values are
// the fixed point of the same order rule, hence the heap's values for every node the heap
// accepts before its stop). What the heap decides is WHERE it stops: at the first node
// on a non-border edge of the window accepted after at least one coarse-coincident node
// (eikmainfwd.jl:724-754). Acceptance follows the keys of the order rule, so the stop
// node is the edge node of smallest key above the first coarse-coincident key, and the
// accepted set is every node of smaller key plus that node. Only when another node has
// exactly the stop node's traveltime (or an edge node ties with the first coarse-coincident
// node) does the heap's internal order decide; those sources are replayed exactly.

// Window, fine source box, the fine problem of the round solver, its slowness and seeds.
__global__ void fine_setup_kernel(ForwardBatch fb, CoarseProblem* fprobs, const double* dsmin, double gate,
                                  int32_t* fseed_lin, double* fseed_tt, double* fslow, double* fkL, uint8_t* fkd) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= fb.nsrc) return;
  const GridDesc& g = fb.g;
  SrcOut& o = fb.out[s];
  const double* src = fb.coordsrc + (size_t)s * g.nd;
  FineInfo fi;
  GridDesc gf;
  const long long nfine = fine_window(fb, src, &fi, &gf);
  o.fine = fi;
  if (nfine > fb.nfmax) {
    atomicOr(fb.err, ERRB_HEAP_OVERFLOW);
    o.nsrcf = 0;
    return;
  }
  const double* vel = fb.vel;
  auto velat_f = [&](int i, int j, int k) { return vel[fine_to_coarse(g, fi, i, j, k)]; };
  int corn[8][3];
  double tc[8], dc[8], vc[8];
  uint32_t warn = 0;
  const int nc = source_box(gf, src, velat_f, corn, tc, dc, vc, &warn);
  o.nsrcf = nc;
  o.nseeds = 0;
  o.nacc = 0;
  o.warn |= warn;
  for (int l = 0; l < nc; l++) {
    o.distcorn[l] = dc[l];
    o.velcorn[l] = vc[l];
    for (int d = 0; d < 3; d++) o.corn[l][d] = corn[l][d];
    fseed_lin[(size_t)s * 8 + l] = (int32_t)lin3(gf, corn[l][0], corn[l][1], corn[l][2]);
    fseed_tt[(size_t)s * 8 + l] = tc[l];
  }
  CoarseProblem& P = fprobs[s];
  P.g = gf;
  P.slow = fslow + (size_t)s * fb.nfmax;
  P.t = fb.fine_tt + (size_t)s * fb.nfmax;
  P.code = fb.fine_code + (size_t)s * fb.nfmax;
  P.kL = fkL + (size_t)s * fb.nfmax;
  P.kd = fkd + (size_t)s * fb.nfmax;
  double dh[3];
  node_dh(gf, 0, dh);
  double hmin = dh[0];
  for (int a = 1; a < gf.nd; a++) hmin = fmin(hmin, dh[a]);
  const double smin = *dsmin;
  uniform_coeffs(gf, &P.c1u, &P.c2u);
  P.delta = gate * hmin * smin;
  P.incmin = 0.999 * (2.0 / 3.0) * hmin * smin / sqrt((double)gf.nd);
}

__global__ void fine_fill_kernel(ForwardBatch fb, const CoarseProblem* fprobs) {
  const long long tot = (long long)fb.nsrc * fb.nfmax;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(q / fb.nfmax);
    const long long l = q - (long long)s * fb.nfmax;
    if (fb.out[s].nsrcf == 0) continue;
    const CoarseProblem& P = fprobs[s];
    const GridDesc& gf = P.g;
    if (l >= npts(gf)) continue;
    const FineInfo& fi = fb.out[s].fine;
    const int i = (int)(l % gf.n[0]), j = (int)((l / gf.n[0]) % gf.n[1]), k = (int)(l / ((long long)gf.n[0] * gf.n[1]));
    const_cast<double*>(P.slow)[l] = fb.slow[fine_to_coarse(fb.g, fi, i, j, k)];
    P.t[l] = EIK_INF;
    P.code[l] = CODE_NONE;
    P.kd[l] = 0;
    const size_t o = (size_t)s * fb.nfmax + l;
    fb.fine_status[o] = 0;
    fb.fine_onh[o] = 0;
  }
}

__device__ __forceinline__ Key fine_key(const CoarseProblem& P, long long l) {
  const double t = P.t[l];
  const uint8_t cb = P.code[l];
  if (cb & CODE_SRC_BIT) return Key{P.kL[l], (int)P.kd[l], t};
  return Key{t, 0, t};
}
__device__ __forceinline__ bool key_lt(const Key& a, const Key& b) { return !key_le(b, a); }

constexpr int SEL_THREADS = 256;

// Block-wide argmin of keys (ties: smaller node index); idx -1 = none.
__device__ void block_min_key(Key* k, long long* idx) {
  __shared__ double sL[SEL_THREADS], st_[SEL_THREADS];
  __shared__ int sd[SEL_THREADS];
  __shared__ long long si[SEL_THREADS];
  const int t = threadIdx.x;
  sL[t] = k->L;
  sd[t] = k->d;
  st_[t] = k->t;
  si[t] = *idx;
  __syncthreads();
  for (int w = SEL_THREADS / 2; w > 0; w >>= 1) {
    if (t < w) {
      const long long ib = si[t + w];
      if (ib >= 0) {
        const Key kb{sL[t + w], sd[t + w], st_[t + w]};
        const Key ka{sL[t], sd[t], st_[t]};
        const long long ia = si[t];
        if (ia < 0 || key_lt(kb, ka) || (!key_lt(ka, kb) && ib < ia)) {
          sL[t] = kb.L;
          sd[t] = kb.d;
          st_[t] = kb.t;
          si[t] = ib;
        }
      }
    }
    __syncthreads();
  }
  *k = Key{sL[0], sd[0], st_[0]};
  *idx = si[0];
  __syncthreads();
}

__device__ __forceinline__ bool fine_less(const CoarseProblem& P, int32_t a, int32_t b) {
  const Key ka = fine_key(P, a), kb = fine_key(P, b);
  if (key_lt(ka, kb)) return true;
  if (key_lt(kb, ka)) return false;
  return a < b;
}

// Acceptance set, FMM order (sorted keys; the source box first, in corner order), coarse
// seeds and status of one source's refined window. One CTA per source.
__global__ void __launch_bounds__(SEL_THREADS) fine_select_kernel(ForwardBatch fb, const CoarseProblem* fprobs,
                                                                  uint8_t* tie) {
  const int s = blockIdx.x;
  const int tid = threadIdx.x;
  SrcOut& o = fb.out[s];
  if (o.nsrcf == 0) {
    if (tid == 0) tie[s] = 0;
    return;
  }
  const CoarseProblem& P = fprobs[s];
  const GridDesc& gf = P.g;
  const FineInfo fi = o.fine;
  const long long n = npts(gf);
  const int nd = gf.nd;
  const size_t base = (size_t)s * fb.nfmax;
  uint8_t* st = fb.fine_status + base;
  uint8_t* onh = fb.fine_onh + base;
  int32_t* order = fb.fine_order + base;
  int32_t* tmp = fb.fine_idx + base;
  auto coords = [&](long long l, int* f) {
    f[0] = (int)(l % gf.n[0]);
    f[1] = (int)((l / gf.n[0]) % gf.n[1]);
    f[2] = (int)(l / ((long long)gf.n[0] * gf.n[1]));
  };
  auto is_cc = [&](long long l) {
    int f[3];
    coords(l, f);
    for (int d = 0; d < nd; d++)
      if (f[d] % fi.ds) return false;
    return true;
  };
  auto is_edge = [&](long long l) {
    int f[3];
    coords(l, f);
    for (int d = 0; d < nd; d++) {
      if (f[d] == 0 && !fi.outmin[d]) return true;
      if (f[d] == gf.n[d] - 1 && !fi.outmax[d]) return true;
    }
    return false;
  };
  // corners of the source box (accepted first, never popped)
  __shared__ long long corner[8];
  __shared__ int ncorner;
  if (tid == 0) {
    ncorner = o.nsrcf;
    for (int c = 0; c < o.nsrcf; c++) corner[c] = lin3(gf, o.corn[c][0], o.corn[c][1], o.corn[c][2]);
  }
  __syncthreads();
  auto is_corner = [&](long long l) {
    for (int c = 0; c < ncorner; c++)
      if (corner[c] == l) return true;
    return false;
  };
  // first coarse-coincident key
  Key kc = key_unreached();
  long long ic = -1;
  for (long long l = tid; l < n; l += SEL_THREADS) {
    if (!(P.t[l] < EIK_INF) || !is_cc(l)) continue;
    const Key k = fine_key(P, l);
    if (ic < 0 || key_lt(k, kc) || (!key_lt(kc, k) && l < ic)) {
      kc = k;
      ic = l;
    }
  }
  block_min_key(&kc, &ic);
  // stop node: the popped edge node of smallest key above kc
  Key ks = key_unreached();
  long long is = -1;
  bool early_edge = false;
  for (long long l = tid; l < n; l += SEL_THREADS) {
    if (!(P.t[l] < EIK_INF) || !is_edge(l) || is_corner(l)) continue;
    const Key k = fine_key(P, l);
    if (ic >= 0 && !key_lt(kc, k)) {
      if (key_lt(k, kc)) early_edge = true;
      continue;
    }
    if (is < 0 || key_lt(k, ks) || (!key_lt(ks, k) && l < is)) {
      ks = k;
      is = l;
    }
  }
  early_edge = __syncthreads_or(early_edge);
  block_min_key(&ks, &is);
  // ties that only the heap's order can settle
  bool amb = false;
  if (ic < 0) amb = true;  // no coarse-coincident node reached: leave it to the replay
  for (long long l = tid; l < n && !amb; l += SEL_THREADS) {
    const double t = P.t[l];
    if (!(t < EIK_INF)) continue;
    if (is >= 0 && l != is && t == ks.t) amb = true;
    if (ic >= 0 && kc.L != -EIK_INF && l != ic && is_edge(l) && !is_corner(l) && t == kc.t) amb = true;
  }
  amb = __syncthreads_or(amb);
  if (tid == 0) tie[s] = amb ? 1 : 0;
  if (amb) return;
  // status and the accepted non-corner nodes (unordered)
  __shared__ unsigned int nlist;
  if (tid == 0) nlist = 0;
  __syncthreads();
  const int nc = ncorner;
  for (long long l = tid; l < n; l += SEL_THREADS) {
    const double t = P.t[l];
    uint8_t sv = 0;
    if (t < EIK_INF) {
      const bool acc = is_corner(l) || is < 0 || l == is || key_lt(fine_key(P, l), ks);
      sv = acc ? 2 : 1;
      if (acc && !is_corner(l)) order[nc + atomicAdd(&nlist, 1u)] = (int32_t)l;
    }
    st[l] = sv;
    onh[l] = 0;
  }
  __syncthreads();
  const int m = (int)nlist;
  // merge sort of order[nc, nc+m) by (key, index): each element finds its rank in the other run
  int32_t* a = order + nc;
  int32_t* b = tmp;
  for (int w = 1; w < m; w *= 2) {
    for (int i = tid; i < m; i += SEL_THREADS) {
      const int run = i / w;
      const int p0 = (run & ~1) * w;
      const int mid = min(p0 + w, m), end = min(p0 + 2 * w, m);
      const int32_t x = a[i];
      int lo, hi;
      if ((run & 1) == 0) {  // left run: count right elements below x
        lo = mid;
        hi = end;
      } else {
        lo = p0;
        hi = mid;
      }
      const int first = lo;
      while (lo < hi) {
        const int md = (lo + hi) >> 1;
        if (fine_less(P, a[md], x)) lo = md + 1;
        else hi = md;
      }
      const int rank = lo - first;
      const int pos = ((run & 1) == 0) ? (i - p0) + rank + p0 : (i - mid) + rank + p0;
      b[pos] = x;
    }
    __syncthreads();
    int32_t* t2 = a;
    a = b;
    b = t2;
  }
  if (a != order + nc)
    for (int i = tid; i < m; i += SEL_THREADS) order[nc + i] = a[i];
  if (tid < nc) order[tid] = (int32_t)corner[tid];
  __syncthreads();
  // coarse seeds in acceptance order
  const int nacc = nc + m;
  __shared__ int wsum[SEL_THREADS / 32];
  __shared__ int carry;
  if (tid == 0) carry = 0;
  __syncthreads();
  for (int b0 = 0; b0 < nacc; b0 += SEL_THREADS) {
    const int p = b0 + tid;
    long long l = -1;
    bool ccf = false;
    if (p < nacc) {
      l = order[p];
      ccf = is_cc(l);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, ccf);
    const int lane = tid & 31, wid = tid >> 5;
    if (lane == 0) wsum[wid] = __popc(bal);
    __syncthreads();
    int off = carry;
    for (int w = 0; w < wid; w++) off += wsum[w];
    off += __popc(bal & ((1u << lane) - 1u));
    if (ccf) {
      onh[l] = 1;
      if (off < fb.seedcap) {
        int f[3];
        coords(l, f);
        fb.seed_lin[(size_t)s * fb.seedcap + off] =
            (int32_t)lin3(fb.g, fi.ijk1[0] + f[0] / fi.ds, fi.ijk1[1] + f[1] / fi.ds, fi.ijk1[2] + f[2] / fi.ds);
        fb.seed_tt[(size_t)s * fb.seedcap + off] = P.t[l];
      } else {
        atomicOr(fb.err, ERRB_SEED_OVERFLOW);
      }
    }
    __syncthreads();
    if (tid == 0)
      for (int w = 0; w < SEL_THREADS / 32; w++) carry += wsum[w];
    __syncthreads();
  }
  if (tid == 0) {
    o.nseeds = carry < fb.seedcap ? carry : fb.seedcap;
    o.nacc = nacc;
    if (is < 0) o.warn |= WARN_FINE_NO_TRIGGER;
    if (early_edge) o.warn |= WARN_BORDER_BEFORE_COARSE;
  }
}

void launch_fine_setup(const ForwardBatch& fb, CoarseProblem* fprobs, const double* dsmin, double gate,
                       int32_t* fseed_lin, double* fseed_tt, double* fine_slow, double* fine_kL, uint8_t* fine_kd,
                       cudaStream_t st) {
  fine_setup_kernel<<<(fb.nsrc + 63) / 64, 64, 0, st>>>(fb, fprobs, dsmin, gate, fseed_lin, fseed_tt, fine_slow,
                                                         fine_kL, fine_kd);
  fine_fill_kernel<<<592, 256, 0, st>>>(fb, fprobs);
}

void launch_fine_select(const ForwardBatch& fb, const CoarseProblem* fprobs, uint8_t* fine_tie, cudaStream_t st) {
  fine_select_kernel<<<fb.nsrc, SEL_THREADS, 0, st>>>(fb, fprobs, fine_tie);
}

// ------------------------------------------------------------------- launchers --
void launch_srcbox(const ForwardBatch& fb, cudaStream_t st) {
  const int T = 128;
  srcbox_kernel<<<(fb.nsrc + T - 1) / T, T, 0, st>>>(fb);
}

size_t fine_smem_bytes(int heapcap) { return (sizeof(double) + sizeof(int32_t)) * (size_t)(heapcap + 1); }

void launch_fine(const ForwardBatch& fb, cudaStream_t st) {
  const size_t sm = fine_smem_bytes(fb.heapcap);
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(fine_fmm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set = true;
  }
  fine_fmm_kernel<<<fb.nsrc, FINE_THREADS, sm, st>>>(fb, nullptr);
}

void launch_fine_replay(const ForwardBatch& fb, const uint8_t* fine_tie, cudaStream_t st) {
  const size_t sm = fine_smem_bytes(fb.heapcap);
  cudaFuncSetAttribute(fine_fmm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  fine_fmm_kernel<<<fb.nsrc, FINE_THREADS, sm, st>>>(fb, fine_tie);
}

}  // namespace eik
