// Coarse-grid forward solve: the reference's heap-ordered FMM main loop
// (ttFMM_core!, src/EikSolv/eikmainfwd.jl:427-823) restated as the fixed point of the
// order rule of stencil.cuh and solved by a block-tiled active-list iteration.
//
// One persistent launch serves many problems (sources, possibly of different grids)
// through one queue of tiles. A CTA takes a tile, stages its traveltimes and keys plus a
// 2-node halo in shared memory, iterates the rule on its active nodes until nothing
// changes (or a pass limit), writes the changed nodes back and queues the neighbouring
// tiles whose halo it changed. The launch ends when no tile is queued or in work.
// Every wait is bounded (global timer), every solve bounded in tile activations; both
// report through an error word instead of trapping.
#include "kernels.cuh"
#include "queue.cuh"

namespace eik {


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

__global__ void queue_init_kernel(SolveArgs a) {
  const long long cap = (long long)a.q.mask + 1;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < cap * QBUCKETS;
       q += (long long)gridDim.x * blockDim.x)
    a.q.seq[q] = (unsigned long long)(q % cap);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < a.ntiles;
       q += (long long)gridDim.x * blockDim.x) {
    a.tile_faces[q] = 0;
    a.tile_flag[q] = 0;
    a.tile_prio[q] = (unsigned long long)__double_as_longlong(EIK_INF);
  }
  if (blockIdx.x == 0 && threadIdx.x < QBUCKETS) {
    a.q.head[threadIdx.x] = 0;
    a.q.tail[threadIdx.x] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *a.pending = 0;
    *a.activations = 0;
    *a.node_evals = 0;
    *a.abort_flag = 0;
  }
}

template <int ND>
__device__ __forceinline__ long long tile_of(const CoarseProblem& P, int i, int j, int k) {
  using C = TileCfg<ND>;
  return (long long)(i / C::TX) + (long long)P.nt[0] * ((long long)(j / C::TY) + (long long)P.nt[1] * (k / C::TZ));
}

// Seeds: fixed traveltimes of the source points (coarse source box or coarse-coincident
// accepted fine nodes); the tiles within two nodes of a seed start the solve.
template <int ND>
__global__ void seed_kernel(SolveArgs a, ForwardBatch fb) {
  const int s = blockIdx.x;
  const CoarseProblem& P = a.probs[s];
  const int ns = fb.out[s].nseeds;
  for (int q = threadIdx.x; q < ns; q += blockDim.x) {
    const long long l = fb.seed_lin[(size_t)s * fb.seedcap + q];
    P.t[l] = fb.seed_tt[(size_t)s * fb.seedcap + q];
    P.code[l] = (uint8_t)(CODE_NONE | CODE_SRC_BIT);
    P.kL[l] = -EIK_INF;
    P.kd[l] = 0;
  }
  __syncthreads();
  __threadfence();
  for (int q = threadIdx.x; q < ns; q += blockDim.x) {
    const long long l = fb.seed_lin[(size_t)s * fb.seedcap + q];
    const int i = (int)(l % P.g.n[0]);
    const int j = (int)((l / P.g.n[0]) % P.g.n[1]);
    const int k = (int)(l / ((long long)P.g.n[0] * P.g.n[1]));
    const int c[3] = {i, j, k};
    const double pr = fb.seed_tt[(size_t)s * fb.seedcap + q];
    enqueue_tile(a, s, tile_of<ND>(P, i, j, k), FACES_ALL, pr);
    for (int ax = 0; ax < ND; ax++)
      for (int d = -2; d <= 2; d += 4) {
        int p[3] = {c[0], c[1], c[2]};
        p[ax] += d;
        if (p[ax] < 0 || p[ax] >= P.g.n[ax]) continue;
        enqueue_tile(a, s, tile_of<ND>(P, p[0], p[1], p[2]), FACES_ALL, pr);
      }
  }
}

// ------------------------------------------------------------------ tile solve --
// One warp owns one tile at a time (its own shared-memory slice, warp-level syncs only),
// so an SM keeps many independent tiles in flight and hides the FP64 latency of the
// update; CTAs only group warps for occupancy.
template <int ND>
struct TileSmem {
  using C = TileCfg<ND>;
  static constexpr int TN = C::TX * C::TY * C::TZ;
  static constexpr int HN = C::HX * C::HY * C::HZ;
  double t[HN];
  double L[HN];       // key level of special nodes
  double slow[TN];
  uint8_t fl[HN];     // bit0 special key, bits 1..4 depth
  uint8_t code[TN];
  uint8_t act[TN];    // to be evaluated (plain stores of 1 from any lane)
  uint8_t dirty[TN];  // changed, to be written back
  int16_t list[TN];
};

template <int ND>
__device__ __forceinline__ int hidx(int x, int y, int z) {
  using C = TileCfg<ND>;
  return (x + C::H) + C::HX * ((y + C::H) + C::HY * (ND == 3 ? z + C::H : 0));
}

template <int ND>
__device__ __forceinline__ void smem_keyLd(const TileSmem<ND>& S, int h, double* L, int* d) {
  const uint8_t f = S.fl[h];
  if (f & 1) {
    *L = S.L[h];
    *d = f >> 1;
  } else {
    *L = S.t[h];
    *d = 0;
  }
}

// Smallest traveltime among the in-grid immediate neighbours of tile node li.
template <int ND>
__device__ __forceinline__ double node_potential(const TileSmem<ND>& S, const GridDesc& g, int ox, int oy,
                                                 int oz, int li) {
  using C = TileCfg<ND>;
  const int x = li % C::TX, y = (li / C::TX) % C::TY, z = li / (C::TX * C::TY);
  const int c[3] = {ox + x, oy + y, oz + z};
  const int hc[3] = {x, y, z};
  double pm = EIK_INF;
#pragma unroll
  for (int ax = 0; ax < ND; ax++)
#pragma unroll
    for (int sh = -1; sh <= 1; sh += 2) {
      if (c[ax] + sh < 0 || c[ax] + sh >= g.n[ax]) continue;
      int q[3] = {hc[0], hc[1], hc[2]};
      q[ax] += sh;
      pm = fmin(pm, S.t[hidx<ND>(q[0], q[1], q[2])]);
    }
  return pm;
}

template <int ND>
__device__ __forceinline__ double eval_node(const TileSmem<ND>& S, const GridDesc& g, int ox, int oy, int oz,
                                            int li, int8_t* cd, Key* kk, bool* neg) {
  using C = TileCfg<ND>;
  const int x = li % C::TX, y = (li / C::TX) % C::TY, z = li / (C::TX * C::TY);
  const int c[3] = {ox + x, oy + y, oz + z};
  const int hc[3] = {x, y, z};
  Nbhd nb;
  nb_clear(nb);
  node_dh(g, c[0], nb.dh);
  nb.slow = S.slow[li];
#pragma unroll
  for (int ax = 0; ax < ND; ax++)
#pragma unroll
    for (int l = 0; l < 2; l++) {
      const int sh = l == 0 ? 1 : -1;
      int p[3] = {c[0], c[1], c[2]};
      p[ax] += sh;
      if (p[ax] < 0 || p[ax] >= g.n[ax]) continue;
      int q[3] = {hc[0], hc[1], hc[2]};
      q[ax] += sh;
      const int h1 = hidx<ND>(q[0], q[1], q[2]);
      double L;
      int d;
      smem_keyLd<ND>(S, h1, &L, &d);
      nb_put1(nb, ax, l, S.t[h1], L, d);
      bool ok = true;
#pragma unroll
      for (int dd = 0; dd < ND; dd++)
        if (p[dd] < 1 || p[dd] > g.n[dd] - 2) ok = false;
      if (ok) {
        q[ax] += sh;
        const int h2 = hidx<ND>(q[0], q[1], q[2]);
        smem_keyLd<ND>(S, h2, &L, &d);
        nb_put2(nb, ax, l, S.t[h2], L, d);
      }
    }
  return prefix_rule<ND>(nb, cd, kk, neg);
}

__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Processes one tile with the 32 lanes of the calling warp. Returns the dirty-face mask
// (bit 6: not converged within the pass limit) and the smallest changed face traveltime.
template <int ND>
__device__ int process_tile(const SolveArgs& a, TileSmem<ND>& S, int prob, long long tile, uint32_t faces,
                            double* fmin_out) {
  using C = TileCfg<ND>;
  constexpr int TN = TileSmem<ND>::TN, HN = TileSmem<ND>::HN;
  constexpr int NPT = (TN + 31) / 32;
  const CoarseProblem& P = a.probs[prob];
  const GridDesc& g = P.g;
  const int tx = (int)(tile % P.nt[0]);
  const int ty = (int)((tile / P.nt[0]) % P.nt[1]);
  const int tz = (int)(tile / ((long long)P.nt[0] * P.nt[1]));
  const int ox = tx * C::TX, oy = ty * C::TY, oz = tz * C::TZ;
  const int lane = threadIdx.x & 31;

  // ---- stage tile + halo
  for (int h = lane; h < HN; h += 32) {
    const int hx = h % C::HX, hy = (h / C::HX) % C::HY, hz = h / (C::HX * C::HY);
    const int gx = ox + hx - C::H, gy = oy + hy - C::H, gz = (ND == 3) ? oz + hz - C::H : 0;
    double tv = EIK_INF, Lv = 0.0;
    uint8_t f = 0;
    if (gx >= 0 && gx < g.n[0] && gy >= 0 && gy < g.n[1] && gz >= 0 && gz < g.n[2]) {
      const long long l = lin3(g, gx, gy, gz);
      // L2-coherent loads: other SMs write these between activations of this tile
      tv = __ldcg(P.t + l);
      const uint8_t cb = __ldcg(P.code + l);
      if (cb & CODE_SRC_BIT) {
        Lv = __ldcg(P.kL + l);
        f = (uint8_t)(1 | (__ldcg(P.kd + l) << 1));
      }
      const bool inter = hx >= C::H && hx < C::H + C::TX && hy >= C::H && hy < C::H + C::TY &&
                         (ND == 2 || (hz >= C::H && hz < C::H + C::TZ));
      if (inter) {
        const int li = (hx - C::H) + C::TX * ((hy - C::H) + C::TY * (ND == 3 ? hz - C::H : 0));
        S.code[li] = cb & 0x7f;
        S.slow[li] = P.slow[l];
      }
    }
    S.t[h] = tv;
    S.L[h] = Lv;
    S.fl[h] = f;
  }
  __syncwarp();
  // ---- initial active set from the dirty faces (source points are never updated)
#pragma unroll
  for (int r = 0; r < NPT; r++) {
    const int li = lane + 32 * r;
    if (li >= TN) continue;
    const int x = li % C::TX, y = (li / C::TX) % C::TY, z = li / (C::TX * C::TY);
    bool act = (faces & FACES_ALL) != 0;
    act = act || ((faces & 1) && x < 2) || ((faces & 2) && x >= C::TX - 2) || ((faces & 4) && y < 2) ||
          ((faces & 8) && y >= C::TY - 2) || ((faces & 16) && z < 2) || ((faces & 32) && z >= C::TZ - 2);
    const int h = hidx<ND>(x, y, z);
    const bool src = (S.fl[h] & 1) && S.L[h] == -EIK_INF;
    const bool inside = ox + x < g.n[0] && oy + y < g.n[1] && oz + z < g.n[2];
    S.act[li] = (act && !src && inside) ? 1 : 0;
    S.dirty[li] = 0;
  }
  double hmin = g.spac[0];
  if (!is_cart(g)) {
    double dh[3];
    node_dh(g, 0, dh);
    hmin = fmin(dh[0], dh[1]);
    if (ND == 3) hmin = fmin(hmin, dh[2]);
  }
  const double gate = a.gate * hmin;
  __syncwarp();

  int fm = 0;
  double fmin_changed = EIK_INF;
  int pass = 0;
  unsigned long long evals = 0;
  bool unconv = false;
  for (;;) {
    // ---- front of the active nodes, gated evaluation list
    double pot[NPT];
    double mypot = EIK_INF;
#pragma unroll
    for (int r = 0; r < NPT; r++) {
      const int li = lane + 32 * r;
      pot[r] = EIK_INF;
      if (li >= TN || !S.act[li]) continue;
      pot[r] = node_potential<ND>(S, g, ox, oy, oz, li);
      if (!(pot[r] < EIK_INF)) S.act[li] = 0;  // no reached neighbour: nothing to compute
      mypot = fmin(mypot, pot[r]);
    }
    const double front = warp_min(mypot);
    if (!(front < EIK_INF)) break;
    int nlist = 0;
#pragma unroll
    for (int r = 0; r < NPT; r++) {
      const int li = lane + 32 * r;
      const bool sel = li < TN && S.act[li] && pot[r] <= front + gate * S.slow[li];
      const unsigned m = __ballot_sync(0xffffffffu, sel);
      if (sel) {
        S.list[nlist + __popc(m & ((1u << lane) - 1u))] = (int16_t)li;
        S.act[li] = 0;
      }
      nlist += __popc(m);
    }
    __syncwarp();
    // ---- evaluate
    double nv[NPT];
    Key nk[NPT];
    uint8_t nc[NPT];
    int nli[NPT];
#pragma unroll
    for (int r = 0; r < NPT; r++) {
      const int e = lane + 32 * r;
      nli[r] = -1;
      if (e >= nlist) continue;
      const int li = S.list[e];
      int8_t cd[3] = {0, 0, 0};
      bool neg = false;
      nv[r] = eval_node<ND>(S, g, ox, oy, oz, li, cd, &nk[r], &neg);
      nc[r] = pack_codes(cd, ND);
      nli[r] = li;
      evals++;
    }
    __syncwarp();
    // ---- apply
#pragma unroll
    for (int r = 0; r < NPT; r++) {
      const int li = nli[r];
      if (li < 0) continue;
      const int x = li % C::TX, y = (li / C::TX) % C::TY, z = li / (C::TX * C::TY);
      const int hm = hidx<ND>(x, y, z);
      double Lo;
      int dold;
      smem_keyLd<ND>(S, hm, &Lo, &dold);
      const double ot = S.t[hm];
      const Key old = Key{Lo, dold, ot};
      const bool same_t = (nv[r] == ot) || (isinf(nv[r]) && isinf(ot));
      const bool tkchange = !(same_t && key_eq(nk[r], old));
      if (!tkchange && nc[r] == S.code[li]) continue;
      S.code[li] = nc[r];
      S.dirty[li] = 1;
      if (!tkchange) continue;
      S.t[hm] = nv[r];
      const bool special = !(nk[r].L == nv[r] && nk[r].d == 0);
      S.fl[hm] = special ? (uint8_t)(1 | (nk[r].d << 1)) : (uint8_t)0;
      S.L[hm] = special ? nk[r].L : 0.0;
      const int xyz[3] = {x, y, z};
      const int T3[3] = {C::TX, C::TY, C::TZ};
      const int o3[3] = {ox, oy, oz};
#pragma unroll
      for (int ax = 0; ax < ND; ax++)
#pragma unroll
        for (int d = -2; d <= 2; d++) {
          if (d == 0) continue;
          int q[3] = {xyz[0], xyz[1], xyz[2]};
          q[ax] += d;
          if (q[ax] < 0 || q[ax] >= T3[ax] || o3[ax] + q[ax] >= g.n[ax]) continue;
          const int lq = q[0] + C::TX * (q[1] + C::TY * q[2]);
          const int hq = hidx<ND>(q[0], q[1], q[2]);
          const bool src = (S.fl[hq] & 1) && S.L[hq] == -EIK_INF;
          if (!src) S.act[lq] = 1;
        }
      int f = 0;
      if (x < 2) f |= 1;
      if (x >= C::TX - 2) f |= 2;
      if (y < 2) f |= 4;
      if (y >= C::TY - 2) f |= 8;
      if (ND == 3 && z < 2) f |= 16;
      if (ND == 3 && z >= C::TZ - 2) f |= 32;
      if (f) {
        fm |= f;
        fmin_changed = fmin(fmin_changed, nv[r]);
      }
    }
    __syncwarp();
    pass++;
    bool anyact = false;
#pragma unroll
    for (int r = 0; r < NPT; r++) {
      const int li = lane + 32 * r;
      anyact = anyact || (li < TN && S.act[li]);
    }
    if (!__any_sync(0xffffffffu, anyact)) break;
    if (pass >= a.max_passes) {
      unconv = true;
      break;
    }
  }
  // ---- write back
#pragma unroll
  for (int r = 0; r < NPT; r++) {
    const int li = lane + 32 * r;
    if (li >= TN || !S.dirty[li]) continue;
    const int x = li % C::TX, y = (li / C::TX) % C::TY, z = li / (C::TX * C::TY);
    const int h = hidx<ND>(x, y, z);
    const long long l = lin3(g, ox + x, oy + y, oz + z);
    P.t[l] = S.t[h];
    const bool special = S.fl[h] & 1;
    P.code[l] = (uint8_t)(S.code[li] | (special ? CODE_SRC_BIT : 0));
    if (special) {
      P.kL[l] = S.L[h];
      P.kd[l] = (uint8_t)(S.fl[h] >> 1);
    }
  }
  // reduce face mask and trigger time over the warp
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) fm |= __shfl_xor_sync(0xffffffffu, fm, o);
  *fmin_out = warp_min(fmin_changed);
  unsigned long long ev = evals;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) ev += __shfl_xor_sync(0xffffffffu, ev, o);
  if (lane == 0 && ev) atomicAdd(a.node_evals, ev);
  return fm | (unconv ? 64 : 0);
}

template <int ND>
__global__ void __launch_bounds__(SOLVE_THREADS, 2) coarse_solve_kernel(SolveArgs a) {
  extern __shared__ __align__(16) unsigned char solve_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  TileSmem<ND>& S = reinterpret_cast<TileSmem<ND>*>(solve_smem)[warp];
  long long idle_since = -1;
  for (;;) {
    int ab = (lane == 0) ? *(volatile int*)a.abort_flag : 0;
    if (__shfl_sync(0xffffffffu, ab, 0)) break;
    unsigned long long its[QCLAIM] = {0, 0, 0, 0};
    const int ngot = q_pop_warp(a, its);
    if (!ngot) {
      int done = (lane == 0) ? (*(volatile int*)a.pending == 0) : 0;
      if (__shfl_sync(0xffffffffu, done, 0)) break;
      if (lane == 0) {
        const long long now = gtimer_ns();
        if (idle_since < 0) idle_since = now;
        if (now - idle_since > a.timeout_ns) {
          atomicOr(a.err, ERRB_QUEUE_TIMEOUT);
          atomicExch(a.abort_flag, 1);
        }
        __nanosleep(200);
      }
      __syncwarp();
      continue;
    }
    idle_since = -1;
    for (int j = 0; j < ngot; j++) {
      const unsigned long long it = its[j];
      const int prob = (int)(it >> 40);
      const long long tile = (long long)(it & ((1ull << 40) - 1));
      const long long gt = a.probs[prob].tbase + tile;
      uint32_t faces = 0;
      if (lane == 0) {
        atomicExch(a.tile_flag + gt, TS_BUSY);
        faces = atomicExch(a.tile_faces + gt, 0u);
        atomicExch(a.tile_prio + gt, (unsigned long long)__double_as_longlong(EIK_INF));
        __threadfence();
        const unsigned long long na = atomicAdd(a.activations, 1ull);
        if (na > a.max_activations) {
          atomicOr(a.err, ERRB_NOT_CONVERGED);
          atomicExch(a.abort_flag, 1);
        }
      }
      faces = __shfl_sync(0xffffffffu, faces, 0);
      double pr;
      const int fm = process_tile<ND>(a, S, prob, tile, faces, &pr);
      __threadfence();
      __syncwarp();
      if (lane == 0) {
        const CoarseProblem& P = a.probs[prob];
        const int tx = (int)(tile % P.nt[0]);
        const int ty = (int)((tile / P.nt[0]) % P.nt[1]);
        const int tz = (int)(tile / ((long long)P.nt[0] * P.nt[1]));
        auto nbt = [&](int x, int y, int z) { return (long long)x + (long long)P.nt[0] * (y + (long long)P.nt[1] * z); };
        if ((fm & 1) && tx > 0) enqueue_tile(a, prob, nbt(tx - 1, ty, tz), 2u, pr);
        if ((fm & 2) && tx + 1 < P.nt[0]) enqueue_tile(a, prob, nbt(tx + 1, ty, tz), 1u, pr);
        if ((fm & 4) && ty > 0) enqueue_tile(a, prob, nbt(tx, ty - 1, tz), 8u, pr);
        if ((fm & 8) && ty + 1 < P.nt[1]) enqueue_tile(a, prob, nbt(tx, ty + 1, tz), 4u, pr);
        if (ND == 3) {
          if ((fm & 16) && tz > 0) enqueue_tile(a, prob, nbt(tx, ty, tz - 1), 32u, pr);
          if ((fm & 32) && tz + 1 < P.nt[2]) enqueue_tile(a, prob, nbt(tx, ty, tz + 1), 16u, pr);
        }
        if (fm & 64) {
          atomicOr(a.tile_faces + gt, FACES_ALL);
          atomicMin(a.tile_prio + gt, (unsigned long long)__double_as_longlong(pr));
          atomicExch(a.tile_flag + gt, TS_BUSY_DIRTY);
        }
        __threadfence();
        finish_tile(a, prob, tile);
      }
      __syncwarp();
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
  const long long N = npts(hprobs[0].g);
  coarse_init_kernel<<<1184, 256, 0, st>>>(dprobs, nprob, N);
  queue_init_kernel<<<296, 256, 0, st>>>(sa);
  if (sa.nd == 3) seed_kernel<3><<<nprob, 128, 0, st>>>(sa, fb);
  else seed_kernel<2><<<nprob, 128, 0, st>>>(sa, fb);
}

void launch_queue_init(const SolveArgs& sa, cudaStream_t st) { queue_init_kernel<<<296, 256, 0, st>>>(sa); }

template <int ND>
static void launch_solve_nd(const SolveArgs& sa, int nsm, cudaStream_t st) {
  const size_t sm = sizeof(TileSmem<ND>) * SOLVE_WARPS;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(coarse_solve_kernel<ND>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    attr = true;
  }
  int per = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, coarse_solve_kernel<ND>, SOLVE_THREADS, sm);
  per = per < 1 ? 1 : per;
  coarse_solve_kernel<ND><<<nsm * per, SOLVE_THREADS, sm, st>>>(sa);
}

void launch_coarse_solve(const SolveArgs& sa, int nsm, cudaStream_t st) {
  if (sa.nd == 3) launch_solve_nd<3>(sa, nsm, st);
  else launch_solve_nd<2>(sa, nsm, st);
}

void launch_picks(const GridDesc& g, const double* t, long long N, int nsrc, const long long* recoff,
                  const double* rec, double* picks, cudaStream_t st) {
  picks_kernel<<<64, 128, 0, st>>>(g, t, N, nsrc, recoff, rec, picks);
}

}  // namespace eik
