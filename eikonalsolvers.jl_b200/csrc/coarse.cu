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

// Push; the caller guarantees at most (mask+1) items are ever in the queue at once.
__device__ bool q_push(const SolveArgs& a, unsigned long long item) {
  const unsigned long long pos = atomicAdd(a.q.tail, 1ull);
  const unsigned long long slot = pos & a.q.mask;
  const long long t0 = gtimer_ns();
  while (ld_volatile(a.q.seq + slot) != pos) {
    if (gtimer_ns() - t0 > a.timeout_ns) {
      atomicOr(a.err, ERRB_QUEUE_TIMEOUT);
      atomicExch(a.abort_flag, 1);
      return false;
    }
    __nanosleep(64);
  }
  a.q.items[slot] = item;
  __threadfence();
  atomicExch(a.q.seq + slot, pos + 1);
  return true;
}

// Try to pop; returns false when the queue looks empty.
__device__ bool q_pop(const SolveArgs& a, unsigned long long* item) {
  for (;;) {
    const unsigned long long h = ld_volatile(a.q.head);
    const unsigned long long t = ld_volatile(a.q.tail);
    if (h >= t) return false;
    if (atomicCAS(a.q.head, h, h + 1) != h) continue;
    const unsigned long long slot = h & a.q.mask;
    const long long t0 = gtimer_ns();
    while (ld_volatile(a.q.seq + slot) != h + 1) {
      if (gtimer_ns() - t0 > a.timeout_ns) {
        atomicOr(a.err, ERRB_QUEUE_TIMEOUT);
        atomicExch(a.abort_flag, 1);
        return false;
      }
      __nanosleep(32);
    }
    *item = ld_volatile(a.q.items + slot);
    __threadfence();
    atomicExch(a.q.seq + slot, h + a.q.mask + 1);
    return true;
  }
}

// Tile states: 0 idle, 1 queued, 2 being processed, 3 being processed and changed again
// by a neighbour meanwhile (re-queued by its processor when it finishes). A tile is never
// processed by two CTAs at once, so a write-back can never overwrite newer values.
constexpr int TS_IDLE = 0, TS_QUEUED = 1, TS_BUSY = 2, TS_BUSY_DIRTY = 3;

__device__ void enqueue_tile(const SolveArgs& a, int prob, long long tile, uint32_t faces) {
  const long long gt = a.probs[prob].tbase + tile;
  atomicOr(a.tile_faces + gt, faces);
  int s = *(volatile int*)(a.tile_flag + gt);
  for (int it = 0; it < 64; it++) {
    if (s == TS_IDLE) {
      const int o = atomicCAS(a.tile_flag + gt, TS_IDLE, TS_QUEUED);
      if (o == TS_IDLE) {
        atomicAdd(a.pending, 1);
        q_push(a, ((unsigned long long)prob << 40) | (unsigned long long)tile);
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
__device__ void finish_tile(const SolveArgs& a, int prob, long long tile) {
  const long long gt = a.probs[prob].tbase + tile;
  const int o = atomicCAS(a.tile_flag + gt, TS_BUSY, TS_IDLE);
  if (o == TS_BUSY) {
    atomicSub(a.pending, 1);
    return;
  }
  // TS_BUSY_DIRTY: stays counted in pending, goes back to the queue
  atomicExch(a.tile_flag + gt, TS_QUEUED);
  q_push(a, ((unsigned long long)prob << 40) | (unsigned long long)tile);
}

// ------------------------------------------------------------------ tile shapes --
template <int ND> struct TileCfg;
template <> struct TileCfg<3> {
  static constexpr int TX = 8, TY = 8, TZ = 8, H = 2;
  static constexpr int HX = TX + 2 * H, HY = TY + 2 * H, HZ = TZ + 2 * H;
};
template <> struct TileCfg<2> {
  static constexpr int TX = 32, TY = 16, TZ = 1, H = 2;
  static constexpr int HX = TX + 2 * H, HY = TY + 2 * H, HZ = 1;
};
constexpr int SOLVE_THREADS = 256;

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
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < (long long)a.q.mask + 1;
       q += (long long)gridDim.x * blockDim.x)
    a.q.seq[q] = (unsigned long long)q;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < a.ntiles;
       q += (long long)gridDim.x * blockDim.x) {
    a.tile_faces[q] = 0;
    a.tile_flag[q] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *a.q.head = 0;
    *a.q.tail = 0;
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
    enqueue_tile(a, s, tile_of<ND>(P, i, j, k), FACES_ALL);
    for (int ax = 0; ax < ND; ax++)
      for (int d = -2; d <= 2; d += 4) {
        int p[3] = {c[0], c[1], c[2]};
        p[ax] += d;
        if (p[ax] < 0 || p[ax] >= P.g.n[ax]) continue;
        enqueue_tile(a, s, tile_of<ND>(P, p[0], p[1], p[2]), FACES_ALL);
      }
  }
}

// ------------------------------------------------------------------ tile solve --
template <int ND>
struct TileSmem {
  using C = TileCfg<ND>;
  static constexpr int TN = C::TX * C::TY * C::TZ;
  static constexpr int HN = C::HX * C::HY * C::HZ;
  double t[HN];
  double L[HN];
  double slow[TN];
  uint8_t fl[HN];  // bit0 special, bits1..7 depth
  uint8_t code[TN];
  uint8_t act[TN];
  uint8_t nxt[TN];
  uint8_t dirty[TN];
};

template <int ND>
__device__ __forceinline__ Key smem_key(const TileSmem<ND>& S, int h) {
  const uint8_t f = S.fl[h];
  if (f & 1) {
    const double L = S.L[h];
    if (L == -EIK_INF) return key_source();
    return Key{L, (int)(f >> 1), S.t[h]};
  }
  return key_normal(S.t[h]);
}

template <int ND>
__device__ void process_tile(const SolveArgs& a, TileSmem<ND>& S, int prob, long long tile, uint32_t faces,
                             int* sh_faces_out, int* sh_unconv) {
  using C = TileCfg<ND>;
  constexpr int TN = TileSmem<ND>::TN, HN = TileSmem<ND>::HN;
  const CoarseProblem& P = a.probs[prob];
  const GridDesc& g = P.g;
  const int tx = (int)(tile % P.nt[0]);
  const int ty = (int)((tile / P.nt[0]) % P.nt[1]);
  const int tz = (int)(tile / ((long long)P.nt[0] * P.nt[1]));
  const int ox = tx * C::TX, oy = ty * C::TY, oz = tz * C::TZ;
  const int tid = threadIdx.x;

  // ---- stage tile + halo
  for (int h = tid; h < HN; h += SOLVE_THREADS) {
    const int hx = h % C::HX, hy = (h / C::HX) % C::HY, hz = h / (C::HX * C::HY);
    const int gx = ox + hx - C::H, gy = oy + hy - C::H, gz = (ND == 3) ? oz + hz - C::H : 0;
    double tv = EIK_INF, Lv = 0.0;
    uint8_t f = 0;
    if (gx >= 0 && gx < g.n[0] && gy >= 0 && gy < g.n[1] && gz >= 0 && gz < g.n[2]) {
      const long long l = lin3(g, gx, gy, gz);
      tv = P.t[l];
      const uint8_t cb = P.code[l];
      if (cb & CODE_SRC_BIT) {
        Lv = P.kL[l];
        f = (uint8_t)(1 | (P.kd[l] << 1));
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
  if (tid == 0) *sh_faces_out = 0;
  __syncthreads();
  // ---- initial active set from the dirty faces
  for (int li = tid; li < TN; li += SOLVE_THREADS) {
    const int x = li % C::TX, y = (li / C::TX) % C::TY, z = li / (C::TX * C::TY);
    const int gx = ox + x, gy = oy + y, gz = oz + z;
    bool act = (faces & FACES_ALL) != 0;
    act = act || ((faces & 1) && x < 2) || ((faces & 2) && x >= C::TX - 2) || ((faces & 4) && y < 2) ||
          ((faces & 8) && y >= C::TY - 2) || ((faces & 16) && z < 2) || ((faces & 32) && z >= C::TZ - 2);
    const int h = (x + C::H) + C::HX * ((y + C::H) + C::HY * (ND == 3 ? z + C::H : 0));
    const bool src = (S.fl[h] & 1) && S.L[h] == -EIK_INF;
    const bool inside = gx < g.n[0] && gy < g.n[1] && gz < g.n[2];
    S.act[li] = (act && !src && inside) ? 1 : 0;
    S.nxt[li] = 0;
    S.dirty[li] = 0;
  }
  __syncthreads();

  constexpr int NPT = (TN + SOLVE_THREADS - 1) / SOLVE_THREADS;
  int pass = 0;
  unsigned long long evals = 0;
  bool any = true;
  while (any) {
    double nv[NPT];
    Key nk[NPT];
    uint8_t nc[NPT];
    bool ch[NPT];
#pragma unroll
    for (int r = 0; r < NPT; r++) {
      ch[r] = false;
      const int li = tid + r * SOLVE_THREADS;
      if (li >= TN || !S.act[li]) continue;
      const int x = li % C::TX, y = (li / C::TX) % C::TY, z = li / (C::TX * C::TY);
      const int c[3] = {ox + x, oy + y, oz + z};
      const int hc[3] = {x + C::H, y + C::H, ND == 3 ? z + C::H : 0};
      Nbhd nb;
      node_dh(g, c[0], nb.dh);
      nb.slow = S.slow[li];
#pragma unroll
      for (int ax = 0; ax < 3; ax++)
#pragma unroll
        for (int l = 0; l < 2; l++) {
          nb.in1[ax][l] = false;
          nb.ok2[ax][l] = false;
          nb.t1[ax][l] = EIK_INF;
          nb.t2[ax][l] = EIK_INF;
          nb.k1[ax][l] = key_unreached();
          nb.k2[ax][l] = key_unreached();
        }
#pragma unroll
      for (int ax = 0; ax < ND; ax++)
#pragma unroll
        for (int l = 0; l < 2; l++) {
          const int sh = l == 0 ? 1 : -1;
          int p[3] = {c[0], c[1], c[2]};
          p[ax] += sh;
          if (p[ax] < 0 || p[ax] >= g.n[ax]) continue;
          nb.in1[ax][l] = true;
          int hp[3] = {hc[0], hc[1], hc[2]};
          hp[ax] += sh;
          const int h1 = hp[0] + C::HX * (hp[1] + C::HY * hp[2]);
          nb.t1[ax][l] = S.t[h1];
          nb.k1[ax][l] = smem_key<ND>(S, h1);
          bool ok = true;
#pragma unroll
          for (int d = 0; d < ND; d++)
            if (p[d] < 1 || p[d] > g.n[d] - 2) ok = false;
          nb.ok2[ax][l] = ok;
          if (ok) {
            hp[ax] += sh;
            const int h2 = hp[0] + C::HX * (hp[1] + C::HY * hp[2]);
            nb.t2[ax][l] = S.t[h2];
            nb.k2[ax][l] = smem_key<ND>(S, h2);
          }
        }
      int8_t cd[3] = {0, 0, 0};
      Key kk;
      bool neg = false;
      const double v = prefix_rule<ND>(nb, cd, &kk, &neg);
      evals++;
      const int hm = hc[0] + C::HX * (hc[1] + C::HY * hc[2]);
      const Key old = smem_key<ND>(S, hm);
      const double ot = S.t[hm];
      const uint8_t pc = pack_codes(cd, ND);
      const bool same_t = (v == ot) || (isinf(v) && isinf(ot));
      nv[r] = v;
      nk[r] = kk;
      nc[r] = pc;
      ch[r] = !(same_t && key_eq(kk, old)) || pc != S.code[li];
    }
    __syncthreads();
    bool anyc = false;
#pragma unroll
    for (int r = 0; r < NPT; r++) {
      if (!ch[r]) continue;
      const int li = tid + r * SOLVE_THREADS;
      const int x = li % C::TX, y = (li / C::TX) % C::TY, z = li / (C::TX * C::TY);
      const int hc[3] = {x + C::H, y + C::H, ND == 3 ? z + C::H : 0};
      const int hm = hc[0] + C::HX * (hc[1] + C::HY * hc[2]);
      const bool tkchange = !(((nv[r] == S.t[hm]) || (isinf(nv[r]) && isinf(S.t[hm]))) &&
                              key_eq(nk[r], smem_key<ND>(S, hm)));
      S.t[hm] = nv[r];
      const bool special = !(nk[r].L == nk[r].t && nk[r].d == 0);
      S.fl[hm] = special ? (uint8_t)(1 | (nk[r].d << 1)) : (uint8_t)0;
      S.L[hm] = special ? nk[r].L : 0.0;
      S.code[li] = nc[r];
      S.dirty[li] = 1;
      if (!tkchange) continue;
      anyc = true;
      const int xyz[3] = {x, y, z};
      const int T3[3] = {C::TX, C::TY, C::TZ};
#pragma unroll
      for (int ax = 0; ax < ND; ax++)
#pragma unroll
        for (int d = -2; d <= 2; d++) {
          if (d == 0) continue;
          int q[3] = {xyz[0], xyz[1], xyz[2]};
          q[ax] += d;
          if (q[ax] < 0 || q[ax] >= T3[ax]) continue;
          const int lq = q[0] + C::TX * (q[1] + C::TY * q[2]);
          S.nxt[lq] = 1;
        }
      int fm = 0;
      if (x < 2) fm |= 1;
      if (x >= C::TX - 2) fm |= 2;
      if (y < 2) fm |= 4;
      if (y >= C::TY - 2) fm |= 8;
      if (ND == 3 && z < 2) fm |= 16;
      if (ND == 3 && z >= C::TZ - 2) fm |= 32;
      if (fm) atomicOr(sh_faces_out, fm);
    }
    __syncthreads();
    bool anyact = false;
    for (int li = tid; li < TN; li += SOLVE_THREADS) {
      const int x = li % C::TX, y = (li / C::TX) % C::TY, z = li / (C::TX * C::TY);
      const int h = (x + C::H) + C::HX * ((y + C::H) + C::HY * (ND == 3 ? z + C::H : 0));
      const bool src = (S.fl[h] & 1) && S.L[h] == -EIK_INF;
      const bool inside = ox + x < g.n[0] && oy + y < g.n[1] && oz + z < g.n[2];
      const uint8_t a2 = (S.nxt[li] && !src && inside) ? 1 : 0;
      S.act[li] = a2;
      S.nxt[li] = 0;
      anyact = anyact || a2;
    }
    (void)anyc;
    pass++;
    any = __syncthreads_or(anyact) != 0;
    if (any && pass >= a.max_passes) {
      if (tid == 0) *sh_unconv = 1;
      break;
    }
  }
  // ---- write back
  for (int li = tid; li < TN; li += SOLVE_THREADS) {
    if (!S.dirty[li]) continue;
    const int x = li % C::TX, y = (li / C::TX) % C::TY, z = li / (C::TX * C::TY);
    const int h = (x + C::H) + C::HX * ((y + C::H) + C::HY * (ND == 3 ? z + C::H : 0));
    const long long l = lin3(g, ox + x, oy + y, oz + z);
    P.t[l] = S.t[h];
    const bool special = S.fl[h] & 1;
    P.code[l] = (uint8_t)(S.code[li] | (special ? CODE_SRC_BIT : 0));
    if (special) {
      P.kL[l] = S.L[h];
      P.kd[l] = (uint8_t)(S.fl[h] >> 1);
    }
  }
  if (evals) atomicAdd(a.node_evals, evals);
}

template <int ND>
__global__ void __launch_bounds__(SOLVE_THREADS) coarse_solve_kernel(SolveArgs a) {
  using C = TileCfg<ND>;
  __shared__ TileSmem<ND> S;
  __shared__ unsigned long long sh_item;
  __shared__ int sh_state;  // 0 work, 1 wait, 2 exit
  __shared__ uint32_t sh_faces_in;
  __shared__ int sh_faces_out, sh_unconv;
  long long idle_since = -1;
  for (;;) {
    if (threadIdx.x == 0) {
      unsigned long long it;
      if (*(volatile int*)a.abort_flag) {
        sh_state = 2;
      } else if (q_pop(a, &it)) {
        sh_state = 0;
        sh_item = it;
        const int prob = (int)(it >> 40);
        const long long tile = (long long)(it & ((1ull << 40) - 1));
        const long long gt = a.probs[prob].tbase + tile;
        atomicExch(a.tile_flag + gt, TS_BUSY);
        sh_faces_in = atomicExch(a.tile_faces + gt, 0u);
        __threadfence();
        const unsigned long long na = atomicAdd(a.activations, 1ull);
        if (na > a.max_activations) {
          atomicOr(a.err, ERRB_NOT_CONVERGED);
          atomicExch(a.abort_flag, 1);
        }
        sh_unconv = 0;
        idle_since = -1;
      } else if (*(volatile int*)a.pending == 0) {
        sh_state = 2;
      } else {
        sh_state = 1;
        const long long now = gtimer_ns();
        if (idle_since < 0) idle_since = now;
        if (now - idle_since > a.timeout_ns) {
          atomicOr(a.err, ERRB_QUEUE_TIMEOUT);
          atomicExch(a.abort_flag, 1);
        }
      }
    }
    __syncthreads();
    const int state = sh_state;
    if (state == 2) break;
    if (state == 1) {
      if (threadIdx.x == 0) __nanosleep(256);
      __syncthreads();
      continue;
    }
    const int prob = (int)(sh_item >> 40);
    const long long tile = (long long)(sh_item & ((1ull << 40) - 1));
    process_tile<ND>(a, S, prob, tile, sh_faces_in, &sh_faces_out, &sh_unconv);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      const CoarseProblem& P = a.probs[prob];
      const int tx = (int)(tile % P.nt[0]);
      const int ty = (int)((tile / P.nt[0]) % P.nt[1]);
      const int tz = (int)(tile / ((long long)P.nt[0] * P.nt[1]));
      const int fm = sh_faces_out;
      auto nbt = [&](int x, int y, int z) { return (long long)x + (long long)P.nt[0] * (y + (long long)P.nt[1] * z); };
      if ((fm & 1) && tx > 0) enqueue_tile(a, prob, nbt(tx - 1, ty, tz), 2u);
      if ((fm & 2) && tx + 1 < P.nt[0]) enqueue_tile(a, prob, nbt(tx + 1, ty, tz), 1u);
      if ((fm & 4) && ty > 0) enqueue_tile(a, prob, nbt(tx, ty - 1, tz), 8u);
      if ((fm & 8) && ty + 1 < P.nt[1]) enqueue_tile(a, prob, nbt(tx, ty + 1, tz), 4u);
      if (ND == 3) {
        if ((fm & 16) && tz > 0) enqueue_tile(a, prob, nbt(tx, ty, tz - 1), 32u);
        if ((fm & 32) && tz + 1 < P.nt[2]) enqueue_tile(a, prob, nbt(tx, ty, tz + 1), 16u);
      }
      if (sh_unconv) {
        atomicOr(a.tile_faces + P.tbase + tile, FACES_ALL);
        atomicExch(a.tile_flag + P.tbase + tile, TS_BUSY_DIRTY);
      }
      __threadfence();
      finish_tile(a, prob, tile);
    }
    __syncthreads();
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

void launch_coarse_solve(const SolveArgs& sa, int nsm, cudaStream_t st) {
  int per = 1;
  if (sa.nd == 3) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, coarse_solve_kernel<3>, SOLVE_THREADS, 0);
    per = per < 1 ? 1 : per;
    coarse_solve_kernel<3><<<nsm * per, SOLVE_THREADS, 0, st>>>(sa);
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, coarse_solve_kernel<2>, SOLVE_THREADS, 0);
    per = per < 1 ? 1 : per;
    coarse_solve_kernel<2><<<nsm * per, SOLVE_THREADS, 0, st>>>(sa);
  }
}

void launch_picks(const GridDesc& g, const double* t, long long N, int nsrc, const long long* recoff,
                  const double* rec, double* picks, cudaStream_t st) {
  picks_kernel<<<64, 128, 0, st>>>(g, t, N, nsrc, recoff, rec, picks);
}

}  // namespace eik
