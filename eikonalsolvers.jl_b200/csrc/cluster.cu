// Forward round solver for small problems, one thread-block cluster per problem, with the
// problem's whole round-solver state in the cluster's distributed shared memory.
//
// The rounds are those of coarse_rounds_kernel (coarse.cu) and every node visit is the same
// process_node (node.cuh); what changes is where the state lives and how rounds are
// separated. On small grids the global solve is latency-bound: a round costs a chain of
// dependent L2 round trips plus a grid barrier, and there are at least as many rounds as the
// grid's graph diameter (about 1200 rounds of ~25 us on a 300x220 grid). Here the traveltime,
// code, cached front, dirty flag and round stamp of every node, and the two worklists, sit in
// the shared memory of the cluster's CTAs (up to 16 SMs x 227 KB), reached through
// distributed shared memory (mapa addresses), and the rounds are separated by the hardware
// cluster barrier (barrier.cluster arrive.release / wait.acquire).
//
// Layout: node l of the problem belongs to CTA (l / 32) mod C of the cluster (C = 2^LGC
// CTAs), at index ((l / 32) / C) * 32 + l mod 32 of that CTA's arrays, so that every front
// spreads over all the CTAs. Each CTA keeps the worklists of its own nodes with their round
// counters (list length, next entry to take, smallest pending front, three rounds deep as in
// the global solve): a CTA takes the entries of its own list, so the visited node's state is
// local, and a node listed for the next round is appended to its owner's list. The cluster's
// threshold and whether a round has any entry are reduced over the CTAs' counters after the
// barrier. Key levels and depths of special nodes and the slowness stay in global memory
// (read at L2); the traveltimes and codes are written back to the problem's global arrays at
// the end, in the layout a global solve leaves them.
//
// Control flow is uniform across the cluster: the round loop ends on a count every thread
// reads after the same barrier, and no CTA leaves before the final barrier, so no CTA reads
// the shared memory of one that has exited. There is no spin-wait (the barrier is the
// hardware's) and the number of rounds is bounded (max_rounds, reported as not converged).
#include <cooperative_groups.h>

#include <algorithm>

#include "kernels.cuh"
#include "node.cuh"
#include "rounds.cuh"

namespace cg = cooperative_groups;

namespace eik {

// Threads per CTA. A round's front gives each CTA a few warps' worth of entries, and the
// round lasts as long as the slowest warp's visit: 256 threads leave the visit 180 registers
// a thread and no spill, which shortens that chain more than 16 warps per CTA would help.
constexpr int CL_THREADS = 256;
constexpr int CL_MAX_LGC = 4;           // clusters of up to 16 CTAs
constexpr int CL_BYTES_PER_NODE = 38;   // t, cached front, two list entries (8 B each), stamp (4), code, dirty

// Round counters of one CTA's worklists.
struct ClusterCtl {
  unsigned int cnt[3];
  unsigned int grab[3];
  unsigned long long nm[3];  // smallest pending front listed for a round (double bits)
  unsigned long long visits[CL_THREADS / 32][8];  // per-warp visit counts by outcome (this CTA's)
};

// The round-solver state of one problem in a cluster's distributed shared memory.
template <int LGC>
struct ClusterNodes {
  double* t_;
  double* tent_;
  int32_t* stamp_;
  uint8_t* code_;
  uint8_t* dirty_;
  __device__ static unsigned rank_of(long long l) { return (unsigned)((l >> 5) & ((1 << LGC) - 1)); }
  __device__ static long long index_of(long long l) { return ((l >> (5 + LGC)) << 5) | (l & 31); }
  // address of element l of this CTA's array `base` as laid out in the CTA that owns l
  template <class T>
  __device__ __forceinline__ T* at(T* base, long long l) const {
    return cg::this_cluster().map_shared_rank(base, rank_of(l)) + index_of(l);
  }
  __device__ __forceinline__ uint8_t dirty(long long l) const { return *(volatile const uint8_t*)at(dirty_, l); }
  __device__ __forceinline__ void set_dirty(long long l, uint8_t v) const { *(volatile uint8_t*)at(dirty_, l) = v; }
  __device__ __forceinline__ double tent(long long l) const { return *(volatile const double*)at(tent_, l); }
  __device__ __forceinline__ void set_tent(long long l, double v) const { *(volatile double*)at(tent_, l) = v; }
  __device__ __forceinline__ uint8_t code(long long l) const { return *(volatile const uint8_t*)at(code_, l); }
  __device__ __forceinline__ void set_code(long long l, uint8_t v) const { *(volatile uint8_t*)at(code_, l) = v; }
  __device__ __forceinline__ double t(long long l) const { return *(volatile const double*)at(t_, l); }
  __device__ __forceinline__ void set_t(long long l, double v) const { *(volatile double*)at(t_, l) = v; }
  __device__ __forceinline__ int32_t stamp(long long l) const { return *(volatile const int32_t*)at(stamp_, l); }
  // orders this thread's earlier writes (shared memory of any CTA of the cluster, and the
  // key levels in global memory) before its later ones, for every thread of the cluster
  __device__ __forceinline__ void fence() const { asm volatile("fence.acq_rel.cluster;" ::: "memory"); }
};

#ifdef EIK_PHASE
// tuning builds only: clock cycles per phase of the cluster rounds, summed over warps (lane 0)
__device__ unsigned long long eik_cphase[8];
extern "C" int eik_cphase_read(unsigned long long* out) {
  return (int)cudaMemcpyFromSymbol(out, eik_cphase, sizeof(unsigned long long) * 8);
}
// and, per round (first 4096), the largest per-warp time in each of phases 1-3 (the round's
// critical warp)
__device__ unsigned long long eik_cwarpmax[3][4096];
extern "C" int eik_cwarpmax_read(unsigned long long* out) {
  return (int)cudaMemcpyFromSymbol(out, eik_cwarpmax, sizeof(unsigned long long) * 3 * 4096);
}
#define CPH_T(v) const long long v = clock64()
#define CPH_ADD(k, t0)                                                                          \
  {                                                                                             \
    const unsigned long long dt_ = (unsigned long long)(clock64() - (t0));                      \
    if ((threadIdx.x & 31) == 0) atomicAdd(&eik_cphase[k], dt_);                                \
    if ((k) >= 1 && (k) <= 3) wsum_[(k) - 1] += dt_;                                           \
  }
#else
#define CPH_T(v)
#define CPH_ADD(k, t0)
#endif

__device__ __forceinline__ unsigned long long cluster_entry(long long l, double front) {
  const float f = front < EIK_INF ? __double2float_rd(front) : __int_as_float(0x7f800000);
  return ((unsigned long long)l << 32) | (unsigned long long)__float_as_uint(f);
}

template <int ND, int LGC>
__global__ void __launch_bounds__(CL_THREADS, 1)
    cluster_rounds_kernel(SolveArgs a, const int32_t* seed_lin, const double* seed_tt, const SrcOut* out,
                          int fine_corners, int seedcap, int cap) {
  cg::cluster_group cl = cg::this_cluster();
  constexpr int C = 1 << LGC;
  const unsigned rank = cl.block_rank();
  const int p = (int)(blockIdx.x >> LGC);
  const int lane = threadIdx.x & 31;
  extern __shared__ __align__(16) unsigned char cl_smem[];
  __shared__ ClusterCtl ctl;
  double* s_t = reinterpret_cast<double*>(cl_smem);
  double* s_tent = s_t + cap;
  unsigned long long* s_list0 = reinterpret_cast<unsigned long long*>(s_tent + cap);
  unsigned long long* s_list1 = s_list0 + cap;
  int32_t* s_stamp = reinterpret_cast<int32_t*>(s_list1 + cap);
  uint8_t* s_code = reinterpret_cast<uint8_t*>(s_stamp + cap);
  uint8_t* s_dirty = s_code + cap;
  const CoarseProblem& P = a.probs[p];
  const GridDesc& g = P.g;
  const long long N = npts(g);
  const ClusterNodes<LGC> m{s_t, s_tent, s_stamp, s_code, s_dirty};

  // initial state of this CTA's nodes (those of a global solve after coarse and round init)
  for (int q = threadIdx.x; q < cap; q += blockDim.x) {
    s_t[q] = EIK_INF;
    s_tent[q] = EIK_INF;
    s_stamp[q] = -1;
    s_code[q] = CODE_NONE;
    s_dirty[q] = 1;
  }
  if (threadIdx.x < 3) {
    ctl.cnt[threadIdx.x] = 0;
    ctl.grab[threadIdx.x] = 0;
    ctl.nm[threadIdx.x] = (unsigned long long)__double_as_longlong(EIK_INF);
  }
  __shared__ unsigned int s_total;
  __shared__ unsigned long long s_nm;
  cl.sync();
  // the list of node l: its owner's (entry index local to the owner)
  auto append = [&](unsigned long long* list, int slot, long long nl, double front) {
    const unsigned owner = ClusterNodes<LGC>::rank_of(nl);
    ClusterCtl* oc = cl.map_shared_rank(&ctl, owner);
    const unsigned int i = atomicAdd(&oc->cnt[slot], 1u);
    cl.map_shared_rank(list, owner)[i] = cluster_entry(nl, front);
  };

  // seeds (as seed_kernel): fixed traveltimes, then the nodes within two steps start round 0
  const int ns = fine_corners ? out[p].nsrcf : out[p].nseeds;
  const int gtid = (int)rank * blockDim.x + threadIdx.x, gthreads = C * blockDim.x;
  for (int q = gtid; q < ns; q += gthreads) {
    const long long l = seed_lin[(size_t)p * seedcap + q];
    m.set_t(l, seed_tt[(size_t)p * seedcap + q]);
    m.set_code(l, (uint8_t)(CODE_NONE | CODE_SRC_BIT));
    P.kL[l] = -EIK_INF;
    P.kd[l] = 0;
  }
  cl.sync();
  for (int q = gtid; q < ns; q += gthreads) {
    const long long l = seed_lin[(size_t)p * seedcap + q];
    const int c[3] = {(int)(l % g.n[0]), (int)((l / g.n[0]) % g.n[1]), (int)(l / ((long long)g.n[0] * g.n[1]))};
    const double tt = seed_tt[(size_t)p * seedcap + q];
    if (tt < EIK_INF) atomicMin(&ctl.nm[0], (unsigned long long)__double_as_longlong(tt));
    for (int ax = 0; ax < ND; ax++)
      for (int d = -2; d <= 2; d++) {
        if (d == 0) continue;
        int pc[3] = {c[0], c[1], c[2]};
        pc[ax] += d;
        if (pc[ax] < 0 || pc[ax] >= g.n[ax]) continue;
        const long long nl = lin3(g, pc[0], pc[1], pc[2]);
        if (atomicExch(m.at(s_stamp, nl), 0) != 0) append(s_list0, 0, nl, tt);
      }
  }
  cl.sync();

  unsigned long long* wvis = ctl.visits[threadIdx.x >> 5];
  clear_visits(wvis, lane);
#ifdef EIK_PHASE
  VisitCount vk[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // lane cycles of the node visit at 7..10
#else
  VisitCount* vk = nullptr;
#endif
  double Tprev = -EIK_INF;
  int r = 0;
  for (; r < a.rs.max_rounds; r++) {
    const int b3 = r % 3, nb3 = (r + 1) % 3;
#ifdef EIK_PHASE
    unsigned long long wsum_[3] = {0, 0, 0};
#endif
    CPH_T(tr0);
    // the cluster's entries and smallest pending front of this round: every CTA reduces the
    // same counters, read after the same barrier and written by no one this round (uniform)
    if (threadIdx.x < 32) {
      unsigned int cn = 0;
      unsigned long long mn = (unsigned long long)__double_as_longlong(EIK_INF);
      if (threadIdx.x < C) {
        const ClusterCtl* oc = cl.map_shared_rank(&ctl, threadIdx.x);
        cn = *(volatile const unsigned int*)&oc->cnt[b3];
        mn = *(volatile const unsigned long long*)&oc->nm[b3];
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        cn += __shfl_xor_sync(0xffffffffu, cn, o);
        const unsigned long long v = __shfl_xor_sync(0xffffffffu, mn, o);
        mn = v < mn ? v : mn;
      }
      if (threadIdx.x == 0) {
        s_total = cn;
        s_nm = mn;
      }
    }
    __syncthreads();
    CPH_ADD(0, tr0);
    const unsigned int ntot = s_total;
    if (ntot == 0) break;
    const double T = fmax(Tprev, __longlong_as_double((long long)s_nm) + P.delta);
    Tprev = T;
    if (rank == 0 && threadIdx.x == 0) atomicAdd(a.activations, (unsigned long long)ntot);
    const unsigned int n = ctl.cnt[b3];  // this CTA's own entries
    unsigned long long* L = (r & 1) ? s_list1 : s_list0;
    unsigned long long* Lnext = (r & 1) ? s_list0 : s_list1;
    for (;;) {
      CPH_T(tp0);
      unsigned int base = 0;
      if (lane == 0) base = atomicAdd(&ctl.grab[b3], 32u);
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= n) break;
      const unsigned int idx = base + lane;
      unsigned dirs = visit_code(VISIT_NONE);
      double front = EIK_INF;
      long long l = 0;
      if (idx < n) {
        const unsigned long long e = L[idx];
        l = (long long)(e >> 32);
        const double ef = (double)__uint_as_float((unsigned int)e);
        const uint8_t dq = m.dirty(l);
        if (ef > T && ef < EIK_INF && !dq) {
          // still waiting and nothing it reads has changed: its front stands
          front = ef;
          dirs = (1u << DIR_SELF) | visit_code(VISIT_STANDS);
        } else {
          dirs = process_node<ND>(m, P, l, T, r, &front, vk);
        }
      }
      __syncwarp();
      count_visits(wvis, dirs, lane);
      CPH_ADD(1, tp0);
      CPH_T(tp1);
      // list the next round's nodes once each (round stamps) with their owners; the stamp
      // exchanges go out together, then the appends
      unsigned keep = 0;
#pragma unroll
      for (int k = 0; k <= DIR_SELF; k++) {
        if (!((dirs >> k) & 1u)) continue;
        const long long nl = dir_lin(g, l, k);
        if (atomicExch(m.at(s_stamp, nl), r + 1) != r + 1) keep |= 1u << k;
      }
      __syncwarp();
      CPH_ADD(2, tp1);
      CPH_T(tp2);
      // the owners' list slots in one batch of remote atomics, then the entries
      unsigned int slot[DIR_SELF + 1];
#pragma unroll
      for (int k = 0; k <= DIR_SELF; k++) {
        slot[k] = 0;
        if (!((keep >> k) & 1u)) continue;
        const long long nl = dir_lin(g, l, k);
        slot[k] = atomicAdd(&cl.map_shared_rank(&ctl, ClusterNodes<LGC>::rank_of(nl))->cnt[nb3], 1u);
      }
#pragma unroll
      for (int k = 0; k <= DIR_SELF; k++) {
        if (!((keep >> k) & 1u)) continue;
        const long long nl = dir_lin(g, l, k);
        cl.map_shared_rank(Lnext, ClusterNodes<LGC>::rank_of(nl))[slot[k]] = cluster_entry(nl, front);
      }
      __syncwarp();
      CPH_ADD(3, tp2);
      // one update of this CTA's smallest pending front per warp
      double fv = keep ? front : EIK_INF;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) fv = fmin(fv, __shfl_xor_sync(0xffffffffu, fv, o));
      if (lane == 0 && fv < EIK_INF &&
          fv < __longlong_as_double((long long)*(volatile const unsigned long long*)&ctl.nm[nb3]))
        atomicMin(&ctl.nm[nb3], (unsigned long long)__double_as_longlong(fv));
    }
#ifdef EIK_PHASE
    if (lane == 0 && r < 4096)
      for (int k = 0; k < 3; k++) atomicMax(&eik_cwarpmax[k][r], wsum_[k]);
#endif
    CPH_T(tb0);
    // this CTA's counters of round r+2 (last read in round r-1)
    if (threadIdx.x == 0) {
      const int c3 = (r + 2) % 3;
      ctl.cnt[c3] = 0;
      ctl.grab[c3] = 0;
      ctl.nm[c3] = (unsigned long long)__double_as_longlong(EIK_INF);
    }
    cl.sync();
    CPH_ADD(4, tb0);
  }

  // results in the problem's global arrays, as a global solve leaves them
  for (int q = threadIdx.x; q < cap; q += blockDim.x) {
    const long long l = ((long long)(q >> 5) << (5 + LGC)) | ((long long)rank << 5) | (q & 31);
    if (l < N) {
      P.t[l] = s_t[q];
      P.code[l] = s_code[q];
    }
  }
  // counters: evaluations, visit outcomes, the largest round count
  flush_visits(wvis, a.rs.visits, a.node_evals, lane);
  if (rank == 0 && threadIdx.x == 0) {
    atomicMax(a.rs.rounds, r);
    if (r >= a.rs.max_rounds) atomicOr(a.err, ERRB_NOT_CONVERGED);
  }
  cl.sync();  // no CTA leaves while another may still read its shared memory
}

__global__ void cluster_counters_kernel(SolveArgs a) {
  if (threadIdx.x == 0) {
    *a.rs.rounds = 0;
    *a.activations = 0;
    *a.node_evals = 0;
    *a.abort_flag = 0;
  }
  if (threadIdx.x < 7) a.rs.visits[threadIdx.x] = 0;
}

static size_t cluster_smem(int cap) { return (size_t)cap * CL_BYTES_PER_NODE; }

static int optin_smem() {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return optin;
}

static cudaLaunchConfig_t cluster_config(int nprob, int lgc, size_t smem, cudaStream_t st, cudaLaunchAttribute* attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(nprob << lgc));
  cfg.blockDim = dim3(CL_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 1u << lgc;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

// Whether clusters of 2^LGC CTAs with the largest shared memory a CTA may take can run on
// this GPU (kernel attributes set once per process, before any capture).
template <int ND, int LGC>
static bool cluster_fits() {
  static const bool fits = [] {
    auto kern = cluster_rounds_kernel<ND, LGC>;
    const int optin = optin_smem();
    if (optin <= 0) return false;
    const size_t smem = (size_t)optin - sizeof(ClusterCtl) - 1024;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess && (1 << LGC) > 8) e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    cudaLaunchAttribute attr[1];
    const cudaLaunchConfig_t cfg = cluster_config(1, LGC, smem, 0, attr);
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, (void*)kern, &cfg) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    return nclusters >= 1;
  }();
  return fits;
}

template <int ND, int LGC>
static cudaError_t cluster_launch(const SolveArgs& sa, int cap, const int32_t* seed_lin, const double* seed_tt,
                                  const SrcOut* out, int fine_corners, int seedcap, cudaStream_t st, bool probe,
                                  bool* ok) {
  *ok = cluster_fits<ND, LGC>();
  if (!*ok || probe) return cudaSuccess;
  cudaLaunchAttribute attr[1];
  const cudaLaunchConfig_t cfg = cluster_config(sa.nprob, LGC, cluster_smem(cap), st, attr);
  return cudaLaunchKernelEx(&cfg, cluster_rounds_kernel<ND, LGC>, sa, seed_lin, seed_tt, out, fine_corners, seedcap,
                            cap);
}

template <int ND>
static cudaError_t cluster_dispatch(int lgc, const SolveArgs& sa, int cap, const int32_t* seed_lin,
                                    const double* seed_tt, const SrcOut* out, int fine_corners, int seedcap,
                                    cudaStream_t st, bool probe, bool* ok) {
  switch (lgc) {
    case 0: return cluster_launch<ND, 0>(sa, cap, seed_lin, seed_tt, out, fine_corners, seedcap, st, probe, ok);
    case 1: return cluster_launch<ND, 1>(sa, cap, seed_lin, seed_tt, out, fine_corners, seedcap, st, probe, ok);
    case 2: return cluster_launch<ND, 2>(sa, cap, seed_lin, seed_tt, out, fine_corners, seedcap, st, probe, ok);
    case 3: return cluster_launch<ND, 3>(sa, cap, seed_lin, seed_tt, out, fine_corners, seedcap, st, probe, ok);
    default: return cluster_launch<ND, 4>(sa, cap, seed_lin, seed_tt, out, fine_corners, seedcap, st, probe, ok);
  }
}

// Cluster size (log2) and per-CTA node capacity for problems of at most nmax nodes: the
// smallest cluster whose shared memory holds them; false when none does.
static bool cluster_shape(long long nmax, int* lgc, int* cap) {
  const int optin = optin_smem();
  const long long room = ((long long)(optin - (int)sizeof(ClusterCtl) - 1024) / CL_BYTES_PER_NODE) & ~31LL;
  for (int k = 0; k <= CL_MAX_LGC; k++) {
    const long long per = ((nmax + (1LL << k) - 1) >> k);
    const long long c = std::max<long long>((per + 31) & ~31LL, 32);
    if (c <= room) {
      *lgc = k;
      *cap = (int)c;
      return true;
    }
  }
  return false;
}

bool cluster_solve_fits(const SolveArgs& sa, long long nmax) {
  int lgc = 0, cap = 0;
  if (sa.nprob < 1 || !cluster_shape(nmax, &lgc, &cap)) return false;
  if ((long long)sa.nprob << lgc > (1LL << 31) - 1) return false;
  bool ok = false;
  if (sa.nd == 3) cluster_dispatch<3>(lgc, sa, cap, nullptr, nullptr, nullptr, 0, 0, 0, true, &ok);
  else cluster_dispatch<2>(lgc, sa, cap, nullptr, nullptr, nullptr, 0, 0, 0, true, &ok);
  return ok;
}

cudaError_t launch_cluster_solve(const SolveArgs& sa, long long nmax, const int32_t* seed_lin, const double* seed_tt,
                                 const SrcOut* out, bool fine_corners, int seedcap, cudaStream_t st, bool* used) {
  *used = false;
  if (!cluster_solve_fits(sa, nmax)) return cudaSuccess;
  int lgc = 0, cap = 0;
  cluster_shape(nmax, &lgc, &cap);
  cluster_counters_kernel<<<1, 32, 0, st>>>(sa);
  bool ok = false;
  const cudaError_t e = sa.nd == 3 ? cluster_dispatch<3>(lgc, sa, cap, seed_lin, seed_tt, out, fine_corners ? 1 : 0,
                                                         seedcap, st, false, &ok)
                                   : cluster_dispatch<2>(lgc, sa, cap, seed_lin, seed_tt, out, fine_corners ? 1 : 0,
                                                         seedcap, st, false, &ok);
  if (e == cudaSuccess && ok) *used = true;
  return e;
}

}  // namespace eik
