// Host runtime of libeikcuda: contexts, resident velocity models, device scratch, and the
// C-ABI entry points declared in include/eikcuda.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/eikcuda.h"
#include "kernels.cuh"
#include "rounds.cuh"
#include "runtime.hpp"

namespace eik {

thread_local std::string tl_error;

int fail(eik_ctx* ctx, int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  tl_error = buf;
  (void)ctx;
  return code;
}



// -------------------------------------------------------------------- scratch --
void* Scratch::get(const std::string& name, size_t bytes, int* rc) {
  auto it = bufs.find(name);
  if (it != bufs.end() && it->second.bytes >= bytes) {
    it->second.used = epoch;
    return it->second.ptr;
  }
  if (it != bufs.end()) {
    cudaFree(it->second.ptr);
    total -= it->second.bytes;
    bufs.erase(it);
  }
  if (total + bytes > budget) release_unused();
  if (total + bytes > budget) {
    *rc = EIK_ERR_OUT_OF_BUDGET;
    return nullptr;
  }
  void* p = nullptr;
  if (cudaMalloc(&p, std::max<size_t>(bytes, 256)) != cudaSuccess) {
    cudaGetLastError();  // clear the allocation error before trying again
    release_unused();
    if (cudaMalloc(&p, std::max<size_t>(bytes, 256)) != cudaSuccess) {
      *rc = EIK_ERR_CUDA;
      return nullptr;
    }
  }
  bufs[name] = Buf{p, bytes, epoch};
  total += bytes;
  return p;
}
void Scratch::release_all() {
  for (auto& kv : bufs) cudaFree(kv.second.ptr);
  bufs.clear();
  total = 0;
}
void Scratch::release_unused() {
  for (auto it = bufs.begin(); it != bufs.end();) {
    if (it->second.used != epoch) {
      cudaFree(it->second.ptr);  // waits for the device work that may still read it
      total -= it->second.bytes;
      it = bufs.erase(it);
    } else {
      ++it;
    }
  }
}

// ----------------------------------------------------------------- grids --
int make_griddesc(eik_ctx* ctx, const eik_grid* g, GridDesc* out) {
  if (!g) return fail(ctx, EIK_ERR_ASSERT, "grid descriptor is NULL");
  GridDesc d;
  std::memset(&d, 0, sizeof d);
  d.kind = g->kind;
  const bool cart = g->kind == EIK_GRID2DCART || g->kind == EIK_GRID3DCART;
  if (g->kind < 0 || g->kind > 3) return fail(ctx, EIK_ERR_ASSERT, "unknown grid kind %d", g->kind);
  d.nd = (g->kind == EIK_GRID2DCART || g->kind == EIK_GRID2DSPHERE) ? 2 : 3;
  if (g->ndim != d.nd) return fail(ctx, EIK_ERR_ASSERT, "2<=ndims(vel)<=3 / grid ndim mismatch");
  for (int a = 0; a < 3; a++) {
    d.n[a] = 1;
    d.spac[a] = 0;
    d.co[a] = 0;
  }
  for (int a = 0; a < d.nd; a++) {
    if (g->grsize[a] <= 0) return fail(ctx, EIK_ERR_ASSERT, "all(grsize.>0)");
    if (g->grsize[a] > (1 << 30)) return fail(ctx, EIK_ERR_UNSUPPORTED, "grid axis too large");
    d.n[a] = (int32_t)g->grsize[a];
    d.co[a] = g->cooinit[a];
    d.spac[a] = cart ? g->spacing[0] : g->spacing[a];
  }
  if (cart && !(g->spacing[0] > 0.0)) return fail(ctx, EIK_ERR_ASSERT, "hgrid>0.0");
  if (g->kind == EIK_GRID2DSPHERE) {
    if (!(g->cooinit[0] >= 0.0)) return fail(ctx, EIK_ERR_ASSERT, "cooinit[1]>=0.0");
    if (!(g->spacing[0] > 0.0)) return fail(ctx, EIK_ERR_ASSERT, "Δr>0.0");
    if (!(g->spacing[1] > 0.0)) return fail(ctx, EIK_ERR_ASSERT, "Δθ>0.0");
  }
  if (g->kind == EIK_GRID3DSPHERE && !(g->cooinit[0] > 0.0)) return fail(ctx, EIK_ERR_ASSERT, "cooinit[1]>0.0");
  for (int a = 0; a < d.nd; a++) d.ax[a] = make_jrange(d.co[a], d.spac[a]);
  if (g->kind == EIK_GRID2DSPHERE) {
    for (int i = 1; i <= d.n[1]; i++) {
      const double th = jr_value(d.ax[1], i);
      if (!(0.0 <= th && th <= 180.0)) return fail(ctx, EIK_ERR_ASSERT, "all(0.0.<=θ.<=180.0)");
    }
  } else if (g->kind == EIK_GRID3DSPHERE) {
    for (int i = 1; i <= d.n[1]; i++) {
      const double th = jr_value(d.ax[1], i);
      if (!(5.0 <= th && th <= 175.0)) return fail(ctx, EIK_ERR_ASSERT, "all(5.0.<=θ.<=175.0)");
    }
    for (int i = 1; i <= d.n[2]; i++) {
      const double ph = jr_value(d.ax[2], i);
      if (!(0.0 <= ph && ph <= 180.0)) return fail(ctx, EIK_ERR_ASSERT, "all(0.0.<=φ.<=180.0)");
    }
  }
  *out = d;
  return EIK_OK;
}

// checksrcrecposition (src/EikSolv/eikchecks.jl:4-50)
int check_positions(eik_ctx* ctx, const GridDesc& g, int64_t nsrc, const double* cs,
                    const int64_t* recoff, const double* rec) {
  for (int d = 0; d < g.nd; d++) {
    const double lo = jr_value(g.ax[d], 1), hi = jr_value(g.ax[d], g.n[d]);
    for (int64_t s = 0; s < nsrc; s++) {
      const double x = cs[s * g.nd + d];
      if (!(lo <= x && x <= hi))
        return fail(ctx, EIK_ERR_ASSERT, "source %lld outside the grid on axis %d", (long long)s, d);
    }
    for (int64_t r = 0; r < recoff[nsrc]; r++) {
      const double x = rec[r * g.nd + d];
      if (!(lo <= x && x <= hi))
        return fail(ctx, EIK_ERR_ASSERT, "receiver %lld outside the grid on axis %d", (long long)r, d);
    }
  }
  for (int64_t s = 0; s < nsrc; s++)
    if (recoff[s + 1] < recoff[s]) return fail(ctx, EIK_ERR_ASSERT, "rec_off must be non-decreasing");
  return EIK_OK;
}

int check_extra(eik_ctx* ctx, const eik_extra* ep) {
  if (ep->radiussmoothgradsrc < 0) return fail(ctx, EIK_ERR_ASSERT, "radiussmoothgradsrc>= 0");
  if (ep->smoothgradkern < 0) return fail(ctx, EIK_ERR_ASSERT, "smoothgradkern>=0");
  if (ep->smoothgradkern > 0 && ep->smoothgradkern % 2 == 0)
    return fail(ctx, EIK_ERR_ERROR, "ExtraParams: smoothgradkern must be an odd number");
  if (ep->parallelkind < 0 || ep->parallelkind > 2)
    return fail(ctx, EIK_ERR_ERROR, "ExtraParams(): 'parallelkind' must be one of :serial, :sharedmem or :distribmem");
  if (ep->refinearoundsrc && (ep->downscalefactor < 1 || ep->noderadius < 0))
    return fail(ctx, EIK_ERR_ASSERT, "GridRefinementPars: downscalefactor>=1, noderadius>=0");
  return EIK_OK;
}

__global__ void slowness_kernel(const double* vel, double* slow, long long n, int* nonpos, double* ssum,
                                unsigned long long* smin) {
  double acc = 0.0, mn = EIK_INF;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = vel[i];
    if (!(v > 0.0)) atomicExch(nonpos, 1);
    slow[i] = 1.0 / v;
    acc += (v > 0.0) ? 1.0 / v : 0.0;
    if (v > 0.0) mn = fmin(mn, 1.0 / v);
  }
  atomicAdd(ssum, acc);
  atomicMin(smin, (unsigned long long)__double_as_longlong(mn));  // positive doubles order as integers
}

void model_refresh(const Model& m, cudaStream_t st) {
  cudaMemsetAsync(m.dstat, 0, 2 * sizeof(double), st);
  cudaMemsetAsync(m.dstat + 2, 0x7f, sizeof(double), st);  // a large positive double
  slowness_kernel<<<592, 256, 0, st>>>(m.vel, m.slow, m.N, reinterpret_cast<int*>(m.dstat), m.dstat + 1,
                                       reinterpret_cast<unsigned long long*>(m.dstat + 2));
}

const void* stage_host(eik_ctx* ctx, const void* src, size_t bytes) {
  if (!ctx->capturing || bytes == 0) return src;
  void* p = nullptr;
  if (cudaMallocHost(&p, bytes) != cudaSuccess) return nullptr;
  std::memcpy(p, src, bytes);
  ctx->stage_arena->push_back(p);
  return p;
}

// Round width and lower-bound increment of every coarse problem from the model's smallest
// slowness, read on the device (the expressions and their order are the host's).
__global__ void problem_scale_kernel(CoarseProblem* dp, int nprob, const double* dsmin, double gate, double hmin,
                                     int nd) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nprob) return;
  const double smin = *dsmin;
  dp[s].delta = gate * hmin * smin;
  dp[s].incmin = 0.999 * (2.0 / 3.0) * hmin * smin / sqrt((double)nd);
}

int model_create(eik_ctx* ctx, const eik_grid* grd, const double* vel, bool dev, eik_model_id* out) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  Model m;
  int rc = make_griddesc(ctx, grd, &m.g);
  if (rc) return rc;
  m.N = npts(m.g);
  const size_t bytes = sizeof(double) * (size_t)m.N;
  if (ctx->scratch.total + ctx->model_bytes + 2 * bytes > ctx->scratch.budget) {
    ctx->scratch.begin_call();  // scratch kept from earlier calls gives way to a resident model
    ctx->scratch.release_unused();
  }
  if (ctx->scratch.total + ctx->model_bytes + 2 * bytes > ctx->scratch.budget)
    return fail(ctx, EIK_ERR_OUT_OF_BUDGET, "model of %zu bytes exceeds the HBM budget", 2 * bytes);
  CUDA_OK(ctx, cudaSetDevice(ctx->device));
  CUDA_OK(ctx, cudaMalloc(&m.vel, bytes));
  CUDA_OK(ctx, cudaMalloc(&m.slow, bytes));
  if (dev) CUDA_OK(ctx, cudaMemcpyAsync(m.vel, vel, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  else CUDA_OK(ctx, cudaMemcpyAsync(m.vel, vel, bytes, cudaMemcpyHostToDevice, ctx->stream));
  CUDA_OK(ctx, cudaMalloc(&m.dstat, 3 * sizeof(double)));
  model_refresh(m, ctx->stream);
  int nonpos = 0;
  CUDA_OK(ctx, cudaMemcpyAsync(&nonpos, m.dstat, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_OK(ctx, cudaMemcpyAsync(&m.smin, m.dstat + 2, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_OK(ctx, cudaStreamSynchronize(ctx->stream));
  if (nonpos) {
    cudaFree(m.vel);
    cudaFree(m.slow);
    cudaFree(m.dstat);
    return fail(ctx, EIK_ERR_ASSERT, "all(vel.>0.0)");
  }
  ctx->model_bytes += 2 * bytes;
  const eik_model_id id = ++ctx->next_model;
  ctx->models[id] = m;
  *out = id;
  return EIK_OK;
}

uint32_t read_err(eik_ctx* ctx, uint32_t* derr) {
  uint32_t h = 0;
  cudaMemcpyAsync(&h, derr, sizeof h, cudaMemcpyDeviceToHost, ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  return h;
}

int err_to_rc(eik_ctx* ctx, uint32_t e) {
  if (!e) return EIK_OK;
  if (e & ERRB_QUEUE_TIMEOUT) return fail(ctx, EIK_ERR_TIMEOUT, "device wait ran out (error word 0x%x)", e);
  if (e & (ERRB_NOT_CONVERGED | ERRB_ADJ_NOT_CONVERGED))
    return fail(ctx, EIK_ERR_NOT_CONVERGED, "iteration limit reached (error word 0x%x)", e);
  if (e & ERRB_SINGULAR) return fail(ctx, EIK_ERR_ERROR, "SingularException in the adjoint solve");
  return fail(ctx, EIK_ERR_UNSUPPORTED, "refined-grid capacity exceeded (error word 0x%x)", e);
}

// -------------------------------------------------------------- forward pipeline --
// Runs the start-up stage and the coarse solve for the sources of several models (nmod >= 1;
// src_off[i]..src_off[i+1] are model i's sources, all models of one dimension) whose
// coordinates are already on the device. The grids may differ in size: every source is a
// problem with its own grid, numbered in the round solver with the largest grid's node
// count as stride, so all of them share one persistent launch. The start-up stage runs per
// model on its slice of the per-source arrays; the refined windows share one launch. On
// return the traveltimes of source s are at fw.t + s*fw.N (its first npts of its model's
// grid; codes at fw.code + s*fw.N).
int forward_multi(eik_ctx* ctx, int nmod, const Model* const* models, const int64_t* src_off, const double* d_cs,
                  const eik_extra& ep, ForwardState* fw, eik_stats* stats) {
  int rc = EIK_OK;
  const int64_t nsrc = src_off[nmod];
  const int nd = models[0]->g.nd;
  long long N = 0;  // stride: the largest grid
  unsigned long long work = 0;
  for (int i = 0; i < nmod; i++) {
    if (models[i]->g.nd != nd) return fail(ctx, EIK_ERR_ASSERT, "models of one call have one dimension");
    N = std::max<long long>(N, models[i]->N);
    work += (unsigned long long)(src_off[i + 1] - src_off[i]) * (unsigned long long)models[i]->N;
  }
  cudaStream_t st = ctx->stream;
  Scratch& S = ctx->scratch;
  ForwardBatch fb;
  std::memset(&fb, 0, sizeof fb);
  fb.g = models[0]->g;
  fb.nsrc = (int32_t)nsrc;
  fb.ds = ep.downscalefactor;
  fb.noderadius = ep.noderadius;
  fb.vel = models[0]->vel;
  fb.slow = models[0]->slow;
  fb.coordsrc = d_cs;
  const bool refine = ep.refinearoundsrc != 0;
  long long win = 1, nfmax = 1;
  for (int d = 0; d < nd; d++) {
    win *= 2LL * ep.noderadius + 2;
    nfmax *= (2LL * ep.noderadius + 1) * ep.downscalefactor + 1;
  }
  fb.seedcap = refine ? (int32_t)std::max<long long>(win, 8) : 8;
  fb.nfmax = refine ? nfmax : 1;
  fb.heapcap = (int32_t)std::min<long long>(refine ? nfmax : 1, 8192);
#define GET(var, type, name, count)                                                  \
  var = (type*)S.get(name, sizeof(type) * (size_t)(count), &rc);                     \
  if (!var) return rc == EIK_ERR_OUT_OF_BUDGET                                       \
                     ? fail(ctx, rc, "scratch '%s' exceeds the HBM budget", name)    \
                     : fail(ctx, rc, "cudaMalloc of scratch '%s' failed", name);
  GET(fb.out, SrcOut, "srcout", nsrc);
  GET(fb.seed_lin, int32_t, "seed_lin", nsrc * fb.seedcap);
  GET(fb.seed_tt, double, "seed_tt", nsrc * fb.seedcap);
  GET(fb.err, uint32_t, "err", 4);
  if (refine) {
    GET(fb.fine_tt, double, "fine_tt", nsrc * fb.nfmax);
    GET(fb.fine_status, uint8_t, "fine_status", nsrc * fb.nfmax);
    GET(fb.fine_code, uint8_t, "fine_code", nsrc * fb.nfmax);
    GET(fb.fine_idx, int32_t, "fine_idx", nsrc * fb.nfmax);
    GET(fb.fine_order, int32_t, "fine_order", nsrc * fb.nfmax);
    GET(fb.fine_onh, uint8_t, "fine_onh", nsrc * fb.nfmax);
  }
  // coarse problems
  double* t;
  uint8_t* code;
  double* kL;
  uint8_t* kd;
  GET(t, double, "t", nsrc * N);
  GET(code, uint8_t, "code", nsrc * N);
  GET(kL, double, "kL", nsrc * N);
  GET(kd, uint8_t, "kd", nsrc * N);
  std::vector<CoarseProblem> hp(nsrc);
  for (int i = 0; i < nmod; i++)
    for (int64_t s = src_off[i]; s < src_off[i + 1]; s++) {
      CoarseProblem& P = hp[s];
      P.g = models[i]->g;
      P.slow = models[i]->slow;
      P.t = t + s * N;
      P.code = code + s * N;
      P.kL = kL + s * N;
      P.kd = kd + s * N;
      P.delta = P.incmin = 0.0;  // set on the device from the model's smallest slowness
      uniform_coeffs(P.g, &P.c1u, &P.c2u);
    }
  CoarseProblem* dp;
  GET(dp, CoarseProblem, "probs", nsrc);
  SolveArgs sa;
  std::memset(&sa, 0, sizeof sa);
  sa.nprob = (int32_t)nsrc;
  sa.nd = nd;
  unsigned long long* ctr;
  GET(ctr, unsigned long long, "solve_ctr", 16);
  sa.activations = ctr;
  sa.node_evals = ctr + 1;
  sa.abort_flag = (int32_t*)(ctr + 2);
  // round-solver state, shared by the refined windows' solve and the coarse solve
  const long long rsn = nsrc * std::max<long long>(N, refine ? fb.nfmax : 1);
  if ((unsigned long long)rsn >= (1ull << 32))
    return fail(ctx, EIK_ERR_OUT_OF_BUDGET, "more than 2^32 node-sources in one call: split the sources");
  GET(sa.rs.stamp, int32_t, "rs_stamp", rsn);
  GET(sa.rs.tent, double, "rs_tent", rsn);
  GET(sa.rs.dirty, uint8_t, "rs_dirty", rsn);
  GET(sa.rs.list[0], unsigned long long, "rs_list0", rsn);
  GET(sa.rs.list[1], unsigned long long, "rs_list1", rsn);
  GET(sa.rs.nextmin, unsigned long long, "rs_nextmin", 3 * nsrc);
  GET(sa.rs.thr, double, "rs_thr", 2 * nsrc);
  {
    unsigned int* rc32;
    GET(rc32, unsigned int, "rs_ctr", 32);
    sa.rs.cnt = rc32;
    sa.rs.grab = rc32 + 3;
    sa.rs.bar = rc32 + 6;
    sa.rs.rounds = (int32_t*)(rc32 + 8);
    sa.rs.visits = reinterpret_cast<unsigned long long*>(rc32 + 12);  // 8-byte aligned: 7 counters
  }
  // round limit: the caller's, else 256 rounds per node of the grid's diameter (a solve
  // takes 2-7 in practice) plus 65536, so that a schedule that fails to settle is stopped in
  // seconds and the call re-run with another (run_with_retry); 2^24 on that re-run
  auto round_limit = [&](long long diam) -> int {
    if (ctx->max_rounds > 0) return ctx->max_rounds;
    if (ctx->retry) return 1 << 24;
    if (ctx->auto_round_limit > 0) return ctx->auto_round_limit;
    return (int)std::min<long long>(1LL << 24, 256LL * diam + 65536);
  };
  long long diam = 0;
  for (int i = 0; i < nmod; i++) {
    long long d = 0;
    for (int a = 0; a < nd; a++) d += models[i]->g.n[a];
    diam = std::max(diam, d);
  }
  sa.rs.max_rounds = round_limit(diam);
  // small problems in thread-block clusters: in 2D by default (1), where it is faster than the
  // global solve (measured: 300x220 x 4 sources 27.7 -> 15.9 ms); in 3D the global solve is
  // faster (44^3 x 16: 33 vs 40 ms, and the refined windows), so only on request (2)
  const bool use_cluster = ctx->cluster_solve == 2 || (ctx->cluster_solve == 1 && nd == 2);
  sa.rs.stride = (unsigned long long)N;
  sa.err = fb.err;
  sa.probs = dp;
  sa.max_activations = ~0ull;
  sa.timeout_ns = 20LL * 1000 * 1000 * 1000;
  // refined windows: one more round-solver problem per source
  CoarseProblem* fprobs = nullptr;
  int32_t* fseed_lin = nullptr;
  double *fseed_tt = nullptr, *fslow = nullptr, *fkL = nullptr;
  uint8_t *fkd = nullptr, *ftie = nullptr;
  if (refine) {
    GET(fprobs, CoarseProblem, "fine_probs", nsrc);
    GET(fseed_lin, int32_t, "fine_seed_lin", nsrc * 8);
    GET(fseed_tt, double, "fine_seed_tt", nsrc * 8);
    GET(fslow, double, "fine_slow", nsrc * fb.nfmax);
    GET(fkL, double, "fine_kL", nsrc * fb.nfmax);
    GET(fkd, uint8_t, "fine_kd", nsrc * fb.nfmax);
    GET(ftie, uint8_t, "fine_tie", nsrc);
  }
#undef GET
  const void* hp_src = stage_host(ctx, hp.data(), sizeof(CoarseProblem) * nsrc);
  if (!hp_src) return fail(ctx, EIK_ERR_CUDA, "cudaMallocHost of a plan's staging copy failed");
  CUDA_OK(ctx, cudaMemcpyAsync(dp, hp_src, sizeof(CoarseProblem) * nsrc, cudaMemcpyHostToDevice, st));
  const double gate = ctx->gate_for(work);
  const int sms = ctx->sms_for(work);
  // model i's slice of the per-source arrays, for the per-model start-up launches
  auto slice = [&](int i) {
    ForwardBatch f = fb;
    const int64_t o = src_off[i];
    f.g = models[i]->g;
    f.vel = models[i]->vel;
    f.slow = models[i]->slow;
    f.nsrc = (int32_t)(src_off[i + 1] - o);
    f.coordsrc = d_cs + o * nd;
    f.out = fb.out + o;
    f.seed_lin = fb.seed_lin + o * fb.seedcap;
    f.seed_tt = fb.seed_tt + o * fb.seedcap;
    if (refine) {
      f.fine_tt = fb.fine_tt + o * fb.nfmax;
      f.fine_status = fb.fine_status + o * fb.nfmax;
      f.fine_code = fb.fine_code + o * fb.nfmax;
      f.fine_idx = fb.fine_idx + o * fb.nfmax;
      f.fine_order = fb.fine_order + o * fb.nfmax;
      f.fine_onh = fb.fine_onh + o * fb.nfmax;
    }
    return f;
  };
  int nlaunch = 0;
  // round widths: about one node's traveltime at the model's largest velocity, times round_gate
  for (int i = 0; i < nmod; i++) {
    const int64_t ni = src_off[i + 1] - src_off[i];
    if (ni == 0) continue;
    double dh[3];
    node_dh(models[i]->g, 0, dh);
    double hmin = dh[0];
    for (int a = 1; a < nd; a++) hmin = std::min(hmin, dh[a]);
    problem_scale_kernel<<<(int)((ni + 127) / 128), 128, 0, st>>>(dp + src_off[i], (int)ni, models[i]->dstat + 2,
                                                                  gate, hmin, nd);
    nlaunch += 1;
  }
  CUDA_OK(ctx, cudaMemsetAsync(fb.err, 0, sizeof(uint32_t) * 4, st));
  CUDA_OK(ctx, cudaMemsetAsync(fb.out, 0, sizeof(SrcOut) * nsrc, st));
  if (!ctx->capturing) cudaEventRecord(ctx->evk[0], st);
  if (refine && ctx->fine_replay) {
    for (int i = 0; i < nmod; i++)
      if (src_off[i + 1] > src_off[i]) {
        launch_fine(slice(i), st);
        nlaunch += 1;
      }
  } else if (refine) {
    // the windows as round-solver problems, then the heap's stop reconstructed from keys
    for (int i = 0; i < nmod; i++) {
      const int64_t o = src_off[i];
      if (src_off[i + 1] == o) continue;
      launch_fine_setup(slice(i), fprobs + o, models[i]->dstat + 2, gate, fseed_lin + o * 8, fseed_tt + o * 8,
                        fslow + o * fb.nfmax, fkL + o * fb.nfmax, fkd + o * fb.nfmax, st);
      nlaunch += 2;
    }
    SolveArgs fsa = sa;
    fsa.probs = fprobs;
    fsa.rs.stride = (unsigned long long)fb.nfmax;
    fsa.activations = sa.activations + 6;  // own counters: the coarse solve's stay separate
    fsa.node_evals = sa.activations + 7;
    fsa.rs.max_rounds = round_limit((long long)nd * ((2LL * ep.noderadius + 1) * ep.downscalefactor + 1));
    // the windows are small: one thread-block cluster each when the GPU has room for it
    bool in_cluster = false;
    if (use_cluster)
      CUDA_OK(ctx, launch_cluster_solve(fsa, fb.nfmax, fseed_lin, fseed_tt, fb.out, true, 8, st, &in_cluster));
    if (in_cluster) {
      nlaunch += 2;
    } else {
      launch_rounds_init(fsa, st);
      launch_rounds_seed(fsa, fseed_lin, fseed_tt, fb.out, true, 8, st);
      CUDA_OK(ctx, launch_coarse_solve(fsa, sms, ctx->ctas_per_sm, ctx->fwd_queue, st));
      nlaunch += 3;
    }
    for (int i = 0; i < nmod; i++) {
      const int64_t o = src_off[i];
      if (src_off[i + 1] == o) continue;
      launch_fine_select(slice(i), fprobs + o, ftie + o, st);
      // stops decided by exact ties: the heap is replayed for the flagged sources only, the
      // flags staying on the device (no host round trip between the stages)
      launch_fine_replay(slice(i), ftie + o, st);
      nlaunch += 2;
    }
    CUDA_OK(ctx, cudaGetLastError());
  } else {
    for (int i = 0; i < nmod; i++)
      if (src_off[i + 1] > src_off[i]) {
        launch_srcbox(slice(i), st);
        nlaunch += 1;
      }
  }
  if (!ctx->capturing) cudaEventRecord(ctx->evk[1], st);
  CUDA_OK(ctx, cudaGetLastError());
  if (use_cluster && cluster_solve_fits(sa, N)) {
    // small grids: one thread-block cluster per source, init and seeds included
    if (!ctx->capturing) cudaEventRecord(ctx->evk[2], st);
    bool in_cluster = false;
    CUDA_OK(ctx, launch_cluster_solve(sa, N, fb.seed_lin, fb.seed_tt, fb.out, false, fb.seedcap, st, &in_cluster));
    if (!in_cluster) return fail(ctx, EIK_ERR_CUDA, "the cluster solve could not be launched");
    if (!ctx->capturing) cudaEventRecord(ctx->evk[3], st);
    CUDA_OK(ctx, cudaGetLastError());
    nlaunch += 2;  // counters, solve
  } else {
    launch_coarse_init(hp.data(), dp, (int)nsrc, fb, sa, st);
    CUDA_OK(ctx, cudaGetLastError());
    if (!ctx->capturing) cudaEventRecord(ctx->evk[2], st);
    CUDA_OK(ctx, launch_coarse_solve(sa, sms, ctx->ctas_per_sm, ctx->fwd_queue, st));
    if (!ctx->capturing) cudaEventRecord(ctx->evk[3], st);
    CUDA_OK(ctx, cudaGetLastError());
    nlaunch += 4;  // coarse init, round init, seeds, solve
  }
  fw->fb = fb;
  fw->sa = sa;
  fw->t = t;
  fw->code = code;
  fw->kL = kL;
  fw->kd = kd;
  fw->N = N;
  fw->nsrc = nsrc;
  fw->fine_tie = (refine && !ctx->fine_replay) ? ftie : nullptr;
  fw->launches = nlaunch;
  fw->gate = gate;
  fw->sms = sms;
  if (stats) stats->launches += nlaunch;
  return EIK_OK;
}

int forward_device(eik_ctx* ctx, const Model& m, int64_t nsrc, const double* d_cs, const eik_extra& ep,
                   ForwardState* fw, eik_stats* stats) {
  const Model* mm = &m;
  const int64_t off[2] = {0, nsrc};
  return forward_multi(ctx, 1, &mm, off, d_cs, ep, fw, stats);
}

int collect_forward_stats(eik_ctx* ctx, ForwardState* fw, eik_stats* stats) {
  unsigned long long ctr[4] = {0, 0, 0, 0};
  uint32_t e = 0;
  int32_t rounds = 0;
  unsigned long long vis[7] = {0, 0, 0, 0, 0, 0, 0};
  cudaMemcpyAsync(ctr + 2, fw->sa.activations, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(vis, fw->sa.rs.visits, sizeof vis, cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(&rounds, fw->sa.rs.rounds, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(&e, fw->fb.err, sizeof e, cudaMemcpyDeviceToHost, ctx->stream);
  std::vector<SrcOut> outs(fw->nsrc);
  cudaMemcpyAsync(outs.data(), fw->fb.out, sizeof(SrcOut) * fw->nsrc, cudaMemcpyDeviceToHost, ctx->stream);
  std::vector<uint8_t> tie(fw->fine_tie ? fw->nsrc : 0);
  if (fw->fine_tie) cudaMemcpyAsync(tie.data(), fw->fine_tie, (size_t)fw->nsrc, cudaMemcpyDeviceToHost, ctx->stream);
  CUDA_OK(ctx, cudaStreamSynchronize(ctx->stream));
  uint32_t warn = 0;
  for (auto& o : outs) warn |= o.warn;
  if (stats) {
    stats->warn_mask |= warn;
    stats->err_mask |= e;
    stats->tile_activations += ctr[2];
    stats->node_evals += ctr[3];
    stats->fwd_rounds += (uint64_t)rounds;
    for (uint8_t f : tie) stats->fine_replays += f ? 1 : 0;
    for (int k = 0; k < 7; k++) stats->fwd_visits[k] += vis[k];
    float a = 0, b = 0;
    cudaEventElapsedTime(&a, ctx->evk[0], ctx->evk[1]);
    cudaEventElapsedTime(&b, ctx->evk[2], ctx->evk[3]);
    stats->fine_ms = a;
    stats->solve_ms = b;
  }
  fw->host_out = std::move(outs);
  return err_to_rc(ctx, e);
}

}  // namespace eik

using namespace eik;

extern "C" {

void eik_extra_defaults(eik_extra* ep) {
  std::memset(ep, 0, sizeof *ep);
  ep->refinearoundsrc = 1;
  ep->downscalefactor = 5;
  ep->noderadius = 3;
  ep->radiussmoothgradsrc = 3;
  ep->smoothgradkern = 0;
  ep->parallelkind = 0;
}

int eik_ctx_create(int device, size_t hbm_budget, eik_ctx** out) {
  if (!out) return fail(nullptr, EIK_ERR_ASSERT, "out is NULL");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(nullptr, EIK_ERR_CUDA, "no CUDA device available");
  if (device < 0 || device >= ndev) return fail(nullptr, EIK_ERR_ASSERT, "device %d out of range", device);
  if (cudaSetDevice(device) != cudaSuccess) return fail(nullptr, EIK_ERR_CUDA, "cudaSetDevice failed");
  eik_ctx* c = new eik_ctx();
  c->device = device;
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  c->nsm = prop.multiProcessorCount;
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  c->scratch.budget = hbm_budget ? hbm_budget : (size_t)(0.9 * (double)fr);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return fail(nullptr, EIK_ERR_CUDA, "cudaStreamCreate failed");
  }
  cudaEventCreate(&c->ev0);
  cudaEventCreate(&c->ev1);
  for (auto& e : c->evk) cudaEventCreate(&e);
  *out = c;
  return EIK_OK;
}

int eik_ctx_destroy(eik_ctx* ctx) {
  if (!ctx) return EIK_OK;
  {
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (ctx->live_plans > 0)
      return fail(ctx, EIK_ERR_ASSERT, "context has %d live plan(s): destroy them first", ctx->live_plans);
  }
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto& kv : ctx->models) {
    cudaFree(kv.second.vel);
    cudaFree(kv.second.slow);
    cudaFree(kv.second.dstat);
  }
  ctx->scratch.release_all();
  cudaEventDestroy(ctx->ev0);
  cudaEventDestroy(ctx->ev1);
  for (auto& e : ctx->evk) cudaEventDestroy(e);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return EIK_OK;
}

void* eik_ctx_stream(eik_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int eik_ctx_set_param(eik_ctx* ctx, const char* name, double value) {
  if (!ctx || !name) return fail(ctx, EIK_ERR_ASSERT, "NULL argument");
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (std::strcmp(name, "round_gate") == 0) {
    if (!(value >= 0.0 && value < 1e6)) return fail(ctx, EIK_ERR_ASSERT, "round_gate must be in [0, 1e6)");
    ctx->round_gate = value;
    return EIK_OK;
  }
  if (std::strcmp(name, "fine_replay") == 0) {
    ctx->fine_replay = value != 0.0;
    return EIK_OK;
  }
  if (std::strcmp(name, "ctas_per_sm") == 0) {
    if (!(value >= 0.0 && value <= 32.0 && value == (double)(int)value))
      return fail(ctx, EIK_ERR_ASSERT, "ctas_per_sm must be an integer in [0, 32]");
    ctx->ctas_per_sm = (int)value;
    return EIK_OK;
  }
  if (std::strcmp(name, "ray_room") == 0) {
    if (!(value >= 0.0 && value <= 100.0)) return fail(ctx, EIK_ERR_ASSERT, "ray_room must be in [0, 100]");
    ctx->ray_room = value;
    return EIK_OK;
  }
  if (std::strcmp(name, "fwd_queue") == 0) {
    if (!(value == -1.0 || value == 0.0 || value == 1.0))
      return fail(ctx, EIK_ERR_ASSERT, "fwd_queue must be -1 (automatic), 0 or 1");
    ctx->fwd_queue = (int)value;
    return EIK_OK;
  }
  if (std::strcmp(name, "auto_round_limit") == 0) {
    if (!(value >= 0.0 && value <= (double)(1 << 24) && value == (double)(long long)value))
      return fail(ctx, EIK_ERR_ASSERT, "auto_round_limit must be an integer in [0, 2^24] (0 = by the grid's size)");
    ctx->auto_round_limit = (int)value;
    return EIK_OK;
  }
  if (std::strcmp(name, "cluster_solve") == 0) {
    if (!(value == 0.0 || value == 1.0 || value == 2.0))
      return fail(ctx, EIK_ERR_ASSERT, "cluster_solve must be 0, 1 or 2");
    ctx->cluster_solve = (int)value;
    return EIK_OK;
  }
  if (std::strcmp(name, "max_rounds") == 0) {
    if (!(value >= 0.0 && value <= (double)(1 << 30) && value == (double)(long long)value))
      return fail(ctx, EIK_ERR_ASSERT, "max_rounds must be an integer in [0, 2^30] (0 = the library's limit)");
    ctx->max_rounds = (int)value;
    return EIK_OK;
  }
  if (std::strcmp(name, "sm_fraction") == 0) {
    if (!(value >= 0.0 && value <= 1.0)) return fail(ctx, EIK_ERR_ASSERT, "sm_fraction must be in [0, 1]");
    ctx->sm_fraction = value;
    return EIK_OK;
  }
  return fail(ctx, EIK_ERR_ASSERT, "unknown parameter '%s'", name);
}

}  // extern "C"

namespace eik {
// A bounded wait on a flag that nothing sets: the wait limit of the persistent solves
// (global timer, then an error bit instead of a trap), exercised on its own.
__global__ void selftest_wait_kernel(const unsigned int* flag, long long timeout_ns, uint32_t* err) {
  const long long t0 = gtimer_ns();
  while (*(volatile const unsigned int*)flag == 0u) {
    if (gtimer_ns() - t0 > timeout_ns) {
      atomicOr(err, ERRB_QUEUE_TIMEOUT);
      return;
    }
    __nanosleep(1000);
  }
}
}  // namespace eik

extern "C" {

int eik_selftest_wait(eik_ctx* ctx, double timeout_s) {
  if (!ctx) return fail(ctx, EIK_ERR_ASSERT, "NULL context");
  if (!(timeout_s >= 1e-3 && timeout_s <= 10.0)) return fail(ctx, EIK_ERR_ASSERT, "timeout_s must be in [0.001, 10]");
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->scratch.begin_call();
  CUDA_OK(ctx, cudaSetDevice(ctx->device));
  int rc = EIK_OK;
  unsigned int* flag = (unsigned int*)ctx->scratch.get("selftest_flag", 2 * sizeof(unsigned int), &rc);
  if (!flag) return fail(ctx, rc, "scratch allocation failed");
  uint32_t* err = flag + 1;
  CUDA_OK(ctx, cudaMemsetAsync(flag, 0, 2 * sizeof(unsigned int), ctx->stream));
  selftest_wait_kernel<<<1, 1, 0, ctx->stream>>>(flag, (long long)(timeout_s * 1e9), err);
  CUDA_OK(ctx, cudaGetLastError());
  return err_to_rc(ctx, read_err(ctx, err));
}

const char* eik_last_error(eik_ctx* ctx) {
  (void)ctx;
  return tl_error.c_str();
}

int eik_model_upload(eik_ctx* ctx, const eik_grid* grd, const double* vel, eik_model_id* out) {
  if (!ctx || !vel || !out) return fail(ctx, EIK_ERR_ASSERT, "NULL argument");
  return model_create(ctx, grd, vel, false, out);
}

int eik_model_upload_device(eik_ctx* ctx, const eik_grid* grd, const double* vel_dev, eik_model_id* out) {
  if (!ctx || !vel_dev || !out) return fail(ctx, EIK_ERR_ASSERT, "NULL argument");
  return model_create(ctx, grd, vel_dev, true, out);
}

int eik_model_release(eik_ctx* ctx, eik_model_id model) {
  if (!ctx) return fail(ctx, EIK_ERR_ASSERT, "NULL context");
  std::lock_guard<std::mutex> lk(ctx->mu);
  auto it = ctx->models.find(model);
  if (it == ctx->models.end()) return fail(ctx, EIK_ERR_ASSERT, "unknown model id %lld", (long long)model);
  if (it->second.plans > 0)
    return fail(ctx, EIK_ERR_ASSERT, "model %lld is used by %d plan(s): destroy them first", (long long)model,
                it->second.plans);
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cudaFree(it->second.vel);
  cudaFree(it->second.slow);
  cudaFree(it->second.dstat);
  ctx->model_bytes -= 2 * sizeof(double) * (size_t)it->second.N;
  ctx->models.erase(it);
  return EIK_OK;
}

int eik_traveltime(eik_ctx* ctx, eik_model_id model, int64_t nsrc, const double* coordsrc,
                   const int64_t* rec_off, const double* rec, const eik_extra* ep_in, double* picks,
                   double* ttgrids, eik_stats* stats) {
  if (!ctx) return fail(ctx, EIK_ERR_ASSERT, "NULL context");
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->scratch.begin_call();
  NvtxRange nvtx_call("eik_traveltime");
  auto it = ctx->models.find(model);
  if (it == ctx->models.end()) return fail(ctx, EIK_ERR_ASSERT, "unknown model id %lld", (long long)model);
  const Model& m = it->second;
  eik_extra ep;
  if (ep_in) ep = *ep_in;
  else eik_extra_defaults(&ep);
  int rc = check_extra(ctx, &ep);
  if (rc) return rc;
  if (nsrc < 0) return fail(ctx, EIK_ERR_ASSERT, "nsrc >= 0");
  if (stats) std::memset(stats, 0, sizeof *stats);
  if (nsrc == 0) return EIK_OK;
  if (!coordsrc || !rec_off || (!rec && rec_off[nsrc] > 0) || (!picks && rec_off[nsrc] > 0))
    return fail(ctx, EIK_ERR_ASSERT, "NULL argument");
  rc = check_positions(ctx, m.g, nsrc, coordsrc, rec_off, rec);
  if (rc) return rc;
  for (int a = 0; a < m.g.nd; a++)
    if (m.g.n[a] < 3) return fail(ctx, EIK_ERR_ERROR, "BoundsError: grid axis %d has fewer than 3 nodes", a);
  CUDA_OK(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const int nd = m.g.nd;
  const long long nrec = rec_off[nsrc];
  double* d_cs = (double*)ctx->scratch.get("in_cs", sizeof(double) * nsrc * nd, &rc);
  long long* d_off = (long long*)ctx->scratch.get("in_off", sizeof(long long) * (nsrc + 1), &rc);
  double* d_rec = (double*)ctx->scratch.get("in_rec", sizeof(double) * std::max<long long>(nrec, 1) * nd, &rc);
  double* d_picks = (double*)ctx->scratch.get("out_picks", sizeof(double) * std::max<long long>(nrec, 1), &rc);
  if (!d_cs || !d_off || !d_rec || !d_picks) return fail(ctx, rc, "scratch allocation failed");
  cudaEventRecord(ctx->ev0, st);
  CUDA_OK(ctx, cudaMemcpyAsync(d_cs, coordsrc, sizeof(double) * nsrc * nd, cudaMemcpyHostToDevice, st));
  CUDA_OK(ctx, cudaMemcpyAsync(d_off, rec_off, sizeof(long long) * (nsrc + 1), cudaMemcpyHostToDevice, st));
  if (nrec) CUDA_OK(ctx, cudaMemcpyAsync(d_rec, rec, sizeof(double) * nrec * nd, cudaMemcpyHostToDevice, st));
  rc = run_with_retry(ctx, stats, [&]() -> int {
    ForwardState fw;
    int r = forward_device(ctx, m, nsrc, d_cs, ep, &fw, stats);
    if (r) return r;
    if (nrec) launch_picks(m.g, fw.t, m.N, (int)nsrc, d_off, d_rec, d_picks, st);
    if (nrec && stats) stats->launches += 1;
    CUDA_OK(ctx, cudaGetLastError());
    if (nrec) CUDA_OK(ctx, cudaMemcpyAsync(picks, d_picks, sizeof(double) * nrec, cudaMemcpyDeviceToHost, st));
    if (ttgrids)
      CUDA_OK(ctx, cudaMemcpyAsync(ttgrids, fw.t, sizeof(double) * nsrc * m.N, cudaMemcpyDeviceToHost, st));
    cudaEventRecord(ctx->ev1, st);
    return collect_forward_stats(ctx, &fw, stats);
  });
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    stats->device_ms = ms;
  }
  return rc;
}

int eik_traveltime_multi(eik_ctx* ctx, int64_t nmodel, const eik_model_id* model_ids, const int64_t* src_off,
                         const double* coordsrc, const int64_t* rec_off, const double* rec, const eik_extra* ep_in,
                         double* picks, double* ttgrids, eik_stats* stats) {
  if (!ctx) return fail(ctx, EIK_ERR_ASSERT, "NULL context");
  if (nmodel < 1 || !model_ids || !src_off) return fail(ctx, EIK_ERR_ASSERT, "nmodel >= 1 and NULL argument");
  if (nmodel > (1 << 20)) return fail(ctx, EIK_ERR_ASSERT, "more than 2^20 models in one call");
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->scratch.begin_call();
  NvtxRange nvtx_call("eik_traveltime_multi");
  std::vector<const Model*> mods(nmodel);
  for (int64_t i = 0; i < nmodel; i++) {
    auto it = ctx->models.find(model_ids[i]);
    if (it == ctx->models.end()) return fail(ctx, EIK_ERR_ASSERT, "unknown model id %lld", (long long)model_ids[i]);
    mods[i] = &it->second;
    if (mods[i]->g.nd != mods[0]->g.nd) return fail(ctx, EIK_ERR_ASSERT, "models of one call have one dimension");
  }
  if (src_off[0] != 0) return fail(ctx, EIK_ERR_ASSERT, "src_off[0] must be 0");
  for (int64_t i = 0; i < nmodel; i++)
    if (src_off[i + 1] < src_off[i]) return fail(ctx, EIK_ERR_ASSERT, "src_off must be non-decreasing");
  const int64_t nsrc = src_off[nmodel];
  eik_extra ep;
  if (ep_in) ep = *ep_in;
  else eik_extra_defaults(&ep);
  int rc = check_extra(ctx, &ep);
  if (rc) return rc;
  if (stats) std::memset(stats, 0, sizeof *stats);
  if (nsrc == 0) return EIK_OK;
  if (!coordsrc || !rec_off || (!rec && rec_off[nsrc] > 0) || (!picks && rec_off[nsrc] > 0))
    return fail(ctx, EIK_ERR_ASSERT, "NULL argument");
  if (rec_off[0] != 0) return fail(ctx, EIK_ERR_ASSERT, "rec_off[0] must be 0");
  const int nd = mods[0]->g.nd;
  // receiver offsets relative to each model's first receiver: model i's at rel[src_off[i] + i ...]
  std::vector<int64_t> rel(nsrc + nmodel);
  for (int64_t i = 0; i < nmodel; i++) {
    const int64_t o = src_off[i], n = src_off[i + 1] - o;
    for (int64_t s = 0; s <= n; s++) rel[o + i + s] = rec_off[o + s] - rec_off[o];
    rc = check_positions(ctx, mods[i]->g, n, coordsrc + o * nd, rel.data() + o + i, rec ? rec + rec_off[o] * nd : rec);
    if (rc) return rc;
    if (n > 0)
      for (int a = 0; a < nd; a++)
        if (mods[i]->g.n[a] < 3) return fail(ctx, EIK_ERR_ERROR, "BoundsError: grid axis %d has fewer than 3 nodes", a);
  }
  CUDA_OK(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const long long nrec = rec_off[nsrc];
  double* d_cs = (double*)ctx->scratch.get("in_cs", sizeof(double) * nsrc * nd, &rc);
  long long* d_off = (long long*)ctx->scratch.get("in_off", sizeof(long long) * (nsrc + nmodel), &rc);
  double* d_rec = (double*)ctx->scratch.get("in_rec", sizeof(double) * std::max<long long>(nrec, 1) * nd, &rc);
  double* d_picks = (double*)ctx->scratch.get("out_picks", sizeof(double) * std::max<long long>(nrec, 1), &rc);
  if (!d_cs || !d_off || !d_rec || !d_picks) return fail(ctx, rc, "scratch allocation failed");
  const void* rel_src = stage_host(ctx, rel.data(), sizeof(int64_t) * rel.size());
  if (!rel_src) return fail(ctx, EIK_ERR_CUDA, "cudaMallocHost of a staging copy failed");
  cudaEventRecord(ctx->ev0, st);
  CUDA_OK(ctx, cudaMemcpyAsync(d_cs, coordsrc, sizeof(double) * nsrc * nd, cudaMemcpyHostToDevice, st));
  CUDA_OK(ctx, cudaMemcpyAsync(d_off, rel_src, sizeof(int64_t) * rel.size(), cudaMemcpyHostToDevice, st));
  if (nrec) CUDA_OK(ctx, cudaMemcpyAsync(d_rec, rec, sizeof(double) * nrec * nd, cudaMemcpyHostToDevice, st));
  rc = run_with_retry(ctx, stats, [&]() -> int {
    ForwardState fw;
    int r = forward_multi(ctx, (int)nmodel, mods.data(), src_off, d_cs, ep, &fw, stats);
    if (r) return r;
    for (int64_t i = 0; i < nmodel; i++) {
      const int64_t o = src_off[i], n = src_off[i + 1] - o;
      if (n == 0 || rec_off[o + n] == rec_off[o]) continue;
      launch_picks(mods[i]->g, fw.t + o * fw.N, fw.N, (int)n, d_off + o + i, d_rec + rec_off[o] * nd,
                   d_picks + rec_off[o], st);
      if (stats) stats->launches += 1;
    }
    CUDA_OK(ctx, cudaGetLastError());
    if (nrec) CUDA_OK(ctx, cudaMemcpyAsync(picks, d_picks, sizeof(double) * nrec, cudaMemcpyDeviceToHost, st));
    if (ttgrids) {
      // each source's grid at its own size, one after another
      double* dst = ttgrids;
      for (int64_t i = 0; i < nmodel; i++) {
        const int64_t o = src_off[i], n = src_off[i + 1] - o;
        if (n == 0) continue;
        const size_t w = sizeof(double) * (size_t)mods[i]->N;
        CUDA_OK(ctx, cudaMemcpy2DAsync(dst, w, fw.t + o * fw.N, sizeof(double) * (size_t)fw.N, w, (size_t)n,
                                       cudaMemcpyDeviceToHost, st));
        dst += n * mods[i]->N;
      }
    }
    cudaEventRecord(ctx->ev1, st);
    return collect_forward_stats(ctx, &fw, stats);
  });
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    stats->device_ms = ms;
  }
  return rc;
}

}  // extern "C"
