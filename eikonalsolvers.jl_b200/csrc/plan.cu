// Captured gradient plans: the whole device pipeline of one eik_gradient call (velocity
// upload and slowness, observations upload, refined start-up, forward round solve, adjoint
// sweep, assembly, result download) recorded once as a CUDA graph and replayed for every
// later evaluation with new velocities and/or observations, as a Hamiltonian Monte Carlo
// chain or a line search does (HMCtraveltimes.jl:84-104 calls eikgradient model after model
// with the same sources and receivers).
//
// What makes the pipeline replayable:
// * it has no host round trip between its stages: the refined start-up's tie flags stay on
//   the device, and the round widths, which depend on the model's smallest slowness, are
//   computed on the device from the slowness statistics that the graph itself recomputes
//   after uploading the velocity;
// * every host array it uploads (problem descriptors, smoothing weights) is staged, while
//   capturing, in pinned memory that the plan owns, and the per-evaluation inputs and
//   outputs go through pinned buffers of the plan;
// * the plan owns its device buffers (its own scratch, set aside from the context's HBM
//   budget), so no later call on the context can move memory that the graph addresses;
// * the model stays put: a plan holds its model (eik_model_release refuses while plans
//   exist) and a replay with a new velocity overwrites that model in place.
// The graph is captured after one ordinary run of the same pipeline has allocated every
// buffer; a replay computes what that run computes, so its results are bit-identical to an
// eik_gradient call on the same inputs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/eikcuda.h"
#include "runtime.hpp"

using namespace eik;

struct eik_plan {
  eik_ctx* ctx = nullptr;
  eik_model_id model = 0;
  int64_t nsrc = 0;
  int nd = 0;
  long long N = 0, nrec = 0;
  int32_t whichgrad = 1;
  Scratch scratch;                 // the plan's device buffers
  std::vector<void*> arena;        // pinned copies of the host arrays the graph uploads
  double *h_vel = nullptr, *h_po = nullptr, *h_so = nullptr;  // pinned per-replay inputs
  double *h_gv = nullptr, *h_gs = nullptr, *h_m = nullptr;    // pinned per-replay outputs
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  GradTail tail;
  size_t reserved = 0;             // HBM set aside from the context's budget
};

namespace {

void free_plan(eik_plan* p) {
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  p->scratch.release_all();
  for (void* a : p->arena) cudaFreeHost(a);
  for (double* h : {p->h_vel, p->h_po, p->h_so, p->h_gv, p->h_gs, p->h_m})
    if (h) cudaFreeHost(h);
  delete p;
}

struct PlanBuffers {
  double *cs, *rec, *po, *so, *gv, *gs, *m;
  long long* off;
};

// One evaluation on the device, from the pinned inputs to the pinned outputs.
int plan_body(eik_ctx* ctx, eik_plan* p, const Model& m, const PlanBuffers& b, const eik_extra& ep) {
  cudaStream_t st = ctx->stream;
  const bool wantvel = p->whichgrad != 2, wantsrc = p->whichgrad != 1;
  CUDA_OK(ctx, cudaMemcpyAsync(m.vel, p->h_vel, sizeof(double) * p->N, cudaMemcpyHostToDevice, st));
  model_refresh(m, st);
  if (p->nrec) {
    CUDA_OK(ctx, cudaMemcpyAsync(b.po, p->h_po, sizeof(double) * p->nrec, cudaMemcpyHostToDevice, st));
    CUDA_OK(ctx, cudaMemcpyAsync(b.so, p->h_so, sizeof(double) * p->nrec, cudaMemcpyHostToDevice, st));
  }
  int rc = gradient_core(ctx, m, p->nsrc, b.cs, b.off, b.rec, b.po, b.so, p->whichgrad, ep, wantvel ? b.gv : nullptr,
                         wantsrc ? b.gs : nullptr, b.m, nullptr, &p->tail);
  if (rc) return rc;
  CUDA_OK(ctx, cudaMemcpyAsync(p->h_m, b.m, sizeof(double), cudaMemcpyDeviceToHost, st));
  if (wantvel) CUDA_OK(ctx, cudaMemcpyAsync(p->h_gv, b.gv, sizeof(double) * p->N, cudaMemcpyDeviceToHost, st));
  if (wantsrc)
    CUDA_OK(ctx, cudaMemcpyAsync(p->h_gs, b.gs, sizeof(double) * p->nsrc * p->nd, cudaMemcpyDeviceToHost, st));
  return EIK_OK;
}

}  // namespace

extern "C" int eik_plan_gradient(eik_ctx* ctx, eik_model_id model, int64_t nsrc, const double* coordsrc,
                                 const int64_t* rec_off, const double* rec, int32_t whichgrad,
                                 const eik_extra* ep_in, eik_plan** out) {
  if (!ctx) return fail(ctx, EIK_ERR_ASSERT, "NULL context");
  if (!out || !coordsrc || !rec_off || !rec) return fail(ctx, EIK_ERR_ASSERT, "NULL argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lk(ctx->mu);
  auto it = ctx->models.find(model);
  if (it == ctx->models.end()) return fail(ctx, EIK_ERR_ASSERT, "unknown model id %lld", (long long)model);
  Model& m = it->second;
  eik_extra ep;
  if (ep_in) ep = *ep_in;
  else eik_extra_defaults(&ep);
  int rc = validate_gradient(ctx, m, nsrc, whichgrad, ep);
  if (rc) return rc;
  rc = check_positions(ctx, m.g, nsrc, coordsrc, rec_off, rec);
  if (rc) return rc;
  CUDA_OK(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  CUDA_OK(ctx, cudaStreamSynchronize(st));
  eik_plan* p = new eik_plan();
  p->ctx = ctx;
  p->model = model;
  p->nsrc = nsrc;
  p->nd = m.g.nd;
  p->N = m.N;
  p->nrec = rec_off[nsrc];
  p->whichgrad = whichgrad;
  const size_t used = ctx->scratch.total + ctx->model_bytes;
  p->scratch.budget = ctx->scratch.budget > used ? ctx->scratch.budget - used : 0;
  const size_t nrec1 = (size_t)std::max<long long>(p->nrec, 1);
  bool ok = cudaMallocHost(&p->h_vel, sizeof(double) * p->N) == cudaSuccess &&
            cudaMallocHost(&p->h_po, sizeof(double) * nrec1) == cudaSuccess &&
            cudaMallocHost(&p->h_so, sizeof(double) * nrec1) == cudaSuccess &&
            cudaMallocHost(&p->h_gv, sizeof(double) * p->N) == cudaSuccess &&
            cudaMallocHost(&p->h_gs, sizeof(double) * nsrc * p->nd) == cudaSuccess &&
            cudaMallocHost(&p->h_m, sizeof(double)) == cudaSuccess;
  if (!ok) {
    free_plan(p);
    return fail(ctx, EIK_ERR_CUDA, "cudaMallocHost of a plan's staging buffers failed");
  }
  // replays without a new velocity upload the model's current one
  if (cudaMemcpy(p->h_vel, m.vel, sizeof(double) * p->N, cudaMemcpyDeviceToHost) != cudaSuccess) {
    free_plan(p);
    return fail(ctx, EIK_ERR_CUDA, "reading the model's velocity failed");
  }
  for (size_t r = 0; r < nrec1; r++) {
    p->h_po[r] = 0.0;
    p->h_so[r] = 1.0;
  }
  // everything below allocates from the plan's own scratch
  std::swap(ctx->scratch, p->scratch);
  PlanBuffers b;
  auto get = [&](const char* name, size_t bytes) { return ctx->scratch.get(name, bytes, &rc); };
  b.cs = (double*)get("plan_cs", sizeof(double) * nsrc * p->nd);
  b.off = (long long*)get("plan_off", sizeof(long long) * (nsrc + 1));
  b.rec = (double*)get("plan_rec", sizeof(double) * nrec1 * p->nd);
  b.po = (double*)get("plan_pickobs", sizeof(double) * nrec1);
  b.so = (double*)get("plan_stdobs", sizeof(double) * nrec1);
  b.gv = (double*)get("plan_gradvel", sizeof(double) * p->N);
  b.gs = (double*)get("plan_gradsrc", sizeof(double) * nsrc * p->nd);
  b.m = (double*)get("plan_misfit", sizeof(double));
  auto give_back = [&](int code) {
    cudaStreamSynchronize(st);  // nothing queued may still use the plan's buffers
    std::swap(ctx->scratch, p->scratch);
    ctx->capturing = false;
    ctx->stage_arena = nullptr;
    free_plan(p);
    return code;
  };
  if (!b.cs || !b.off || !b.rec || !b.po || !b.so || !b.gv || !b.gs || !b.m)
    return give_back(fail(ctx, rc ? rc : EIK_ERR_CUDA, "plan buffers exceed the HBM budget"));
  // sources and receivers are fixed for the plan: uploaded once, outside the graph
  if (cudaMemcpyAsync(b.cs, coordsrc, sizeof(double) * nsrc * p->nd, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(b.off, rec_off, sizeof(long long) * (nsrc + 1), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      (p->nrec && cudaMemcpyAsync(b.rec, rec, sizeof(double) * p->nrec * p->nd, cudaMemcpyHostToDevice, st) !=
                      cudaSuccess))
    return give_back(fail(ctx, EIK_ERR_CUDA, "upload of the plan's sources and receivers failed"));
  // 1) an ordinary run allocates every buffer the pipeline uses and checks that it runs
  rc = plan_body(ctx, p, m, b, ep);
  if (rc) return give_back(rc);
  if (cudaStreamSynchronize(st) != cudaSuccess) return give_back(fail(ctx, EIK_ERR_CUDA, "plan dry run failed"));
  rc = gradient_tail_stats(ctx, p->tail, nullptr);
  if (rc) return give_back(rc);
  // 2) the same pipeline, captured
  ctx->capturing = true;
  ctx->stage_arena = &p->arena;
  cudaError_t ce = cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed);
  if (ce != cudaSuccess) return give_back(fail(ctx, EIK_ERR_CUDA, "cudaStreamBeginCapture: %s", cudaGetErrorString(ce)));
  rc = plan_body(ctx, p, m, b, ep);
  cudaGraph_t graph = nullptr;
  ce = cudaStreamEndCapture(st, &graph);
  p->graph = graph;
  ctx->capturing = false;
  ctx->stage_arena = nullptr;
  if (rc) return give_back(rc);
  if (ce != cudaSuccess || !graph)
    return give_back(fail(ctx, EIK_ERR_CUDA, "stream capture of the pipeline failed: %s", cudaGetErrorString(ce)));
  ce = cudaGraphInstantiate(&p->exec, graph, 0);
  if (ce != cudaSuccess)
    return give_back(fail(ctx, EIK_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(ce)));
  std::swap(ctx->scratch, p->scratch);
  // the plan's device memory leaves the context's budget until the plan is destroyed
  p->reserved = p->scratch.total;
  ctx->scratch.budget = ctx->scratch.budget > p->reserved ? ctx->scratch.budget - p->reserved : 0;
  m.plans++;
  ctx->live_plans++;
  *out = p;
  return EIK_OK;
}

extern "C" int eik_plan_run(eik_plan* p, const double* vel, const double* pickobs, const double* stdobs,
                            double* gradvel, double* gradsrc, double* misfit, eik_stats* stats) {
  if (!p) return fail(nullptr, EIK_ERR_ASSERT, "NULL plan");
  eik_ctx* ctx = p->ctx;
  if (p->nrec && (!pickobs || !stdobs)) return fail(ctx, EIK_ERR_ASSERT, "NULL argument");
  std::lock_guard<std::mutex> lk(ctx->mu);
  NvtxRange nvtx_call("eik_plan_run");
  auto it = ctx->models.find(p->model);
  if (it == ctx->models.end()) return fail(ctx, EIK_ERR_ASSERT, "the plan's model is gone");
  Model& m = it->second;
  if (stats) std::memset(stats, 0, sizeof *stats);
  if (vel) {
    for (long long i = 0; i < p->N; i++)
      if (!(vel[i] > 0.0)) return fail(ctx, EIK_ERR_ASSERT, "all(vel.>0.0)");
    std::memcpy(p->h_vel, vel, sizeof(double) * p->N);
  }
  if (p->nrec) {
    std::memcpy(p->h_po, pickobs, sizeof(double) * p->nrec);
    std::memcpy(p->h_so, stdobs, sizeof(double) * p->nrec);
  }
  CUDA_OK(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  cudaEventRecord(ctx->ev0, st);
  CUDA_OK(ctx, cudaGraphLaunch(p->exec, st));
  cudaEventRecord(ctx->ev1, st);
  CUDA_OK(ctx, cudaStreamSynchronize(st));
  const int rc = gradient_tail_stats(ctx, p->tail, stats);
  CUDA_OK(ctx, cudaMemcpy(&m.smin, m.dstat + 2, sizeof(double), cudaMemcpyDeviceToHost));
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    stats->device_ms = ms;
    stats->launches += p->tail.fw.launches;  // the forward's kernels (the adjoint's are counted above)
  }
  if (rc) return rc;
  if (misfit) *misfit = *p->h_m;
  if (gradvel && p->whichgrad != 2) std::memcpy(gradvel, p->h_gv, sizeof(double) * p->N);
  if (gradsrc && p->whichgrad != 1) std::memcpy(gradsrc, p->h_gs, sizeof(double) * p->nsrc * p->nd);
  return EIK_OK;
}

extern "C" int eik_plan_destroy(eik_plan* p) {
  if (!p) return EIK_OK;
  eik_ctx* ctx = p->ctx;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  auto it = ctx->models.find(p->model);
  if (it != ctx->models.end()) it->second.plans--;
  ctx->live_plans--;
  ctx->scratch.budget += p->reserved;
  free_plan(p);
  return EIK_OK;
}
