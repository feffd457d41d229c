// Host-side state of libeikcuda contexts (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/eikcuda.h"
#include "kernels.cuh"
#include <nvtx3/nvToolsExt.h>

#define CUDA_OK(ctx, call)                                                                      \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      return eik::fail(ctx, EIK_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));      \
  } while (0)

namespace eik {

// Grow-only named device buffers, bounded by the context's HBM budget.
// Named device buffers kept from call to call (grown on demand) under an HBM budget. A
// call that would exceed the budget, or whose cudaMalloc fails, first frees the buffers no
// part of the current call has taken (begin_call starts a call), then tries once more.
// A named NVTX range over a scope (header-only NVTX 3: a no-op unless a profiler is
// attached). Entry points open one for their whole call, which ends after the device work.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

struct Scratch {
  struct Buf {
    void* ptr;
    size_t bytes;
    unsigned used;  // epoch of the last call that took it
  };
  std::map<std::string, Buf> bufs;
  size_t total = 0;
  size_t budget = 0;
  unsigned epoch = 1;
  void begin_call() { epoch++; }
  void* get(const std::string& name, size_t bytes, int* rc);
  void release_all();
  void release_unused();
};

struct Model {
  GridDesc g;
  long long N = 0;
  double* vel = nullptr;   // device
  double* slow = nullptr;  // device, 1.0/vel
  double smin = 0.0;       // smallest slowness of the model (round width of the forward solve)
  double* dstat = nullptr; // device: [non-positive flag, Σ slowness, smallest slowness]
  int plans = 0;           // captured plans that hold this model's buffers
};

// Device results of the forward stage of one call.
struct ForwardState {
  ForwardBatch fb;
  SolveArgs sa;
  double* t = nullptr;
  uint8_t* code = nullptr;
  double* kL = nullptr;
  uint8_t* kd = nullptr;
  long long N = 0;
  long long nsrc = 0;
  const uint8_t* fine_tie = nullptr;  // per-source replay flags of the refined start-up (device)
  int launches = 0;                   // kernels the forward stage launched
  double gate = 2.0;                  // round width used (units of smallest spacing x slowness)
  int sms = 1;                        // SMs of the persistent solves of this call
  std::vector<SrcOut> host_out;
};

int fail(eik_ctx* ctx, int code, const char* fmt, ...);
int make_griddesc(eik_ctx* ctx, const eik_grid* g, GridDesc* out);
int forward_device(eik_ctx* ctx, const Model& m, int64_t nsrc, const double* d_cs, const eik_extra& ep,
                   ForwardState* fw, eik_stats* stats);
// The forward of the sources of several models of one dimension (model i: sources
// src_off[i]..src_off[i+1]) in one pipeline; fw->N is then the largest grid's node count,
// the stride of the per-source arrays.
int forward_multi(eik_ctx* ctx, int nmod, const Model* const* models, const int64_t* src_off, const double* d_cs,
                  const eik_extra& ep, ForwardState* fw, eik_stats* stats);
int collect_forward_stats(eik_ctx* ctx, ForwardState* fw, eik_stats* stats);
int check_positions(eik_ctx* ctx, const GridDesc& g, int64_t nsrc, const double* cs, const int64_t* recoff,
                    const double* rec);
int check_extra(eik_ctx* ctx, const eik_extra* ep);
int err_to_rc(eik_ctx* ctx, uint32_t e);
// Recomputes a model's slowness and its device statistics from its velocity (stream-ordered,
// no host synchronisation, so it can be part of a captured graph).
void model_refresh(const Model& m, cudaStream_t st);
// Source of a host-to-device copy of `bytes` at `src` inside the pipeline: `src` itself, or,
// while a plan is being captured, a pinned copy owned by the plan (a graph replays its
// copies from the same host address, so that address must outlive the call).
const void* stage_host(eik_ctx* ctx, const void* src, size_t bytes);

// What is left to read back after a gradient pipeline has run: the forward's device state
// and the adjoint's warning word and round counter.
struct GradTail {
  ForwardState fw;
  uint32_t* dwarn = nullptr;
  int32_t* arounds = nullptr;
  int launches = 0;
};
int gradient_tail_stats(eik_ctx* ctx, GradTail& tail, eik_stats* stats);
int validate_gradient(eik_ctx* ctx, const Model& m, int64_t nsrc, int32_t whichgrad, const eik_extra& ep);
// Forward + adjoint + assembly for nsrc sources whose inputs are on the device; outputs
// (each nullable) stay on the device. tail_out (nullable) receives what to read back.
// One chunk of the sources of a gradient call that is split to fit the HBM budget: its place
// in the call and the state handed from chunk to chunk (the ordered group sums of the field
// and of the misfit, and the group buffer as the previous chunk left it). The sum state
// arrays start at zero; first_group/gcur start at 1/0 and are advanced on the host.
struct GradChunk {
  int s0 = 0;            // index of the chunk's first source in the call
  int nsrc_total = 0;
  bool final_chunk = true;
  double* acc = nullptr;  // N: current group's partial sum of the field
  double* tot = nullptr;  // N: sum of the finished groups
  double* macc = nullptr; // misfit: current group / finished groups
  double* mtot = nullptr;
  double* prevbuf = nullptr;  // N: final field of the previous chunk's last source
  bool prev_valid = false;
  int first_group = 1;
  int gcur = 0;
};
// Device bytes one gradient call of nsrc sources takes from the context's scratch budget
// (the named buffers the forward and adjoint stages allocate), and the fixed part that does
// not grow with the sources.
void gradient_footprint(const Model& m, const eik_extra& ep, long long nrec, int32_t whichgrad,
                        size_t* per_source, size_t* fixed);
// Explicit source groups of one call (host offsets, ngroups + 1 values from 0 to nsrc):
// each group has its own gradient buffer, carry-over and outputs (gradient field, misfit),
// as a call of that group's sources alone.
struct GroupSpec {
  int64_t ngroups;
  const int64_t* off;
};
// Source groups of distribsrcs (eikutils.jl:171-190): first source of the group of s.
int host_group_start(int nsrc, int nw, int s);
int gradient_core(eik_ctx* ctx, const Model& m, int64_t nsrc, const double* d_cs, const long long* d_off,
                  const double* d_rec, const double* d_po, const double* d_so, int32_t whichgrad,
                  const eik_extra& ep, double* d_gradvel, double* d_gradsrc, double* d_misfit, eik_stats* stats,
                  GradTail* tail_out, GradChunk* chunk = nullptr, const GroupSpec* groups = nullptr);

}  // namespace eik

struct eik_ctx {
  int device = 0;
  int nsm = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // whole call
  cudaEvent_t evk[6] = {};                    // start-up stage, coarse solve, adjoint solve
  double round_gate = 0.0;  // forward round width in units of (smallest spacing x smallest slowness); 0 = by size
  int ctas_per_sm = 0;       // resident CTAs per SM of the forward solve (0 = as many as fit)
  int fwd_queue = -1;        // per-warp evaluation queue of the forward solve: -1 by size, 0 off, 1 on
  int cluster_solve = 1;     // small problems in one thread-block cluster each: 1 in 2D, 2 in any dimension, 0 never
  int max_rounds = 0;        // round limit of the persistent solves (0 = the library's, see forward_multi)
  int retry = 0;             // a pipeline run again after the automatic round limit: wider rounds, limit 2^24
  int auto_round_limit = 0;  // the automatic round limit of a first run (0 = by the grid's diameter)
  double sm_fraction = 0.0; // share of the SMs the persistent (cooperative) solves use; 0 = by size
  double ray_room = 3.0;     // room of a ray in its first tracing pass, in straight-line lengths
  bool fine_replay = false; // refined start-up by exact heap replay for every source (else only on ties)
  // Launch parameters of a call whose coarse solve has `work` node-sources: the values set
  // on the context, else chosen by size. Small calls are bound by their rounds (each closed
  // by a grid barrier over all resident CTAs), so they take wider rounds on fewer SMs.
  static constexpr unsigned long long SMALL_WORK = 1ull << 22;
  double gate_for(unsigned long long work) const {
    const double g = round_gate > 0.0 ? round_gate : (work < SMALL_WORK ? 8.0 : 2.0);
    return retry ? 1.5 * g : g;
  }
  int sms_for(unsigned long long work) const {
    const double f = sm_fraction > 0.0 ? sm_fraction : (work < SMALL_WORK ? 0.25 : 1.0);
    const int n = (int)(f * (double)nsm + 0.5);
    return n < 1 ? 1 : (n > nsm ? nsm : n);
  }
  std::mutex mu;
  eik::Scratch scratch;
  bool capturing = false;                    // the pipeline is being captured into a plan's graph
  std::vector<void*>* stage_arena = nullptr; // pinned host copies made while capturing
  int live_plans = 0;
  size_t model_bytes = 0;
  eik_model_id next_model = 0;
  std::map<eik_model_id, eik::Model> models;
};

namespace eik {
// Runs one pipeline (`call`, which returns an EIK_* code); when its forward solve stopped at
// the library's automatic round limit (no max_rounds set), runs it once more with wider
// rounds and the full limit. The solve's result is the fixed point of the order rule, the
// same under every schedule, so the second run gives what the first would have.
template <class F>
int run_with_retry(eik_ctx* ctx, eik_stats* stats, F call) {
  int rc = call();
  if (rc == EIK_ERR_NOT_CONVERGED && ctx->max_rounds == 0) {
    ctx->retry = 1;
    rc = call();
    ctx->retry = 0;
    if (stats) stats->retries += 1;
  }
  return rc;
}
}  // namespace eik
