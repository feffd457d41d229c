// Host-side state of libeikcuda contexts (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/eikcuda.h"
#include "kernels.cuh"

#define CUDA_OK(ctx, call)                                                                      \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      return eik::fail(ctx, EIK_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));      \
  } while (0)

namespace eik {

// Grow-only named device buffers, bounded by the context's HBM budget.
struct Scratch {
  struct Buf {
    void* ptr;
    size_t bytes;
  };
  std::map<std::string, Buf> bufs;
  size_t total = 0;
  size_t budget = 0;
  void* get(const std::string& name, size_t bytes, int* rc);
  void release_all();
};

struct Model {
  GridDesc g;
  long long N = 0;
  double* vel = nullptr;   // device
  double* slow = nullptr;  // device, 1.0/vel
  double smin = 0.0;       // smallest slowness of the model (round width of the forward solve)
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
  std::vector<SrcOut> host_out;
};

int fail(eik_ctx* ctx, int code, const char* fmt, ...);
int make_griddesc(eik_ctx* ctx, const eik_grid* g, GridDesc* out);
int forward_device(eik_ctx* ctx, const Model& m, int64_t nsrc, const double* d_cs, const eik_extra& ep,
                   ForwardState* fw, eik_stats* stats);
int collect_forward_stats(eik_ctx* ctx, ForwardState* fw, eik_stats* stats);
int check_positions(eik_ctx* ctx, const GridDesc& g, int64_t nsrc, const double* cs, const int64_t* recoff,
                    const double* rec);
int check_extra(eik_ctx* ctx, const eik_extra* ep);
int err_to_rc(eik_ctx* ctx, uint32_t e);

}  // namespace eik

struct eik_ctx {
  int device = 0;
  int nsm = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // whole call
  cudaEvent_t evk[6] = {};                    // start-up stage, coarse solve, adjoint solve
  double round_gate = 2.0;  // forward round width in units of (smallest spacing x smallest slowness)
  double sm_fraction = 1.0; // share of the SMs the persistent (cooperative) solves of this context use
  bool fine_replay = false; // refined start-up by exact heap replay for every source (else only on ties)
  int solve_sms() const {
    const int n = (int)(sm_fraction * (double)nsm + 0.5);
    return n < 1 ? 1 : (n > nsm ? nsm : n);
  }
  std::mutex mu;
  eik::Scratch scratch;
  size_t model_bytes = 0;
  eik_model_id next_model = 0;
  std::map<eik_model_id, eik::Model> models;
};
