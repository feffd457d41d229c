// Device-side interfaces between the kernels of libeikcuda and its host runtime.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "common.cuh"

namespace eik {

// Refined-grid window of one source (createfinegrid, eikmainfwd.jl:950-1104), 0-based.
struct FineInfo {
  int32_t ds;
  int32_t ijk1[3];    // coarse index of the window origin
  int32_t nf[3];      // fine grid size
  int32_t outmin[3];  // window clipped at the model's lower border on this axis
  int32_t outmax[3];
};

// Per-source results of the start-up stage.
struct SrcOut {
  FineInfo fine;
  int32_t nseeds;       // coarse source points (traveltimes fixed before the coarse solve)
  int32_t nsrcf;        // source-box corners (of the fine grid if refined, else coarse)
  int32_t nacc;         // accepted fine nodes at the stop (refined only)
  uint32_t warn;
  int32_t corn[8][3];   // source-box corners
  double distcorn[8];
  double velcorn[8];
};

struct ForwardBatch {
  GridDesc g;               // coarse grid
  int32_t nsrc;
  int32_t ds, noderadius;
  int32_t seedcap;          // capacity of seed lists per source
  long long nfmax;          // capacity of fine arrays per source
  int32_t heapcap;          // shared-memory heap capacity (fine FMM)
  const double* vel;        // coarse velocity
  const double* slow;       // 1/vel
  const double* coordsrc;   // nsrc x nd
  SrcOut* out;
  int32_t* seed_lin;        // nsrc x seedcap: coarse node index
  double* seed_tt;          // nsrc x seedcap
  double* fine_tt;          // nsrc x nfmax
  uint8_t* fine_status;
  uint8_t* fine_code;
  int32_t* fine_idx;        // heap handle positions
  int32_t* fine_order;      // accepted fine nodes in FMM order
  uint8_t* fine_onh;        // accepted fine node coincides with a coarse node
  uint32_t* err;
};

// One coarse solve: a source on a grid. Several problems share one persistent launch.
struct CoarseProblem {
  GridDesc g;
  const double* slow;
  double* t;       // traveltime
  uint8_t* code;   // packed derivative codes; bit 7: special key (source or non-causal)
  double* kL;      // key level of special nodes (-inf for source points)
  uint8_t* kd;     // key depth of special nodes
  double delta;    // round width of the forward solve (traveltime units)
  double incmin;   // smallest increment of the local update over a neighbour: (2/3) h s_min / sqrt(nd)
  double c1u, c2u; // Cartesian grids: the local solver's coefficients 1/h^2 and 9/(4h^2); 0 otherwise
};

// The coefficients of a grid with the same spacing h on every axis, computed with the
// local solver's own expressions (so they are the values it would compute per call).
EIK_HD void uniform_coeffs(const GridDesc& g, double* c1u, double* c2u) {
  if (is_cart(g)) {
    const double h = g.spac[0];
    *c1u = 1.0 / (h * h);
    *c2u = 9.0 / (4.0 * (h * h));
  } else {
    *c1u = *c2u = 0.0;
  }
}

// Worklists and thresholds of the round-synchronous forward solve. Nodes are numbered
// globally over the problems of a call: problem * N + node.
struct RoundState {
  int32_t* stamp;               // per node: last round it was listed for
  double* tent;                 // per node: value of its last evaluation
  uint8_t* dirty;               // per node: something it reads changed since that evaluation
  unsigned long long* list[2];  // entries of the current and the next round (node id << 32 | front)
  unsigned int* cnt;            // [3] list length per round (mod 3)
  unsigned int* grab;           // [3] next list entry to take per round (mod 3)
  unsigned long long* nextmin;  // [3][nprob] smallest pending potential (double bits)
  double* thr;                  // [2][nprob] threshold of the previous / current round
  unsigned int* bar;            // [2] grid barrier: arrivals, generation
  unsigned long long stride;    // node ids: problem * stride + node
  int32_t* rounds;              // rounds run
  unsigned long long* visits;   // [7] outcomes of the forward's list visits
  int32_t max_rounds;
};

struct SolveArgs {
  const CoarseProblem* probs;
  int32_t nprob;
  int32_t nd;
  unsigned long long* activations;  // list entries visited
  unsigned long long max_activations;
  unsigned long long* node_evals;
  uint32_t* err;
  int32_t* abort_flag;
  long long timeout_ns;
  RoundState rs;
};


// launchers (defined in the .cu files)
void launch_srcbox(const ForwardBatch& fb, cudaStream_t st);
void launch_fine(const ForwardBatch& fb, cudaStream_t st);
size_t fine_smem_bytes(int heapcap);
void launch_coarse_init(const CoarseProblem* hprobs, const CoarseProblem* dprobs, int nprob,
                        const ForwardBatch& fb, const SolveArgs& sa, cudaStream_t st);
// Round-solver state reset, and seeding from per-problem seed lists (fixed values).
void launch_rounds_init(const SolveArgs& sa, cudaStream_t st);
void launch_rounds_seed(const SolveArgs& sa, const int32_t* seed_lin, const double* seed_tt, const SrcOut* out,
                        bool fine_corners, int seedcap, cudaStream_t st);
// Refined start-up as a fixed point: window set-up, the fine problems' arrays, the
// acceptance set at the reference's stop, and the exact heap replay for the sources
// whose stop is decided by a tie (flags in fine_tie, nonzero = replay needed).
void launch_fine_setup(const ForwardBatch& fb, CoarseProblem* fprobs, const double* dsmin, double gate,
                       int32_t* fseed_lin, double* fseed_tt, double* fine_slow, double* fine_kL, uint8_t* fine_kd,
                       cudaStream_t st);
void launch_fine_select(const ForwardBatch& fb, const CoarseProblem* fprobs, uint8_t* fine_tie, cudaStream_t st);
void launch_fine_replay(const ForwardBatch& fb, const uint8_t* fine_tie, cudaStream_t st);
// ctas_per_sm: resident CTAs per SM of the persistent launch (0 = as many as fit);
// queue: per-warp evaluation queue 1 = on, 0 = off, -1 = chosen by the launch's size
cudaError_t launch_coarse_solve(const SolveArgs& sa, int nsm, int ctas_per_sm, int queue, cudaStream_t st);
// The forward solve of small problems (every problem at most nmax nodes), one thread-block
// cluster per problem with its state in distributed shared memory, seeds and counters
// included (it replaces round init, seeding and launch_coarse_solve). *used = false when no
// cluster of this GPU holds such a problem (nothing launched: use the global solve).
cudaError_t launch_cluster_solve(const SolveArgs& sa, long long nmax, const int32_t* seed_lin, const double* seed_tt,
                                 const SrcOut* out, bool fine_corners, int seedcap, cudaStream_t st, bool* used);
bool cluster_solve_fits(const SolveArgs& sa, long long nmax);
void launch_picks(const GridDesc& g, const double* t, long long N, int nsrc, const long long* recoff,
                  const double* rec, double* picks, cudaStream_t st);
// Gaussian smoothing of a gradient field (smoothgradkern = l, odd): weights on the host,
// then one launch from in to out (distinct buffers); d_w holds gaussian_weights(l, nd).
std::vector<double> gaussian_weights(int l, int dim);
cudaError_t launch_smoothgrad(const GridDesc& g, int l, const double* d_w, const double* in, double* out,
                              cudaStream_t st);

}  // namespace eik
