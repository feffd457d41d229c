// Oracle: CPU restatement of EikonalSolvers.jl 0.15.3's forward (2nd-order FMM)
// and discrete-adjoint path. TEST INFRASTRUCTURE ONLY: the GPU library never
// links or calls this code; tests, smoke() and bench.py's cpu_baseline leg use
// it as the checker and as the timed CPU baseline.
//
// Every function cites the reference file:line it follows (paths relative to
// the EikonalSolvers.jl project root). Julia semantics that decide bitwise
// results are mirrored explicitly: x^2 == x*x, no FMA contraction (build with
// -ffp-contract=off), left-to-right evaluation, `rem` == fmod, ranges built
// like Base.range(start=..., step=..., length=...).
#pragma once
#include <cstdint>
#include <cstddef>
#include <vector>
#include <string>
#include <stdexcept>
#include <array>

namespace eikor {

using i64 = int64_t;

// ---------------------------------------------------------------- errors --
// AssertionError / ErrorException of the reference become OracleError.
struct OracleError : std::runtime_error {
  int code;  // 1 = assertion (AssertionError), 2 = error() call (ErrorException)
  OracleError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
[[noreturn]] void jl_assert_fail(const std::string& what);
[[noreturn]] void jl_error(const std::string& what);
#define EIKOR_ASSERT(cond, msg) do { if (!(cond)) ::eikor::jl_assert_fail(msg); } while (0)

// Warning bits mirroring the reference's @warn sites.
enum WarnBits : uint32_t {
  WARN_NEG_DISCRIMINANT = 1u << 0,   // eikforward2D.jl:342, eikforward3D.jl:429
  WARN_SRC_HALFWAY_SHIFT = 1u << 1,  // eikmainfwd.jl:1298
  WARN_BORDER_BEFORE_COARSE = 1u << 2,  // eikmainfwd.jl:731
  WARN_SRCPOS_ALIGNED_SHIFT = 1u << 3,  // eikmaingrad.jl:1250
  WARN_SRC_ON_NODE_DERIV = 1u << 4,     // eikmaingrad.jl:1260
  WARN_FINE_NO_TRIGGER = 1u << 5,       // fine FMM exhausted the heap without a stop
};

// ------------------------------------------------------- Julia numerics --
// Base.range(start=a, step=st, length=n)[i] for Float64 (twiceprecision.jl):
// rational start/step are evaluated as the correctly rounded (n0 + (i-1)*ns)/den.
struct JRange {
  double a = 0, st = 0;
  i64 len = 0;
  bool rational = false;
  i64 start_n = 0, step_n = 0, den = 1;
  void init(double a_, double st_, i64 len_);
  double operator()(i64 i1) const;  // 1-based
  double last() const { return (*this)(len); }
};

double jl_rem(double x, double y);   // Base.rem for Float64 == C fmod
double jl_mod(double x, double y);   // Base.mod for Float64
double jl_div(double x, double y);   // Base.div(x,y) (RoundToZero) for Float64
bool isapprox_default(double x, double y);  // x ≈ y, rtol = sqrt(eps)
double deg2rad(double x);
double cosd(double x);
double sind(double x);

// ----------------------------------------------------------------- grids --
// eikstructs.jl:33-219. kind: 0 Grid2DCart, 1 Grid3DCart, 2 Grid2DSphere, 3 Grid3DSphere.
enum GridKind { G2DCART = 0, G3DCART = 1, G2DSPH = 2, G3DSPH = 3 };
struct Grid {
  int kind = 0;
  int nd = 2;
  i64 n[3] = {1, 1, 1};
  double spac[3] = {0, 0, 0};   // hgrid (all axes) or (Δr, Δθ[, Δφ]) in degrees
  double cooinit[3] = {0, 0, 0};
  JRange ax[3];                  // x,y,z or r,θ,φ node coordinates
  bool cart() const { return kind == G2DCART || kind == G3DCART; }
  bool sph() const { return !cart(); }
  i64 npts() const { return n[0] * n[1] * n[2]; }
  double hgrid() const { return spac[0]; }
  // column-major linear index of 1-based (i,j,k) -- eikutils.jl:6-19
  i64 lin(const i64* ijk) const {
    return (ijk[0] - 1) + n[0] * ((ijk[1] - 1) + n[1] * (nd == 3 ? (ijk[2] - 1) : 0));
  }
  void cart_of(i64 l, i64* ijk) const {  // eikutils.jl:24-43, 1-based output
    ijk[0] = l % n[0] + 1;
    i64 r = l / n[0];
    ijk[1] = r % n[1] + 1;
    ijk[2] = (nd == 3) ? r / n[1] + 1 : 1;
  }
};
Grid make_grid(int kind, const i64* grsize, const double* spacing, const double* cooinit);

struct ExtraParams {  // eikstructs.jl:246-282
  bool refinearoundsrc = true;
  int parallelkind = 0;  // 0 serial, 1 sharedmem, 2 distribmem (2 not supported for gradients)
  i64 radiussmoothgradsrc = 3;
  i64 smoothgradkern = 0;
  i64 downscalefactor = 5;
  i64 noderadius = 3;
  int nthreads = 1;       // threads used for :sharedmem (Threads.nthreads())
};

// --------------------------------------------------------------- binheap --
// BinHeaps.jl:56-62, 313-485: min-heap with handle -> position map.
struct BinHeapMin {
  i64 Nmax = 0, Nh = 0;
  std::vector<double> nodes;   // 1-based storage (index 0 unused)
  std::vector<i64> handles;
  std::vector<int32_t> idxhan; // indexed by handle (0-based linear node + 1)
  void init(i64 nmax);
  void swap_nodes(i64 p, i64 q);
  void min_heapify(i64 i);
  void insert(double val, i64 handle);
  void update(double val, i64 handle);
  void pop(i64& handle, double& val);
  double topval() const { return nodes[1]; }
};

// ---------------------------------------------------- CSR derivative mats --
struct CSR {  // eikstructs.jl:305-324 (VecSPDerivMat)
  i64 nrows = 0, ncols = 0;
  std::vector<i64> iptr;   // size nrows+1, 0-based offsets
  std::vector<int32_t> j;  // 0-based column (FMM position)
  std::vector<double> v;
};

// --------------------------------------------------------------- FMM vars --
struct FMMVars {  // eikstructs.jl:430-488
  Grid grd;
  std::vector<double> ttime;
  std::vector<uint8_t> status;
  BinHeapMin bheap;
  bool refinearoundsrc = false;
  // source points (1-based ijk, one row per point): SourceBoxParams / SourcePtsFromFineGrid
  std::vector<std::array<i64, 3>> ijksrc;
  std::vector<double> velcorn, distcorn;
  double xyzsrc[3] = {0, 0, 0};
  bool is_srcbox = true;  // false: points came from a fine grid
};

struct AdjointVars {  // eikstructs.jl:381-406, 328-358, 286-300
  Grid grd;
  std::vector<int32_t> lfmm2grid;  // FMM position -> linear node + 1 (0 = unset)
  std::vector<int32_t> lgrid2fmm;  // linear node -> FMM position + 1
  std::vector<double> fmmtt;       // traveltime in FMM order (-1 = unset)
  std::vector<uint8_t> onsrccols, onhpoints;
  std::vector<int8_t> code;        // N x nd, row-major by node
  i64 lastcomputedtt = 0;
  i64 nsize0[3], nsize1[3];        // Deriv[d].Nsize
  CSR D[3];
  void init(const Grid& g);
  void reset_for_run();
};

struct SrcRefinVars {  // eikstructs.jl:492-500
  i64 downscalefactor = 5;
  i64 ijkorigincoarse[3] = {1, 1, 1};
  bool outijk_min[3] = {false, false, false};
  bool outijk_max[3] = {false, false, false};
  std::vector<i64> nearneigh_idxcoarse;  // fine linear -> coarse-window column (1-based)
  i64 window_n[3] = {1, 1, 1};
  std::vector<double> velcart_fine;
  Grid grd_fine;
};

// Per-run counters used by tests and by the GPU-parity analysis.
struct FMMStats {
  std::vector<int32_t>* batch_of = nullptr;  // optional: batch index per coarse node (0 = source)
  i64 pops = 0;
  i64 nonmonotone_pops = 0;  // popped value smaller than an earlier popped value
  i64 max_batch = 0;
  uint32_t warn = 0;
};

// ----------------------------------------------------------- forward API --
double calcttpt_2ndord(const FMMVars& fv, const double* vel, const i64* ijk, int8_t* codeD,
                       uint32_t* warn);
void sourceboxloctt(FMMVars& fv, const double* vel, const double* srcpos, uint32_t* warn);
void findenclosingbox(const Grid& g, const double* xyzsrc, std::vector<std::array<i64, 3>>& out);
double distance2points(const Grid& g, const double* a, const double* b);
void createfinegrid(const Grid& g, const double* xyzsrc, const double* vel, i64 ds, i64 noderadius,
                    SrcRefinVars& srv);
void ttFMM_core(FMMVars& fv, const double* vel, AdjointVars* adj, FMMVars* coarse,
                AdjointVars* adjcoarse, SrcRefinVars* srv, FMMStats* st);
// Runs one source (eikmainfwd.jl:230-326). When adj != nullptr and refinement is on, the
// fine-grid state is returned through the *_fine outputs.
void ttFMM_hiord(FMMVars& fv, const double* vel, const double* src, AdjointVars* adj,
                 const ExtraParams& ep, FMMVars* fine_out, AdjointVars* adjfine_out,
                 SrcRefinVars* srv_out, FMMStats* st);
double interpolate_receiver(const std::vector<double>& tt, const Grid& g, const double* pt);
void interp_coeffs(const Grid& g, const double* pt, double* coeff, i64 (*ijk)[3], int* ncoe);
void createsparsederivativematrices(const Grid& g, AdjointVars& adj, const std::vector<uint8_t>& status);

// ----------------------------------------------------------- top-level API --
void checksrcrecposition(const Grid& g, i64 nsrc, const double* coordsrc, const i64* recoff,
                         const double* rec);
void eiktraveltime(const Grid& g, const double* vel, i64 nsrc, const double* coordsrc,
                   const i64* recoff, const double* rec, const ExtraParams& ep, double* picks,
                   double* ttgrids, uint32_t* warn);
void eikgradient(const Grid& g, const double* vel, i64 nsrc, const double* coordsrc,
                 const i64* recoff, const double* rec, const double* pickobs, const double* stdobs,
                 int whichgrad, const ExtraParams& ep, double* gradvel, double* gradsrc,
                 double* misfit, uint32_t* warn);
void smoothgradaroundsrc(std::vector<double>& grad, const double* xyzsrc, const Grid& g, i64 radiuspx);
void smoothgradient(i64 l, const Grid& g, std::vector<double>& grad);

// tracerays (eikutils.jl:201-328), oracle/rays.cpp. npts per receiver (recoff order),
// points concatenated row-major.
void tracerays(const Grid& g, const double* ttgrids, i64 nsrc, const double* coordsrc, const i64* recoff,
               const double* rec, double steplen, i64 max_steps, std::vector<i64>& npts, std::vector<double>& pts);

}  // namespace eikor
