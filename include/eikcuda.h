/*
 * libeikcuda: B200 (sm_100a) implementation of the forward and discrete-adjoint hot path
 * of EikonalSolvers.jl 0.15.3, behind a plain C ABI.
 *
 * The reference has no FFI of its own (it is pure Julia); the seam these entry points
 * replace is the per-source-group worker pair that all three `parallelkind` branches call:
 *   ttforwsomesrc   (src/EikSolv/eikmainfwd.jl:152-199)  -> eik_traveltime
 *   calcgradsomesrc (src/EikSolv/eikmaingrad.jl:174-258) -> eik_gradient
 * so that the public Julia API keeps its signatures:
 *   eiktraveltime  (src/EikSolv/eikmainfwd.jl:33-143)
 *   eikgradient    (src/EikSolv/eikmaingrad.jl:31-164)
 *   eikttimemisfit (src/EikSolv/eikmaingrad.jl:1302-1328)
 *
 * Conventions
 *  - Arrays are FP64. Grids are column-major with x fastest (Julia's layout, cart2lin in
 *    src/EikSolv/eikutils.jl:6-19); indices in this ABI are 0-based.
 *  - coordsrc is nsrc x ndim row-major (source s at coordsrc[s*ndim .. s*ndim+ndim-1]).
 *  - Receivers of all sources are concatenated row-major; rec_off[0..nsrc] are offsets
 *    (receiver r of source s is row rec_off[s]+r). Picks, pickobs and stdobs follow rec_off.
 *  - Spherical grids take θ, φ in degrees, as the reference.
 *  - All host buffers are caller-owned; outputs are preallocated by the caller.
 *    Device memory is owned by the context; models stay resident until released.
 *  - Return value: EIK_OK or a negative EIK_ERR_*; eik_last_error() gives the message of
 *    the calling thread's last failure on that context.
 */
#ifndef EIKCUDA_H
#define EIKCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EIK_OK 0
#define EIK_ERR_ASSERT (-1)        /* an @assert of the reference failed (AssertionError) */
#define EIK_ERR_ERROR (-2)         /* an error() call of the reference (ErrorException) */
#define EIK_ERR_CUDA (-3)          /* CUDA runtime failure */
#define EIK_ERR_NOT_CONVERGED (-4) /* iteration limit reached */
#define EIK_ERR_OUT_OF_BUDGET (-5) /* request does not fit the context's HBM budget */
#define EIK_ERR_TIMEOUT (-6)       /* a bounded device wait ran out */
#define EIK_ERR_UNSUPPORTED (-7)   /* configuration outside what this build implements */

/* Grid kinds (src/EikSolv/eikstructs.jl:33-219). */
#define EIK_GRID2DCART 0
#define EIK_GRID3DCART 1
#define EIK_GRID2DSPHERE 2
#define EIK_GRID3DSPHERE 3

/* whichgrad (eikmaingrad.jl:40): :gradvel, :gradsrcloc, :gradvelandsrcloc */
#define EIK_GRADVEL 1
#define EIK_GRADSRCLOC 2
#define EIK_GRADVELANDSRCLOC 3

/* Warning bits (the reference's @warn sites). */
#define EIK_WARN_NEG_DISCRIMINANT 0x1u     /* eikforward2D.jl:342 / eikforward3D.jl:429 */
#define EIK_WARN_SRC_HALFWAY_SHIFT 0x2u    /* eikmainfwd.jl:1298 */
#define EIK_WARN_BORDER_BEFORE_COARSE 0x4u /* eikmainfwd.jl:731 */
#define EIK_WARN_SRCPOS_ALIGNED_SHIFT 0x8u /* eikmaingrad.jl:1250 */
#define EIK_WARN_SRC_ON_NODE_DERIV 0x10u   /* eikmaingrad.jl:1260 */
#define EIK_WARN_FINE_NO_TRIGGER 0x20u     /* refined grid covered the model: no edge stop */

typedef struct eik_ctx eik_ctx;
typedef int64_t eik_model_id;

/* Grid2DCart/Grid3DCart: spacing = {hgrid, hgrid, hgrid};
 * Grid2DSphere: {Δr, Δθ, -}; Grid3DSphere: {Δr, Δθ, Δφ}. Unused entries are ignored. */
typedef struct {
  int32_t kind;
  int32_t ndim;
  int64_t grsize[3];
  double spacing[3];
  double cooinit[3];
} eik_grid;

/* ExtraParams / GridRefinementPars (src/EikSolv/eikstructs.jl:230-282). parallelkind is
 * accepted and ignored: every call batches all its sources on the device. */
typedef struct {
  int32_t refinearoundsrc;      /* default 1 */
  int32_t downscalefactor;      /* default 5 */
  int32_t noderadius;           /* default 3 */
  int32_t radiussmoothgradsrc;  /* default 3 */
  int32_t smoothgradkern;       /* default 0 (odd when > 0) */
  int32_t parallelkind;         /* 0 serial, 1 sharedmem, 2 distribmem */
  int32_t nthreads;             /* Threads.nthreads() of the caller; with :sharedmem the
                                   gradient's sources form min(nsrc, nthreads) consecutive
                                   groups with separate gradient buffers (distribsrcs,
                                   eikutils.jl:171-190). 0 or 1: one group. */
  int32_t reserved;
} eik_extra;

typedef struct {
  uint32_t warn_mask;        /* EIK_WARN_* */
  uint32_t err_mask;         /* device error word of the last launch (0 = none) */
  uint64_t tile_activations; /* forward solve: listed nodes visited over all rounds */
  uint64_t node_evals;       /* coarse node updates evaluated */
  double device_ms;          /* device time of the call (CUDA events) */
  double fine_ms;            /* start-up stage: refined-grid FMM or source box (CUDA events) */
  double solve_ms;           /* coarse forward solve kernel (CUDA events) */
  double adj_ms;             /* adjoint dataflow solve kernel (CUDA events) */
  uint64_t adj_rounds;       /* rounds of the adjoint sweep */
  uint64_t launches;         /* kernels this call launched */
  uint64_t fwd_rounds;       /* rounds of the forward solve */
  uint64_t fine_replays;      /* sources whose refined start-up needed the exact heap replay */
  uint64_t fwd_visits[7];    /* forward list visits by outcome: value cached above the front,
                                source point, nothing reached, bound above the front,
                                evaluated above the front, evaluated unchanged, changed */
  uint64_t chunks;           /* gradient calls split to fit the HBM budget: pipelines run (else 0) */
  uint64_t retries;          /* pipelines run again after the automatic round limit (see max_rounds) */
} eik_stats;

/* Fills the reference defaults of ExtraParams(). */
void eik_extra_defaults(eik_extra* ep);

/* Creates a context on CUDA device `device`. hbm_budget bounds the device memory the
 * context may hold (0 = 90% of the device's free memory). */
int eik_ctx_create(int device, size_t hbm_budget, eik_ctx** out);
int eik_ctx_destroy(eik_ctx* ctx);
const char* eik_last_error(eik_ctx* ctx);
/* The CUDA stream (cudaStream_t) all work of this context runs on, for callers that order
 * their own work or events against it. */
void* eik_ctx_stream(eik_ctx* ctx);
/* Scheduling parameters of a context (results do not depend on them, only the amount of
 * work does): "round_gate" = width of a forward round in units of (smallest node spacing x
 * smallest slowness); "sm_fraction" = share of the SMs that the persistent solve kernels of
 * this context occupy, in (0, 1] (contexts whose calls overlap on one GPU, as in a serving
 * loop, each take a share so that their solves can be resident together). For both, 0 (the
 * default) = chosen per call by its size: calls of fewer than 2^22 node-sources (nsrc x grid
 * nodes) take round_gate 8 on a quarter of the SMs, larger ones round_gate 2 on all of them; "ctas_per_sm" = resident CTAs per SM of the forward solve, an integer, 0 (the
 * default) = as many as fit; "fwd_queue" = how the forward solve's warps work through their
 * entries: 1 = evaluations queued per warp and run 32 at a time, 0 = each in place, -1 (the
 * default) = the queue from 2^27 node-sources per launch up; "ray_room" = room of a ray in
 * the single tracing pass, in multiples of its straight-line length (default 3; rays that
 * outgrow it are traced again); "fine_replay" = 1 replays the refined start-up's heap for every
 * source instead of only where an exact tie decides its stop (default 0); "max_rounds" = round
 * limit of the persistent forward and adjoint solves, an integer; a solve that reaches it
 * stops on the device and the call returns EIK_ERR_NOT_CONVERGED, the context staying usable.
 * 0 (the default) = the library's: for a forward solve 256 rounds per node of its grid's
 * diameter (the sum of its sizes) plus 65 536, and a call whose forward solve reaches that
 * limit runs once more with wider rounds and a limit of 2^24 (eik_stats.retries; the result
 * does not depend on the schedule), 2^26 for the adjoint; "auto_round_limit" = that
 * automatic limit of a first run, an integer, 0 (the default) = by the grid's diameter; "cluster_solve" = how problems
 * small enough for one thread-block cluster's shared memory (the refined windows, grids up to
 * ~97 000 nodes) are solved: 1 (the default) = 2D ones in one cluster each (faster there),
 * 2 = in any dimension, 0 = always the persistent global solve. Returns EIK_ERR_ASSERT for an unknown name or a value out of
 * range. */
int eik_ctx_set_param(eik_ctx* ctx, const char* name, double value);

/* No counterpart in the reference: failure-detection self-test. Runs, on the context's
 * stream, one device wait of the kind the persistent solves use (bounded by the global
 * timer) on a flag that nothing sets, with a limit of timeout_s seconds (in [0.001, 10]),
 * and returns what such a wait reports when it runs out: EIK_ERR_TIMEOUT, the kernel having
 * returned and the context staying usable. */
int eik_selftest_wait(eik_ctx* ctx, double timeout_s);

/* Uploads a velocity model (host, column-major, FP64) and keeps it resident. Checks
 * all(vel.>0) (eikmainfwd.jl:45). */
int eik_model_upload(eik_ctx* ctx, const eik_grid* grd, const double* vel, eik_model_id* out);
/* Same, from a device pointer of this context's device. */
int eik_model_upload_device(eik_ctx* ctx, const eik_grid* grd, const double* vel_dev, eik_model_id* out);
int eik_model_release(eik_ctx* ctx, eik_model_id model);

/* No counterpart in the reference: device bytes that one eik_gradient pipeline of nsrc
 * sources and nrec receivers in all takes from the context's HBM budget (the forward and
 * adjoint state of every source plus the fixed part). A serving loop uses it for admission;
 * eik_gradient splits a call whose footprint exceeds the budget. */
int eik_gradient_bytes(eik_ctx* ctx, eik_model_id model, int64_t nsrc, int64_t nrec, const eik_extra* ep,
                       int32_t whichgrad, uint64_t* bytes);

/* Replaces ttforwsomesrc (eikmainfwd.jl:152-199) for all nsrc sources at once.
 * picks: rec_off[nsrc] values. ttgrids: nullable, nsrc x N traveltime grids (returntt). */
int eik_traveltime(eik_ctx* ctx, eik_model_id model, int64_t nsrc, const double* coordsrc,
                   const int64_t* rec_off, const double* rec, const eik_extra* ep, double* picks,
                   double* ttgrids, eik_stats* stats);

/* No counterpart in the reference as one call: ttforwsomesrc (eikmainfwd.jl:152-199) for the
 * sources of several models of one dimension, whose grids may differ in size, in one
 * pipeline (one persistent solve for all of them). Model model_ids[i] takes sources
 * src_off[i]..src_off[i+1]-1 (src_off[0] = 0, non-decreasing, nmodel+1 values); coordsrc,
 * rec_off (rec_off[0] = 0), rec and picks run over all sources in that order, as in
 * eik_traveltime. ttgrids: nullable, each source's grid at its own model's node count, one
 * after another. Every source's results are bit-identical to eik_traveltime of its model
 * alone. */
int eik_traveltime_multi(eik_ctx* ctx, int64_t nmodel, const eik_model_id* model_ids, const int64_t* src_off,
                         const double* coordsrc, const int64_t* rec_off, const double* rec, const eik_extra* ep,
                         double* picks, double* ttgrids, eik_stats* stats);

/* Replaces calcgradsomesrc (eikmaingrad.jl:174-258) with the sources in one group (the
 * :serial order). gradvel: nullable N values; gradsrc: nullable nsrc x ndim; misfit: the
 * summed 0.5*Σ(t-obs)²/σ² of the group. A call whose device footprint (eik_gradient_bytes)
 * exceeds the context's HBM budget runs as several pipelines over consecutive chunks of its
 * sources, recomputing each chunk's traveltimes instead of keeping all of them, with the
 * gradient carried between sources (the reference's per-group buffer) and the ordered sums
 * handed from chunk to chunk: the result is the one-pipeline result bit for bit
 * (eik_stats.chunks gives the number of pipelines). */
int eik_gradient(eik_ctx* ctx, eik_model_id model, int64_t nsrc, const double* coordsrc,
                 const int64_t* rec_off, const double* rec, const double* pickobs,
                 const double* stdobs, int32_t whichgrad, const eik_extra* ep, double* gradvel,
                 double* gradsrc, double* misfit, eik_stats* stats);

/* Same as eik_gradient with inputs and outputs in this context's device memory (for callers
 * that keep observations and results on the GPU: autodiff wrappers, serving). rec_off stays
 * on the host. gradvel_dev: N values, gradsrc_dev: nsrc x ndim, misfit_dev: 1 value; each
 * nullable. Returns when the results are written. */
int eik_gradient_device(eik_ctx* ctx, eik_model_id model, int64_t nsrc, const double* coordsrc_dev,
                        const int64_t* rec_off, const double* rec_dev, const double* pickobs_dev,
                        const double* stdobs_dev, int32_t whichgrad, const eik_extra* ep,
                        double* gradvel_dev, double* gradsrc_dev, double* misfit_dev, eik_stats* stats);

/* No counterpart in the reference as one call: calcgradsomesrc (eikmaingrad.jl:174-258) for
 * several independent gradient evaluations on one model in one pipeline (a serving loop
 * merging requests). Group g is sources group_off[g]..group_off[g+1]-1 (group_off[0] = 0,
 * every group non-empty) with its own gradient buffer and carry-over, as the reference's one
 * worker group; its results equal eik_gradient of those sources alone with one group
 * (:serial), bit for bit. coordsrc, rec_off, rec, pickobs, stdobs run over all sources as in
 * eik_gradient; ep applies to every group (its parallelkind and nthreads are not used).
 * gradvel: nullable, ngroups x N (group g's field at g*N); gradsrc: nullable, nsrc x ndim;
 * misfit: nullable, ngroups values. The call is not split into chunks: one that exceeds the
 * HBM budget returns EIK_ERR_OUT_OF_BUDGET. */
int eik_gradient_groups(eik_ctx* ctx, eik_model_id model, int64_t ngroups, const int64_t* group_off,
                        const double* coordsrc, const int64_t* rec_off, const double* rec, const double* pickobs,
                        const double* stdobs, int32_t whichgrad, const eik_extra* ep, double* gradvel,
                        double* gradsrc, double* misfit, eik_stats* stats);

/* Captured gradient plans (no counterpart in the reference; for callers that evaluate
 * eikgradient model after model with the same sources and receivers, as the HMC problem
 * callables of HMCtraveltimes.jl:84-104 do). eik_plan_gradient validates like eik_gradient,
 * runs the pipeline once and captures it as a CUDA graph for fixed model, sources,
 * receivers, whichgrad and extraparams (and the context's scheduling parameters at that
 * time). The plan owns its device buffers, taken from the context's HBM budget until
 * eik_plan_destroy. eik_plan_run replays it: vel (host, column-major, nullable) replaces the
 * model's velocity in place first (the model keeps it afterwards; NULL keeps the current
 * one), pickobs/stdobs are the observations of this evaluation (rec_off[nsrc] values each);
 * outputs as eik_gradient. Results are bit-identical to eik_gradient on the same inputs.
 * While a plan exists its model cannot be released and its context cannot be destroyed
 * (EIK_ERR_ASSERT). Replays of plans of one context are serialised with its other calls. */
typedef struct eik_plan eik_plan;
int eik_plan_gradient(eik_ctx* ctx, eik_model_id model, int64_t nsrc, const double* coordsrc,
                      const int64_t* rec_off, const double* rec, int32_t whichgrad, const eik_extra* ep,
                      eik_plan** out);
int eik_plan_run(eik_plan* plan, const double* vel, const double* pickobs, const double* stdobs,
                 double* gradvel, double* gradsrc, double* misfit, eik_stats* stats);
int eik_plan_destroy(eik_plan* plan);

/* Replaces tracerays (eikutils.jl:201-328): for every receiver of every source the ray from
 * the receiver to the source, following the cubic B-spline gradient of the source's
 * traveltime grid in steps of steplen*h (steplen on Grid2DSphere); Grid3DSphere errors as in
 * the reference. ttgrids: host, nsrc x N column-major grids (as eik_traveltime returns them).
 * ray_npts (out): rec_off[nsrc] point counts. paths (nullable): room for paths_cap points of
 * ndim doubles; the rays are written there, concatenated in receiver order, when they fit,
 * else EIK_ERR_OUT_OF_BUDGET is returned with ray_npts filled (call again with a larger
 * buffer). A ray that needs more than 2^24 steps fails with EIK_ERR_NOT_CONVERGED. */
int eik_tracerays(eik_ctx* ctx, const eik_grid* grd, int64_t nsrc, const double* ttgrids,
                  const double* coordsrc, const int64_t* rec_off, const double* rec, double steplen,
                  int64_t* ray_npts, double* paths, int64_t paths_cap, eik_stats* stats);
/* Traveltimes (picks as eik_traveltime) and rays in one device pipeline: the traveltime
 * grids stay in device memory between the solve and the ray tracing. */
int eik_traveltime_rays(eik_ctx* ctx, eik_model_id model, int64_t nsrc, const double* coordsrc,
                        const int64_t* rec_off, const double* rec, const eik_extra* ep, double steplen,
                        double* picks, int64_t* ray_npts, double* paths, int64_t paths_cap,
                        eik_stats* stats);

/* No counterpart in the reference. Misfit 0.5*Σ_s Σ_r (t - obs)²/σ² of nsrc traveltime
 * grids that are already in device memory (ttgrids_dev: nsrc x N, as eik_traveltime
 * returns them), with receivers, observations and the result also in device memory and
 * rec_off on the host. It allocates no device memory: for callers that may not call
 * cudaMalloc (a framework op under the framework's own allocator, a sampler callback that
 * must not change the device's memory map). Its scratch is a fixed ~1 MB array in the
 * library, so nsrc is limited to 65536 (larger calls fail with EIK_ERR_OUT_OF_BUDGET).
 * All calls on a device share that array: calls that overlap on the GPU race, so
 * serialise them. Every call runs on `stream` (a cudaStream_t; NULL = legacy default
 * stream), copies rec_off from the host, reads its error word back into host memory and
 * synchronises `stream` before it returns: it blocks the calling host thread until the
 * result is written, and no call can run while its stream is being captured into a graph. */
int eik_ttimemisfit_noalloc(const eik_grid* grd, int64_t nsrc, const double* ttgrids_dev,
                            const int64_t* rec_off, const double* rec_dev, const double* pickobs_dev,
                            const double* stdobs_dev, double* misfit_dev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* EIKCUDA_H */
