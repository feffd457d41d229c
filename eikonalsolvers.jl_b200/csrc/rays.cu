// Ray tracing on device-resident traveltime grids: tracerays / tracerays_singlesrc
// (src/EikSolv/eikutils.jl:201-328).
//
// The reference interpolates each traveltime grid with Interpolations.jl's cubic B-spline
// (`BSpline(Cubic())` = `Cubic(Line(OnGrid()))`, scaled to the grid axes) and walks from
// every receiver against the interpolated gradient, one step of steplen*h (steplen on a
// Grid2DSphere) at a time, clamped into the grid, until it is within h*sqrt(2) (Δr*sqrt(2))
// of the source; the last point is replaced by the source.
//
// The interpolant and the per-line / per-ray work are in rays.cuh (host/device code). The
// filter runs one thread per line, axis after axis. The arithmetic is the oracle's,
// operation for operation, so Cartesian rays are bit-identical to it (the spherical step
// also calls sin, cos and atan2).
//
// Tracing: one thread per ray, in one pass that writes every ray into a room of three times
// its straight-line length plus 16 points and counts its points; a compaction kernel then
// moves the rays to their places in the output (the rare ray that outgrows its room makes the
// pass run again, each ray with exactly its room). A ray longer than the step limit sets an
// error bit and stops.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/eikcuda.h"
#include "rays.cuh"
#include "runtime.hpp"

namespace eik {

constexpr int RAY_THREADS = 128;

__global__ void spline_load_kernel(SplineArgs s, const double* tt, long long N) {
  const long long tot = N * s.nsrc;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x)
    spline_load_one(s, tt, N, q);
}

// One Thomas sweep per line along axis ax (one thread per line).
__global__ void spline_axis_kernel(SplineArgs s, int ax, const double* cp) {
  long long cnt[3];
  const long long tot = spline_lines(s, ax, cnt) * s.nsrc;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x)
    spline_line(s, ax, cp, q);
}

// Rays from their rooms in the slab to their places in the output, one block per ray.
__global__ void ray_compact_kernel(const double* slab, const long long* soff, const long long* npts,
                                   const long long* outoff, double* out, long long nray, int nd) {
  for (long long r = blockIdx.x; r < nray; r += gridDim.x) {
    const long long n = npts[r] * nd;
    const double* src = slab + soff[r] * nd;
    double* dst = out + outoff[r] * nd;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
  }
}

template <int ND>
__global__ void __launch_bounds__(RAY_THREADS) trace_kernel(RayArgs a, int write) {
  const long long nray = a.recoff[a.nsrc];
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < nray; r += (long long)gridDim.x * blockDim.x)
    trace_one<ND>(a, r, write);
}

// Thomas factors of the constant system (1/6, 2/3, 1/6) of size k, as the oracle computes them.
static std::vector<double> thomas_factors(long long k) {
  std::vector<double> cp((size_t)(k > 0 ? k : 1));
  const double a = 1.0 / 6.0, b = 2.0 / 3.0, cc = 1.0 / 6.0;
  if (k > 0) cp[0] = cc / b;
  for (long long i = 1; i < k; i++) cp[(size_t)i] = cc / (b - a * cp[(size_t)(i - 1)]);
  return cp;
}

// Rays of nsrc sources whose traveltime grids (nsrc x N) are at d_tt on the device; the
// other inputs are on the device too except rec_off (host). ray_npts (host) receives the
// point counts; paths (host, nullable) the points when paths_cap is large enough.
int trace_device(eik_ctx* ctx, const GridDesc& g, int64_t nsrc, const double* d_tt, const double* d_cs,
                 const long long* d_off, const double* d_rec, const double* h_cs, const int64_t* rec_off,
                 const double* h_rec, double steplen, int64_t* ray_npts, double* paths, int64_t paths_cap,
                 eik_stats* stats) {
  int rc = EIK_OK;
  cudaStream_t st = ctx->stream;
  Scratch& S = ctx->scratch;
  if (g.kind == G3DSPH)
    return fail(ctx, EIK_ERR_ERROR, "tracerays_singlesrc(): ray tracing for spherical grids not yet implemented.");
  for (int d = 0; d < g.nd; d++)
    if (g.n[d] < 2) return fail(ctx, EIK_ERR_ERROR, "tracerays: every grid axis needs at least 2 nodes");
  if (!(steplen > 0.0)) return fail(ctx, EIK_ERR_ASSERT, "steplen > 0");
  SplineArgs sp;
  sp.nd = g.nd;
  sp.nsrc = (int)nsrc;
  for (int d = 0; d < 3; d++) {
    sp.n[d] = g.n[d];
    sp.m[d] = d < g.nd ? g.n[d] + 2 : 1;
  }
  sp.cstride = sp.m[0] * sp.m[1] * sp.m[2];
  sp.coef_size = sp.cstride * nsrc;
  const long long N = npts(g), nray = rec_off[nsrc];
#define GET(var, type, name, count)                                                  \
  var = (type*)S.get(name, sizeof(type) * (size_t)(count), &rc);                     \
  if (!var) return rc == EIK_ERR_OUT_OF_BUDGET                                       \
                     ? fail(ctx, rc, "scratch '%s' exceeds the HBM budget", name)    \
                     : fail(ctx, rc, "cudaMalloc of scratch '%s' failed", name);
  double* coef;
  double* cpd;
  long long *d_np, *d_oo;
  uint32_t* d_err;
  GET(coef, double, "ray_coef", sp.cstride * nsrc);
  GET(cpd, double, "ray_thomas", (long long)g.n[0] + g.n[1] + g.n[2]);
  GET(d_np, long long, "ray_npts", std::max<long long>(nray, 1));
  GET(d_oo, long long, "ray_off", std::max<long long>(nray, 1));
  GET(d_err, uint32_t, "ray_err", 1);
  {
    std::vector<double> all;
    for (int d = 0; d < g.nd; d++) {
      sp.cp[d] = cpd + all.size();
      const std::vector<double> f = thomas_factors(g.n[d] - 2);
      all.insert(all.end(), f.begin(), f.end());
    }
    CUDA_OK(ctx, cudaMemcpyAsync(cpd, all.data(), sizeof(double) * all.size(), cudaMemcpyHostToDevice, st));
  }
  sp.coef = coef;
  sp.err = d_err;
  CUDA_OK(ctx, cudaMemsetAsync(d_err, 0, sizeof(uint32_t), st));
  spline_load_kernel<<<ctx->nsm * 8, 256, 0, st>>>(sp, d_tt, N);
  for (int ax = 0; ax < g.nd; ax++) spline_axis_kernel<<<ctx->nsm * 4, 128, 0, st>>>(sp, ax, sp.cp[ax]);
  RayArgs ra;
  ra.g = g;
  ra.nsrc = (int)nsrc;
  for (int d = 0; d < 3; d++) ra.m[d] = sp.m[d];
  ra.cstride = sp.cstride;
  ra.coef_size = sp.coef_size;
  ra.pts_size = 0;
  ra.coef = coef;
  ra.coordsrc = d_cs;
  ra.recoff = d_off;
  ra.rec = d_rec;
  ra.rstep = is_cart(g) ? steplen * g.spac[0] : steplen;
  ra.thrdist = g.spac[0] * sqrt(2.0);
  ra.max_steps = 1LL << 24;
  ra.outoff = d_oo;
  ra.cap = nullptr;
  ra.npts = d_np;
  ra.pts = nullptr;
  ra.err = d_err;
  const int nblk = (int)std::max<long long>(1, std::min<long long>((nray + RAY_THREADS - 1) / RAY_THREADS, 1 << 16));
  int launches = 0;
  auto launch = [&](int write) {
    if (!nray) return;
    if (g.nd == 3) trace_kernel<3><<<nblk, RAY_THREADS, 0, st>>>(ra, write);
    else trace_kernel<2><<<nblk, RAY_THREADS, 0, st>>>(ra, write);
    launches++;
  };
  std::vector<long long> cnt((size_t)std::max<long long>(nray, 1), 0);
  auto read_counts = [&]() -> int {
    uint32_t herr = 0;
    CUDA_OK(ctx, cudaGetLastError());
    if (nray) CUDA_OK(ctx, cudaMemcpyAsync(cnt.data(), d_np, sizeof(long long) * nray, cudaMemcpyDeviceToHost, st));
    CUDA_OK(ctx, cudaMemcpyAsync(&herr, d_err, sizeof herr, cudaMemcpyDeviceToHost, st));
    CUDA_OK(ctx, cudaStreamSynchronize(st));
    if (herr & ERRB_RAY_ADDR) return fail(ctx, EIK_ERR_ERROR, "ray kernels: an address check failed (0x%x)", herr);
    if (herr & ERRB_RAY_STEPS)
      return fail(ctx, EIK_ERR_NOT_CONVERGED, "a ray did not reach its source within 2^24 steps");
    return EIK_OK;
  };
  if (!paths) {  // counts only
    launch(0);
    rc = read_counts();
    if (rc) return rc;
    for (long long r = 0; r < nray; r++) ray_npts[r] = cnt[(size_t)r];
    if (stats) stats->launches += 1 + g.nd + launches;
    return EIK_OK;
  }
  // one pass that writes every ray into a room of ray_room (3) times its straight-line length
  // (in steps) plus 16 points; the rays that outgrow their room are traced again below
  std::vector<long long> room((size_t)std::max<long long>(nray, 1)), soff((size_t)std::max<long long>(nray, 1));
  long long slab = 0;
  for (int64_t s = 0; s < nsrc; s++)
    for (long long r = rec_off[s]; r < rec_off[s + 1]; r++) {
      const double dist = distance2points(g, h_rec + r * g.nd, h_cs + s * g.nd);
      const double est = std::isfinite(dist) ? ctx->ray_room * dist / ra.rstep : 0.0;
      room[(size_t)r] = (est < 1e7 ? (long long)est : 10000000LL) + 16;
      soff[(size_t)r] = slab;
      slab += room[(size_t)r];
    }
  long long* d_room;
  double* d_slab;
  GET(d_room, long long, "ray_room", std::max<long long>(nray, 1));
  GET(d_slab, double, "ray_slab", std::max<long long>(slab, 1) * g.nd);
  if (nray) {
    CUDA_OK(ctx, cudaMemcpyAsync(d_room, room.data(), sizeof(long long) * nray, cudaMemcpyHostToDevice, st));
    CUDA_OK(ctx, cudaMemcpyAsync(d_oo, soff.data(), sizeof(long long) * nray, cudaMemcpyHostToDevice, st));
  }
  ra.cap = d_room;
  ra.pts = d_slab;
  ra.pts_size = slab * g.nd;
  launch(1);
  rc = read_counts();
  if (rc) return rc;
  std::vector<long long> off((size_t)std::max<long long>(nray, 1), 0);
  long long total = 0;
  bool outgrown = false;
  for (long long r = 0; r < nray; r++) {
    ray_npts[r] = cnt[(size_t)r];
    off[(size_t)r] = total;
    total += cnt[(size_t)r];
    outgrown = outgrown || cnt[(size_t)r] > room[(size_t)r];
  }
  if (total > paths_cap)
    return fail(ctx, EIK_ERR_OUT_OF_BUDGET, "the rays have %lld points, paths has room for %lld", total,
                (long long)paths_cap);
  double* d_pts;
  long long* d_xoff;
  GET(d_pts, double, "ray_pts", std::max<long long>(total, 1) * g.nd);
  GET(d_xoff, long long, "ray_xoff", std::max<long long>(nray, 1));
#undef GET
  if (nray) CUDA_OK(ctx, cudaMemcpyAsync(d_xoff, off.data(), sizeof(long long) * nray, cudaMemcpyHostToDevice, st));
  if (!outgrown) {
    ray_compact_kernel<<<(int)std::min<long long>(std::max<long long>(nray, 1), 1 << 16), 128, 0, st>>>(
        d_slab, d_oo, d_np, d_xoff, d_pts, nray, g.nd);
    launches++;
  } else {  // trace every ray again, each with exactly its room
    if (nray) {
      CUDA_OK(ctx, cudaMemcpyAsync(d_room, cnt.data(), sizeof(long long) * nray, cudaMemcpyHostToDevice, st));
      CUDA_OK(ctx, cudaMemcpyAsync(d_oo, off.data(), sizeof(long long) * nray, cudaMemcpyHostToDevice, st));
    }
    ra.pts = d_pts;
    ra.pts_size = total * g.nd;
    launch(1);
    rc = read_counts();
    if (rc) return rc;
  }
  CUDA_OK(ctx, cudaGetLastError());
  CUDA_OK(ctx, cudaMemcpyAsync(paths, d_pts, sizeof(double) * total * g.nd, cudaMemcpyDeviceToHost, st));
  CUDA_OK(ctx, cudaStreamSynchronize(st));
  if (stats) stats->launches += 1 + g.nd + launches;
  return EIK_OK;
}

}  // namespace eik

using namespace eik;

namespace {

int check_ray_inputs(eik_ctx* ctx, const GridDesc& g, int64_t nsrc, const double* coordsrc, const int64_t* rec_off,
                     const double* rec, int64_t* ray_npts) {
  if (nsrc < 1) return fail(ctx, EIK_ERR_ASSERT, "nsrc >= 1");
  if (!coordsrc || !rec_off || !ray_npts || (!rec && rec_off[nsrc] > 0)) return fail(ctx, EIK_ERR_ASSERT, "NULL argument");
  if (rec_off[0] != 0) return fail(ctx, EIK_ERR_ASSERT, "rec_off[0] must be 0");
  for (int64_t s = 0; s < nsrc; s++)
    if (rec_off[s + 1] < rec_off[s]) return fail(ctx, EIK_ERR_ASSERT, "rec_off must be non-decreasing");
  for (int64_t i = 0; i < nsrc * g.nd; i++)
    if (!std::isfinite(coordsrc[i])) return fail(ctx, EIK_ERR_ASSERT, "coordsrc must be finite");
  for (int64_t i = 0; i < rec_off[nsrc] * g.nd; i++)
    if (!std::isfinite(rec[i])) return fail(ctx, EIK_ERR_ASSERT, "coordrec must be finite");
  return EIK_OK;
}

}  // namespace

extern "C" int eik_tracerays(eik_ctx* ctx, const eik_grid* grd, int64_t nsrc, const double* ttgrids,
                             const double* coordsrc, const int64_t* rec_off, const double* rec, double steplen,
                             int64_t* ray_npts, double* paths, int64_t paths_cap, eik_stats* stats) {
  if (!ctx) return fail(ctx, EIK_ERR_ASSERT, "NULL context");
  if (!grd || !ttgrids) return fail(ctx, EIK_ERR_ASSERT, "NULL argument");
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->scratch.begin_call();
  NvtxRange nvtx_call("eik_tracerays");
  if (stats) std::memset(stats, 0, sizeof *stats);
  GridDesc g;
  int rc = make_griddesc(ctx, grd, &g);
  if (rc) return rc;
  rc = check_ray_inputs(ctx, g, nsrc, coordsrc, rec_off, rec, ray_npts);
  if (rc) return rc;
  CUDA_OK(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const long long N = npts(g), nrec = rec_off[nsrc];
  double* d_tt = (double*)ctx->scratch.get("ray_tt", sizeof(double) * N * nsrc, &rc);
  double* d_cs = (double*)ctx->scratch.get("in_cs", sizeof(double) * nsrc * g.nd, &rc);
  long long* d_off = (long long*)ctx->scratch.get("in_off", sizeof(long long) * (nsrc + 1), &rc);
  double* d_rec = (double*)ctx->scratch.get("in_rec", sizeof(double) * std::max<long long>(nrec, 1) * g.nd, &rc);
  if (!d_tt || !d_cs || !d_off || !d_rec) return fail(ctx, rc ? rc : EIK_ERR_CUDA, "scratch allocation failed");
  cudaEventRecord(ctx->ev0, st);
  CUDA_OK(ctx, cudaMemcpyAsync(d_tt, ttgrids, sizeof(double) * N * nsrc, cudaMemcpyHostToDevice, st));
  CUDA_OK(ctx, cudaMemcpyAsync(d_cs, coordsrc, sizeof(double) * nsrc * g.nd, cudaMemcpyHostToDevice, st));
  CUDA_OK(ctx, cudaMemcpyAsync(d_off, rec_off, sizeof(long long) * (nsrc + 1), cudaMemcpyHostToDevice, st));
  if (nrec) CUDA_OK(ctx, cudaMemcpyAsync(d_rec, rec, sizeof(double) * nrec * g.nd, cudaMemcpyHostToDevice, st));
  rc = trace_device(ctx, g, nsrc, d_tt, d_cs, d_off, d_rec, coordsrc, rec_off, rec, steplen, ray_npts, paths, paths_cap, stats);
  cudaEventRecord(ctx->ev1, st);
  cudaStreamSynchronize(st);
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    stats->device_ms = ms;
  }
  return rc;
}

extern "C" int eik_traveltime_rays(eik_ctx* ctx, eik_model_id model, int64_t nsrc, const double* coordsrc,
                                   const int64_t* rec_off, const double* rec, const eik_extra* ep_in, double steplen,
                                   double* picks, int64_t* ray_npts, double* paths, int64_t paths_cap,
                                   eik_stats* stats) {
  if (!ctx) return fail(ctx, EIK_ERR_ASSERT, "NULL context");
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->scratch.begin_call();
  NvtxRange nvtx_call("eik_traveltime_rays");
  auto it = ctx->models.find(model);
  if (it == ctx->models.end()) return fail(ctx, EIK_ERR_ASSERT, "unknown model id %lld", (long long)model);
  const Model& m = it->second;
  eik_extra ep;
  if (ep_in) ep = *ep_in;
  else eik_extra_defaults(&ep);
  int rc = check_extra(ctx, &ep);
  if (rc) return rc;
  if (stats) std::memset(stats, 0, sizeof *stats);
  rc = check_ray_inputs(ctx, m.g, nsrc, coordsrc, rec_off, rec, ray_npts);
  if (rc) return rc;
  if (!picks && rec_off[nsrc] > 0) return fail(ctx, EIK_ERR_ASSERT, "NULL argument");
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
  if (!d_cs || !d_off || !d_rec || !d_picks) return fail(ctx, rc ? rc : EIK_ERR_CUDA, "scratch allocation failed");
  cudaEventRecord(ctx->ev0, st);
  CUDA_OK(ctx, cudaMemcpyAsync(d_cs, coordsrc, sizeof(double) * nsrc * nd, cudaMemcpyHostToDevice, st));
  CUDA_OK(ctx, cudaMemcpyAsync(d_off, rec_off, sizeof(long long) * (nsrc + 1), cudaMemcpyHostToDevice, st));
  if (nrec) CUDA_OK(ctx, cudaMemcpyAsync(d_rec, rec, sizeof(double) * nrec * nd, cudaMemcpyHostToDevice, st));
  ForwardState fw;
  rc = forward_device(ctx, m, nsrc, d_cs, ep, &fw, stats);
  if (rc) return rc;
  if (nrec) launch_picks(m.g, fw.t, m.N, (int)nsrc, d_off, d_rec, d_picks, st);
  CUDA_OK(ctx, cudaGetLastError());
  if (nrec) CUDA_OK(ctx, cudaMemcpyAsync(picks, d_picks, sizeof(double) * nrec, cudaMemcpyDeviceToHost, st));
  rc = collect_forward_stats(ctx, &fw, stats);
  if (rc) return rc;
  // the traveltime grids never leave the device
  rc = trace_device(ctx, m.g, nsrc, fw.t, d_cs, d_off, d_rec, coordsrc, rec_off, rec, steplen, ray_npts, paths, paths_cap, stats);
  cudaEventRecord(ctx->ev1, st);
  cudaStreamSynchronize(st);
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    stats->device_ms = ms;
    stats->launches += nrec ? 1 : 0;
  }
  return rc;
}
