// Traveltime misfit of traveltime grids already on the device, with no device allocation.
//
// Who needs this: code that evaluates the misfit inside a host program that owns all
// device memory and does not let its operators call cudaMalloc: a framework's custom op
// running under the framework's caching allocator, or a sampler callback (Julia, JAX) that
// must not change the device's memory map or synchronise the device the way cudaMalloc and
// cudaFree can. Those callers bring their own input and output buffers; the little scratch
// this computation needs (the receiver offsets and one partial sum per source) lives in a
// fixed array compiled into the library instead of being allocated.
//
// The fixed array is shared by every call of the process on that device and keeps the
// last call's contents. Two calls whose work overlaps on the GPU (different streams, or
// different host threads) race on it and give wrong results: serialise them.
// The first call on each device does a one-time set-up (it looks up the array's device
// address with cudaGetSymbolAddress). Every call copies the receiver offsets from host
// memory, reads its error word back to the host and synchronises its stream: it blocks the
// calling thread until the misfit is written, and cannot run inside a stream capture.
#include <mutex>

#include "../../include/eikcuda.h"
#include "kernels.cuh"
#include "runtime.hpp"

namespace eik {

// Largest number of sources one call accepts.
constexpr int64_t NOALLOC_MAX_SOURCES = 65536;

// Layout of the fixed scratch: error word | receiver offsets (max+1) | per-source sums (max).
constexpr size_t NA_ERR_OFF = 0;
constexpr size_t NA_RECOFF_OFF = 256;
constexpr size_t NA_PART_OFF = NA_RECOFF_OFF + sizeof(long long) * (NOALLOC_MAX_SOURCES + 1 + 31);
constexpr size_t NA_BYTES = NA_PART_OFF + sizeof(double) * NOALLOC_MAX_SOURCES;

// ~1 MB, held by every GPU that loads the library until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

// Device addresses of the fixed scratch per device (the array's name is only a host-side
// handle in host code; passing it to a kernel would address the wrong memory).
static std::mutex g_na_mu;
static void* g_na_addr[256] = {};

static int noalloc_scratch(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(nullptr, EIK_ERR_CUDA, "cudaGetDevice failed: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= 256) return fail(nullptr, EIK_ERR_CUDA, "device index %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_na_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(nullptr, EIK_ERR_CUDA, "cudaGetSymbolAddress of the fixed scratch failed: %s",
                  cudaGetErrorString(e));
    g_na_addr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_na_addr[dev]);
  return EIK_OK;
}

// One thread per source, receivers in order: Σ_r (pick - obs)² / σ², the pick being the
// reference's bilinear / trilinear receiver interpolation (eikforward2D.jl:17-87,
// eikforward3D.jl:17-140; corner (i+1,j,k+1) weighted xd*(1-yd)*(1-zd) as there).
// A receiver outside the grid sets the error word (checksrcrecposition, eikchecks.jl:4-50).
__global__ void noalloc_misfit_sources_kernel(GridDesc g, int nsrc, const double* tt, long long N,
                                              const long long* recoff, const double* rec, const double* pickobs,
                                              const double* stdobs, double* part, unsigned int* err) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsrc) return;
  const double* t = tt + (size_t)s * N;
  double m = 0.0;
  for (long long r = recoff[s]; r < recoff[s + 1]; r++) {
    const double* p = rec + r * g.nd;
    bool inside = true;
    for (int d = 0; d < g.nd; d++) {
      const double lo = jr_value(g.ax[d], 1), hi = jr_value(g.ax[d], g.n[d]);
      if (!(lo <= p[d] && p[d] <= hi)) inside = false;
    }
    if (!inside) {
      atomicOr(err, 1u);
      continue;
    }
    double pick;
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
      pick = t[a] * (1.0 - xd) * (1.0 - yd) + t[a + 1] * (1.0 - yd) * xd + t[a + g.n[0]] * (1.0 - xd) * yd +
             t[a + g.n[0] + 1] * xd * yd;
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
      auto T = [&](int a, int b, int c) { return t[lin3(g, (int)i - 1 + a, (int)j - 1 + b, (int)k - 1 + c)]; };
      pick = T(0, 0, 0) * (1 - xd) * (1 - yd) * (1 - zd) + T(1, 0, 0) * xd * (1 - yd) * (1 - zd) +
             T(0, 1, 0) * (1 - xd) * yd * (1 - zd) + T(0, 0, 1) * (1 - xd) * (1 - yd) * zd +
             T(1, 1, 0) * xd * yd * (1 - zd) + T(0, 1, 1) * (1 - xd) * yd * zd +
             T(1, 0, 1) * xd * (1 - yd) * (1 - zd) + T(1, 1, 1) * xd * yd * zd;
    }
    const double pd = pick - pickobs[r];
    m += (pd * pd) / (stdobs[r] * stdobs[r]);
  }
  part[s] = m;
}

// 0.5 * Σ_s m_s in source order (eikttimemisfit, eikmaingrad.jl:1302-1328).
__global__ void noalloc_misfit_sum_kernel(int nsrc, const double* part, const unsigned int* err, double* out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  if (*err) return;
  double tot = 0.0;
  for (int s = 0; s < nsrc; s++) tot += 0.5 * part[s];
  *out = tot;
}

}  // namespace eik

using namespace eik;

extern "C" int eik_ttimemisfit_noalloc(const eik_grid* grd, int64_t nsrc, const double* ttgrids_dev,
                                       const int64_t* rec_off, const double* rec_dev, const double* pickobs_dev,
                                       const double* stdobs_dev, double* misfit_dev, void* stream) {
  GridDesc g;
  int rc = make_griddesc(nullptr, grd, &g);
  if (rc) return rc;
  if (nsrc < 1) return fail(nullptr, EIK_ERR_ASSERT, "nsrc >= 1");
  if (nsrc > NOALLOC_MAX_SOURCES)
    return fail(nullptr, EIK_ERR_OUT_OF_BUDGET,
                "eik_ttimemisfit_noalloc: %lld sources exceed its fixed scratch of %lld sources; "
                "split the call or use eik_traveltime", (long long)nsrc, (long long)NOALLOC_MAX_SOURCES);
  if (!ttgrids_dev || !rec_off || !misfit_dev) return fail(nullptr, EIK_ERR_ASSERT, "NULL argument");
  if (rec_off[0] != 0) return fail(nullptr, EIK_ERR_ASSERT, "rec_off[0] must be 0");
  for (int64_t s = 0; s < nsrc; s++)
    if (rec_off[s + 1] < rec_off[s]) return fail(nullptr, EIK_ERR_ASSERT, "rec_off must be non-decreasing");
  if (rec_off[nsrc] > 0 && (!rec_dev || !pickobs_dev || !stdobs_dev))
    return fail(nullptr, EIK_ERR_ASSERT, "NULL argument");
  unsigned char* base = nullptr;
  rc = noalloc_scratch(&base);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned int* err = reinterpret_cast<unsigned int*>(base + NA_ERR_OFF);
  long long* d_off = reinterpret_cast<long long*>(base + NA_RECOFF_OFF);
  double* part = reinterpret_cast<double*>(base + NA_PART_OFF);
  // the error word must start at zero; offsets and partial sums are fully rewritten
  CUDA_OK(nullptr, cudaMemsetAsync(err, 0, sizeof(unsigned int), st));
  CUDA_OK(nullptr, cudaMemcpyAsync(d_off, rec_off, sizeof(long long) * (size_t)(nsrc + 1), cudaMemcpyHostToDevice, st));
  const int T = 128;
  noalloc_misfit_sources_kernel<<<(int)((nsrc + T - 1) / T), T, 0, st>>>(g, (int)nsrc, ttgrids_dev, npts(g), d_off,
                                                                        rec_dev, pickobs_dev, stdobs_dev, part, err);
  noalloc_misfit_sum_kernel<<<1, 1, 0, st>>>((int)nsrc, part, err, misfit_dev);
  CUDA_OK(nullptr, cudaGetLastError());
  unsigned int herr = 0;
  CUDA_OK(nullptr, cudaMemcpyAsync(&herr, err, sizeof herr, cudaMemcpyDeviceToHost, st));
  CUDA_OK(nullptr, cudaStreamSynchronize(st));
  if (herr) return fail(nullptr, EIK_ERR_ASSERT, "a receiver position is outside the grid");
  return EIK_OK;
}
