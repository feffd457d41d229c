// Ray tracing (tracerays, src/EikSolv/eikutils.jl:201-328): the per-line and per-ray work
// of the kernels in rays.cu as host/device functions, so that the same code also runs on
// the host (its tests compile it with the address and alignment sanitizers).
//
// Interpolant: Interpolations.jl's `BSpline(Cubic())` = `Cubic(Line(OnGrid()))` on the
// grid axes. Padded coefficients (one node more on each side of every axis); with the Line
// boundary rows (zero second difference at both ends) the first and last coefficients of a
// line equal the data and the interior ones solve the constant tridiagonal system
// (1/6, 2/3, 1/6); each axis is filtered in turn, one line at a time, by a Thomas sweep in
// place (the sweep factors depend only on the position along the line and come from the
// host). Evaluation takes the 4^d coefficients around clamp(floor(u), 1, n-1) with the cubic
// B-spline weights; the gradient uses the derivative weights along its axis divided by the
// spacing.
#pragma once

#include <cstddef>
#include <cstdint>

#include "common.cuh"

#if defined(__CUDA_ARCH__)
#define RAY_LD(p) __ldg(p)
#define RAY_OR(p, v) atomicOr((p), (v))
#else
#define RAY_LD(p) (*(p))
#define RAY_OR(p, v) (*(p) |= (v))
#endif

namespace eik {

constexpr uint32_t ERRB_RAY_STEPS = 1u << 20;
constexpr uint32_t ERRB_RAY_ADDR = 1u << 21;  // an address check failed (the access was skipped)

// p[0..count) lies inside [base, base + size) and p is aligned for T.
template <typename T>
EIK_HD bool ray_span_ok(const T* p, long long count, const T* base, long long size) {
  return p >= base && count >= 0 && p + count <= base + size &&
         ((unsigned long long)(uintptr_t)p % alignof(T)) == 0;
}

struct SplineArgs {
  int nd;
  long long n[3], m[3];
  long long cstride;  // coefficients per source
  int nsrc;
  double* coef;
  long long coef_size;  // doubles at coef (nsrc * cstride)
  const double* cp[3];  // Thomas factors per axis (n[a]-2 values)
  uint32_t* err;
};

// Data value q (source-major, column-major grid) into its padded coefficient position.
EIK_HD void spline_load_one(const SplineArgs& s, const double* tt, long long N, long long q) {
  const long long src = q / N, l = q - src * N;
  const long long i = l % s.n[0], j = (l / s.n[0]) % s.n[1], k = l / (s.n[0] * s.n[1]);
  const long long k1 = s.nd == 3 ? k + 1 : 0;
  double* dst = s.coef + src * s.cstride + (i + 1) + s.m[0] * ((j + 1) + s.m[1] * k1);
  if (!ray_span_ok<double>(dst, 1, s.coef, s.coef_size)) {
    RAY_OR(s.err, ERRB_RAY_ADDR);
    return;
  }
  *dst = tt[q];
}

// Lines along axis ax: every padded position of the axes before ax (already filtered, pads
// included) and the data positions of the axes after it; per source.
EIK_HD long long spline_lines(const SplineArgs& s, int ax, long long* cnt) {
  for (int d = 0; d < 3; d++) {
    if (d == ax || d >= s.nd) cnt[d] = 1;
    else cnt[d] = d < ax ? s.m[d] : s.n[d];
  }
  return cnt[0] * cnt[1] * cnt[2];
}

// The Thomas sweep of line q (of lines * nsrc) along axis ax, in place.
EIK_HD void spline_line(const SplineArgs& s, int ax, const double* cp, long long q) {
  long long cnt[3];
  const long long lines = spline_lines(s, ax, cnt);
  const long long n = s.n[ax];
  const long long st = ax == 0 ? 1 : (ax == 1 ? s.m[0] : s.m[0] * s.m[1]);
  const double a = 1.0 / 6.0, b = 2.0 / 3.0;
  const long long src = q / lines, li = q - src * lines;
  long long p[3] = {li % cnt[0], (li / cnt[0]) % cnt[1], li / (cnt[0] * cnt[1])};
  for (int d = ax + 1; d < s.nd; d++) p[d] += 1;  // data positions of the later axes
  p[ax] = 0;
  if (s.nd == 2) p[2] = 0;
  double* c = s.coef + src * s.cstride + p[0] + s.m[0] * (p[1] + s.m[1] * p[2]);
  if (!ray_span_ok<double>(c, 1, s.coef, s.coef_size) || !ray_span_ok<double>(c + (n + 1) * st, 1, s.coef, s.coef_size)) {
    RAY_OR(s.err, ERRB_RAY_ADDR);
    return;
  }
  const long long k = n - 2;
  if (k > 0) {
    double prev = 0.0;
    for (long long i = 0; i < k; i++) {
      double d = c[(i + 2) * st];
      if (i == 0) d = d - a * c[1 * st];
      if (i == k - 1) d = d - a * c[n * st];
      prev = (i == 0) ? d / b : (d - a * prev) / (b - a * cp[i - 1]);
      c[(i + 2) * st] = prev;
    }
    for (long long i = k - 2; i >= 0; i--) c[(i + 2) * st] = c[(i + 2) * st] - cp[i] * c[(i + 3) * st];
  }
  c[0] = 2.0 * c[1 * st] - c[2 * st];
  c[(n + 1) * st] = 2.0 * c[n * st] - c[(n - 1) * st];
}

struct RayArgs {
  GridDesc g;
  int nsrc;
  long long m[3], cstride;
  long long coef_size;   // doubles at coef
  long long pts_size;    // doubles at pts (second pass)
  const double* coef;
  const double* coordsrc;
  const long long* recoff;
  const double* rec;
  double rstep, thrdist;
  long long max_steps;
  const long long* outoff;  // writing: first point of every ray
  const long long* cap;     // writing: room (points) of every ray at outoff
  long long* npts;          // points of every ray
  double* pts;
  uint32_t* err;
};

EIK_HD void bweights(double dl, double* w, double* dw) {
  const double om = 1.0 - dl;
  w[0] = (om * om * om) / 6.0;
  w[1] = 2.0 / 3.0 - dl * dl + (dl * dl * dl) / 2.0;
  w[2] = 2.0 / 3.0 - om * om + (om * om * om) / 2.0;
  w[3] = (dl * dl * dl) / 6.0;
  dw[0] = -(om * om) / 2.0;
  dw[1] = 1.5 * (dl * dl) - 2.0 * dl;
  dw[2] = 2.0 * om - 1.5 * (om * om);
  dw[3] = (dl * dl) / 2.0;
}

template <int ND>
EIK_HD bool spline_gradient(const RayArgs& a, const double* c, const double* x, double* grad) {
  long long ix[3] = {1, 1, 1};
  double w[3][4], dw[3][4];
  for (int d = 0; d < ND; d++) {
    const double u = (x[d] - a.g.co[d]) / a.g.spac[d] + 1.0;
    const double fu = floor(u);
    // clamp in floating point first: the conversion of a value out of range is undefined
    long long i = fu < 1.0 ? 1 : (fu > (double)(a.g.n[d] - 1) ? (long long)(a.g.n[d] - 1) : (long long)fu);
    ix[d] = i;
    bweights(u - (double)i, w[d], dw[d]);
  }
  // every coefficient is loaded once; each gradient component keeps its own row / plane /
  // total sums, accumulated in the same order as a component-by-component evaluation
  double acc[3] = {0.0, 0.0, 0.0};
  if (ND == 2) {
    for (int bb = 0; bb < 4; bb++) {
      const double* crow = c + (ix[0] - 1) + a.m[0] * (ix[1] - 1 + bb);
      if (!ray_span_ok<double>(crow, 4, a.coef, a.coef_size)) return false;
      double row[2] = {0.0, 0.0};
      for (int aa = 0; aa < 4; aa++) {
        const double cv = RAY_LD(crow + aa);
        row[0] = row[0] + dw[0][aa] * cv;
        row[1] = row[1] + w[0][aa] * cv;
      }
      acc[0] = acc[0] + w[1][bb] * row[0];
      acc[1] = acc[1] + dw[1][bb] * row[1];
    }
  } else {
    for (int cc = 0; cc < 4; cc++) {
      double plane[3] = {0.0, 0.0, 0.0};
      for (int bb = 0; bb < 4; bb++) {
        const double* crow = c + (ix[0] - 1) + a.m[0] * ((ix[1] - 1 + bb) + a.m[1] * (ix[2] - 1 + cc));
        if (!ray_span_ok<double>(crow, 4, a.coef, a.coef_size)) return false;
        double rd = 0.0, rw = 0.0;  // rows with the derivative / value weights along x
        for (int aa = 0; aa < 4; aa++) {
          const double cv = RAY_LD(crow + aa);
          rd = rd + dw[0][aa] * cv;
          rw = rw + w[0][aa] * cv;
        }
        plane[0] = plane[0] + w[1][bb] * rd;
        plane[1] = plane[1] + dw[1][bb] * rw;
        plane[2] = plane[2] + w[1][bb] * rw;
      }
      acc[0] = acc[0] + w[2][cc] * plane[0];
      acc[1] = acc[1] + w[2][cc] * plane[1];
      acc[2] = acc[2] + dw[2][cc] * plane[2];
    }
  }
  for (int gd = 0; gd < ND; gd++) grad[gd] = acc[gd] / a.g.spac[gd];
  return true;
}

constexpr double RAD2DEG = 180.0 / 3.141592653589793;  // rad2deg(x) = x*(180/π)

// One step from pt (eikutils.jl:274-309), into nw, clamped into the grid.
template <int ND>
EIK_HD bool ray_step(const RayArgs& a, const double* c, const double* pt, double* nw) {
  double gr[3] = {0.0, 0.0, 0.0};
  if (!spline_gradient<ND>(a, c, pt, gr)) return false;
  if (is_cart(a.g)) {
    double s = 0.0;
    for (int d = 0; d < ND; d++) s = (d == 0) ? gr[d] * gr[d] : s + gr[d] * gr[d];
    const double nrm = sqrt(s);
    for (int d = 0; d < ND; d++) nw[d] = pt[d] - a.rstep * (gr[d] / nrm);
  } else {  // Grid2DSphere (eikutils.jl:284-303)
    const double rcur = pt[0];
    const double th = pt[1] * DEG2RAD;
    const double dfdx = cos(th) * gr[0] - (1.0 / rcur) * sin(th) * (gr[1] * RAD2DEG);
    const double dfdy = sin(th) * gr[0] + (1.0 / rcur) * cos(th) * (gr[1] * RAD2DEG);
    const double nrm = sqrt(dfdx * dfdx + dfdy * dfdy);
    double sn, cs;
    sincosd(pt[1], &sn, &cs);
    const double px = pt[0] * cs, py = pt[0] * sn;
    const double nx = px - a.rstep * (dfdx / nrm), ny = py - a.rstep * (dfdy / nrm);
    nw[0] = sqrt(nx * nx + ny * ny);
    nw[1] = atan2(ny, nx) * RAD2DEG;
  }
  for (int d = 0; d < ND; d++) {
    const double lo = a.g.co[d], hi = jr_value(a.g.ax[d], a.g.n[d]);
    if (nw[d] < lo) nw[d] = lo;
    else if (nw[d] > hi) nw[d] = hi;
  }
  return true;
}

// Ray r: counts its points into npts[r] and, when write is set, writes those that fit in
// its room cap[r] at outoff[r] (a ray longer than its room is counted in full; the caller
// traces it again with enough room).
template <int ND>
EIK_HD void trace_one(const RayArgs& a, long long r, int write) {
  int s = 0;
  while (s < a.nsrc && a.recoff[s + 1] <= r) s++;
  if (s >= a.nsrc) {
    RAY_OR(a.err, ERRB_RAY_ADDR);
    return;
  }
  const double* c = a.coef + (long long)s * a.cstride;
  const double* src = a.coordsrc + (long long)s * ND;
  double pt[3] = {0.0, 0.0, 0.0}, nw[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < ND; d++) pt[d] = a.rec[r * ND + d];
  double* out = nullptr;
  const long long room = write ? a.cap[r] : 0;
  if (write && room > 0) {
    out = a.pts + a.outoff[r] * ND;
    if (!ray_span_ok<double>(out, room * ND, a.pts, a.pts_size)) {
      RAY_OR(a.err, ERRB_RAY_ADDR);
      return;
    }
    for (int d = 0; d < ND; d++) out[d] = pt[d];
  }
  double dist = distance2points(a.g, pt, src);
  long long np = 1;
  while (dist >= a.thrdist) {
    if (np > a.max_steps) {
      RAY_OR(a.err, ERRB_RAY_STEPS);
      break;
    }
    if (!ray_step<ND>(a, c, pt, nw)) {
      RAY_OR(a.err, ERRB_RAY_ADDR);
      return;
    }
    for (int d = 0; d < ND; d++) {
      pt[d] = nw[d];
      if (np < room) out[np * ND + d] = nw[d];
    }
    dist = distance2points(a.g, pt, src);
    np++;
  }
  if (np <= room) {  // the last point is the source (eikutils.jl:319)
    for (int d = 0; d < ND; d++) out[(np - 1) * ND + d] = src[d];
  }
  a.npts[r] = np;
}

}  // namespace eik
