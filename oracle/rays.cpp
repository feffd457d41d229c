// Oracle of tracerays / tracerays_singlesrc (src/EikSolv/eikutils.jl:201-328). TEST
// INFRASTRUCTURE ONLY (see eikoracle.hpp).
//
// The reference interpolates each traveltime grid with Interpolations.jl's
// `scale(interpolate(ttime, BSpline(Cubic())), axes...)` (eikutils.jl:230-246) and
// follows -grad(T) from each receiver in steps of steplen*h (steplen on Grid2DSphere)
// until the ray is within h*sqrt(2) (Δr*sqrt(2)) of the source (eikutils.jl:262-323).
// Interpolations.jl is a dependency that is not vendored and has no version pin in the
// reference's Project.toml; this file restates its published cubic B-spline algorithm:
//  * `Cubic()` is `Cubic(Line(OnGrid()))`: the coefficient array is padded by one node on
//    each side; the interior rows are c[i-1]/6 + 2c[i]/3 + c[i+1]/6 = A[i], the two
//    boundary rows c[0] - 2c[1] + c[2] = 0 and c[n+1] - 2c[n] + c[n-1] = 0 (zero second
//    difference). Substituting the boundary rows into the first and last interior rows
//    gives c[1] = A[1] and c[n] = A[n] exactly, so each line is a tridiagonal system for
//    c[2..n-1] with constant diagonals (1/6, 2/3, 1/6), solved here by the Thomas
//    algorithm, axis after axis (the B-spline tensor product is separable);
//  * evaluation at index coordinate u = (x - x0)/Δ + 1 uses the four coefficients
//    ix-1..ix+2 around ix = clamp(floor(u), 1, n-1) with the cubic B-spline weights of
//    δ = u - ix; the gradient w.r.t. a coordinate takes the derivative weights along that
//    axis divided by its spacing.
// The algebra is exact; its floating-point rounding is this restatement's (the reference's
// LU + Woodbury solve rounds differently), so parity with Julia is at rounding level, not
// bitwise. The GPU kernels follow the operations of this file one for one.
#include <cmath>
#include <vector>

#include "eikoracle.hpp"

namespace eikor {

namespace {

struct Spline {
  int nd = 2;
  i64 n[3] = {1, 1, 1};  // data nodes per axis
  i64 m[3] = {1, 1, 1};  // padded: n + 2 on the interpolated axes
  std::vector<double> c;
  i64 at(i64 q0, i64 q1, i64 q2) const { return q0 + m[0] * (q1 + m[1] * q2); }
};

// Thomas sweep factors of the constant-diagonal system (1/6, 2/3, 1/6) of size k.
std::vector<double> thomas_factors(i64 k) {
  std::vector<double> cp((size_t)std::max<i64>(k, 1));
  const double a = 1.0 / 6.0, b = 2.0 / 3.0, cc = 1.0 / 6.0;
  if (k > 0) cp[0] = cc / b;
  for (i64 i = 1; i < k; i++) cp[(size_t)i] = cc / (b - a * cp[(size_t)(i - 1)]);
  return cp;
}

// One line of n data values at c[s], c[s+st], ... (padded positions 1..n); writes the
// padded coefficients 0..n+1.
void prefilter_line(double* c, i64 st, i64 n, const std::vector<double>& cp, std::vector<double>& dp) {
  const double a = 1.0 / 6.0, b = 2.0 / 3.0;
  const i64 k = n - 2;  // unknowns c[2..n-1]
  if (k > 0) {
    // right-hand sides with the known ends moved over
    for (i64 i = 0; i < k; i++) {
      double d = c[(i + 2) * st];
      if (i == 0) d = d - a * c[1 * st];
      if (i == k - 1) d = d - a * c[n * st];
      dp[(size_t)i] = (i == 0) ? d / b : (d - a * dp[(size_t)(i - 1)]) / (b - a * cp[(size_t)(i - 1)]);
    }
    c[(k + 1) * st] = dp[(size_t)(k - 1)];
    for (i64 i = k - 2; i >= 0; i--) c[(i + 2) * st] = dp[(size_t)i] - cp[(size_t)i] * c[(i + 3) * st];
  }
  c[0] = 2.0 * c[1 * st] - c[2 * st];
  c[(n + 1) * st] = 2.0 * c[n * st] - c[(n - 1) * st];
}

Spline make_spline(const Grid& g, const double* tt) {
  Spline S;
  S.nd = g.nd;
  for (int d = 0; d < 3; d++) {
    S.n[d] = g.n[d];
    S.m[d] = (d < g.nd) ? g.n[d] + 2 : 1;
  }
  S.c.assign((size_t)(S.m[0] * S.m[1] * S.m[2]), 0.0);
  const i64 off2 = g.nd == 3 ? 1 : 0;
  for (i64 k = 0; k < g.n[2]; k++)
    for (i64 j = 0; j < g.n[1]; j++)
      for (i64 i = 0; i < g.n[0]; i++)
        S.c[(size_t)S.at(i + 1, j + 1, k + off2)] = tt[i + g.n[0] * (j + g.n[1] * k)];
  std::vector<double> dp;
  for (int ax = 0; ax < g.nd; ax++) {
    const i64 n = g.n[ax];
    const std::vector<double> cp = thomas_factors(n - 2);
    dp.assign((size_t)std::max<i64>(n, 1), 0.0);
    const i64 st = ax == 0 ? 1 : (ax == 1 ? S.m[0] : S.m[0] * S.m[1]);
    // every line along ax (all padded positions of the other axes: the pads of the axes
    // already filtered are lines too)
    for (i64 q2 = 0; q2 < S.m[2]; q2++)
      for (i64 q1 = 0; q1 < S.m[1]; q1++)
        for (i64 q0 = 0; q0 < S.m[0]; q0++) {
          const i64 q[3] = {q0, q1, q2};
          if (q[ax] != 0) continue;
          bool inner = true;  // axes not yet filtered: only the data positions
          for (int d = ax + 1; d < g.nd; d++)
            if (q[d] < 1 || q[d] > g.n[d]) inner = false;
          if (!inner) continue;
          prefilter_line(S.c.data() + S.at(q0, q1, q2), st, n, cp, dp);
        }
  }
  return S;
}

// Cubic B-spline weights (value) and their derivatives at offset δ in [0, 1].
void bweights(double dl, double* w, double* dw) {
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

// Interpolations.gradient(itp, x...) of the scaled interpolant.
void spline_gradient(const Spline& S, const Grid& g, const double* x, double* grad) {
  i64 ix[3] = {1, 1, 1};
  double w[3][4], dw[3][4];
  for (int d = 0; d < g.nd; d++) {
    const double u = (x[d] - g.cooinit[d]) / g.spac[d] + 1.0;
    i64 i = (i64)std::floor(u);
    if (i < 1) i = 1;
    if (i > S.n[d] - 1) i = S.n[d] - 1;
    ix[d] = i;
    bweights(u - (double)i, w[d], dw[d]);
  }
  for (int gd = 0; gd < g.nd; gd++) {
    double acc = 0.0;
    if (g.nd == 2) {
      for (int b = 0; b < 4; b++) {
        const double wb = (gd == 1) ? dw[1][b] : w[1][b];
        double row = 0.0;
        for (int a = 0; a < 4; a++) {
          const double wa = (gd == 0) ? dw[0][a] : w[0][a];
          row = row + wa * S.c[(size_t)S.at(ix[0] - 1 + a, ix[1] - 1 + b, 0)];
        }
        acc = acc + wb * row;
      }
    } else {
      for (int cc = 0; cc < 4; cc++) {
        const double wc = (gd == 2) ? dw[2][cc] : w[2][cc];
        double plane = 0.0;
        for (int b = 0; b < 4; b++) {
          const double wb = (gd == 1) ? dw[1][b] : w[1][b];
          double row = 0.0;
          for (int a = 0; a < 4; a++) {
            const double wa = (gd == 0) ? dw[0][a] : w[0][a];
            row = row + wa * S.c[(size_t)S.at(ix[0] - 1 + a, ix[1] - 1 + b, ix[2] - 1 + cc)];
          }
          plane = plane + wb * row;
        }
        acc = acc + wc * plane;
      }
    }
    grad[gd] = acc / g.spac[gd];
  }
}

double dist2pts(const Grid& g, const double* a, const double* b) {
  if (g.cart()) {
    double s = 0.0;
    for (int d = 0; d < g.nd; d++) {
      const double t = a[d] - b[d];
      s = (d == 0) ? t * t : s + t * t;
    }
    return std::sqrt(s);
  }
  // Grid2DSphere, degrees (eikutils.jl:54-65)
  return std::sqrt((a[0] * a[0] + b[0] * b[0]) - ((2.0 * a[0]) * b[0]) * cosd(a[1] - b[1]));
}

constexpr double RAD2DEG = 180.0 / 3.141592653589793;  // rad2deg(x) = x*(180/π)

// One step from pt (eikutils.jl:274-309), written into nw.
void ray_step(const Spline& S, const Grid& g, double rstep, const double* pt, double* nw) {
  double gr[3];
  spline_gradient(S, g, pt, gr);
  if (g.cart()) {
    double s = 0.0;
    for (int d = 0; d < g.nd; d++) s = (d == 0) ? gr[d] * gr[d] : s + gr[d] * gr[d];
    const double nrm = std::sqrt(s);
    for (int d = 0; d < g.nd; d++) nw[d] = pt[d] - rstep * (gr[d] / nrm);
  } else {
    const double rcur = pt[0];
    const double th = deg2rad(pt[1]);
    const double dfdx = std::cos(th) * gr[0] - (1.0 / rcur) * std::sin(th) * (gr[1] * RAD2DEG);
    const double dfdy = std::sin(th) * gr[0] + (1.0 / rcur) * std::cos(th) * (gr[1] * RAD2DEG);
    const double nrm = std::sqrt(dfdx * dfdx + dfdy * dfdy);
    const double px = pt[0] * cosd(pt[1]), py = pt[0] * sind(pt[1]);
    const double nx = px - rstep * (dfdx / nrm), ny = py - rstep * (dfdy / nrm);
    nw[0] = std::sqrt(nx * nx + ny * ny);
    nw[1] = std::atan2(ny, nx) * RAD2DEG;
  }
  for (int d = 0; d < g.nd; d++) {
    const double lo = g.cooinit[d], hi = g.ax[d].last();
    if (nw[d] < lo) nw[d] = lo;
    else if (nw[d] > hi) nw[d] = hi;
  }
}

}  // namespace

// tracerays (eikutils.jl:201-213): rays of every receiver of every source, concatenated
// (points row-major, nd values each); npts[r] = points of ray r (receivers in recoff order).
void tracerays(const Grid& g, const double* ttgrids, i64 nsrc, const double* coordsrc, const i64* recoff,
               const double* rec, double steplen, i64 max_steps, std::vector<i64>& npts, std::vector<double>& pts) {
  if (g.kind == G3DSPH) jl_error("tracerays_singlesrc(): ray tracing for spherical grids not yet implemented.");
  for (int d = 0; d < g.nd; d++)
    if (g.n[d] < 2) jl_error("tracerays: every grid axis needs at least 2 nodes");
  const double rstep = g.cart() ? steplen * g.spac[0] : steplen;
  const double thrdist = g.spac[0] * std::sqrt(2.0);
  const i64 N = g.npts();
  npts.assign((size_t)recoff[nsrc], 0);
  pts.clear();
  for (i64 s = 0; s < nsrc; s++) {
    const Spline S = make_spline(g, ttgrids + s * N);
    const double* src = coordsrc + s * g.nd;
    for (i64 r = recoff[s]; r < recoff[s + 1]; r++) {
      double pt[3] = {0, 0, 0}, nw[3] = {0, 0, 0};
      for (int d = 0; d < g.nd; d++) pt[d] = rec[r * g.nd + d];
      const size_t start = pts.size();
      for (int d = 0; d < g.nd; d++) pts.push_back(pt[d]);
      double dist = dist2pts(g, pt, src);
      i64 np = 1;
      while (dist >= thrdist) {
        if (np > max_steps) jl_error("tracerays: ray did not reach the source within the step limit");
        ray_step(S, g, rstep, pt, nw);
        for (int d = 0; d < g.nd; d++) {
          pt[d] = nw[d];
          pts.push_back(nw[d]);
        }
        dist = dist2pts(g, pt, src);
        np++;
      }
      // the last point is the source (eikutils.jl:319)
      for (int d = 0; d < g.nd; d++) pts[start + (size_t)((np - 1) * g.nd + d)] = src[d];
      npts[(size_t)r] = np;
    }
  }
}

}  // namespace eikor
