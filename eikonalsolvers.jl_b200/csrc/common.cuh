// Shared device/host definitions of libeikcuda: grid descriptor, Julia-range node
// coordinates, source-box geometry and small numeric helpers.
//
// Layout in HBM: every per-node array is column-major with x fastest, matching the
// reference's Julia arrays (cart2lin, src/EikSolv/eikutils.jl:6-19): l = i + n1*(j + n2*k)
// with 0-based (i, j, k).
#pragma once

#include <cstdint>
#include <math.h>

#include "stencil.cuh"

namespace eik {

enum GridKind : int32_t { G2DCART = 0, G3DCART = 1, G2DSPH = 2, G3DSPH = 3 };

// Float64 Base.range(start=a, step=st, length=n)[i]: rational start/step are evaluated as
// the correctly rounded (start_n + (i-1)*step_n)/den, others as a + (i-1)*st rounded once
// from double-double.
struct JRange {
  double a, st;
  long long sn, tn, den;
  int32_t rational;
  int32_t pad;
};

EIK_HD double jr_value(const JRange& r, long long i1) {
  if (r.rational) {
    const long long num = r.sn + (i1 - 1) * r.tn;
    return (double)num / (double)r.den;
  }
  const double u = (double)(i1 - 1);
  const double p = u * r.st;
  const double pe = fma(u, r.st, -p);
  const double s = r.a + p;
  const double bb = s - r.a;
  const double se = (r.a - (s - bb)) + (p - bb);
  return s + (se + pe);
}

struct GridDesc {
  int32_t kind, nd;
  int32_t n[3];      // 1 for unused axes
  int32_t pad;
  double spac[3];    // hgrid on every axis (Cartesian) or (Δr, Δθ°, Δφ°)
  double co[3];      // cooinit
  JRange ax[3];
};

EIK_HD bool is_cart(const GridDesc& g) { return g.kind == G2DCART || g.kind == G3DCART; }
EIK_HD long long npts(const GridDesc& g) { return (long long)g.n[0] * g.n[1] * g.n[2]; }
EIK_HD long long lin3(const GridDesc& g, int i, int j, int k) {
  return (long long)i + (long long)g.n[0] * ((long long)j + (long long)g.n[1] * k);
}
constexpr double DEG2RAD = 3.141592653589793 / 180.0;  // deg2rad(x) = x*(π/180)

// Node spacing per axis at radial index i (0-based) (eikforward2D.jl:115-119,
// eikforward3D.jl:168-172: no sinθ factor on the φ axis).
EIK_HD void node_dh(const GridDesc& g, int i, double* dh) {
  if (is_cart(g)) {
    dh[0] = dh[1] = dh[2] = g.spac[0];
  } else {
    const double r = jr_value(g.ax[0], i + 1);
    dh[0] = g.spac[0];
    dh[1] = r * (g.spac[1] * DEG2RAD);
    dh[2] = (g.nd == 3) ? r * (g.spac[2] * DEG2RAD) : 0.0;
  }
}

// ------------------------------------------------------------- source box helpers --
// Base.rem / div for Float64 (findenclosingbox uses divrem).
EIK_HD double jl_div(double x, double y) {
  const double r = fmod(x, y);
  return nearbyint((x - r) / y);
}

// Degree sine/cosine with exact reduction by quarter turns (cosd/sind).
EIK_HD void sincosd(double x, double* s, double* c) {
  double r = fmod(x, 360.0);
  if (r < 0) r += 360.0;
  const int q = (int)floor((r + 45.0) / 90.0);
  const double y = (r - 90.0 * q) * DEG2RAD;
  const double sy = sin(y), cy = cos(y);
  switch (q & 3) {
    case 0: *s = sy; *c = cy; break;
    case 1: *s = cy; *c = -sy; break;
    case 2: *s = -sy; *c = -cy; break;
    default: *s = -cy; *c = sy; break;
  }
}

// distance2points (eikutils.jl:47-73); Grid3DSphere as chord length via
// sphericaldeg2cartesian (utils.jl:344-349) (the reference errors there).
EIK_HD double distance2points(const GridDesc& g, const double* a, const double* b) {
  if (is_cart(g)) {
    double s = 0.0;
    for (int d = 0; d < g.nd; d++) {
      const double t = a[d] - b[d];
      s = (d == 0) ? t * t : s + t * t;
    }
    return sqrt(s);
  }
  if (g.kind == G2DSPH) {
    double sn, cs;
    sincosd(a[1] - b[1], &sn, &cs);
    return sqrt((a[0] * a[0] + b[0] * b[0]) - ((2.0 * a[0]) * b[0]) * cs);
  }
  double s1t, c1t, s1p, c1p, s2t, c2t, s2p, c2p;
  sincosd(a[1], &s1t, &c1t);
  sincosd(a[2], &s1p, &c1p);
  sincosd(b[1], &s2t, &c2t);
  sincosd(b[2], &s2p, &c2p);
  const double x1 = a[0] * s1t * c1p, y1 = a[0] * s1t * s1p, z1 = a[0] * c1t;
  const double x2 = b[0] * s2t * c2p, y2 = b[0] * s2t * s2p, z2 = b[0] * c2t;
  const double dx = x1 - x2, dy = y1 - y2, dz = z1 - z2;
  return sqrt((dx * dx + dy * dy) + dz * dz);
}

// findenclosingbox (eikmainfwd.jl:1114-1186): 1 corner when the point is on a node
// (all remainders within 1e-8), else 2^nd corners in the reference's order. Corners are
// 0-based (i,j,k). Returns the number of corners.
EIK_HD int findenclosingbox(const GridDesc& g, const double* x, int (*corn)[3]) {
  int ijk[3] = {0, 0, 0};
  bool onnode = true;
  for (int d = 0; d < g.nd; d++) {
    const double dx = x[d] - g.co[d];
    const double q = jl_div(dx, g.spac[d]);
    const double rem = fmod(dx, g.spac[d]);
    ijk[d] = (int)floor(q);  // 0-based (reference: floor+1, 1-based)
    if (ijk[d] < 0) ijk[d] = 0;                  // positions are validated to lie inside the
    if (ijk[d] > g.n[d] - 1) ijk[d] = g.n[d] - 1;  // grid; the clamp only guards rounding
    if (!(fabs(rem) <= 1e-8)) onnode = false;
  }
  if (onnode) {
    corn[0][0] = ijk[0];
    corn[0][1] = ijk[1];
    corn[0][2] = ijk[2];
    return 1;
  }
  for (int d = 0; d < g.nd; d++)
    if (ijk[d] == g.n[d] - 1) ijk[d] -= 1;
  if (g.nd == 2) {
    const int o[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};
    for (int l = 0; l < 4; l++) {
      corn[l][0] = ijk[0] + o[l][0];
      corn[l][1] = ijk[1] + o[l][1];
      corn[l][2] = 0;
    }
    return 4;
  }
  const int o[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                       {1, 1, 0}, {0, 1, 1}, {1, 0, 1}, {1, 1, 1}};
  for (int l = 0; l < 8; l++)
    for (int d = 0; d < 3; d++) corn[l][d] = ijk[d] + o[l][d];
  return 8;
}

// Julia Base.rat (twiceprecision.jl) and range construction, usable on device to build the
// fine grid's coordinate ranges.
EIK_HD void jl_rat(double x, long long* num, long long* den) {
  double y = x;
  long long a = 1, d = 1, b = 0, c = 0;
  const double m = 16777216.0;
  const long long mi = 16777216;
  while (fabs(y) <= m) {
    const long long f = (long long)trunc(y);
    y -= (double)f;
    const long long an = f * a + c;
    c = a;
    a = an;
    const long long bn = f * b + d;
    d = b;
    b = bn;
    const long long aa = a < 0 ? -a : a, ab = b < 0 ? -b : b;
    if (!((aa > ab ? aa : ab) <= mi)) {
      *num = c;
      *den = d;
      return;
    }
    if ((double)a / (double)b == x) break;
    y = 1.0 / y;
  }
  *num = a;
  *den = b;
}
EIK_HD long long gcdll(long long a, long long b) {
  a = a < 0 ? -a : a;
  b = b < 0 ? -b : b;
  while (b) {
    const long long t = a % b;
    a = b;
    b = t;
  }
  return a;
}
EIK_HD JRange make_jrange(double a, double st) {
  JRange r;
  r.a = a;
  r.st = st;
  r.sn = 0;
  r.tn = 0;
  r.den = 1;
  r.rational = 0;
  r.pad = 0;
  long long sn, sd, tn, td;
  jl_rat(a, &sn, &sd);
  jl_rat(st, &tn, &td);
  if (sd != 0 && td != 0 && (double)sn / (double)sd == a && (double)tn / (double)td == st) {
    const long long den = sd / gcdll(sd, td) * td;
    const double m = 9007199254740992.0;
    if (fabs((double)den * a) <= m && fabs((double)den * st) <= m && den % sd == 0 && den % td == 0) {
      r.rational = 1;
      r.den = den;
      r.sn = sn * (den / sd);
      r.tn = tn * (den / td);
    }
  }
  return r;
}

// ------------------------------------------------------------------ error words --
enum ErrBits : uint32_t {
  ERRB_NOT_CONVERGED = 1u << 0,
  ERRB_QUEUE_TIMEOUT = 1u << 1,
  ERRB_HEAP_OVERFLOW = 1u << 2,
  ERRB_BATCH_OVERFLOW = 1u << 3,   // more than 128 equal minima popped at once
  ERRB_SEED_OVERFLOW = 1u << 4,
  ERRB_ADJ_NOT_CONVERGED = 1u << 5,
  ERRB_SINGULAR = 1u << 6,
};
enum WarnBits : uint32_t {
  WARN_NEG_DISCRIMINANT = 1u << 0,
  WARN_SRC_HALFWAY_SHIFT = 1u << 1,
  WARN_BORDER_BEFORE_COARSE = 1u << 2,
  WARN_SRCPOS_ALIGNED_SHIFT = 1u << 3,
  WARN_SRC_ON_NODE_DERIV = 1u << 4,
  WARN_FINE_NO_TRIGGER = 1u << 5,
};

}  // namespace eik
