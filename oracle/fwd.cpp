// Oracle forward path: grids, binary heap, local 2nd-order solver, source box,
// refined grid around the source, FMM core, receiver interpolation and the
// FMM-ordered derivative matrices. Test infrastructure only (see eikoracle.hpp).
#include "eikoracle.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <limits>

namespace eikor {

static const double HUGE_TT = std::numeric_limits<double>::infinity();  // typemax(Float64)

void jl_assert_fail(const std::string& what) { throw OracleError(1, "AssertionError: " + what); }
void jl_error(const std::string& what) { throw OracleError(2, what); }

// ------------------------------------------------------------------ Julia numerics --
// Base.rat (twiceprecision.jl): continued-fraction rational approximation bounded by
// maxintfloat(Float32).
static void jl_rat(double x, i64& num, i64& den) {
  double y = x;
  i64 a = 1, d = 1, b = 0, c = 0;
  const double m = 16777216.0;
  const i64 mi = 16777216;
  while (std::fabs(y) <= m) {
    i64 f = (i64)std::trunc(y);
    y -= (double)f;
    i64 an = f * a + c;
    c = a;
    a = an;
    i64 bn = f * b + d;
    d = b;
    b = bn;
    if (!(std::max(std::llabs(a), std::llabs(b)) <= mi)) {
      num = c;
      den = d;
      return;
    }
    if ((double)a / (double)b == x) break;
    y = 1.0 / y;
  }
  num = a;
  den = b;
}

static i64 gcd64(i64 a, i64 b) {
  a = std::llabs(a);
  b = std::llabs(b);
  while (b) {
    i64 t = a % b;
    a = b;
    b = t;
  }
  return a;
}

void JRange::init(double a_, double st_, i64 len_) {
  a = a_;
  st = st_;
  len = len_;
  rational = false;
  i64 sn, sd, tn, td;
  jl_rat(a, sn, sd);
  jl_rat(st, tn, td);
  if (sd != 0 && td != 0 && (double)sn / (double)sd == a && (double)tn / (double)td == st) {
    i64 den_ = sd / gcd64(sd, td) * td;
    const double m = 9007199254740992.0;  // maxintfloat(Float64)
    if (std::fabs((double)den_ * a) <= m && std::fabs((double)den_ * st) <= m && den_ % sd == 0 &&
        den_ % td == 0) {
      rational = true;
      den = den_;
      start_n = sn * (den_ / sd);
      step_n = tn * (den_ / td);
    }
  }
}

double JRange::operator()(i64 i1) const {
  if (rational) {
    __int128 num = (__int128)start_n + (__int128)(i1 - 1) * step_n;
    const __int128 lim = (__int128)1 << 53;
    if (num <= lim && num >= -lim) return (double)(i64)num / (double)den;
    return (double)((long double)num / (long double)den);
  }
  // a + (i-1)*st evaluated in double-double, then rounded once
  double u = (double)(i1 - 1);
  double p = u * st;
  double pe = std::fma(u, st, -p);
  double s = a + p;
  double bb = s - a;
  double se = (a - (s - bb)) + (p - bb);
  return s + (se + pe);
}

double jl_rem(double x, double y) { return std::fmod(x, y); }

double jl_mod(double x, double y) {
  double r = std::fmod(x, y);
  if (r == 0.0) return std::copysign(0.0, y);
  if ((r > 0) != (y > 0)) return r + y;
  return r;
}

double jl_div(double x, double y) {
  double r = std::fmod(x, y);
  return std::nearbyint((x - r) / y);
}

bool isapprox_default(double x, double y) {
  if (x == y) return true;
  if (!std::isfinite(x) || !std::isfinite(y)) return false;
  const double rtol = 1.4901161193847656e-8;  // sqrt(eps(Float64))
  return std::fabs(x - y) <= rtol * std::max(std::fabs(x), std::fabs(y));
}

double deg2rad(double x) { return x * (3.141592653589793 / 180.0); }

// Degree-argument sine/cosine with exact reduction by quarter turns.
static void sincosd(double x, double* s, double* c) {
  double r = std::fmod(x, 360.0);
  if (r < 0) r += 360.0;
  int q = (int)std::floor((r + 45.0) / 90.0);
  double y = r - 90.0 * q;  // y in [-45, 45)
  double yr = deg2rad(y);
  double sy = std::sin(yr), cy = std::cos(yr);
  switch (q & 3) {
    case 0: *s = sy; *c = cy; break;
    case 1: *s = cy; *c = -sy; break;
    case 2: *s = -sy; *c = -cy; break;
    default: *s = -cy; *c = sy; break;
  }
}
double cosd(double x) { double s, c; sincosd(x, &s, &c); return c; }
double sind(double x) { double s, c; sincosd(x, &s, &c); return s; }

// ------------------------------------------------------------------------- grids --
// eikstructs.jl:33-219 constructors (with their asserts).
Grid make_grid(int kind, const i64* grsize, const double* spacing, const double* cooinit) {
  Grid g;
  g.kind = kind;
  g.nd = (kind == G2DCART || kind == G2DSPH) ? 2 : 3;
  for (int d = 0; d < 3; d++) {
    g.n[d] = 1;
    g.spac[d] = 0;
    g.cooinit[d] = 0;
  }
  for (int d = 0; d < g.nd; d++) {
    g.n[d] = grsize[d];
    g.cooinit[d] = cooinit[d];
    EIKOR_ASSERT(grsize[d] > 0, "all(grsize.>0)");
  }
  if (g.cart()) {
    EIKOR_ASSERT(spacing[0] > 0.0, "hgrid>0.0");
    for (int d = 0; d < g.nd; d++) g.spac[d] = spacing[0];
  } else {
    for (int d = 0; d < g.nd; d++) g.spac[d] = spacing[d];
    if (kind == G2DSPH) {
      EIKOR_ASSERT(cooinit[0] >= 0.0, "cooinit[1]>=0.0");
      EIKOR_ASSERT(spacing[0] > 0.0, "Δr>0.0");
      EIKOR_ASSERT(spacing[1] > 0.0, "Δθ>0.0");
    } else {
      EIKOR_ASSERT(cooinit[0] > 0.0, "cooinit[1]>0.0");
    }
  }
  for (int d = 0; d < g.nd; d++) g.ax[d].init(g.cooinit[d], g.spac[d], g.n[d]);
  if (kind == G2DSPH) {
    for (i64 i = 1; i <= g.n[1]; i++) {
      double th = g.ax[1](i);
      EIKOR_ASSERT(0.0 <= th && th <= 180.0, "all(0.0.<=θ.<=180.0)");
    }
  } else if (kind == G3DSPH) {
    for (i64 i = 1; i <= g.n[1]; i++) {
      double th = g.ax[1](i);
      EIKOR_ASSERT(5.0 <= th && th <= 175.0, "all(5.0.<=θ.<=175.0)");
    }
    for (i64 i = 1; i <= g.n[2]; i++) {
      double ph = g.ax[2](i);
      EIKOR_ASSERT(0.0 <= ph && ph <= 180.0, "all(0.0.<=φ.<=180.0)");
    }
  }
  return g;
}

// ------------------------------------------------------------------------ binheap --
// BinHeaps.jl:313-485
void BinHeapMin::init(i64 nmax) {
  Nmax = nmax;
  Nh = 0;
  nodes.assign(nmax + 2, 0.0);
  handles.assign(nmax + 2, 0);
  idxhan.assign(nmax + 2, 0);
}
void BinHeapMin::swap_nodes(i64 p, i64 q) {  // BinHeaps.jl:89-109
  double tn = nodes[p];
  i64 th = handles[p];
  nodes[p] = nodes[q];
  nodes[q] = tn;
  handles[p] = handles[q];
  handles[q] = th;
  idxhan[handles[p]] = (int32_t)p;
  idxhan[handles[q]] = (int32_t)q;
}
void BinHeapMin::min_heapify(i64 i) {  // BinHeaps.jl:362-386
  for (;;) {
    i64 l = 2 * i, r = 2 * i + 1, smallest;
    if (l <= Nh && nodes[l] < nodes[i]) smallest = l;
    else smallest = i;
    if (r <= Nh && nodes[r] < nodes[smallest]) smallest = r;
    if (smallest == i) return;
    swap_nodes(i, smallest);
    i = smallest;
  }
}
void BinHeapMin::insert(double val, i64 handle) {  // BinHeaps.jl:437-460
  EIKOR_ASSERT(Nmax > Nh, "h.Nmax>h.Nh[]");
  Nh += 1;
  nodes[Nh] = val;
  handles[Nh] = handle;
  idxhan[handle] = (int32_t)Nh;
  i64 i = Nh;
  while (i > 1 && nodes[i / 2] > nodes[i]) {
    swap_nodes(i, i / 2);
    i = i / 2;
  }
}
void BinHeapMin::update(double val, i64 handle) {  // BinHeaps.jl:394-430
  i64 i = idxhan[handle];
  nodes[i] = val;
  while (i > 1 && nodes[i / 2] > nodes[i]) {
    swap_nodes(i, i / 2);
    i = i / 2;
  }
  if (i < Nh) min_heapify(i);
}
void BinHeapMin::pop(i64& handle, double& val) {  // BinHeaps.jl:467-485
  handle = handles[1];
  val = nodes[1];
  nodes[1] = nodes[Nh];
  handles[1] = handles[Nh];
  idxhan[handles[Nh]] = 1;
  nodes[Nh] = 0.0;
  handles[Nh] = 0;
  idxhan[handle] = 0;
  Nh -= 1;
  min_heapify(1);
}

// --------------------------------------------------------- local 2nd-order solver --
// Node spacing per axis at node i (eikforward2D.jl:115-119, eikforward3D.jl:168-172).
static inline void node_spacing(const Grid& g, i64 i1, double* dh) {
  if (g.cart()) {
    dh[0] = dh[1] = dh[2] = g.spac[0];
  } else {
    double r = g.ax[0](i1);
    dh[0] = g.spac[0];
    dh[1] = r * deg2rad(g.spac[1]);
    dh[2] = (g.nd == 3) ? r * deg2rad(g.spac[2]) : 0.0;
  }
}

// isonbord (eikutils.jl:129-162) evaluated at the neighbour position nb.
static inline void isonbord(const Grid& g, const i64* nb, bool& onb1, bool& onb2) {
  onb1 = false;
  onb2 = false;
  for (int d = 0; d < g.nd; d++) {
    if (nb[d] < 1 || nb[d] > g.n[d]) onb1 = true;
    if (nb[d] < 2 || nb[d] > g.n[d] - 1) onb2 = true;
  }
}

// calcttpt_2ndord! (eikforward2D.jl:98-433, eikforward3D.jl:151-532); one body for 2D/3D.
double calcttpt_2ndord(const FMMVars& fv, const double* vel, const i64* ijk, int8_t* codeD,
                       uint32_t* warn) {
  const Grid& g = fv.grd;
  const int nd = g.nd;
  double dh[3];
  node_spacing(g, ijk[0], dh);
  const double slowcurpt = 1.0 / vel[g.lin(ijk)];
  const double* tt = fv.ttime.data();
  const uint8_t* status = fv.status.data();

  double alpha = 0.0, beta = 0.0, gamma = -(slowcurpt * slowcurpt);
  for (int d = 0; d < nd; d++) codeD[d] = 0;

  for (int axis = 0; axis < nd; axis++) {
    bool use1stord = false, use2ndord = false;
    double chosenval1 = HUGE_TT, chosenval2 = HUGE_TT;
    for (int l = 0; l < 2; l++) {
      const int sh = (l == 0) ? 1 : -1;
      i64 nb[3] = {ijk[0], ijk[1], ijk[2]};
      nb[axis] += sh;
      bool onb1, onb2;
      isonbord(g, nb, onb1, onb2);
      if (!onb1 && status[g.lin(nb)] == 2) {
        double testval1 = tt[g.lin(nb)];
        if (testval1 < chosenval1) {
          chosenval1 = testval1;
          use1stord = true;
          codeD[axis] = (int8_t)(-sh);
          i64 nb2[3] = {ijk[0], ijk[1], ijk[2]};
          nb2[axis] += 2 * sh;
          if (!onb2 && status[g.lin(nb2)] == 2) {
            double testval2 = tt[g.lin(nb2)];
            if (testval2 <= chosenval1) {
              chosenval2 = testval2;
              use2ndord = true;
              codeD[axis] = (int8_t)(-2 * sh);
            } else {
              chosenval2 = HUGE_TT;
              use2ndord = false;
              codeD[axis] = (int8_t)(-sh);
            }
          }
        }
      }
    }
    const double deltah = dh[axis];
    if (use2ndord && use1stord) {
      double tmpa2 = (1.0 / 3.0) * (4.0 * chosenval1 - chosenval2);
      double curalpha = 9.0 / (4.0 * (deltah * deltah));
      alpha += curalpha;
      beta += (-2.0 * curalpha) * tmpa2;
      gamma += curalpha * (tmpa2 * tmpa2);
    } else if (use1stord) {
      double curalpha = 1.0 / (deltah * deltah);
      alpha += curalpha;
      beta += (-2.0 * curalpha) * chosenval1;
      gamma += curalpha * (chosenval1 * chosenval1);
    }
  }
  double sqarg = beta * beta - (4.0 * alpha) * gamma;

  if (sqarg < 0.0) {  // revert to 1st order on every axis
    for (int d = 0; d < nd; d++) codeD[d] = 0;
    alpha = 0.0;
    beta = 0.0;
    gamma = -(slowcurpt * slowcurpt);
    for (int axis = 0; axis < nd; axis++) {
      bool use1stord = false;
      double chosenval1 = HUGE_TT;
      for (int l = 0; l < 2; l++) {
        const int sh = (l == 0) ? 1 : -1;
        i64 nb[3] = {ijk[0], ijk[1], ijk[2]};
        nb[axis] += sh;
        bool onb1, onb2;
        isonbord(g, nb, onb1, onb2);
        if (!onb1 && status[g.lin(nb)] == 2) {
          double testval1 = tt[g.lin(nb)];
          if (testval1 < chosenval1) {
            chosenval1 = testval1;
            use1stord = true;
            codeD[axis] = (int8_t)(-sh);
          }
        }
      }
      if (use1stord) {
        const double deltah = dh[axis];
        double curalpha = 1.0 / (deltah * deltah);
        alpha += curalpha;
        beta += (-2.0 * curalpha) * chosenval1;
        gamma += curalpha * (chosenval1 * chosenval1);
      }
    }
    sqarg = beta * beta - (4.0 * alpha) * gamma;
  }

  if (sqarg < 0.0) {  // still negative: one-dimensional update
    if (warn) *warn |= WARN_NEG_DISCRIMINANT;
    for (int d = 0; d < nd; d++) codeD[d] = 0;
    double cv[3] = {HUGE_TT, HUGE_TT, HUGE_TT};
    for (int axis = 0; axis < nd; axis++) {
      for (int l = 0; l < 2; l++) {
        const int sh = (l == 0) ? 1 : -1;
        i64 nb[3] = {ijk[0], ijk[1], ijk[2]};
        nb[axis] += sh;
        bool onb1, onb2;
        isonbord(g, nb, onb1, onb2);
        if (!onb1 && status[g.lin(nb)] == 2) {
          double testval1 = tt[g.lin(nb)];
          if (testval1 < cv[axis]) {
            cv[axis] = testval1;
            codeD[axis] = (int8_t)(-sh);
          }
        }
      }
    }
    int idcv = 0;
    for (int d = 1; d < nd; d++)
      if (cv[d] < cv[idcv]) idcv = d;
    double soughtt = (dh[idcv] * slowcurpt) + cv[idcv];
    int8_t keep = codeD[idcv];
    for (int d = 0; d < nd; d++) codeD[d] = 0;
    codeD[idcv] = keep;
    return soughtt;
  }

  double tmpsq = std::sqrt(sqarg);
  double s1 = (-beta + tmpsq) / (2.0 * alpha);
  double s2 = (-beta - tmpsq) / (2.0 * alpha);
  return (s2 > s1) ? s2 : s1;
}

// ------------------------------------------------------------------ source box --
// distance2points (eikutils.jl:47-73). Grid3DSphere has no implementation in the
// reference (error at eikutils.jl:72); completed as the chord length through
// sphericaldeg2cartesian (utils.jl:344-349).
double distance2points(const Grid& g, const double* a, const double* b) {
  if (g.cart()) {
    double s = 0.0;
    for (int d = 0; d < g.nd; d++) {
      double t = a[d] - b[d];
      if (d == 0) s = t * t;
      else s = s + t * t;
    }
    return std::sqrt(s);
  }
  if (g.kind == G2DSPH) {
    double r1 = a[0], t1 = a[1], r2 = b[0], t2 = b[1];
    return std::sqrt((r1 * r1 + r2 * r2) - ((2.0 * r1) * r2) * cosd(t1 - t2));
  }
  double x1 = a[0] * sind(a[1]) * cosd(a[2]), y1 = a[0] * sind(a[1]) * sind(a[2]),
         z1 = a[0] * cosd(a[1]);
  double x2 = b[0] * sind(b[1]) * cosd(b[2]), y2 = b[0] * sind(b[1]) * sind(b[2]),
         z2 = b[0] * cosd(b[1]);
  double dx = x1 - x2, dy = y1 - y2, dz = z1 - z2;
  return std::sqrt((dx * dx + dy * dy) + dz * dz);
}

// findenclosingbox (eikmainfwd.jl:1114-1186). Grid3DSphere spacing completed with
// (Δr, Δθ, Δφ) (the reference has no branch for it at :1122-1131).
void findenclosingbox(const Grid& g, const double* xyzsrc, std::vector<std::array<i64, 3>>& out) {
  const int nd = g.nd;
  double rem[3];
  i64 ijk[3] = {1, 1, 1};
  for (int d = 0; d < nd; d++) {
    double x = xyzsrc[d] - g.cooinit[d];
    double q = jl_div(x, g.spac[d]);
    rem[d] = jl_rem(x, g.spac[d]);
    ijk[d] = (i64)std::floor(q) + 1;
  }
  bool allzero = true;
  for (int d = 0; d < nd; d++)
    if (!(std::fabs(rem[d]) <= 1e-8)) allzero = false;
  out.clear();
  if (allzero) {
    out.push_back({ijk[0], ijk[1], nd == 3 ? ijk[2] : 1});
    return;
  }
  for (int d = 0; d < nd; d++)
    if (ijk[d] == g.n[d]) ijk[d] -= 1;
  if (nd == 2) {
    static const int off2[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};
    for (auto& o : off2) out.push_back({ijk[0] + o[0], ijk[1] + o[1], 1});
  } else {
    static const int off3[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                                   {1, 1, 0}, {0, 1, 1}, {1, 0, 1}, {1, 1, 1}};
    for (auto& o : off3) out.push_back({ijk[0] + o[0], ijk[1] + o[1], ijk[2] + o[2]});
  }
}

// sourceboxloctt! (eikmainfwd.jl:1195-1322). The halfway shift recomputes the corner
// distances from the *unshifted* position (:1314), so only xyzsrc and a warning change.
void sourceboxloctt(FMMVars& fv, const double* vel, const double* srcpos, uint32_t* warn) {
  const Grid& g = fv.grd;
  const int nd = g.nd;
  findenclosingbox(g, srcpos, fv.ijksrc);
  fv.is_srcbox = true;
  const size_t nc = fv.ijksrc.size();
  fv.velcorn.assign(nc, 0.0);
  fv.distcorn.assign(nc, 0.0);
  for (int d = 0; d < 3; d++) fv.xyzsrc[d] = (d < nd) ? srcpos[d] : 0.0;
  for (size_t l = 0; l < nc; l++) {
    const i64* ijk = fv.ijksrc[l].data();
    i64 lin = g.lin(ijk);
    fv.status[lin] = 2;
    double xyzpt[3];
    for (int d = 0; d < nd; d++) xyzpt[d] = g.ax[d](ijk[d]);
    double dc = distance2points(g, xyzpt, srcpos);
    fv.velcorn[l] = vel[lin];
    fv.distcorn[l] = dc;
    fv.ttime[lin] = dc / vel[lin];
  }
  if (nc > 1) {
    double srcshift;
    if (g.cart()) srcshift = 1e-4 * g.spac[0];
    else if (g.kind == G2DSPH) srcshift = 1e-4 * std::min(g.spac[0], g.spac[1]);
    else srcshift = 1e-4 * std::min(std::min(g.spac[0], g.spac[1]), g.spac[2]);
    bool any = false;
    bool half[3] = {false, false, false};
    for (int d = 0; d < nd; d++) {
      double r = jl_rem(srcpos[d] - g.cooinit[d], g.spac[d]);
      half[d] = isapprox_default(r, g.spac[d] / 2.0);
      any = any || half[d];
    }
    if (any) {
      if (warn) *warn |= WARN_SRC_HALFWAY_SHIFT;
      for (int d = 0; d < nd; d++)
        if (half[d]) fv.xyzsrc[d] = srcpos[d] + srcshift;
      // corner distances/times recomputed with srcpos: identical values
    }
  }
}

// ------------------------------------------------------------ refined fine grid --
// createfinegrid (eikmainfwd.jl:950-1104). The Grid3DSphere branch errors in the
// reference (:1092); completed as spacing/ds on every axis.
void createfinegrid(const Grid& g, const double* xyzsrc, const double* vel, i64 ds, i64 noderadius,
                    SrcRefinVars& srv) {
  const int nd = g.nd;
  std::vector<std::array<i64, 3>> corn;
  findenclosingbox(g, xyzsrc, corn);
  i64 ijk1[3] = {1, 1, 1}, ijk2[3] = {1, 1, 1};
  for (int d = 0; d < nd; d++) {
    i64 mn = corn[0][d], mx = corn[0][d];
    for (auto& c : corn) {
      mn = std::min(mn, c[d]);
      mx = std::max(mx, c[d]);
    }
    i64 v1 = mn - noderadius, v2 = mx + noderadius;
    srv.outijk_min[d] = v1 < 1;
    srv.outijk_max[d] = v2 > g.n[d];
    ijk1[d] = srv.outijk_min[d] ? 1 : v1;
    ijk2[d] = srv.outijk_max[d] ? g.n[d] : v2;
  }
  srv.downscalefactor = ds;
  i64 nf[3] = {1, 1, 1};
  for (int d = 0; d < nd; d++) {
    nf[d] = (ijk2[d] - ijk1[d]) * ds + 1;
    srv.window_n[d] = ijk2[d] - ijk1[d] + 1;
    srv.ijkorigincoarse[d] = ijk1[d];
  }
  for (int d = nd; d < 3; d++) {
    srv.window_n[d] = 1;
    srv.ijkorigincoarse[d] = 1;
  }
  const i64 nfine = nf[0] * nf[1] * nf[2];
  srv.nearneigh_idxcoarse.assign(nfine, 0);
  srv.velcart_fine.assign(nfine, 0.0);
  for (i64 lf = 0; lf < nfine; lf++) {
    i64 fi[3] = {lf % nf[0] + 1, (lf / nf[0]) % nf[1] + 1, lf / (nf[0] * nf[1]) + 1};
    i64 ic[3] = {1, 1, 1};
    for (int d = 0; d < nd; d++) {
      i64 di = (fi[d] - 1) / ds;
      i64 ri = fi[d] - di * ds;
      ic[d] = ((double)ri >= (double)ds / 2.0 + 1.0) ? di + 2 : di + 1;
    }
    i64 jcol = (ic[0] - 1) + srv.window_n[0] * ((ic[1] - 1) + srv.window_n[1] * (ic[2] - 1));
    srv.nearneigh_idxcoarse[lf] = jcol + 1;
    i64 gijk[3] = {ijk1[0] + ic[0] - 1, ijk1[1] + ic[1] - 1, nd == 3 ? ijk1[2] + ic[2] - 1 : 1};
    srv.velcart_fine[lf] = vel[g.lin(gijk)];
  }
  double sp[3], co[3];
  for (int d = 0; d < nd; d++) {
    co[d] = g.ax[d](ijk1[d]);
    sp[d] = g.spac[d] / (double)ds;
  }
  srv.grd_fine = make_grid(g.kind, nf, sp, co);
}

// isacoarsegridnode (eikutils.jl:78-119)
static inline bool isacoarsegridnode(const Grid& fg, const i64* ijk, const SrcRefinVars& srv,
                                     i64* out) {
  for (int d = 0; d < fg.nd; d++)
    if ((ijk[d] - 1) % srv.downscalefactor != 0) return false;
  for (int d = 0; d < fg.nd; d++) out[d] = (ijk[d] - 1) / srv.downscalefactor + srv.ijkorigincoarse[d];
  if (fg.nd == 2) out[2] = 1;
  return true;
}

// ----------------------------------------------------------------- adjoint vars --
void AdjointVars::init(const Grid& g) {
  grd = g;
  const i64 n = g.npts();
  lfmm2grid.assign(n, 0);
  lgrid2fmm.assign(n, 0);
  fmmtt.assign(n, -1.0);
  onsrccols.assign(n, 0);
  onhpoints.assign(n, 0);
  code.assign(n * g.nd, 0);
  lastcomputedtt = 0;
  for (int d = 0; d < 3; d++) nsize0[d] = nsize1[d] = n;
}
// eikmainfwd.jl:257-279 (lfmm2grid is deliberately *not* cleared)
void AdjointVars::reset_for_run() {
  const i64 n = grd.npts();
  for (int d = 0; d < 3; d++) nsize0[d] = nsize1[d] = n;
  std::fill(onsrccols.begin(), onsrccols.end(), 0);
  std::fill(onhpoints.begin(), onhpoints.end(), 0);
  std::fill(fmmtt.begin(), fmmtt.end(), -1.0);
  lastcomputedtt = 0;
  std::fill(code.begin(), code.end(), 0);
}

// ---------------------------------------------------------------------- FMM core --
// ttFMM_core! (eikmainfwd.jl:427-823)
void ttFMM_core(FMMVars& fv, const double* vel, AdjointVars* adj, FMMVars* coarse,
                AdjointVars* adjcoarse, SrcRefinVars* srv, FMMStats* st) {
  const bool refsrc = srv != nullptr;
  const Grid& g = fv.grd;
  const int nd = g.nd;
  const i64 N = g.npts();
  const std::vector<std::array<i64, 3>> ijksrc = fv.ijksrc;
  const i64 naccinit = (i64)ijksrc.size();
  uint32_t* warn = st ? &st->warn : nullptr;
  static const int neigh2[4][3] = {{1, 0, 0}, {0, 1, 0}, {-1, 0, 0}, {0, -1, 0}};
  static const int neigh3[6][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {-1, 0, 0}, {0, -1, 0}, {0, 0, -1}};
  const int nneigh = (nd == 2) ? 4 : 6;
  auto NEI = [&](int ne, int d) { return nd == 2 ? neigh2[ne][d] : neigh3[ne][d]; };
  int8_t idD[3] = {0, 0, 0};

  if (adj) {  // eikmainfwd.jl:500-547
    adj->lastcomputedtt = naccinit;
    for (i64 l = 0; l < naccinit; l++) {
      i64 lin = g.lin(ijksrc[l].data());
      adj->lfmm2grid[l] = (int32_t)(lin + 1);
      adj->fmmtt[l] = fv.ttime[lin];
      adj->onsrccols[l] = 1;
      for (int d = 0; d < nd; d++) adj->nsize0[d] -= 1;
    }
  }

  std::vector<std::array<i64, 3>> ijksrc_coarse;
  i64 counter_adjcoarse = 0;
  if (refsrc) {  // eikmainfwd.jl:554-581
    for (i64 l = 0; l < naccinit; l++) {
      i64 ijkc[3];
      if (isacoarsegridnode(g, ijksrc[l].data(), *srv, ijkc)) {
        i64 lf = g.lin(ijksrc[l].data());
        i64 lc = coarse->grd.lin(ijkc);
        coarse->ttime[lc] = fv.ttime[lf];
        coarse->status[lc] = fv.status[lf];
        ijksrc_coarse.push_back({ijkc[0], ijkc[1], ijkc[2]});
        if (adj) adj->onhpoints[l] = 1;
      }
    }
  }

  auto inbounds = [&](const i64* p) {
    for (int d = 0; d < nd; d++)
      if (p[d] < 1 || p[d] > g.n[d]) return false;
    return true;
  };

  // initial narrow band (eikmainfwd.jl:590-621)
  for (i64 l = 0; l < naccinit; l++) {
    for (int ne = 0; ne < nneigh; ne++) {
      i64 cur[3] = {ijksrc[l][0], ijksrc[l][1], ijksrc[l][2]};
      for (int d = 0; d < nd; d++) cur[d] += NEI(ne, d);
      if (!inbounds(cur)) continue;
      i64 han = g.lin(cur);
      if (fv.status[han] == 0) {
        double tmptt = calcttpt_2ndord(fv, vel, cur, idD, warn);
        fv.bheap.insert(tmptt, han + 1);
        fv.status[han] = 1;
        if (adj)
          for (int d = 0; d < nd; d++) adj->code[han * nd + d] = idD[d];
      }
    }
  }

  // main loop (eikmainfwd.jl:627-814)
  i64 node = naccinit;  // 1-based FMM position counter
  double maxpopped = -HUGE_TT;
  bool firstwarning = true;
  std::vector<std::array<i64, 3>> popped;
  popped.reserve(128);
  const bool rec_batch = st && st->batch_of && !refsrc;
  if (rec_batch) {
    st->batch_of->assign(N, -1);
    for (i64 l = 0; l < naccinit; l++) (*st->batch_of)[g.lin(ijksrc[l].data())] = 0;
  }
  int32_t batchno = 0;
  for (i64 iter = 1; iter <= N - naccinit; iter++) {
    if (fv.bheap.Nh < 1) break;
    popped.clear();
    batchno++;
    bool sameminval = true;
    while (sameminval) {
      node += 1;
      if (fv.bheap.Nh < 1) break;
      i64 acchan1;
      double tmptt;
      fv.bheap.pop(acchan1, tmptt);
      sameminval = (fv.bheap.topval() == tmptt);
      const i64 acchan = acchan1 - 1;
      i64 acc[3];
      g.cart_of(acchan, acc);
      fv.status[acchan] = 2;
      fv.ttime[acchan] = tmptt;
      if (rec_batch) (*st->batch_of)[acchan] = batchno;
      if (st) {
        st->pops++;
        if (tmptt < maxpopped) st->nonmonotone_pops++;
      }
      if (tmptt > maxpopped) maxpopped = tmptt;
      if (adj) {
        adj->lfmm2grid[node - 1] = (int32_t)(acchan + 1);
        adj->fmmtt[node - 1] = tmptt;
        adj->lastcomputedtt = node;
      }
      if (refsrc) {
        i64 ijkc[3];
        if (isacoarsegridnode(g, acc, *srv, ijkc)) {
          i64 lc = coarse->grd.lin(ijkc);
          coarse->ttime[lc] = fv.ttime[acchan];
          coarse->status[lc] = fv.status[acchan];
          ijksrc_coarse.push_back({ijkc[0], ijkc[1], ijkc[2]});
          if (adj) {
            adj->onhpoints[node - 1] = 1;
            adjcoarse->lfmm2grid[counter_adjcoarse] = (int32_t)(lc + 1);
            adjcoarse->fmmtt[counter_adjcoarse] = fv.ttime[acchan];
            counter_adjcoarse++;
          }
        }
        bool onedge = false;
        for (int d = 0; d < nd; d++) {
          if (acc[d] == 1 && !srv->outijk_min[d]) onedge = true;
          if (acc[d] == g.n[d] && !srv->outijk_max[d]) onedge = true;
        }
        if (onedge) {
          bool anycoarse = false;
          for (auto s : coarse->status)
            if (s > 0) {
              anycoarse = true;
              break;
            }
          if (!anycoarse) {
            if (firstwarning) {
              if (warn) *warn |= WARN_BORDER_BEFORE_COARSE;
              firstwarning = false;
            }
            continue;
          }
          if (adj) createsparsederivativematrices(g, *adj, fv.status);
          for (auto& s : coarse->status)
            if (s == 1) s = 0;
          coarse->ijksrc = ijksrc_coarse;
          coarse->is_srcbox = false;
          return;
        }
      }
      if ((i64)popped.size() >= 128) jl_error("BoundsError: more than 128 equal minima popped at once");
      popped.push_back({acc[0], acc[1], acc[2]});
      if (st && (i64)popped.size() > st->max_batch) st->max_batch = (i64)popped.size();
    }
    for (auto& a : popped) {
      for (int ne = 0; ne < nneigh; ne++) {
        i64 cur[3] = {a[0], a[1], a[2]};
        for (int d = 0; d < nd; d++) cur[d] += NEI(ne, d);
        if (!inbounds(cur)) continue;
        i64 han = g.lin(cur);
        if (fv.status[han] == 0) {
          double tmptt = calcttpt_2ndord(fv, vel, cur, idD, warn);
          fv.bheap.insert(tmptt, han + 1);
          fv.status[han] = 1;
          if (adj)
            for (int d = 0; d < nd; d++) adj->code[han * nd + d] = idD[d];
        } else if (fv.status[han] == 1) {
          double tmptt = calcttpt_2ndord(fv, vel, cur, idD, warn);
          fv.bheap.update(tmptt, han + 1);
          if (adj)
            for (int d = 0; d < nd; d++) adj->code[han * nd + d] = idD[d];
        }
      }
    }
  }
  if (refsrc && warn) *warn |= WARN_FINE_NO_TRIGGER;
  if (adj) createsparsederivativematrices(g, *adj, fv.status);
}

// ttFMM_hiord! + runrefinementaroundsrc! (eikmainfwd.jl:230-405)
void ttFMM_hiord(FMMVars& fv, const double* vel, const double* src, AdjointVars* adj,
                 const ExtraParams& ep, FMMVars* fine_out, AdjointVars* adjfine_out,
                 SrcRefinVars* srv_out, FMMStats* st) {
  const Grid& g = fv.grd;
  std::fill(fv.ttime.begin(), fv.ttime.end(), HUGE_TT);
  std::fill(fv.status.begin(), fv.status.end(), (uint8_t)0);
  if (adj) adj->reset_for_run();
  uint32_t* warn = st ? &st->warn : nullptr;
  if (fv.refinearoundsrc) {
    SrcRefinVars local_srv;
    SrcRefinVars& srv = srv_out ? *srv_out : local_srv;
    createfinegrid(g, src, vel, ep.downscalefactor, ep.noderadius, srv);
    FMMVars local_fine;
    FMMVars& fine = fine_out ? *fine_out : local_fine;
    fine.grd = srv.grd_fine;
    const i64 nfine = fine.grd.npts();
    fine.ttime.assign(nfine, HUGE_TT);
    fine.status.assign(nfine, 0);
    fine.bheap.init(nfine);
    fine.refinearoundsrc = false;
    AdjointVars local_adjf;
    AdjointVars* adjf = nullptr;
    if (adj) {
      adjf = adjfine_out ? adjfine_out : &local_adjf;
      adjf->init(fine.grd);
    }
    sourceboxloctt(fine, srv.velcart_fine.data(), src, warn);
    ttFMM_core(fine, srv.velcart_fine.data(), adjf, &fv, adj, &srv, st);
  } else {
    sourceboxloctt(fv, vel, src, warn);
  }
  ttFMM_core(fv, vel, adj, nullptr, nullptr, nullptr, st);
}

// ------------------------------------------------------------ receiver interpolation --
// bilinear_interp / trilinear_interp (eikforward2D.jl:17-87, eikforward3D.jl:17-140).
struct InterpCell {
  i64 i, j, k;
  double xd, yd, zd;
};
static InterpCell interp_cell(const Grid& g, const double* pt) {
  InterpCell c{1, 1, 1, 0, 0, 0};
  if (g.nd == 2) {
    double xh = (pt[0] - g.cooinit[0]) / g.spac[0];
    double yh = (pt[1] - g.cooinit[1]) / g.spac[1];
    i64 i = (i64)std::floor(xh + 1), j = (i64)std::floor(yh + 1);
    if (i == g.n[0]) i -= 1;
    else if (i > g.n[0]) i -= 2;
    if (j == g.n[1]) j -= 1;
    else if (j > g.n[1]) j -= 2;
    c.i = i;
    c.j = j;
    c.xd = xh - (double)(i - 1);
    c.yd = yh - (double)(j - 1);
  } else {
    double dx = g.spac[0], dy = g.spac[1], dz = g.spac[2];
    double xh = (pt[0] - g.cooinit[0]) / dx, yh = (pt[1] - g.cooinit[1]) / dy,
           zh = (pt[2] - g.cooinit[2]) / dz;
    double x = pt[0] - g.cooinit[0], y = pt[1] - g.cooinit[1], z = pt[2] - g.cooinit[2];
    i64 i = (i64)std::floor(xh + 1), j = (i64)std::floor(yh + 1), k = (i64)std::floor(zh + 1);
    if (i == g.n[0]) i -= 1;
    else if (i > g.n[0]) i -= 2;
    if (j == g.n[1]) j -= 1;
    else if (j > g.n[1]) j -= 2;
    if (k == g.n[2]) k -= 1;
    else if (k > g.n[2]) k -= 2;
    double x0 = (double)(i - 1) * dx, y0 = (double)(j - 1) * dy, z0 = (double)(k - 1) * dz;
    double x1 = (double)i * dx, y1 = (double)j * dy, z1 = (double)k * dz;
    c.i = i;
    c.j = j;
    c.k = k;
    c.xd = (x - x0) / (x1 - x0);
    c.yd = (y - y0) / (y1 - y0);
    c.zd = (z - z0) / (z1 - z0);
  }
  return c;
}

double interpolate_receiver(const std::vector<double>& tt, const Grid& g, const double* pt) {
  InterpCell c = interp_cell(g, pt);
  if (g.nd == 2) {
    i64 a[3] = {c.i, c.j, 1}, b[3] = {c.i + 1, c.j, 1}, e[3] = {c.i, c.j + 1, 1},
        f[3] = {c.i + 1, c.j + 1, 1};
    double xd = c.xd, yd = c.yd;
    return tt[g.lin(a)] * (1.0 - xd) * (1.0 - yd) + tt[g.lin(b)] * (1.0 - yd) * xd +
           tt[g.lin(e)] * (1.0 - xd) * yd + tt[g.lin(f)] * xd * yd;
  }
  double xd = c.xd, yd = c.yd, zd = c.zd;
  auto T = [&](int di, int dj, int dk) {
    i64 p[3] = {c.i + di, c.j + dj, c.k + dk};
    return tt[g.lin(p)];
  };
  // corner (i+1,j,k+1) carries the weight xd*(1-yd)*(1-zd) (eikforward3D.jl:133)
  return T(0, 0, 0) * (1 - xd) * (1 - yd) * (1 - zd) + T(1, 0, 0) * xd * (1 - yd) * (1 - zd) +
         T(0, 1, 0) * (1 - xd) * yd * (1 - zd) + T(0, 0, 1) * (1 - xd) * (1 - yd) * zd +
         T(1, 1, 0) * xd * yd * (1 - zd) + T(0, 1, 1) * (1 - xd) * yd * zd +
         T(1, 0, 1) * xd * (1 - yd) * (1 - zd) + T(1, 1, 1) * xd * yd * zd;
}

void interp_coeffs(const Grid& g, const double* pt, double* coeff, i64 (*ijk)[3], int* ncoe) {
  InterpCell c = interp_cell(g, pt);
  if (g.nd == 2) {
    double xd = c.xd, yd = c.yd;
    coeff[0] = (1.0 - xd) * (1.0 - yd);
    coeff[1] = (1.0 - yd) * xd;
    coeff[2] = (1.0 - xd) * yd;
    coeff[3] = xd * yd;
    static const int o[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};
    for (int l = 0; l < 4; l++) {
      ijk[l][0] = c.i + o[l][0];
      ijk[l][1] = c.j + o[l][1];
      ijk[l][2] = 1;
    }
    *ncoe = 4;
    return;
  }
  double xd = c.xd, yd = c.yd, zd = c.zd;
  coeff[0] = (1 - xd) * (1 - yd) * (1 - zd);
  coeff[1] = xd * (1 - yd) * (1 - zd);
  coeff[2] = (1 - xd) * yd * (1 - zd);
  coeff[3] = (1 - xd) * (1 - yd) * zd;
  coeff[4] = xd * yd * (1 - zd);
  coeff[5] = (1 - xd) * yd * zd;
  coeff[6] = xd * (1 - yd) * (1 - zd);  // eikforward3D.jl:102
  coeff[7] = xd * yd * zd;
  static const int o[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                              {1, 1, 0}, {0, 1, 1}, {1, 0, 1}, {1, 1, 1}};
  for (int l = 0; l < 8; l++)
    for (int d = 0; d < 3; d++) ijk[l][d] = (d == 0 ? c.i : d == 1 ? c.j : c.k) + o[l][d];
  *ncoe = 8;
}

// ------------------------------------------------------ FMM-ordered derivative matrices --
// createsparsederivativematrices! + setcoeffderiv! + addrowCSRmat!
// (eikmainfwd.jl:827-946, eikmaingrad.jl:946-1131). Grid3DSphere errors in the reference
// (eikmainfwd.jl:887, eikmaingrad.jl:1079); completed with the θ/φ arc spacings used by the
// local solver (r_i·deg2rad(Δθ), r_i·deg2rad(Δφ)).
void createsparsederivativematrices(const Grid& g, AdjointVars& adj, const std::vector<uint8_t>& status) {
  const int nd = g.nd;
  const i64 npts = g.npts();
  i64 nptsonsrc = 0;
  for (auto b : adj.onsrccols) nptsonsrc += b;
  for (i64 i = 0; i < npts; i++) {
    int32_t ifm = adj.lfmm2grid[i];
    if (ifm == 0) {
      for (int d = 0; d < nd; d++) {
        adj.nsize0[d] = i - nptsonsrc;
        adj.nsize1[d] = i;
      }
      break;
    }
    adj.lgrid2fmm[ifm - 1] = (int32_t)(i + 1);
  }
  const i64 nrows = adj.nsize0[0];
  for (int d = 0; d < nd; d++) {
    CSR& D = adj.D[d];
    D.nrows = nrows;
    D.ncols = adj.nsize1[d];
    D.iptr.assign(nrows + 1, 0);
    D.j.clear();
    D.v.clear();
    D.j.reserve(nrows * 2);
    D.v.reserve(nrows * 2);
  }
  for (i64 irow = 0; irow < nrows; irow++) {
    const i64 iptorig = adj.lfmm2grid[irow + nptsonsrc] - 1;
    i64 ijk[3];
    g.cart_of(iptorig, ijk);
    const bool acc = status[iptorig] == 2;
    double r_i = g.sph() ? g.ax[0](ijk[0]) : 0.0;
    for (int d = 0; d < nd; d++) {
      CSR& D = adj.D[d];
      int code = acc ? adj.code[iptorig * nd + d] : 0;
      if (code == 0) {
        D.iptr[irow + 1] = D.iptr[irow];
        continue;
      }
      int abscode = std::abs(code);
      int nnzcol = abscode + 1;
      int signcod = (code > 0) ? -1 : 1;
      double h;
      if (g.cart() || d == 0) h = g.spac[d];
      else h = r_i * deg2rad(g.spac[d]);
      double c1[2] = {-1.0 / h, 1.0 / h};
      double c2[3] = {-3.0 / (2.0 * h), 4.0 / (2.0 * h), -1.0 / (2.0 * h)};
      i64 cols[3];
      double vals[3];
      for (int p = 0; p < nnzcol; p++) {
        i64 q[3] = {ijk[0], ijk[1], ijk[2]};
        q[d] += (i64)signcod * p;
        double cf = (abscode == 1) ? c1[p] : c2[p];
        vals[p] = (double)signcod * cf;
        cols[p] = adj.lgrid2fmm[g.lin(q)];  // 1-based FMM position
      }
      int perm[3] = {0, 1, 2};
      std::sort(perm, perm + nnzcol, [&](int a, int b) { return cols[a] < cols[b]; });
      for (int p = 0; p < nnzcol; p++) {
        D.j.push_back((int32_t)(cols[perm[p]] - 1));
        D.v.push_back(vals[perm[p]]);
      }
      D.iptr[irow + 1] = D.iptr[irow] + nnzcol;
    }
  }
}

}  // namespace eikor
