// Runs the ray kernels' per-line and per-ray code (eikonalsolvers.jl_b200/csrc/rays.cuh)
// on the host, in the order the kernels run it, for tests/test_rays_host.py, which
// compiles it with the address and undefined-behaviour (alignment) sanitizers.
// Usage: rays_host_harness META TT CS OFF REC OUT (raw little-endian float64 / int64 files:
// META = kind nd n0 n1 n2 spacing0..2 cooinit0..2 steplen; OUT = point counts then points).
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <cmath>
#include "rays.cuh"
using namespace eik;
static std::vector<double> readd(const char* f) { FILE* p = fopen(f, "rb"); std::vector<double> v; double x; while (fread(&x, 8, 1, p) == 1) v.push_back(x); fclose(p); return v; }
static std::vector<long long> readl(const char* f) { FILE* p = fopen(f, "rb"); std::vector<long long> v; long long x; while (fread(&x, 8, 1, p) == 1) v.push_back(x); fclose(p); return v; }
int main(int argc, char** argv) {
  // meta: kind nd n0 n1 n2 h0 h1 h2 co0 co1 co2 steplen
  std::vector<double> meta = readd(argv[1]);
  std::vector<double> tt = readd(argv[2]), cs = readd(argv[3]), rec = readd(argv[5]);
  std::vector<long long> off = readl(argv[4]);
  GridDesc g; std::memset(&g, 0, sizeof g);
  g.kind = (int)meta[0]; g.nd = (int)meta[1];
  for (int d = 0; d < 3; d++) { g.n[d] = (int)meta[2 + d]; g.spac[d] = meta[5 + d]; g.co[d] = meta[8 + d]; }
  for (int d = 0; d < g.nd; d++) g.ax[d] = make_jrange(g.co[d], g.spac[d]);
  const double steplen = meta[11];
  const long long nsrc = (long long)off.size() - 1, N = (long long)g.n[0] * g.n[1] * g.n[2], nray = off[nsrc];
  SplineArgs sp; sp.nd = g.nd; sp.nsrc = (int)nsrc;
  for (int d = 0; d < 3; d++) { sp.n[d] = g.n[d]; sp.m[d] = d < g.nd ? g.n[d] + 2 : 1; }
  sp.cstride = sp.m[0] * sp.m[1] * sp.m[2];
  std::vector<double> coef(sp.cstride * nsrc), cpd;
  std::vector<std::vector<double>> cps(3);
  for (int d = 0; d < g.nd; d++) {
    long long k = g.n[d] - 2; std::vector<double> c(k > 0 ? k : 1, 0.0);
    if (k > 0) c[0] = (1.0/6.0) / (2.0/3.0);
    for (long long i = 1; i < k; i++) c[i] = (1.0/6.0) / (2.0/3.0 - (1.0/6.0) * c[i-1]);
    cps[d] = c; sp.cp[d] = cps[d].data();
  }
  sp.coef = coef.data(); sp.coef_size = sp.cstride * nsrc; uint32_t serr = 0; sp.err = &serr;
  for (long long q = 0; q < N * nsrc; q++) spline_load_one(sp, tt.data(), N, q);
  for (int ax = 0; ax < g.nd; ax++) { long long cnt[3]; long long L = spline_lines(sp, ax, cnt) * nsrc; for (long long q = 0; q < L; q++) spline_line(sp, ax, sp.cp[ax], q); }
  RayArgs ra; std::memset(&ra, 0, sizeof ra);
  ra.g = g; ra.nsrc = (int)nsrc; for (int d = 0; d < 3; d++) ra.m[d] = sp.m[d]; ra.cstride = sp.cstride; ra.coef_size = sp.coef_size;
  ra.coef = coef.data(); ra.coordsrc = cs.data(); ra.recoff = off.data(); ra.rec = rec.data();
  ra.rstep = is_cart(g) ? steplen * g.spac[0] : steplen; ra.thrdist = g.spac[0] * sqrt(2.0); ra.max_steps = 1LL << 24;
  std::vector<long long> np(nray), oo(nray); uint32_t err = 0; ra.npts = np.data(); ra.outoff = oo.data(); ra.err = &err;
  for (long long r = 0; r < nray; r++) { if (g.nd == 3) trace_one<3>(ra, r, 0); else trace_one<2>(ra, r, 0); }
  long long tot = 0; for (long long r = 0; r < nray; r++) { oo[r] = tot; tot += np[r]; }
  // writing pass with a room of exactly the counted points for odd rays and a generous one
  // (the counted points plus 7) for even rays, in the layout of a slab
  std::vector<long long> room(nray), soff(nray); long long slab = 0;
  for (long long r = 0; r < nray; r++) { room[r] = np[r] + ((r % 2) ? 0 : 7); soff[r] = slab; slab += room[r]; }
  std::vector<double> sl(slab * g.nd); ra.pts = sl.data(); ra.pts_size = slab * g.nd; ra.cap = room.data(); ra.outoff = soff.data();
  std::vector<long long> np2(nray); ra.npts = np2.data();
  for (long long r = 0; r < nray; r++) { if (g.nd == 3) trace_one<3>(ra, r, 1); else trace_one<2>(ra, r, 1); }
  for (long long r = 0; r < nray; r++) if (np2[r] != np[r]) { printf("count mismatch\n"); return 3; }
  std::vector<double> pts(tot * g.nd);
  for (long long r = 0; r < nray; r++) std::memcpy(pts.data() + oo[r] * g.nd, sl.data() + soff[r] * g.nd, sizeof(double) * np[r] * g.nd);
  FILE* o = fopen(argv[6], "wb"); fwrite(np.data(), 8, nray, o); fwrite(pts.data(), 8, pts.size(), o); fclose(o);
  printf("rays %lld points %lld err %u spline_err %u\n", nray, tot, err, serr);
  return 0;
}
