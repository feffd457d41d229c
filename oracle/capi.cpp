// C entry points of the oracle, bound from Python by oracle/eikoracle.py (ctypes).
// Test infrastructure only. Layouts: vel is column-major (x fastest); coordsrc is
// nsrc x nd row-major; receivers of all sources are concatenated row-major with
// offsets recoff[0..nsrc]; picks/pickobs/stdobs follow recoff.
#include "eikoracle.hpp"

#include <cstdio>
#include <cstring>

using namespace eikor;

namespace {
int report(const std::exception& e, char* errbuf, int errlen, int code) {
  if (errbuf && errlen > 0) {
    std::snprintf(errbuf, (size_t)errlen, "%s", e.what());
  }
  return code;
}
ExtraParams make_ep(int refine, int64_t ds, int64_t noderadius, int64_t rsmooth, int64_t kern,
                    int parallelkind, int nthreads) {
  ExtraParams ep;
  if (rsmooth < 0) jl_assert_fail("radiussmoothgradsrc>= 0");
  if (kern < 0) jl_assert_fail("smoothgradkern>=0");
  if (kern > 0 && kern % 2 == 0) jl_error("ExtraParams: smoothgradkern must be an odd number");
  if (parallelkind < 0 || parallelkind > 2)
    jl_error("ExtraParams(): 'parallelkind' must be one of :serial, :sharedmem or :distribmem");
  ep.refinearoundsrc = refine != 0;
  ep.downscalefactor = ds;
  ep.noderadius = noderadius;
  ep.radiussmoothgradsrc = rsmooth;
  ep.smoothgradkern = kern;
  ep.parallelkind = parallelkind;
  ep.nthreads = nthreads < 1 ? 1 : nthreads;
  return ep;
}
}  // namespace

extern "C" {

int eikor_traveltime(int kind, const int64_t* grsize, const double* spacing, const double* cooinit,
                     const double* vel, int64_t nsrc, const double* coordsrc, const int64_t* recoff,
                     const double* rec, int refine, int64_t ds, int64_t noderadius,
                     int parallelkind, int nthreads, double* picks, double* ttgrids,
                     uint32_t* warn, char* errbuf, int errlen) {
  try {
    Grid g = make_grid(kind, grsize, spacing, cooinit);
    ExtraParams ep = make_ep(refine, ds, noderadius, 3, 0, parallelkind, nthreads);
    if (warn) *warn = 0;
    eiktraveltime(g, vel, nsrc, coordsrc, recoff, rec, ep, picks, ttgrids, warn);
    return 0;
  } catch (const OracleError& e) {
    return report(e, errbuf, errlen, e.code);
  } catch (const std::exception& e) {
    return report(e, errbuf, errlen, 3);
  }
}

int eikor_gradient(int kind, const int64_t* grsize, const double* spacing, const double* cooinit,
                   const double* vel, int64_t nsrc, const double* coordsrc, const int64_t* recoff,
                   const double* rec, const double* pickobs, const double* stdobs, int whichgrad,
                   int refine, int64_t ds, int64_t noderadius, int64_t rsmooth, int64_t kern,
                   int parallelkind, int nthreads, double* gradvel, double* gradsrc,
                   double* misfit, uint32_t* warn, char* errbuf, int errlen) {
  try {
    Grid g = make_grid(kind, grsize, spacing, cooinit);
    ExtraParams ep = make_ep(refine, ds, noderadius, rsmooth, kern, parallelkind, nthreads);
    if (warn) *warn = 0;
    eikgradient(g, vel, nsrc, coordsrc, recoff, rec, pickobs, stdobs, whichgrad, ep, gradvel,
                gradsrc, misfit, warn);
    return 0;
  } catch (const OracleError& e) {
    return report(e, errbuf, errlen, e.code);
  } catch (const std::exception& e) {
    return report(e, errbuf, errlen, 3);
  }
}

// One source, forward with adjoint bookkeeping: coarse traveltimes, derivative codes
// (N x nd, row-major by node), FMM position of every node (1-based, 0 = unset) and the
// coarse source points. stats = {pops, nonmonotone_pops, max_batch, nsrcpts, warn}.
// The fine-grid state (if refinement is on) is returned through fine_* when the caller's
// capacity fine_cap is large enough (fine_n receives the fine grid size either way).
int eikor_forward_debug(int kind, const int64_t* grsize, const double* spacing,
                        const double* cooinit, const double* vel, const double* src, int refine,
                        int64_t ds, int64_t noderadius, double* tt, int8_t* codes,
                        int32_t* fmmpos, int64_t* srcpts, int64_t srcpts_cap, int64_t* stats,
                        int64_t* fine_n, int64_t fine_cap, double* fine_tt, uint8_t* fine_status,
                        int32_t* fine_fmmpos, int64_t* fine_nacc, int32_t* batch_out, char* errbuf,
                        int errlen) {
  try {
    Grid g = make_grid(kind, grsize, spacing, cooinit);
    ExtraParams ep = make_ep(refine, ds, noderadius, 3, 0, 0, 1);
    FMMVars fv;
    fv.grd = g;
    fv.ttime.assign(g.npts(), 0.0);
    fv.status.assign(g.npts(), 0);
    fv.bheap.init(g.npts());
    fv.refinearoundsrc = ep.refinearoundsrc;
    AdjointVars adj;
    adj.init(g);
    FMMVars fine;
    AdjointVars adjf;
    SrcRefinVars srv;
    FMMStats st;
    std::vector<int32_t> batches;
    if (batch_out) st.batch_of = &batches;
    ttFMM_hiord(fv, vel, src, &adj, ep, &fine, &adjf, &srv, &st);
    const int64_t N = g.npts();
    if (batch_out)
      for (int64_t i = 0; i < N; i++) batch_out[i] = batches.empty() ? -1 : batches[i];
    std::memcpy(tt, fv.ttime.data(), sizeof(double) * N);
    std::memcpy(codes, adj.code.data(), (size_t)(N * g.nd));
    for (int64_t i = 0; i < N; i++) fmmpos[i] = adj.lgrid2fmm[i];
    int64_t ns = (int64_t)fv.ijksrc.size();
    for (int64_t l = 0; l < ns && l < srcpts_cap; l++) srcpts[l] = g.lin(fv.ijksrc[l].data());
    stats[0] = st.pops;
    stats[1] = st.nonmonotone_pops;
    stats[2] = st.max_batch;
    stats[3] = ns;
    stats[4] = st.warn;
    if (fine_n) {
      for (int d = 0; d < 3; d++) fine_n[d] = ep.refinearoundsrc ? fine.grd.n[d] : 0;
      if (ep.refinearoundsrc) {
        const int64_t nf = fine.grd.npts();
        if (fine_nacc) *fine_nacc = adjf.lastcomputedtt;
        if (nf <= fine_cap) {
          if (fine_tt) std::memcpy(fine_tt, fine.ttime.data(), sizeof(double) * nf);
          if (fine_status) std::memcpy(fine_status, fine.status.data(), (size_t)nf);
          if (fine_fmmpos) {
            // position by node, from the FMM order of the accepted fine nodes
            for (int64_t i = 0; i < nf; i++) fine_fmmpos[i] = 0;
            for (int64_t p = 0; p < adjf.lastcomputedtt; p++)
              fine_fmmpos[adjf.lfmm2grid[p] - 1] = (int32_t)(p + 1);
          }
        }
      }
    }
    return 0;
  } catch (const OracleError& e) {
    return report(e, errbuf, errlen, e.code);
  } catch (const std::exception& e) {
    return report(e, errbuf, errlen, 3);
  }
}

// Julia-range node coordinate (Base.range(start, step, length)[i]) for tests.
double eikor_range_value(double start, double step, int64_t len, int64_t i1) {
  JRange r;
  r.init(start, step, len);
  return r(i1);
}

int eikor_smoothgradient(int kind, const int64_t* grsize, const double* spacing,
                         const double* cooinit, int64_t l, double* grad, char* errbuf, int errlen) {
  try {
    Grid g = make_grid(kind, grsize, spacing, cooinit);
    std::vector<double> v(grad, grad + g.npts());
    smoothgradient(l, g, v);
    std::memcpy(grad, v.data(), sizeof(double) * g.npts());
    return 0;
  } catch (const OracleError& e) {
    return report(e, errbuf, errlen, e.code);
  } catch (const std::exception& e) {
    return report(e, errbuf, errlen, 3);
  }
}

// Rays: pass 1 (pts NULL or cap too small) returns the point counts in npts and the total
// in *total; pass 2 with cap >= total also writes the points.
int eikor_tracerays(int kind, const int64_t* grsize, const double* spacing, const double* cooinit,
                    const double* ttgrids, int64_t nsrc, const double* coordsrc, const int64_t* recoff,
                    const double* rec, double steplen, int64_t max_steps, int64_t* npts, double* pts,
                    int64_t cap, int64_t* total, char* errbuf, int errlen) {
  try {
    Grid g = make_grid(kind, grsize, spacing, cooinit);
    std::vector<i64> np;
    std::vector<double> pp;
    tracerays(g, ttgrids, nsrc, coordsrc, recoff, rec, steplen, max_steps, np, pp);
    i64 tot = 0;
    for (size_t r = 0; r < np.size(); r++) {
      npts[r] = np[r];
      tot += np[r];
    }
    *total = tot;
    if (pts && cap >= tot) std::memcpy(pts, pp.data(), sizeof(double) * pp.size());
    return 0;
  } catch (const OracleError& e) {
    return report(e, errbuf, errlen, e.code);
  } catch (const std::exception& e) {
    return report(e, errbuf, errlen, 3);
  }
}

}  // extern "C"
