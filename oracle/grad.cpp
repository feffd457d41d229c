// Oracle adjoint path: projection operator, 2·diag(D t)·D products, sparse
// back-substitution, fine-grid chain rule, source-location derivative, source
// smoothing and the public eiktraveltime/eikgradient drivers.
// Test infrastructure only (see eikoracle.hpp).
#include "eikoracle.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <atomic>
#include <functional>
#include <thread>

namespace eikor {

// Compressed sparse column matrix built like SparseArrays.sparse(I,J,V,m,n):
// rows sorted inside each column, duplicates summed.
struct CSC {
  i64 m = 0, n = 0;
  std::vector<i64> colptr;
  std::vector<i64> rowval;
  std::vector<double> nzval;
};
static CSC sparse_from_triplets(const std::vector<i64>& I, const std::vector<i64>& J,
                                const std::vector<double>& V, i64 m, i64 n) {
  CSC A;
  A.m = m;
  A.n = n;
  std::vector<i64> idx(I.size());
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](i64 a, i64 b) {
    if (J[a] != J[b]) return J[a] < J[b];
    return I[a] < I[b];
  });
  A.colptr.assign(n + 1, 0);
  for (size_t q = 0; q < idx.size(); q++) {
    i64 k = idx[q];
    if (!A.rowval.empty() && q > 0 && J[idx[q - 1]] == J[k] && I[idx[q - 1]] == I[k]) {
      A.nzval.back() += V[k];
      continue;
    }
    A.rowval.push_back(I[k]);
    A.nzval.push_back(V[k]);
    A.colptr[J[k] + 1]++;
  }
  for (i64 c = 0; c < n; c++) A.colptr[c + 1] += A.colptr[c];
  return A;
}

// calcprojttfmmord (eikmaingrad.jl:878-937): rows = receivers, columns = FMM positions.
static CSC calcprojttfmmord(const Grid& g, const AdjointVars& adj, i64 nrec, const double* rec) {
  std::vector<i64> I, J;
  std::vector<double> V;
  for (i64 r = 0; r < nrec; r++) {
    double pt[3];
    for (int d = 0; d < g.nd; d++) pt[d] = rec[r * g.nd + d];
    double coeff[8];
    i64 ijk[8][3];
    int nc;
    interp_coeffs(g, pt, coeff, ijk, &nc);
    for (int l = 0; l < nc; l++) {
      i64 iorig = g.lin(ijk[l]);
      I.push_back(r);
      J.push_back((i64)adj.lgrid2fmm[iorig] - 1);
      V.push_back(coeff[l]);
    }
  }
  return sparse_from_triplets(I, J, V, nrec, g.npts());
}

// calc2diagDttD (eikmaingrad.jl:751-868)
struct TwoDtt {
  CSR R;          // rows x reduced columns (non-source), columns 0-based reduced index
  CSC S;          // rows x source columns
};
static TwoDtt calc2diagDttD(const CSR& D, const double* tt, const std::vector<uint8_t>& onsrccols) {
  TwoDtt out;
  const i64 nrows = D.nrows;
  i64 nsrcpts = 0;
  for (auto b : onsrccols) nsrcpts += b;
  std::vector<i64> idxrowred(onsrccols.size());
  std::vector<i64> srcrank(onsrccols.size());
  i64 q = 0, s = 0;
  for (size_t p = 0; p < onsrccols.size(); p++) {
    if (onsrccols[p]) {
      s++;
      idxrowred[p] = q;  // unused for source columns
    } else {
      q++;
      idxrowred[p] = q;
    }
    srcrank[p] = s;
  }
  out.R.nrows = nrows;
  out.R.ncols = D.ncols - nsrcpts;
  out.R.iptr.assign(nrows + 1, 0);
  std::vector<i64> SI, SJ;
  std::vector<double> SV;
  for (i64 i = 0; i < nrows; i++) {
    double tmp1 = 0.0;
    for (i64 l = D.iptr[i]; l < D.iptr[i + 1]; l++) tmp1 += D.v[l] * tt[D.j[l]];
    out.R.iptr[i + 1] = out.R.iptr[i];
    for (i64 l = D.iptr[i]; l < D.iptr[i + 1]; l++) {
      i64 j = D.j[l];
      double val = (2.0 * tmp1) * D.v[l];
      if (!onsrccols[j]) {
        out.R.iptr[i + 1] += 1;
        out.R.j.push_back((int32_t)(idxrowred[j] - 1));
        out.R.v.push_back(val);
      } else {
        SI.push_back(i);
        SJ.push_back(srcrank[j] - 1);
        SV.push_back(val);
      }
    }
  }
  out.S = sparse_from_triplets(SI, SJ, SV, nrows, nsrcpts);
  return out;
}

static CSC csc_add(const CSC& A, const CSC& B) {
  std::vector<i64> I, J;
  std::vector<double> V;
  for (i64 c = 0; c < A.n; c++)
    for (i64 k = A.colptr[c]; k < A.colptr[c + 1]; k++) {
      I.push_back(A.rowval[k]);
      J.push_back(c);
      V.push_back(A.nzval[k]);
    }
  for (i64 c = 0; c < B.n; c++)
    for (i64 k = B.colptr[c]; k < B.colptr[c + 1]; k++) {
      I.push_back(B.rowval[k]);
      J.push_back(c);
      V.push_back(B.nzval[k]);
    }
  return sparse_from_triplets(I, J, V, A.m, A.n);
}

// solveadjointeq (eikmaingrad.jl:488-535): LHS = Σ_d transpose(CSR_d) as CSC, then the
// column-oriented backward substitution of SparseArrays' UpperTriangular solve.
// B is column-major nrhs columns of length n (overwritten with the solution).
static void solveadjointeq(const std::vector<const CSR*>& R, double* B, i64 nrhs) {
  const i64 n = R[0]->nrows;
  // Column c of LHS = row c of the CSR matrices; entries summed over d in order.
  std::vector<i64> colptr(n + 1, 0);
  std::vector<i64> rows;
  std::vector<double> vals;
  rows.reserve(n * 4);
  vals.reserve(n * 4);
  std::vector<std::pair<i64, double>> tmp;
  for (i64 c = 0; c < n; c++) {
    tmp.clear();
    for (const CSR* M : R)
      for (i64 l = M->iptr[c]; l < M->iptr[c + 1]; l++) {
        i64 r = M->j[l];
        bool found = false;
        for (auto& e : tmp)
          if (e.first == r) {
            e.second = e.second + M->v[l];
            found = true;
            break;
          }
        if (!found) tmp.push_back({r, 0.0 + M->v[l]});
      }
    std::sort(tmp.begin(), tmp.end(), [](auto& a, auto& b) { return a.first < b.first; });
    for (auto& e : tmp) {
      rows.push_back(e.first);
      vals.push_back(e.second);
    }
    colptr[c + 1] = (i64)rows.size();
  }
  for (i64 k = 0; k < nrhs; k++) {
    double* x = B + k * n;
    for (i64 j = n - 1; j >= 0; j--) {
      i64 i1 = colptr[j], i2 = colptr[j + 1] - 1;
      i64 ii = i2;
      while (ii >= i1 && rows[ii] > j) ii--;
      if (ii < i1 || rows[ii] != j) jl_error("SingularException in adjoint triangular solve");
      double bj = x[j] / vals[ii];
      x[j] = bj;
      for (i64 i = ii - 1; i >= i1; i--) x[rows[i]] -= bj * vals[i];
    }
  }
}

// partderivttsrcpos (eikmaingrad.jl:1235-1273)
static void partderivttsrcpos(int nd, const double* xyzpt, const double* inpsrc, double vel,
                              double hgrid, double* deriv, uint32_t* warn) {
  const double shift = 1e-6 * hgrid;
  double src[3];
  for (int d = 0; d < nd; d++) {
    double align = jl_mod(inpsrc[d], hgrid);
    if (align <= 2.220446049250313e-16) {
      src[d] = inpsrc[d] + shift;
      if (warn) *warn |= WARN_SRCPOS_ALIGNED_SHIFT;
    } else {
      src[d] = inpsrc[d];
    }
  }
  double ss = 0.0;
  for (int d = 0; d < nd; d++) {
    double t = xyzpt[d] - src[d];
    ss = (d == 0) ? t * t : ss + t * t;
  }
  double denom = vel * std::sqrt(ss);
  if (denom == 0.0) {
    if (warn) *warn |= WARN_SRC_ON_NODE_DERIV;
    for (int d = 0; d < nd; d++) deriv[d] = 0.0;
    return;
  }
  for (int d = 0; d < nd; d++) deriv[d] = -(xyzpt[d] - src[d]) / denom;
}

// Fine-grid adjoint pieces (computestuff_finegrid!, eikmaingrad.jl:540-632).
struct FineAdj {
  i64 naccpts = 0, nsrc = 0, nh = 0;
  std::vector<i64> idxonH;        // FMM positions of h points (coarse-coincident)
  std::vector<double> lambda;     // (naccpts-nsrc) x nh, column-major
  std::vector<double> duh_dtaus;  // nh x nsrc, column-major
  std::vector<double> H_A;        // nh x nsrc dense (0/1)
};
static FineAdj computestuff_finegrid(const AdjointVars& adj) {
  FineAdj F;
  const i64 N = adj.grd.npts();
  F.naccpts = adj.lastcomputedtt;
  i64 firstneg = N;
  for (i64 i = 0; i < N; i++)
    if (adj.fmmtt[i] < 0.0) {
      firstneg = i;
      break;
    }
  EIKOR_ASSERT(firstneg == F.naccpts, "findfirst(adjvars.fmmord.ttime .< 0.0)-1 == Naccpts");
  const i64 na = F.naccpts;
  std::vector<uint8_t> onsrc(adj.onsrccols.begin(), adj.onsrccols.begin() + na);
  for (i64 p = 0; p < na; p++) F.nsrc += onsrc[p];
  for (i64 p = 0; p < na; p++)
    if (adj.onhpoints[p]) F.idxonH.push_back(p);
  F.nh = (i64)F.idxonH.size();
  const int nd = adj.grd.nd;
  std::vector<TwoDtt> tw(nd);
  std::vector<const CSR*> Rs;
  for (int d = 0; d < nd; d++) tw[d] = calc2diagDttD(adj.D[d], adj.fmmtt.data(), onsrc);
  for (int d = 0; d < nd; d++) Rs.push_back(&tw[d].R);
  const i64 nr = na - F.nsrc;
  // reduced column index of FMM positions
  std::vector<i64> red(na, -1), srck(na, -1);
  i64 q = 0, s = 0;
  for (i64 p = 0; p < na; p++) {
    if (onsrc[p]) srck[p] = s++;
    else red[p] = q++;
  }
  F.lambda.assign(nr * F.nh, 0.0);
  F.H_A.assign(F.nh * F.nsrc, 0.0);
  for (i64 l = 0; l < F.nh; l++) {
    i64 p = F.idxonH[l];
    if (onsrc[p]) F.H_A[l + F.nh * srck[p]] = 1.0;
    else F.lambda[red[p] + nr * l] = -1.0;  // rhs = copy(-transpose(H_Breg))
  }
  if (nr > 0) solveadjointeq(Rs, F.lambda.data(), F.nh);
  CSC S = tw[0].S;
  for (int d = 1; d < nd; d++) S = csc_add(S, tw[d].S);
  F.duh_dtaus.assign(F.nh * F.nsrc, 0.0);
  for (i64 k = 0; k < F.nsrc; k++)
    for (i64 e = S.colptr[k]; e < S.colptr[k + 1]; e++) {
      i64 i = S.rowval[e];
      double v = S.nzval[e];
      for (i64 h = 0; h < F.nh; h++) F.duh_dtaus[h + F.nh * k] += F.lambda[i + nr * h] * v;
    }
  return F;
}

// calc_duh_dva_finegrid! (eikmaingrad.jl:636-741); returns nh x nh column-major.
static std::vector<double> calc_duh_dva_finegrid(const FineAdj& F, const FMMVars& fine,
                                                 const AdjointVars& adj, const SrcRefinVars& srv) {
  const i64 na = F.naccpts, nsrc = F.nsrc, nh = F.nh, noff = na - nsrc;
  std::vector<double> duh_dwq(nh * na, 0.0);  // nh x na col-major
  for (i64 p = 0; p < noff; p++) {
    i64 iorig = adj.lfmm2grid[p + nsrc] - 1;
    double v = srv.velcart_fine[iorig];
    double v3 = v * v * v;
    for (i64 h = 0; h < nh; h++) duh_dwq[h + nh * (p + nsrc)] = 2.0 * F.lambda[p + noff * h] / v3;
  }
  std::vector<double> dtaus_dwa(nsrc);
  for (i64 l = 0; l < nsrc; l++)
    dtaus_dwa[l] = (-fine.distcorn[l]) * (1.0 / (fine.velcorn[l] * fine.velcorn[l]));
  for (i64 p = 0; p < nsrc; p++)
    for (i64 h = 0; h < nh; h++) duh_dwq[h + nh * p] += F.duh_dtaus[h + nh * p] * dtaus_dwa[p];
  for (i64 p = 0; p < nsrc; p++)
    for (i64 h = 0; h < nh; h++) duh_dwq[h + nh * p] += F.H_A[h + nh * p] * dtaus_dwa[p];
  std::vector<double> out(nh * nh, 0.0);
  for (i64 j = 0; j < nh; j++) {
    i64 q = F.idxonH[j];
    i64 qorig = srv.nearneigh_idxcoarse[adj.lfmm2grid[q] - 1];
    for (i64 p = 0; p < na; p++) {
      i64 porig = adj.lfmm2grid[p] - 1;
      if (srv.nearneigh_idxcoarse[porig] == qorig)
        for (i64 h = 0; h < nh; h++) out[h + nh * j] += duh_dwq[h + nh * p];
    }
  }
  return out;
}

// calcgrads_singlesrc! (eikmaingrad.jl:274-484). whichgrad: 1 vel, 2 srcloc, 3 both.
static double calcgrads_singlesrc(std::vector<double>& gradvel1, double* gradsrcpos1,
                                  const FMMVars& fv, const AdjointVars& adj, const double* xyzsrc,
                                  i64 nrec, const double* rec, const double* pickobs,
                                  const double* stdobs, const double* vel, const Grid& g,
                                  int whichgrad, bool refinearoundsrc, const FMMVars* fine,
                                  const AdjointVars* adjfine, const SrcRefinVars* srv,
                                  uint32_t* warn) {
  const int nd = g.nd;
  const i64 N = g.npts();
  CSC P = calcprojttfmmord(g, adj, nrec, rec);
  const double* tt = adj.fmmtt.data();
  std::vector<double> Pt(nrec, 0.0);
  for (i64 c = 0; c < P.n; c++)
    for (i64 k = P.colptr[c]; k < P.colptr[c + 1]; k++) Pt[P.rowval[k]] += P.nzval[k] * tt[c];
  std::vector<double> pickdiff(nrec), fact(nrec);
  double misfit1src = 0.0;
  for (i64 r = 0; r < nrec; r++) {
    pickdiff[r] = Pt[r] - pickobs[r];
    double sd2 = stdobs[r] * stdobs[r];
    misfit1src += (pickdiff[r] * pickdiff[r]) / sd2;
    fact[r] = pickdiff[r] / sd2;
  }
  i64 nsrc = 0;
  for (i64 p = 0; p < N; p++) nsrc += adj.onsrccols[p];
  std::vector<i64> red(N, -1), srck(N, -1);
  {
    i64 q = 0, s = 0;
    for (i64 p = 0; p < N; p++) {
      if (adj.onsrccols[p]) srck[p] = s++;
      else red[p] = q++;
    }
  }
  std::vector<TwoDtt> tw(nd);
  std::vector<const CSR*> Rs;
  for (int d = 0; d < nd; d++) tw[d] = calc2diagDttD(adj.D[d], tt, adj.onsrccols);
  for (int d = 0; d < nd; d++) Rs.push_back(&tw[d].R);
  const i64 nr = N - nsrc;
  std::vector<double> lambda(nr, 0.0);
  std::vector<double> dpsi_dus(nsrc, 0.0);
  for (i64 c = 0; c < N; c++) {
    double acc = 0.0, accA = 0.0;
    for (i64 k = P.colptr[c]; k < P.colptr[c + 1]; k++) {
      if (adj.onsrccols[c]) accA += P.nzval[k] * fact[P.rowval[k]];
      else acc += (-P.nzval[k]) * fact[P.rowval[k]];
    }
    if (adj.onsrccols[c]) dpsi_dus[srck[c]] = accA;
    else lambda[red[c]] = acc;
  }
  solveadjointeq(Rs, lambda.data(), 1);
  CSC S = tw[0].S;
  for (int d = 1; d < nd; d++) S = csc_add(S, tw[d].S);
  std::vector<double> y(nsrc, 0.0);  // ∂ψ∂up_∂up∂us
  for (i64 k = 0; k < nsrc; k++) {
    double a = 0.0;
    for (i64 e = S.colptr[k]; e < S.colptr[k + 1]; e++) a += S.nzval[e] * lambda[S.rowval[e]];
    y[k] = a;
  }

  FineAdj F;
  if (refinearoundsrc) F = computestuff_finegrid(*adjfine);

  if (whichgrad == 2 || whichgrad == 3) {
    if (g.sph()) jl_error("type " + std::string(g.nd == 2 ? "Grid2DSphere" : "Grid3DSphere") +
                          " has no field hgrid");
    std::vector<double> dus_dsr;  // npts x nd (row-major)
    i64 npts;
    if (!refinearoundsrc) {
      npts = nsrc;
      dus_dsr.assign(npts * nd, 0.0);
      for (i64 p = 0; p < npts; p++) {
        double xyzpt[3];
        for (int d = 0; d < nd; d++) xyzpt[d] = g.ax[d](fv.ijksrc[p][d]);
        double velsrc = vel[g.lin(fv.ijksrc[p].data())];
        partderivttsrcpos(nd, xyzpt, xyzsrc, velsrc, g.hgrid(), &dus_dsr[p * nd], warn);
      }
    } else {
      const Grid& gf = srv->grd_fine;
      const i64 nsf = F.nsrc;
      std::vector<double> dtaus_dsr(nsf * nd, 0.0);
      for (i64 p = 0; p < nsf; p++) {
        double xyzpt[3];
        for (int d = 0; d < nd; d++) xyzpt[d] = gf.ax[d](fine->ijksrc[p][d]);
        double velsrc = srv->velcart_fine[gf.lin(fine->ijksrc[p].data())];
        partderivttsrcpos(nd, xyzpt, xyzsrc, velsrc, gf.hgrid(), &dtaus_dsr[p * nd], warn);
      }
      npts = F.nh;
      dus_dsr.assign(npts * nd, 0.0);
      for (i64 h = 0; h < F.nh; h++)
        for (int d = 0; d < nd; d++) {
          double t1 = 0.0, t2 = 0.0;
          for (i64 k = 0; k < nsf; k++) {
            t1 += F.duh_dtaus[h + F.nh * k] * dtaus_dsr[k * nd + d];
            t2 += F.H_A[h + F.nh * k] * dtaus_dsr[k * nd + d];
          }
          dus_dsr[h * nd + d] = t1 + t2;
        }
    }
    for (int d = 0; d < nd; d++) {
      double a = 0.0, b = 0.0;
      for (i64 p = 0; p < npts; p++) {
        a += dus_dsr[p * nd + d] * y[p];
        b += dus_dsr[p * nd + d] * dpsi_dus[p];
      }
      gradsrcpos1[d] = a + b;
    }
  }

  if (whichgrad == 1 || whichgrad == 3) {
    for (i64 p = 0; p < nr; p++) {
      i64 iorig = adj.lfmm2grid[p + nsrc] - 1;
      double v = vel[iorig];
      gradvel1[iorig] = 2.0 * lambda[p] / (v * v * v);
    }
    std::vector<double> T2Va(nsrc, 0.0), T1Va(nsrc, 0.0);
    if (!refinearoundsrc) {
      for (i64 l = 0; l < nsrc; l++) {
        double dd = (-fv.distcorn[l]) * (1.0 / (fv.velcorn[l] * fv.velcorn[l]));
        T2Va[l] = dd * y[l];
        T1Va[l] = dd * dpsi_dus[l];
      }
    } else {
      std::vector<double> duh_dva = calc_duh_dva_finegrid(F, *fine, *adjfine, *srv);
      const i64 nh = F.nh;
      EIKOR_ASSERT(nh == nsrc, "size(dus_dva,1)==length(∂ψ∂up_∂up∂us)");
      for (i64 j = 0; j < nh; j++) {
        double a = 0.0, b = 0.0;
        for (i64 h = 0; h < nh; h++) {
          a += duh_dva[h + nh * j] * y[h];
          b += duh_dva[h + nh * j] * dpsi_dus[h];
        }
        T2Va[j] = a;
        T1Va[j] = b;
      }
    }
    for (i64 l = 0; l < nsrc; l++) gradvel1[g.lin(fv.ijksrc[l].data())] += T2Va[l];
    for (i64 l = 0; l < nsrc; l++) gradvel1[g.lin(fv.ijksrc[l].data())] += T1Va[l];
  }
  return misfit1src;
}

// smoothgradaroundsrc! (utils.jl:121-338). The off-grid 3D k-range is built from the x
// index (utils.jl:257-258, :307-308), kept as in the reference. The Grid3DSphere branch
// errors in the reference (:288-290); completed with the grid's own size fields.
void smoothgradaroundsrc(std::vector<double>& grad, const double* xyzsrc, const Grid& g,
                         i64 radiuspx) {
  if (radiuspx == 0) return;
  if (radiuspx < 0) jl_error("smoothgradaroundsrc!(): 'radius'<0 ");
  std::vector<std::array<i64, 3>> c;
  findenclosingbox(g, xyzsrc, c);
  const int nd = g.nd;
  double rmax = (double)radiuspx * g.spac[0];
  i64 imin, imax, jmin, jmax, kmin = 1, kmax = 1;
  if (c.size() == 1) {
    imin = c[0][0] - radiuspx;
    imax = c[0][0] + radiuspx;
    jmin = c[0][1] - radiuspx;
    jmax = c[0][1] + radiuspx;
    if (nd == 3) {
      kmin = c[0][2] - radiuspx;
      kmax = c[0][2] + radiuspx;
    }
  } else {
    imin = c[0][0] - radiuspx;
    imax = c[1][0] + radiuspx;
    jmin = c[0][1] - radiuspx;
    jmax = c[2][1] + radiuspx;
    if (nd == 3) {
      kmin = c[0][0] - radiuspx;
      kmax = c[3][0] + radiuspx;
    }
  }
  double xs[3] = {0, 0, 0};
  if (g.cart()) {
    for (int d = 0; d < nd; d++) xs[d] = xyzsrc[d];
  } else if (nd == 2) {
    xs[0] = xyzsrc[0] * cosd(xyzsrc[1]);
    xs[1] = xyzsrc[0] * sind(xyzsrc[1]);
  } else {
    xs[0] = xyzsrc[0] * sind(xyzsrc[1]) * cosd(xyzsrc[2]);
    xs[1] = xyzsrc[0] * sind(xyzsrc[1]) * sind(xyzsrc[2]);
    xs[2] = xyzsrc[0] * cosd(xyzsrc[1]);
  }
  for (i64 k = kmin; k <= kmax; k++)
    for (i64 j = jmin; j <= jmax; j++)
      for (i64 i = imin; i <= imax; i++) {
        if (i < 1 || i > g.n[0] || j < 1 || j > g.n[1]) continue;
        if (nd == 3 && (k < 1 || k > g.n[2])) continue;
        double xc[3] = {0.0, 0.0, 0.0};
        if (g.cart()) {
          xc[0] = g.ax[0](i);
          xc[1] = g.ax[1](j);
          if (nd == 3) xc[2] = g.ax[2](k);
        } else if (nd == 2) {
          double r = g.ax[0](i), th = g.ax[1](j);
          xc[0] = r * cosd(th);
          xc[1] = r * sind(th);
        } else {
          double r = g.ax[0](i), th = g.ax[1](j), ph = g.ax[2](k);
          xc[0] = r * sind(th) * cosd(ph);
          xc[1] = r * sind(th) * sind(ph);
          xc[2] = r * cosd(th);
        }
        double r;
        if (nd == 2) {
          double a = xc[0] - xs[0], b = xs[1] - xc[1];
          r = std::sqrt(a * a + b * b);
        } else {
          double a = xc[0] - xs[0], b = xs[1] - xc[1], e = xs[2] - xc[2];
          r = std::sqrt((a * a + b * b) + e * e);
        }
        if (r <= rmax) {
          double att = r / rmax;
          i64 p[3] = {i, j, k};
          grad[g.lin(p)] *= att;
        }
      }
}

// smoothgradient + gaussian_kernel + smoothimg (utils.jl:22-96).
void smoothgradient(i64 l, const Grid& g, std::vector<double>& grad) {
  // drop singleton dimensions
  std::vector<i64> sz;
  for (int d = 0; d < g.nd; d++)
    if (g.n[d] != 1) sz.push_back(g.n[d]);
  const int dim = (int)sz.size();
  const i64 half = l / 2;
  // kernel
  i64 kn = 1;
  for (int d = 0; d < dim; d++) kn *= l;
  std::vector<double> ker(kn);
  double s = ((double)l / 2.0) - std::sqrt((double)l / 2.0);
  double ksum = 0.0;
  for (i64 q = 0; q < kn; q++) {
    i64 rr = 0, t = q;
    for (int d = 0; d < dim; d++) {
      i64 jd = t % l + 1;
      t /= l;
      i64 pos = jd - (l / 2 + 1);
      rr += pos * pos;
    }
    double r = std::sqrt((double)rr);
    ker[q] = std::exp(-(r * r) / (2.0 * s));
  }
  for (i64 q = 0; q < kn; q++) ksum += ker[q];
  for (i64 q = 0; q < kn; q++) ker[q] = ker[q] / ksum;
  // padded image
  std::vector<i64> pd(dim);
  i64 np = 1;
  for (int d = 0; d < dim; d++) {
    pd[d] = sz[d] + l;
    np *= pd[d];
  }
  std::vector<double> pad(np, 0.0), filt(np, 0.0);
  auto padlin = [&](const i64* c) {
    i64 li = 0, m = 1;
    for (int d = 0; d < dim; d++) {
      li += (c[d] - 1) * m;
      m *= pd[d];
    }
    return li;
  };
  const i64 N = g.npts();
  for (i64 q = 0; q < N; q++) {
    i64 c[3], t = q;
    for (int d = 0; d < dim; d++) {
      c[d] = t % sz[d] + 1 + half;
      t /= sz[d];
    }
    pad[padlin(c)] = grad[q];
  }
  const i64 lk = l / 2 + 1;
  for (i64 q = 0; q < np; q++) {
    i64 I[3], t = q;
    for (int d = 0; d < dim; d++) {
      I[d] = t % pd[d] + 1;
      t /= pd[d];
    }
    bool inner = true;
    for (int d = 0; d < dim; d++)
      if (!(I[d] >= lk && I[d] <= pd[d] - lk + 1)) inner = false;
    if (inner) {
      double acc = 0.0;
      for (i64 kq = 0; kq < kn; kq++) {
        i64 J[3], tk = kq;
        bool in = true;
        for (int d = 0; d < dim; d++) {
          J[d] = tk % l - half;
          tk /= l;
          i64 p = I[d] + J[d];
          if (p < 1 || p > pd[d]) in = false;
        }
        if (!in) continue;
        i64 P[3];
        for (int d = 0; d < dim; d++) P[d] = I[d] + J[d];
        acc += pad[padlin(P)] * ker[kq];
      }
      filt[q] = acc;
    } else {
      filt[q] = pad[q];
    }
  }
  for (i64 q = 0; q < N; q++) {
    i64 c[3], t = q;
    for (int d = 0; d < dim; d++) {
      c[d] = t % sz[d] + 1 + half;
      t /= sz[d];
    }
    grad[q] = filt[padlin(c)];
  }
}

// ------------------------------------------------------------------- drivers --
// distribsrcs (eikutils.jl:171-190): inclusive 0-based [first,last] per group
static std::vector<std::pair<i64, i64>> distribsrcs(i64 nsrc, i64 nw) {
  std::vector<i64> sizes;
  if (nsrc >= nw) {
    i64 dis = nsrc / nw;
    sizes.assign(nw, dis);
    i64 resto = nsrc % nw;
    for (i64 i = 0; i < resto; i++) sizes[i] += 1;
  } else {
    sizes.assign(nsrc, 1);
  }
  std::vector<std::pair<i64, i64>> g;
  i64 c = 0;
  for (i64 s : sizes) {
    g.push_back({c, c + s - 1});
    c += s;
  }
  return g;
}

// checksrcrecposition (eikchecks.jl:4-50)
void checksrcrecposition(const Grid& g, i64 nsrc, const double* coordsrc, const i64* recoff,
                         const double* rec) {
  const int nd = g.nd;
  for (int d = 0; d < nd; d++) {
    double lo = g.ax[d](1), hi = g.ax[d].last();
    for (i64 s = 0; s < nsrc; s++) {
      double x = coordsrc[s * nd + d];
      EIKOR_ASSERT(lo <= x && x <= hi, "source position outside the grid");
    }
    for (i64 r = 0; r < recoff[nsrc]; r++) {
      double x = rec[r * nd + d];
      EIKOR_ASSERT(lo <= x && x <= hi, "receiver position outside the grid");
    }
  }
}

static FMMVars make_fmmvars(const Grid& g, bool refine) {
  FMMVars fv;
  fv.grd = g;
  fv.ttime.assign(g.npts(), 0.0);
  fv.status.assign(g.npts(), 0);
  fv.bheap.init(g.npts());
  fv.refinearoundsrc = refine;
  fv.is_srcbox = !refine;
  return fv;
}

// Threads.@threads over source groups (:sharedmem): groups are handed out to nthreads
// worker threads; each group runs exactly as in the serial driver.
static void parallel_groups(int ng, int nthreads, const std::function<void(int)>& fn) {
  if (nthreads <= 1 || ng <= 1) {
    for (int gi = 0; gi < ng; gi++) fn(gi);
    return;
  }
  std::atomic<int> next(0);
  std::vector<std::thread> pool;
  for (int t = 0; t < std::min(nthreads, ng); t++)
    pool.emplace_back([&]() {
      for (int gi = next++; gi < ng; gi = next++) fn(gi);
    });
  for (auto& th : pool) th.join();
}

// eiktraveltime + ttforwsomesrc (eikmainfwd.jl:33-199)
void eiktraveltime(const Grid& g, const double* vel, i64 nsrc, const double* coordsrc,
                   const i64* recoff, const double* rec, const ExtraParams& ep, double* picks,
                   double* ttgrids, uint32_t* warn) {
  const i64 N = g.npts();
  for (i64 i = 0; i < N; i++) EIKOR_ASSERT(vel[i] > 0.0, "all(vel.>0.0)");
  checksrcrecposition(g, nsrc, coordsrc, recoff, rec);
  auto groups = (ep.parallelkind == 0) ? distribsrcs(nsrc, 1) : distribsrcs(nsrc, std::max(1, ep.nthreads));
  if (nsrc == 0) return;
  std::vector<uint32_t> gwarn(groups.size(), 0);
  std::vector<std::string> gerr(groups.size());
  const int ng = (int)groups.size();
  parallel_groups(ng, ep.nthreads, [&](int gi) {
    try {
      FMMVars fv = make_fmmvars(g, ep.refinearoundsrc);
      FMMStats st;
      for (i64 s = groups[gi].first; s <= groups[gi].second; s++) {
        ttFMM_hiord(fv, vel, coordsrc + s * g.nd, nullptr, ep, nullptr, nullptr, nullptr, &st);
        for (i64 r = recoff[s]; r < recoff[s + 1]; r++) picks[r] = interpolate_receiver(fv.ttime, g, rec + r * g.nd);
        if (ttgrids) std::memcpy(ttgrids + s * N, fv.ttime.data(), sizeof(double) * N);
      }
      gwarn[gi] = st.warn;
    } catch (const std::exception& e) {
      gerr[gi] = e.what();
    }
  });
  for (int gi = 0; gi < ng; gi++) {
    if (!gerr[gi].empty()) throw OracleError(2, gerr[gi]);
    if (warn) *warn |= gwarn[gi];
  }
}

// calcgradsomesrc (eikmaingrad.jl:174-258) for sources [s0, s1]
static void calcgradsomesrc(const Grid& g, const double* vel, i64 s0, i64 s1, const double* coordsrc,
                            const i64* recoff, const double* rec, const double* pickobs,
                            const double* stdobs, int whichgrad, const ExtraParams& ep,
                            std::vector<double>& gradvelall, double* gradsrcpos, double& totmisf,
                            uint32_t* warn) {
  const i64 N = g.npts();
  std::vector<double> gradvel1(N, 0.0);
  gradvelall.assign(N, 0.0);
  FMMVars fv = make_fmmvars(g, ep.refinearoundsrc);
  AdjointVars adj;
  adj.init(g);
  totmisf = 0.0;
  FMMStats st;
  for (i64 s = s0; s <= s1; s++) {
    const double* src = coordsrc + s * g.nd;
    FMMVars fine;
    AdjointVars adjf;
    SrcRefinVars srv;
    ttFMM_hiord(fv, vel, src, &adj, ep, &fine, &adjf, &srv, &st);
    double* gsp = gradsrcpos ? gradsrcpos + s * g.nd : nullptr;
    double tmp[3];
    const i64 nrec = recoff[s + 1] - recoff[s];
    double m = calcgrads_singlesrc(gradvel1, gsp ? gsp : tmp, fv, adj, src, nrec, rec + recoff[s] * g.nd,
                                   pickobs + recoff[s], stdobs + recoff[s], vel, g, whichgrad,
                                   ep.refinearoundsrc, &fine, &adjf, &srv, &st.warn);
    totmisf += 0.5 * m;
    if (whichgrad == 1 || whichgrad == 3) {
      smoothgradaroundsrc(gradvel1, src, g, ep.radiussmoothgradsrc);
      for (i64 i = 0; i < N; i++) gradvelall[i] += gradvel1[i];
    }
  }
  if (warn) *warn |= st.warn;
}

// eikgradient (eikmaingrad.jl:31-164)
void eikgradient(const Grid& g, const double* vel, i64 nsrc, const double* coordsrc,
                 const i64* recoff, const double* rec, const double* pickobs, const double* stdobs,
                 int whichgrad, const ExtraParams& ep, double* gradvel, double* gradsrc,
                 double* misfit, uint32_t* warn) {
  EIKOR_ASSERT(whichgrad >= 1 && whichgrad <= 3, "Symbol 'whichgrad' not in (:gradvel, :gradsrcloc, :gradvelandsrcloc)");
  const i64 N = g.npts();
  for (i64 i = 0; i < N; i++) EIKOR_ASSERT(vel[i] > 0.0, "all(vel.>0.0)");
  for (i64 r = 0; r < recoff[nsrc]; r++) (void)stdobs[r];
  checksrcrecposition(g, nsrc, coordsrc, recoff, rec);
  if (ep.parallelkind == 2) jl_error("BoundsError: :distribmem gradient path returns 3 values into 2");
  auto groups = (ep.parallelkind == 0) ? distribsrcs(nsrc, 1) : distribsrcs(nsrc, std::max(1, ep.nthreads));
  const int ng = (int)groups.size();
  std::vector<std::vector<double>> gall(ng);
  std::vector<double> gmisf(ng, 0.0);
  std::vector<uint32_t> gwarn(ng, 0);
  std::vector<std::string> gerr(ng);
  parallel_groups(ng, ep.nthreads, [&](int gi) {
    try {
      calcgradsomesrc(g, vel, groups[gi].first, groups[gi].second, coordsrc, recoff, rec, pickobs,
                      stdobs, whichgrad, ep, gall[gi], gradsrc, gmisf[gi], &gwarn[gi]);
    } catch (const std::exception& e) {
      gerr[gi] = e.what();
    }
  });
  for (int gi = 0; gi < ng; gi++)
    if (!gerr[gi].empty()) throw OracleError(2, gerr[gi]);
  std::vector<double> tot(N, 0.0);
  double m = 0.0;
  for (int gi = 0; gi < ng; gi++) {
    if (gi == 0) {
      tot = gall[0];
      m = gmisf[0];
    } else {
      for (i64 i = 0; i < N; i++) tot[i] = tot[i] + gall[gi][i];
      m = m + gmisf[gi];
    }
    if (warn) *warn |= gwarn[gi];
  }
  if (ep.smoothgradkern > 0) smoothgradient(ep.smoothgradkern, g, tot);
  if (gradvel) std::memcpy(gradvel, tot.data(), sizeof(double) * N);
  if (misfit) *misfit = m;
}

}  // namespace eikor
