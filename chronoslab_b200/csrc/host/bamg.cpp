// Host BAMG prolongation: least-squares interpolation of the test space from
// coarse neighbours chosen by a maximum-volume selection.  Restates the
// reference's algorithm (sources/Preconditioner/AMG/prolong/):
//   cpt_ProlMEX_BAMG.m:33-66        argument preparation
//   MEX_BAMG_Prol/BAMG.cpp:119-225  per-row neighbourhood growth and fit
//   add_new_neighs.cpp              breadth-first rings on the strength pattern
//   maxVol.cpp / maxVol_inner.cpp   rank-revealing Householder selection + swaps
//   Reduce_IntSet.cpp               shrinking the set while the row norm is large
// The dense least-squares fit uses a Householder QR of our own in place of
// LAPACK dgels; results agree with it to rounding.
#include <algorithm>
#include <cmath>
#include <vector>

#include "host.h"
#include "../errors.h"

namespace chronos {
namespace {

constexpr double kRelaxFac = 1.5;   // BAMG_params.h: RELAX_FAC

// Dense row-major scratch of one fine row: rows = candidate coarse nodes,
// columns = test vectors.
struct RowWork {
  std::vector<int> neigh, int_list, mark;
  std::vector<double> Z;            // n_int x ntv, row-major
  std::vector<double> w, coef, col, row, qr;
};

inline double dnrm2(int n, const double *x) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += x[i] * x[i];
  return std::sqrt(s);
}

// One breadth-first ring: every unmarked strong neighbour of ring [b, e).
void add_ring(const HostCSR &S, int b, int e, std::vector<int> &neigh, std::vector<int> &mark) {
  for (int r = b; r < e; ++r) {
    const int j = neigh[r];
    for (int64_t k = S.rp[j]; k < S.rp[j + 1]; ++k) {
      const int c = S.ci[k];
      if (!mark[c]) { mark[c] = 1; neigh.push_back(c); }
    }
  }
}

// Householder vector of v (length n) into w, normalised so that the
// reflection is I - 2 w w^T; zero vector -> w = 0.
void householder(int n, const double *v, double *w) {
  double n2 = 0.0;
  for (int i = 0; i < n; ++i) { w[i] = v[i]; n2 += v[i] * v[i]; }
  const double nv = std::sqrt(n2);
  if (nv == 0.0) { for (int i = 0; i < n; ++i) w[i] = 0.0; return; }
  double nw;
  if (w[0] == 0.0) { w[0] = nv; nw = std::sqrt(2.0 * n2); }
  else if (w[0] > 0.0) { nw = std::sqrt(2.0 * (w[0] * nv + n2)); w[0] += nv; }
  else { nw = std::sqrt(2.0 * (-w[0] * nv + n2)); w[0] -= nv; }
  const double inv = 1.0 / nw;
  for (int i = 0; i < n; ++i) w[i] *= inv;
}

inline void reflect(int n, const double *w, double *v) {
  double f = 0.0;
  for (int i = 0; i < n; ++i) f += w[i] * v[i];
  const double a = -2.0 * f;
  for (int i = 0; i < n; ++i) v[i] += a * w[i];
}

// Row of maximal norm over columns [c0, m) among rows [r0, n) moved to r0
// (first maximum wins); returns its norm and the original position.
void pivot_row(double *Z, int m, int r0, int n, int c0, std::vector<int> &list, double *nrm) {
  int best = r0;
  double bn = dnrm2(m - c0, Z + (size_t)r0 * m + c0);
  for (int r = r0 + 1; r < n; ++r) {
    double t = dnrm2(m - c0, Z + (size_t)r * m + c0);
    if (t > bn) { bn = t; best = r; }
  }
  if (best != r0) {
    for (int j = 0; j < m; ++j) std::swap(Z[(size_t)best * m + j], Z[(size_t)r0 * m + j]);
    std::swap(list[r0], list[best]);
  }
  *nrm = bn;
}

// Maximum-volume choice of at most min(n, m, mmax) rows of Z (n x m).  On
// return list[0..rank) are the chosen rows.  Z is overwritten.
int max_volume(int mmax, double condmax, int itmax, double delta, int n, int m, double *Z,
               std::vector<int> &list, RowWork &wk) {
  const int maxrank = std::min(std::min(n, m), mmax);
  wk.w.resize(m);
  int rank = 1;
  double sv_max;
  pivot_row(Z, m, 0, n, 0, list, &sv_max);
  householder(m, Z, wk.w.data());
  for (int r = 0; r < n; ++r) reflect(m, wk.w.data(), Z + (size_t)r * m);
  while (rank < maxrank) {
    ++rank;
    double nrm;
    pivot_row(Z, m, rank - 1, n, rank - 1, list, &nrm);
    const double an = std::fabs(nrm);
    const double cond = an > 1e-15 ? sv_max / an : condmax + 1.0;
    if (cond > condmax) { --rank; break; }
    householder(m - rank + 1, Z + (size_t)(rank - 1) * m + rank - 1, wk.w.data());
    for (int r = rank - 1; r < n; ++r)
      reflect(m - rank + 1, wk.w.data(), Z + (size_t)r * m + rank - 1);
  }
  // Rows [0, rank) now form a lower-triangular L (columns [0, rank)); the rest
  // B.  Z <- B L^{-1} for the remaining rows.
  const int nb = n - rank;
  double *B = Z + (size_t)rank * m;
  for (int i = rank - 1; i >= 0; --i)
    for (int k = nb - 1; k >= 0; --k) {
      double *zr = B + (size_t)k * m;
      zr[i] /= Z[(size_t)i * m + i];
      for (int j = i - 1; j >= 0; --j) zr[j] -= Z[(size_t)i * m + j] * zr[i];
    }
  // Swap rows while some |z_ij| > 1 + delta (largest first, column-major scan).
  auto find_max = [&](int &ir, int &jc) {
    ir = 0; jc = 0;
    double best = 0.0;
    for (int j = 0; j < rank; ++j)
      for (int i = 0; i < nb; ++i) {
        double v = std::fabs(B[(size_t)i * m + j]);
        if (v > best) { best = v; ir = i; jc = j; }
      }
    return best;
  };
  wk.col.resize(std::max(nb, 1));
  wk.row.resize(std::max(rank, 1));
  int ir, jc, it = 0;
  double zmax = find_max(ir, jc);
  while (zmax > 1.0 + delta && it < itmax) {
    ++it;
    for (int i = 0; i < nb; ++i) wk.col[i] = B[(size_t)i * m + jc];
    wk.col[ir] -= 1.0;
    const double fac = 1.0 / B[(size_t)ir * m + jc];
    for (int j = 0; j < rank; ++j) wk.row[j] = B[(size_t)ir * m + j] * fac;
    wk.row[jc] += fac;
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < rank; ++j) B[(size_t)i * m + j] -= wk.col[i] * wk.row[j];
    std::swap(list[ir + rank], list[jc]);
    zmax = find_max(ir, jc);
  }
  return rank;
}

// Least squares min || T w - t ||: T is ntv x rank with column k = TV row of
// chosen[k].  coef[0..rank) <- w; coef[rank..ntv) <- the residual components
// (as LAPACK dgels leaves them), whose norm is the fit error.
void lsq_fit(int ntv, int rank, const double *TV, const int *chosen, const double *t,
             RowWork &wk) {
  wk.qr.assign((size_t)ntv * rank, 0.0);
  for (int k = 0; k < rank; ++k)
    for (int r = 0; r < ntv; ++r) wk.qr[(size_t)k * ntv + r] = TV[(size_t)chosen[k] * ntv + r];
  wk.coef.assign(t, t + ntv);
  double *Q = wk.qr.data(), *b = wk.coef.data();
  for (int j = 0; j < rank; ++j) {
    double *c = Q + (size_t)j * ntv;
    double nrm2 = 0.0;
    for (int i = j + 1; i < ntv; ++i) nrm2 += c[i] * c[i];
    const double alpha = c[j];
    if (nrm2 == 0.0) continue;                       // H = I (tau = 0)
    const double beta = -std::copysign(std::sqrt(alpha * alpha + nrm2), alpha);
    const double tau = (beta - alpha) / beta, scal = 1.0 / (alpha - beta);
    for (int i = j + 1; i < ntv; ++i) c[i] *= scal;   // v = [1, c[j+1..]]
    c[j] = beta;
    auto apply = [&](double *x) {
      double s = x[j];
      for (int i = j + 1; i < ntv; ++i) s += c[i] * x[i];
      s *= tau;
      x[j] -= s;
      for (int i = j + 1; i < ntv; ++i) x[i] -= s * c[i];
    };
    for (int jj = j + 1; jj < rank; ++jj) apply(Q + (size_t)jj * ntv);
    apply(b);
  }
  for (int j = rank - 1; j >= 0; --j) {              // R w = (Q^T t)[0..rank)
    double s = b[j];
    for (int k = j + 1; k < rank; ++k) s -= Q[(size_t)k * ntv + j] * b[k];
    b[j] = s / Q[(size_t)j * ntv + j];
  }
}

// Loads the TV rows of the coarse candidates among neigh[1..) into Z.
int load_candidates(const std::vector<int> &neigh, const std::vector<int> &fc, const double *TV,
                    int ntv, RowWork &wk) {
  wk.int_list.clear();
  for (size_t i = 1; i < neigh.size(); ++i)
    if (fc[neigh[i]] >= 0) wk.int_list.push_back(neigh[i]);
  const int n_int = (int)wk.int_list.size();
  wk.Z.resize((size_t)std::max(n_int, 1) * ntv);
  for (int i = 0; i < n_int; ++i)
    for (int j = 0; j < ntv; ++j) wk.Z[(size_t)i * ntv + j] = TV[(size_t)wk.int_list[i] * ntv + j];
  return n_int;
}

// Fit with the best basis of at most mmax candidates.
int fit_row(int mmax, const BamgParams &p, int inod, const std::vector<int> &fc,
            const double *TV, int ntv, RowWork &wk, double *res_row, double *row_nrm,
            bool *has_candidates) {
  const int n_int = load_candidates(wk.neigh, fc, TV, ntv, wk);
  *has_candidates = n_int > 0;
  if (n_int == 0) {
    *res_row = dnrm2(ntv, TV + (size_t)inod * ntv);
    *row_nrm = 0.0;
    return 0;
  }
  int rank = max_volume(mmax, p.maxcond, p.itmax_vol, p.tol_vol, n_int, ntv, wk.Z.data(),
                        wk.int_list, wk);
  std::sort(wk.int_list.begin(), wk.int_list.begin() + rank);
  lsq_fit(ntv, rank, TV, wk.int_list.data(), TV + (size_t)inod * ntv, wk);
  *res_row = dnrm2(ntv - rank, wk.coef.data() + rank);
  *row_nrm = dnrm2(rank, wk.coef.data());
  return rank;
}

// Reduce_IntSet.cpp: drop one interpolation point at a time while the row
// norm exceeds `limit`.
int reduce_set(double limit, const BamgParams &p, int inod, int rank, const std::vector<int> &fc,
               const double *TV, int ntv, RowWork &wk, double *row_nrm) {
  while (*row_nrm > limit) {
    if (rank <= 1) { rank = 0; break; }
    const int n_int = load_candidates(wk.neigh, fc, TV, ntv, wk);
    rank = max_volume(rank - 1, p.maxcond, p.itmax_vol, p.tol_vol, n_int, ntv, wk.Z.data(),
                      wk.int_list, wk);
    std::sort(wk.int_list.begin(), wk.int_list.begin() + rank);
    lsq_fit(ntv, rank, TV, wk.int_list.data(), TV + (size_t)inod * ntv, wk);
    *row_nrm = dnrm2(rank, wk.coef.data());
  }
  return rank;
}

}  // namespace

namespace {

// One fine row (BAMG.cpp:119-225): neighbourhood rings, fit, set reduction.
// Appends the row's columns and values; returns its c_mark.
int bamg_row(const BamgParams &p, const HostCSR &S, const std::vector<int> &fc, const double *TV,
             int ntv, int inod, RowWork &wk, std::vector<int> &cols, std::vector<double> &vals) {
  const int mmax = p.mmax;
  int cmark = 0;
  wk.neigh.assign(1, inod);
  wk.mark[inod] = 1;
  int b = 0, e = 1, distance = 0;
  while (distance < p.dist_min) {
    ++distance;
    add_ring(S, b, e, wk.neigh, wk.mark);
    if ((int)wk.neigh.size() == e) break;
    b = e;
    e = (int)wk.neigh.size();
  }
  const double bnorm = dnrm2(ntv, TV + (size_t)inod * ntv);
  const double res_ass = p.eps * bnorm;
  double res_row = 0.0, row_nrm = 0.0;
  int rank = 0;
  bool more = true;
  while (more) {
    bool has_cand;
    rank = fit_row(mmax, p, inod, fc, TV, ntv, wk, &res_row, &row_nrm, &has_cand);
    if (row_nrm < p.maxrownrm && (res_row < res_ass || rank == ntv)) {
      more = false;
    } else if (distance < p.dist_max) {
      ++distance;
      const int before = (int)wk.neigh.size();
      add_ring(S, b, e, wk.neigh, wk.mark);
      if ((int)wk.neigh.size() == before) {
        more = false;
        if (!has_cand) {
          cmark = 1;
        } else {
          if (row_nrm > kRelaxFac * p.maxrownrm)
            rank = reduce_set(kRelaxFac * p.maxrownrm, p, inod, rank, fc, TV, ntv, wk, &row_nrm);
          res_row = rank == 0 ? bnorm : dnrm2(ntv - rank, wk.coef.data() + rank);
          if (!(res_row < res_ass)) cmark = 1;
        }
      }
      b = e;
      e = (int)wk.neigh.size();
    } else {
      more = false;
      if (row_nrm > kRelaxFac * p.maxrownrm)
        rank = reduce_set(kRelaxFac * p.maxrownrm, p, inod, rank, fc, TV, ntv, wk, &row_nrm);
      res_row = rank == 0 ? bnorm : dnrm2(ntv - rank, wk.coef.data() + rank);
      if (res_row > res_ass) cmark = 1;
    }
  }
  for (int k = 0; k < rank; ++k) {
    if (wk.coef[k] == 0.0) continue;              // explicit zeros are dropped
    cols.push_back(fc[wk.int_list[k]]);
    vals.push_back(wk.coef[k]);
  }
  for (int v : wk.neigh) wk.mark[v] = 0;
  return cmark;
}

}  // namespace

void bamg_rows_host(const BamgParams &p, const HostCSR &S, const std::vector<int> &fc,
                    const double *TV, int ntv, const std::vector<int> &rows,
                    std::vector<std::vector<int>> &rcols, std::vector<std::vector<double>> &rvals,
                    std::vector<int> &c_mark) {
  const int n = S.nrows;
#pragma omp parallel num_threads(p.nthreads)
  {
    RowWork wk;
    wk.mark.assign(n, 0);
#pragma omp for schedule(dynamic, 32)
    for (int r = 0; r < (int)rows.size(); ++r) {
      const int inod = rows[r];
      rcols[inod].clear();
      rvals[inod].clear();
      if (fc[inod] >= 0) {
        rcols[inod].assign(1, fc[inod]);
        rvals[inod].assign(1, 1.0);
        c_mark[inod] = 0;
        continue;
      }
      c_mark[inod] = bamg_row(p, S, fc, TV, ntv, inod, wk, rcols[inod], rvals[inod]);
    }
  }
}

HostCSR bamg_prolongation(const BamgParams &p, const HostCSR &S, const std::vector<int> &fc,
                          int nc, const double *TV, int ntv, std::vector<int> &c_mark) {
  const int n = S.nrows;
  c_mark.assign(n, 0);
  std::vector<std::vector<int>> rcols(n);
  std::vector<std::vector<double>> rvals(n);
  std::vector<int> rows(n);
  for (int i = 0; i < n; ++i) rows[i] = i;
  bamg_rows_host(p, S, fc, TV, ntv, rows, rcols, rvals, c_mark);
  HostCSR P;
  P.nrows = n;
  P.ncols = nc;
  P.rp.assign((size_t)n + 1, 0);
  for (int i = 0; i < n; ++i) P.rp[i + 1] = P.rp[i] + (int64_t)rcols[i].size();
  P.ci.resize(P.rp[n]);
  P.v.resize(P.rp[n]);
#pragma omp parallel for num_threads(p.nthreads) schedule(static, 4096)
  for (int i = 0; i < n; ++i) {
    std::copy(rcols[i].begin(), rcols[i].end(), P.ci.begin() + P.rp[i]);
    std::copy(rvals[i].begin(), rvals[i].end(), P.v.begin() + P.rp[i]);
  }
  return P;
}

}  // namespace chronos
