// Adaptive symmetric FSAI pattern search on the host: for each row i, grow the
// strictly-lower pattern of G one Kaporin-gradient step at a time and re-solve
// the local SPD system, until the Kaporin decrease stalls or nstep steps are
// taken.  Restates the reference's algorithm
// (sources/Preconditioner/AMG/smoother/MEX_SYM_AFSAI/cpt_afsai_coef.cpp):
//   kap_grad        :227-312   gradient over candidate columns < i
//   ri_sortsplit    :40-89     partial selection of the step_size largest
//   gather_fullsys  :144-223   local system A[P,P] and rhs -A[P,i]
//   cpt_afsai_coef  :316-543   refinement loop, exit test, row scaling
// with the local Cholesky solve written here (LAPACK dpotrf/dpotrs in the
// reference).  tau = 0 (afsai_cpp.m:46): no dropping.
//
// Magnitudes.  Under g++/libstdc++ the reference's unqualified abs(double)
// binds to C's int abs, so |x| is computed as |(int)x| (truncation toward
// zero; outside the int range the x86 conversion yields INT_MIN, which abs
// leaves negative).  This affects the candidate ranking (:51,58) and the exit
// test (:466).  ref_abs = true reproduces it (the reference's actual output);
// ref_abs = false uses fabs.
#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "host.h"
#include "../errors.h"

namespace chronos {
namespace {

inline double mag(double x, bool ref_abs) {
  if (!ref_abs) return std::fabs(x);
  if (!(x > -2147483649.0 && x < 2147483648.0)) return -2147483648.0;
  int i = (int)x;
  return (double)(i < 0 ? -i : i);
}

// Brings the ncut largest magnitudes of R[0..n) to the front (quickselect
// partition with the first element as pivot, as ri_sortsplit).
void select_largest(int n, int ncut, double *R, int *I, bool ref_abs) {
  int first = 1, last = n;
  if (ncut < first || ncut > last) return;
  while (true) {
    int mid = first;
    const double pivot = mag(R[mid - 1], ref_abs);
    for (int j = first + 1; j <= last; ++j) {
      if (mag(R[j - 1], ref_abs) > pivot) {
        ++mid;
        std::swap(R[mid - 1], R[j - 1]);
        std::swap(I[mid - 1], I[j - 1]);
      }
    }
    std::swap(R[mid - 1], R[first - 1]);
    std::swap(I[mid - 1], I[first - 1]);
    if (mid == ncut) return;
    if (mid > ncut) last = mid - 1;
    else first = mid + 1;
  }
}

struct Work {
  // pattern (IWN[0..mrow)) followed by candidates, and the candidates'
  // gradients: n slots each, written before they are read, so left
  // uninitialised (zero-filling 12 bytes per row and thread was a visible
  // share of the search at a million rows)
  std::unique_ptr<int[]> pat;
  std::unique_ptr<double[]> grad;
  std::vector<int> mark;       // per column: -1 in pattern, >0 candidate slot, 0 free
  std::vector<double> M;       // mmax x mmax, column-major lower triangle
  std::vector<double> y, ysav; // current solution / saved right-hand side
};

// Gradient of the Kaporin number over candidate columns j < i not in the
// pattern; keeps the lfil largest and appends them to the pattern (sorted).
void grow_pattern(const HostCSR &A, int i, int lfil, int &mrow, Work &w, bool ref_abs) {
  int nw = 0;
  int *pat = w.pat.get();
  int *mark = w.mark.data();
  for (int64_t k = A.rp[i]; k < A.rp[i + 1] && A.ci[k] < i; ++k) {
    const int c = A.ci[k];
    if (mark[c] >= 0) {
      ++nw;
      mark[c] = nw;
      pat[mrow + nw - 1] = c;
      w.grad[nw - 1] = A.v[k];
    }
  }
  for (int p = 0; p < mrow; ++p) {
    const int r = pat[p];
    const double yr = w.y[p];
    for (int64_t k = A.rp[r]; k < A.rp[r + 1]; ++k) {
      const int c = A.ci[k];
      if (c >= i) continue;
      const int s = mark[c];
      if (s == 0) {
        ++nw;
        mark[c] = nw;
        pat[mrow + nw - 1] = c;
        w.grad[nw - 1] = yr * A.v[k];
      } else if (s > 0) {
        w.grad[s - 1] += yr * A.v[k];
      }
    }
  }
  const int ncut = std::min(lfil, nw);
  select_largest(nw, ncut, w.grad.get(), pat + mrow, ref_abs);
  for (int p = mrow; p < mrow + ncut; ++p) mark[pat[p]] = -1;
  for (int p = mrow + ncut; p < mrow + nw; ++p) mark[pat[p]] = 0;
  mrow += ncut;
  std::sort(pat, pat + mrow);
}

// Lower triangle of A[P,P] (column k from row P[k], entries P[j] >= P[k]) into
// M (ld = mmax), and rhs = -A[i, P].  Returns false when row i holds no entry
// left of the diagonal (the null right-hand side).
bool gather_system(const HostCSR &A, int i, int mrow, int mmax, Work &w) {
  const int *P = w.pat.get();
  for (int c = 0; c < mrow; ++c) {
    const int r = P[c];
    int64_t k = A.rp[r];
    const int64_t ke = A.rp[r + 1];
    double *col = w.M.data() + (size_t)c * mmax;
    for (int j = c; j < mrow; ++j) {
      while (k < ke && A.ci[k] < P[j]) ++k;
      col[j] = (k < ke && A.ci[k] == P[j]) ? A.v[k] : 0.0;
    }
  }
  int64_t k = A.rp[i];
  const int64_t ke = A.rp[i + 1];
  if (k >= ke || A.ci[k] >= i) return false;
  for (int j = 0; j < mrow; ++j) {
    while (k < ke && A.ci[k] < P[j]) ++k;
    w.y[j] = (k < ke && A.ci[k] == P[j]) ? -A.v[k] : 0.0;
  }
  return true;
}

// In-place Cholesky (lower, column-major, ld) and solve; false on breakdown.
bool chol_factor(int m, int ld, double *M) {
  for (int j = 0; j < m; ++j) {
    double d = M[(size_t)j * ld + j];
    for (int k = 0; k < j; ++k) d -= M[(size_t)k * ld + j] * M[(size_t)k * ld + j];
    if (!(d > 0.0)) return false;
    d = std::sqrt(d);
    M[(size_t)j * ld + j] = d;
    for (int r = j + 1; r < m; ++r) {
      double s = M[(size_t)j * ld + r];
      for (int k = 0; k < j; ++k) s -= M[(size_t)k * ld + r] * M[(size_t)k * ld + j];
      M[(size_t)j * ld + r] = s / d;
    }
  }
  return true;
}

void chol_solve(int m, int ld, const double *L, double *b) {
  for (int r = 0; r < m; ++r) {
    double s = b[r];
    for (int k = 0; k < r; ++k) s -= L[(size_t)k * ld + r] * b[k];
    b[r] = s / L[(size_t)r * ld + r];
  }
  for (int r = m - 1; r >= 0; --r) {
    double s = b[r];
    for (int k = r + 1; k < m; ++k) s -= L[(size_t)r * ld + k] * b[k];
    b[r] = s / L[(size_t)r * ld + r];
  }
}

inline double dot(int n, const double *a, const double *b) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

}  // namespace

FsaiResult fsai_adaptive(const HostCSR &A, int nstep, int step_size, double eps, int nthreads,
                         bool ref_abs) {
  const int n = A.nrows;
  const int mmax = nstep * step_size;
  const int kmax = 1 + mmax;
  std::vector<int> rowlen(n, 0);
  // each row's columns and values, written before they are read (not zeroed:
  // n * kmax * 12 bytes)
  std::unique_ptr<int[]> cols(new int[(size_t)std::max(n, 1) * kmax]);
  std::unique_ptr<double[]> vals(new double[(size_t)std::max(n, 1) * kmax]);
  int posdef_all = 1;

#pragma omp parallel num_threads(std::max(1, nthreads)) reduction(& : posdef_all)
  {
    Work w;
    w.pat.reset(new int[std::max(n, 1)]);
    w.grad.reset(new double[std::max(n, 1)]);
    w.mark.assign((size_t)n, 0);
    w.M.assign((size_t)std::max(mmax, 1) * std::max(mmax, 1), 0.0);
    w.y.assign((size_t)mmax + 1, 0.0);
    w.ysav.assign((size_t)mmax + 1, 0.0);
    int posdef = 1;
#pragma omp for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
      int mrow = 0;
      int istep = 0;
      double dk_old = 0.0;
      bool refine = nstep >= 1;
      while (refine) {
        ++istep;
        const int mold = mrow;
        grow_pattern(A, i, step_size, mrow, w, ref_abs);
        if (mrow > mold) {
          const bool has_rhs = gather_system(A, i, mrow, mmax, w);
          if (has_rhs && mrow > 0) {
            if (!chol_factor(mrow, mmax, w.M.data())) {
              posdef = 0;
            } else {
              w.ysav = w.y;
              chol_solve(mrow, mmax, w.M.data(), w.y.data());
            }
          }
          const double dk_new = dot(mrow, w.y.data(), w.ysav.data());
          if (istep == nstep) {
            refine = false;
          } else {
            refine = (mag(dk_new - dk_old, ref_abs) >= eps * dk_old) && (dk_new != 0.0);
            dk_old = dk_new;
          }
        } else {
          refine = false;
        }
      }
      // Row scaling 1/sqrt(a_ii - A_iP A_PP^{-1} A_Pi)
      double aii = 0.0;
      bool found = false;
      for (int64_t k = A.rp[i]; k < A.rp[i + 1] && A.ci[k] <= i; ++k)
        if (A.ci[k] == i) { aii = A.v[k]; found = true; break; }
      double scal = 0.0;
      if (!found) posdef = 0;
      else scal = aii - dot(mrow, w.ysav.data(), w.y.data());
      if (scal < 0.0) {
        posdef = 0;
        if (mrow > 0 && found) {
          gather_system(A, i, mrow, mmax, w);
          if (chol_factor(mrow, mmax, w.M.data())) {
            w.ysav = w.y;
            chol_solve(mrow, mmax, w.M.data(), w.y.data());
            scal = aii - dot(mrow, w.ysav.data(), w.y.data());
          }
        }
      }
      if (scal <= 0.0) { posdef = 0; scal = 1.0; }
      scal = 1.0 / std::sqrt(scal);
      int *oc = cols.get() + (size_t)i * kmax;
      double *ov = vals.get() + (size_t)i * kmax;
      for (int p = 0; p < mrow; ++p) {
        oc[p] = w.pat[p];
        ov[p] = scal * w.y[p];
        w.mark[w.pat[p]] = 0;
      }
      oc[mrow] = i;
      ov[mrow] = scal;
      rowlen[i] = mrow + 1;
    }
    posdef_all &= posdef;
  }
  FsaiResult out;
  out.posdef = posdef_all != 0;
  HostCSR &G = out.G;
  G.nrows = G.ncols = n;
  G.rp.assign((size_t)n + 1, 0);
  for (int i = 0; i < n; ++i) G.rp[i + 1] = G.rp[i] + rowlen[i];
  G.ci.resize(G.rp[n]);
  G.v.resize(G.rp[n]);
#pragma omp parallel for num_threads(std::max(1, nthreads)) schedule(static)
  for (int i = 0; i < n; ++i) {
    std::copy(cols.get() + (size_t)i * kmax, cols.get() + (size_t)i * kmax + rowlen[i],
              G.ci.begin() + G.rp[i]);
    std::copy(vals.get() + (size_t)i * kmax, vals.get() + (size_t)i * kmax + rowlen[i],
              G.v.begin() + G.rp[i]);
  }
  return out;
}

}  // namespace chronos
