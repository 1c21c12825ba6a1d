// Host coarsening of the solve path: strength of connection, Dirichlet-node
// marking and the sequential PMIS sweep, restated from the reference's MATLAB
// (sources/Preconditioner/AMG/coarsen/): coarsen.m:30-76,
// mark_isolated_nodes.m:1-8, cpt_SoC_dom.m:25-63, cpt_SoC_cla.m:107-159,
// cpt_PMIS.m:1-102.  Plus the MT19937 stream MATLAB's rng(0) draws from, the
// thin Householder QR used for qr(TV,0) and CSR transposes.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>

#include "host.h"
#include "../errors.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace chronos {

// ---- MT19937 -----------------------------------------------------------------
void MT19937::seed_(uint32_t s) {
  mt_[0] = s;
  for (int i = 1; i < 624; ++i)
    mt_[i] = 1812433253u * (mt_[i - 1] ^ (mt_[i - 1] >> 30)) + (uint32_t)i;
  mti_ = 624;
}

uint32_t MT19937::next_u32() {
  static const uint32_t mag01[2] = {0u, 0x9908b0dfu};
  if (mti_ >= 624) {
    int k = 0;
    for (; k < 624 - 397; ++k) {
      uint32_t y = (mt_[k] & 0x80000000u) | (mt_[k + 1] & 0x7fffffffu);
      mt_[k] = mt_[k + 397] ^ (y >> 1) ^ mag01[y & 1u];
    }
    for (; k < 623; ++k) {
      uint32_t y = (mt_[k] & 0x80000000u) | (mt_[k + 1] & 0x7fffffffu);
      mt_[k] = mt_[k + (397 - 624)] ^ (y >> 1) ^ mag01[y & 1u];
    }
    uint32_t y = (mt_[623] & 0x80000000u) | (mt_[0] & 0x7fffffffu);
    mt_[623] = mt_[396] ^ (y >> 1) ^ mag01[y & 1u];
    mti_ = 0;
  }
  uint32_t y = mt_[mti_++];
  y ^= (y >> 11);
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= (y >> 18);
  return y;
}

// ---- CSR transposes ---------------------------------------------------------
// Transpose of A with rows ascending in each column.  Parallel over blocks
// of rows: every thread counts the columns of its block, the positions are
// laid out column by column in block order, and every thread scatters its
// block -- the same output as the sequential pass.
HostCSR csr_transpose(const HostCSR &A) {
  HostCSR T;
  T.nrows = A.ncols;
  T.ncols = A.nrows;
  T.rp.assign((size_t)T.nrows + 1, 0);
  const int64_t nnz = A.nnz();
  const int nc = A.ncols;
  int nt = 1;
#ifdef _OPENMP
  nt = std::max(1, std::min(omp_get_max_threads(), (int)(nnz / 262144) + 1));
#endif
  std::vector<int> rb(nt + 1);
  for (int t = 0; t <= nt; ++t) rb[t] = (int)((int64_t)A.nrows * t / nt);
  std::vector<std::vector<int64_t>> pos(nt, std::vector<int64_t>(nc, 0));
#pragma omp parallel for num_threads(nt) schedule(static, 1)
  for (int t = 0; t < nt; ++t)
    for (int64_t k = A.rp[rb[t]]; k < A.rp[rb[t + 1]]; ++k) pos[t][A.ci[k]]++;
  int64_t run = 0;
  for (int c = 0; c < nc; ++c) {
    for (int t = 0; t < nt; ++t) {
      const int64_t cnt = pos[t][c];
      pos[t][c] = run;
      run += cnt;
    }
    T.rp[(size_t)c + 1] = run;
  }
  T.ci.resize(nnz);
  T.v.resize(nnz);
  const bool vals = !A.v.empty();
#pragma omp parallel for num_threads(nt) schedule(static, 1)
  for (int t = 0; t < nt; ++t) {
    std::vector<int64_t> &p = pos[t];
    for (int i = rb[t]; i < rb[t + 1]; ++i)
      for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        const int64_t d = p[A.ci[k]]++;
        T.ci[d] = i;
        T.v[d] = vals ? A.v[k] : 0.0;
      }
  }
  return T;
}


// ---- strength of connection ------------------------------------------------
static std::vector<double> diagonal(const HostCSR &A) {
  std::vector<double> d(A.nrows, 0.0);
  for (int i = 0; i < A.nrows; ++i)
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] == i) d[i] = A.v[k];
  return d;
}

HostCSR soc_matrix(const HostCSR &A, const char *soc_type, double tau) {
  const int n = A.nrows;
  std::string t(soc_type);
  for (auto &c : t) c = (char)toupper(c);
  HostCSR S;
  S.nrows = S.ncols = n;
  S.rp.assign((size_t)n + 1, 0);
  std::vector<double> d = diagonal(A);
  if (t == "DOM") {
    // cpt_SoC_dom.m:26-47: s_ij = |a_ij| / sqrt(d_i d_j), strong if s_ij > tau.
    CHRONOS_REQUIRE(tau >= 0, CHRONOS_ENOTSUP, "DOM strength with tau < 0 is outside this path");
    // rows counted, then filled, in parallel (the same entries in row order)
    auto strong = [&](int i, int64_t k, double &s) {
      const double a = A.v[k];
      if (a == 0.0) return false;
      s = std::fabs(a) / std::sqrt(d[i] * d[A.ci[k]]);
      return s > tau;
    };
#pragma omp parallel for schedule(static, 4096)
    for (int i = 0; i < n; ++i) {
      int64_t c = 0;
      double s;
      for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) c += strong(i, k, s) ? 1 : 0;
      S.rp[(size_t)i + 1] = c;
    }
    for (int i = 0; i < n; ++i) S.rp[(size_t)i + 1] += S.rp[i];
    S.ci.resize(S.rp[n]);
    S.v.resize(S.rp[n]);
#pragma omp parallel for schedule(static, 4096)
    for (int i = 0; i < n; ++i) {
      int64_t o = S.rp[i];
      double s;
      for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
        if (strong(i, k, s)) { S.ci[o] = A.ci[k]; S.v[o] = s; ++o; }
    }
    return S;
  }
  if (t == "CLA") {
    // cpt_SoC_cla.m:109-159.  Column minimum of the off-diagonal part counts
    // implicit zeros (MATLAB min over a sparse column).
    std::vector<double> minc(n, 0.0), maxabs(n, 0.0);
    std::vector<int64_t> cnt(n, 0);
    for (int i = 0; i < n; ++i)
      for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        int j = A.ci[k];
        double a = A.v[k];
        if (j == i || a == 0.0) continue;
        if (cnt[j] == 0) minc[j] = a; else minc[j] = std::min(minc[j], a);
        maxabs[j] = std::max(maxabs[j], std::fabs(a));
        cnt[j]++;
      }
    bool all_nonneg = true;
    for (int j = 0; j < n; ++j) {
      if (cnt[j] < n) minc[j] = std::min(minc[j], 0.0);   // implicit zeros
      if (minc[j] < 0) all_nonneg = false;
    }
    for (int j = 0; j < n; ++j) {
      if (minc[j] == 0.0) minc[j] = 1.0;
      if (maxabs[j] == 0.0) maxabs[j] = 1.0;
    }
    for (int i = 0; i < n; ++i) {
      bool have_diag = false;
      for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        double a = A.v[k];
        if (a == 0.0) continue;
        int j = A.ci[k];
        double s = all_nonneg ? std::fabs(a) / std::max(maxabs[i], maxabs[j])
                              : a / std::max(minc[i], minc[j]);
        double val = s > tau ? s : 0.0;
        if (j == i) { val += 1.0; have_diag = true; }     // S + speye(nn)
        if (val != 0.0) { S.ci.push_back(j); S.v.push_back(val); }
      }
      if (!have_diag) {                                   // diagonal of speye
        auto pos = std::lower_bound(S.ci.begin() + S.rp[i], S.ci.end(), i) - S.ci.begin();
        S.ci.insert(S.ci.begin() + pos, i);
        S.v.insert(S.v.begin() + pos, 1.0);
      }
      S.rp[i + 1] = (int64_t)S.ci.size();
    }
    return S;
  }
  throw Error(CHRONOS_ENOTSUP, "SoC type " + t + " is outside this path (DOM, CLA)");
}

// ---- PMIS -------------------------------------------------------------------
std::vector<int> pmis_split(const HostCSR &A, const HostCSR &S, MT19937 &rng, int *nc_out) {
  const int n = S.nrows;
  // mark_isolated_nodes.m: columns of A with a single nonzero -> Dirichlet (-2)
  std::vector<int> colcnt(n, 0);
  for (int i = 0; i < A.nrows; ++i)
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.v[k] != 0.0) colcnt[A.ci[k]]++;
  std::vector<int> fc(n, 0);
  for (int j = 0; j < n; ++j)
    if (colcnt[j] == 1) fc[j] = -2;

  // S without its diagonal (rows counted, then filled, in parallel); its
  // transpose gives the columns S(:,inod)
  HostCSR So;
  So.nrows = So.ncols = n;
  So.rp.assign((size_t)n + 1, 0);
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < n; ++i) {
    int64_t c = 0;
    for (int64_t k = S.rp[i]; k < S.rp[i + 1]; ++k) c += (S.ci[k] != i && S.v[k] != 0.0);
    So.rp[(size_t)i + 1] = c;
  }
  for (int i = 0; i < n; ++i) So.rp[(size_t)i + 1] += So.rp[i];
  So.ci.resize(So.rp[n]);
  So.v.assign(So.rp[n], 1.0);
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < n; ++i) {
    int64_t o = So.rp[i];
    for (int64_t k = S.rp[i]; k < S.rp[i + 1]; ++k)
      if (S.ci[k] != i && S.v[k] != 0.0) So.ci[o++] = S.ci[k];
  }
  HostCSR St = csr_transpose(So);                 // row j of St = column j of S
  // S_sym = |S| + |S'|: union of the patterns of row j of S and of S'
  std::vector<int64_t> sym_rp((size_t)n + 1, 0);
  auto merge = [&](int j, int *out) {
    int64_t a = So.rp[j], ae = So.rp[j + 1], b = St.rp[j], be = St.rp[j + 1], m = 0;
    while (a < ae || b < be) {
      const int ca = a < ae ? So.ci[a] : INT32_MAX, cb = b < be ? St.ci[b] : INT32_MAX;
      const int c = std::min(ca, cb);
      if (out) out[m] = c;
      ++m;
      if (ca == c) ++a;
      if (cb == c) ++b;
    }
    return m;
  };
#pragma omp parallel for schedule(static, 4096)
  for (int j = 0; j < n; ++j) sym_rp[(size_t)j + 1] = merge(j, nullptr);
  for (int j = 0; j < n; ++j) sym_rp[(size_t)j + 1] += sym_rp[j];
  std::vector<int> sym_ci(sym_rp[n]);
#pragma omp parallel for schedule(static, 4096)
  for (int j = 0; j < n; ++j) merge(j, sym_ci.data() + sym_rp[j]);
  // nod_weight = sum(S ~= 0, 1)' + rand(nn,1)
  std::vector<double> w(n), wfree(n);
  for (int j = 0; j < n; ++j) w[j] = (double)(St.rp[j + 1] - St.rp[j]);
  for (int j = 0; j < n; ++j) w[j] += rng.next_res53();
  for (int j = 0; j < n; ++j) {
    if (fc[j] == -2) fc[j] = -1;
    wfree[j] = fc[j] == -1 ? -1.0 : w[j];
  }
  // cpt_PMIS.m's sweep makes an undecided node coarse once no undecided
  // neighbour (in S + S') outweighs it, and then makes the nodes it strongly
  // influences fine -- a coarse node included, which only a lighter node can
  // do.  The outcome therefore does not depend on the order of the sweep
  // (the weights differ: integer counts plus 53-bit random fractions), and
  // rounds give it in parallel: every undecided node that outweighs all its
  // undecided neighbours turns coarse (no two of them are neighbours), then
  // the nodes they influence turn fine, until no node is undecided.
  std::vector<int> und, next, newc;
  und.reserve(n);
  for (int j = 0; j < n; ++j)
    if (fc[j] == 0) und.push_back(j);
  std::vector<char> pick(n, 0);
  while (!und.empty()) {
    const int64_t m = (int64_t)und.size();
#pragma omp parallel for schedule(static, 1024)
    for (int64_t q = 0; q < m; ++q) {
      const int i = und[q];
      const double wi = w[i];
      bool is_coarse = true;
      for (int64_t k = sym_rp[i]; k < sym_rp[i + 1]; ++k)
        if (wfree[sym_ci[k]] > wi) { is_coarse = false; break; }
      pick[i] = is_coarse ? 1 : 0;
    }
    newc.clear();
    for (int64_t q = 0; q < m; ++q)
      if (pick[und[q]]) newc.push_back(und[q]);
    CHRONOS_REQUIRE(!newc.empty(), CHRONOS_EINVAL, "PMIS made no progress (equal node weights)");
    for (int i : newc) {
      fc[i] = 1;
      wfree[i] = -1.0;
    }
    const int64_t nn = (int64_t)newc.size();
#pragma omp parallel for schedule(static, 256)
    for (int64_t q = 0; q < nn; ++q) {
      const int i = newc[q];
      for (int64_t k = St.rp[i]; k < St.rp[i + 1]; ++k) {
        const int j = St.ci[k];
#pragma omp atomic write
        fc[j] = -1;
#pragma omp atomic write
        wfree[j] = -1.0;
      }
    }
    next.clear();
    for (int64_t q = 0; q < m; ++q)
      if (fc[und[q]] == 0) next.push_back(und[q]);
    und.swap(next);
    for (int i : newc) pick[i] = 0;
  }
  int nc = 0, nf = 0;
  for (int j = 0; j < n; ++j) {
    if (fc[j] > 0) fc[j] = ++nc;
    else fc[j] = -(++nf);
  }
  *nc_out = nc;
  return fc;
}

// ---- thin QR ------------------------------------------------------------------
// Householder QR with LAPACK's sign convention (beta = -sign(x1)*||x||); Q is
// accumulated explicitly into X (n x k, column-major).  Each reflector's
// projections on the other columns are independent: they run in parallel
// over the columns, each dot product summed in index order as a sequential
// loop would, and the column updates in parallel over the rows, so the result
// does not depend on the thread count.
void qr_orthonormalize(int n, int k, double *X) {
  if (k == 0 || n == 0) return;
  std::vector<double> V((size_t)n * k, 0.0), tau(k, 0.0), s(k, 0.0);
  std::vector<double> R(X, X + (size_t)n * k);
  const bool big = n > 65536;
  // s[jj] = tau_j * (v_j . M_jj) over rows j.. for columns jj0..k-1 of M
  auto project = [&](const double *v, const double *M, int j, int jj0) {
#pragma omp parallel for schedule(static, 1) if (big && k - jj0 > 1)
    for (int jj = jj0; jj < k; ++jj) {
      const double *cc = M + (size_t)jj * n;
      double t = 0;
      for (int i = j; i < n; ++i) t += v[i] * cc[i];
      s[jj] = t * tau[j];
    }
  };
  // M_jj -= s[jj] v_j over rows j.. for columns jj0..k-1
  auto update = [&](const double *v, double *M, int j, int jj0) {
#pragma omp parallel for schedule(static) if (big)
    for (int i = j; i < n; ++i)
      for (int jj = jj0; jj < k; ++jj) M[(size_t)jj * n + i] -= s[jj] * v[i];
  };
  for (int j = 0; j < k && j < n; ++j) {
    double *c = &R[(size_t)j * n];
    double nrm2 = 0;
    for (int i = j + 1; i < n; ++i) nrm2 += c[i] * c[i];
    double alpha = c[j];
    double *v = &V[(size_t)j * n];
    if (nrm2 == 0.0) { tau[j] = 0.0; v[j] = 1.0; continue; }
    double beta = -std::copysign(std::sqrt(alpha * alpha + nrm2), alpha);
    tau[j] = (beta - alpha) / beta;
    double scal = 1.0 / (alpha - beta);
    v[j] = 1.0;
#pragma omp parallel for schedule(static) if (big)
    for (int i = j + 1; i < n; ++i) {
      v[i] = c[i] * scal;
      c[i] = 0.0;
    }
    c[j] = beta;
    if (j + 1 < k) {
      project(v, R.data(), j, j + 1);
      update(v, R.data(), j, j + 1);
    }
  }
  // Q = H_0 H_1 ... H_{k-1} applied to the first k columns of I
#pragma omp parallel for schedule(static) if (big)
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < k; ++j) X[(size_t)j * n + i] = (i == j) ? 1.0 : 0.0;
  for (int j = std::min(k, n) - 1; j >= 0; --j) {
    const double *v = &V[(size_t)j * n];
    project(v, X, j, 0);
    update(v, X, j, 0);
  }
}

}  // namespace chronos
