// BAMG prolongation on the GPU: the least-squares interpolation of
// host/bamg.cpp (restating MEX_BAMG_Prol/BAMG.cpp:119-225, add_new_neighs.cpp,
// maxVol.cpp, maxVol_inner.cpp, Reduce_IntSet.cpp), one thread per fine row.
//
// The host restatement is the reference here, bit for bit: every row runs the
// same operations in the same order -- breadth-first rings on the strength
// pattern in the pattern's column order, the maximum-volume selection with
// Householder reflections (first maximum wins every pivot and swap search),
// the back substitution and swap phase, the Householder least-squares fit,
// the set reduction -- with each product and sum rounded on its own (this
// file is compiled without fused multiply-adds, the host code with
// -ffp-contract=off), IEEE division and square root on both sides.  The ring
// search replaces the host's node marks (an array of n per thread) by a
// per-thread open-addressing set, which changes nothing in the order the
// neighbours are listed.
//
// Each thread works in its own slice of a global scratch area whose sizes
// are capped (512 to 8192 neighbours, by level size); a row whose neighbourhood would
// outgrow its slice stops, is flagged, and is computed by the host
// restatement, so the caps never change the result.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "hier.h"
#include "internal.h"

namespace chronos {

namespace {

constexpr int kBamgMaxTv = 16;               // test vectors
constexpr int64_t kBamgScratchBytes = int64_t(2) << 30;   // all threads' scratch together
constexpr double kRelaxFacDev = 1.5;         // BAMG_params.h: RELAX_FAC
constexpr int kBamgThreads = 128;

struct BamgDevParams {
  int itmax_vol, dist_min, dist_max, mmax, ntv;
  double maxcond, maxrownrm, tol_vol, eps;
  int maxneigh, hashsize;      // neighbours per thread; set slots (power of two, > 2 maxneigh)
};

// One thread's scratch.
struct RowScratch {
  int maxneigh, hmask;
  int *neigh, *int_list, *hash;
  double *Z, *col;
  double w[kBamgMaxTv], row[kBamgMaxTv], coef[kBamgMaxTv];
  double qr[kBamgMaxTv * kBamgMaxTv];
  int nneigh;
  bool overflow;
};

__device__ double d_nrm2(int n, const double *x) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += x[i] * x[i];
  return sqrt(s);
}

// Inserts node c into the thread's set; true when it was not there.
__device__ bool set_insert(RowScratch &w, int c) {
  unsigned h = ((unsigned)c * 2654435761u) & w.hmask;
  for (int probe = 0; probe <= w.hmask; ++probe) {
    const int v = w.hash[h];
    if (v == 0) { w.hash[h] = c + 1; return true; }
    if (v == c + 1) return false;
    h = (h + 1) & w.hmask;
  }
  return false;                                // full: more slots than maxneigh keeps this unreachable
}

// Empties the set.  Every key but the one that overflowed is listed in
// neigh, in insertion order; removing them newest first restores, at each
// step, the table as it was just after that key went in, so each one is
// found on its own probe path.  After an overflow the whole table is cleared.
__device__ void set_clear(RowScratch &w) {
  if (w.overflow) {
    for (int i = 0; i <= w.hmask; ++i) w.hash[i] = 0;
    return;
  }
  for (int i = w.nneigh - 1; i >= 0; --i) {
    unsigned h = ((unsigned)w.neigh[i] * 2654435761u) & w.hmask;
    while (w.hash[h] != 0) {
      if (w.hash[h] == w.neigh[i] + 1) { w.hash[h] = 0; break; }
      h = (h + 1) & w.hmask;
    }
  }
}

// add_ring: every unlisted strong neighbour of ring [b, e), in order.
__device__ void d_add_ring(const int *__restrict__ srp, const int *__restrict__ sci, int b, int e,
                           RowScratch &w) {
  for (int r = b; r < e && !w.overflow; ++r) {
    const int j = w.neigh[r];
    for (int k = srp[j]; k < srp[j + 1]; ++k) {
      const int c = sci[k];
      if (set_insert(w, c)) {
        if (w.nneigh == w.maxneigh) { w.overflow = true; return; }
        w.neigh[w.nneigh++] = c;
      }
    }
  }
}

__device__ void d_householder(int n, const double *v, double *wv) {
  double n2 = 0.0;
  for (int i = 0; i < n; ++i) { wv[i] = v[i]; n2 += v[i] * v[i]; }
  const double nv = sqrt(n2);
  if (nv == 0.0) { for (int i = 0; i < n; ++i) wv[i] = 0.0; return; }
  double nw;
  if (wv[0] == 0.0) { wv[0] = nv; nw = sqrt(2.0 * n2); }
  else if (wv[0] > 0.0) { nw = sqrt(2.0 * (wv[0] * nv + n2)); wv[0] += nv; }
  else { nw = sqrt(2.0 * (-wv[0] * nv + n2)); wv[0] -= nv; }
  const double inv = 1.0 / nw;
  for (int i = 0; i < n; ++i) wv[i] *= inv;
}

__device__ void d_reflect(int n, const double *wv, double *v) {
  double f = 0.0;
  for (int i = 0; i < n; ++i) f += wv[i] * v[i];
  const double a = -2.0 * f;
  for (int i = 0; i < n; ++i) v[i] += a * wv[i];
}

__device__ void d_pivot_row(double *Z, int m, int r0, int n, int c0, int *list, double *nrm) {
  int best = r0;
  double bn = d_nrm2(m - c0, Z + (size_t)r0 * m + c0);
  for (int r = r0 + 1; r < n; ++r) {
    const double t = d_nrm2(m - c0, Z + (size_t)r * m + c0);
    if (t > bn) { bn = t; best = r; }
  }
  if (best != r0) {
    for (int j = 0; j < m; ++j) {
      const double t = Z[(size_t)best * m + j];
      Z[(size_t)best * m + j] = Z[(size_t)r0 * m + j];
      Z[(size_t)r0 * m + j] = t;
    }
    const int t = list[r0];
    list[r0] = list[best];
    list[best] = t;
  }
  *nrm = bn;
}

__device__ int d_max_volume(int mmax, double condmax, int itmax, double delta, int n, int m,
                            RowScratch &w) {
  double *Z = w.Z;
  int *list = w.int_list;
  const int maxrank = min(min(n, m), mmax);
  int rank = 1;
  double sv_max;
  d_pivot_row(Z, m, 0, n, 0, list, &sv_max);
  d_householder(m, Z, w.w);
  for (int r = 0; r < n; ++r) d_reflect(m, w.w, Z + (size_t)r * m);
  while (rank < maxrank) {
    ++rank;
    double nrm;
    d_pivot_row(Z, m, rank - 1, n, rank - 1, list, &nrm);
    const double an = fabs(nrm);
    const double cond = an > 1e-15 ? sv_max / an : condmax + 1.0;
    if (cond > condmax) { --rank; break; }
    d_householder(m - rank + 1, Z + (size_t)(rank - 1) * m + rank - 1, w.w);
    for (int r = rank - 1; r < n; ++r) d_reflect(m - rank + 1, w.w, Z + (size_t)r * m + rank - 1);
  }
  const int nb = n - rank;
  double *B = Z + (size_t)rank * m;
  for (int i = rank - 1; i >= 0; --i)
    for (int k = nb - 1; k >= 0; --k) {
      double *zr = B + (size_t)k * m;
      zr[i] /= Z[(size_t)i * m + i];
      for (int j = i - 1; j >= 0; --j) zr[j] -= Z[(size_t)i * m + j] * zr[i];
    }
  auto find_max = [&](int &ir, int &jc) {
    ir = 0;
    jc = 0;
    double best = 0.0;
    for (int j = 0; j < rank; ++j)
      for (int i = 0; i < nb; ++i) {
        const double v = fabs(B[(size_t)i * m + j]);
        if (v > best) { best = v; ir = i; jc = j; }
      }
    return best;
  };
  int ir, jc, it = 0;
  double zmax = find_max(ir, jc);
  while (zmax > 1.0 + delta && it < itmax) {
    ++it;
    for (int i = 0; i < nb; ++i) w.col[i] = B[(size_t)i * m + jc];
    w.col[ir] -= 1.0;
    const double fac = 1.0 / B[(size_t)ir * m + jc];
    for (int j = 0; j < rank; ++j) w.row[j] = B[(size_t)ir * m + j] * fac;
    w.row[jc] += fac;
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < rank; ++j) B[(size_t)i * m + j] -= w.col[i] * w.row[j];
    const int t = list[ir + rank];
    list[ir + rank] = list[jc];
    list[jc] = t;
    zmax = find_max(ir, jc);
  }
  return rank;
}

__device__ void d_lsq_fit(int ntv, int rank, const double *__restrict__ TV, const int *chosen,
                          const double *t, RowScratch &w) {
  double *Q = w.qr, *b = w.coef;
  for (int k = 0; k < rank; ++k)
    for (int r = 0; r < ntv; ++r) Q[(size_t)k * ntv + r] = TV[(size_t)chosen[k] * ntv + r];
  for (int r = 0; r < ntv; ++r) b[r] = t[r];
  for (int j = 0; j < rank; ++j) {
    double *c = Q + (size_t)j * ntv;
    double nrm2 = 0.0;
    for (int i = j + 1; i < ntv; ++i) nrm2 += c[i] * c[i];
    const double alpha = c[j];
    if (nrm2 == 0.0) continue;
    const double beta = -copysign(sqrt(alpha * alpha + nrm2), alpha);
    const double tau = (beta - alpha) / beta, scal = 1.0 / (alpha - beta);
    for (int i = j + 1; i < ntv; ++i) c[i] *= scal;
    c[j] = beta;
    for (int jj = j + 1; jj <= rank; ++jj) {      // jj == rank: the right-hand side
      double *x = jj < rank ? Q + (size_t)jj * ntv : b;
      double s = x[j];
      for (int i = j + 1; i < ntv; ++i) s += c[i] * x[i];
      s *= tau;
      x[j] -= s;
      for (int i = j + 1; i < ntv; ++i) x[i] -= s * c[i];
    }
  }
  for (int j = rank - 1; j >= 0; --j) {
    double s = b[j];
    for (int k = j + 1; k < rank; ++k) s -= Q[(size_t)k * ntv + j] * b[k];
    b[j] = s / Q[(size_t)j * ntv + j];
  }
}

__device__ int d_load_candidates(const int *__restrict__ fc, const double *__restrict__ TV,
                                 int ntv, RowScratch &w) {
  int n_int = 0;
  for (int i = 1; i < w.nneigh; ++i)
    if (fc[w.neigh[i]] >= 0) w.int_list[n_int++] = w.neigh[i];
  for (int i = 0; i < n_int; ++i)
    for (int j = 0; j < ntv; ++j) w.Z[(size_t)i * ntv + j] = TV[(size_t)w.int_list[i] * ntv + j];
  return n_int;
}

__device__ void d_sort_small(int *a, int n) {            // insertion sort (distinct ints)
  for (int i = 1; i < n; ++i) {
    const int v = a[i];
    int j = i - 1;
    while (j >= 0 && a[j] > v) { a[j + 1] = a[j]; --j; }
    a[j + 1] = v;
  }
}

__device__ int d_fit_row(int mmax, const BamgDevParams &p, int inod, const int *__restrict__ fc,
                         const double *__restrict__ TV, RowScratch &w, double *res_row,
                         double *row_nrm, bool *has_candidates) {
  const int ntv = p.ntv;
  const int n_int = d_load_candidates(fc, TV, ntv, w);
  *has_candidates = n_int > 0;
  if (n_int == 0) {
    *res_row = d_nrm2(ntv, TV + (size_t)inod * ntv);
    *row_nrm = 0.0;
    return 0;
  }
  const int rank = d_max_volume(mmax, p.maxcond, p.itmax_vol, p.tol_vol, n_int, ntv, w);
  d_sort_small(w.int_list, rank);
  d_lsq_fit(ntv, rank, TV, w.int_list, TV + (size_t)inod * ntv, w);
  *res_row = d_nrm2(ntv - rank, w.coef + rank);
  *row_nrm = d_nrm2(rank, w.coef);
  return rank;
}

__device__ int d_reduce_set(double limit, const BamgDevParams &p, int inod, int rank,
                            const int *__restrict__ fc, const double *__restrict__ TV,
                            RowScratch &w, double *row_nrm) {
  const int ntv = p.ntv;
  while (*row_nrm > limit) {
    if (rank <= 1) { rank = 0; break; }
    const int n_int = d_load_candidates(fc, TV, ntv, w);
    rank = d_max_volume(rank - 1, p.maxcond, p.itmax_vol, p.tol_vol, n_int, ntv, w);
    d_sort_small(w.int_list, rank);
    d_lsq_fit(ntv, rank, TV, w.int_list, TV + (size_t)inod * ntv, w);
    *row_nrm = d_nrm2(rank, w.coef);
  }
  return rank;
}

// Per fine row: out_cnt entries (column, value) in out_col / out_val[row *
// ntv ...]; c_mark; status 1 when the row outgrew the thread's scratch (the
// host computes it).  Coarse rows are the host's business too (one entry).
__global__ void __launch_bounds__(kBamgThreads)
k_bamg_rows(int n, const int *__restrict__ srp, const int *__restrict__ sci,
            const int *__restrict__ fc, const double *__restrict__ TV, BamgDevParams p,
            int *iscr, double *dscr, int *out_cnt, int *out_col, double *out_val, int *c_mark,
            int *status) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nthr = gridDim.x * blockDim.x;
  const int ntv = p.ntv;
  RowScratch w;
  const int mn = p.maxneigh;
  w.maxneigh = mn;
  w.hmask = p.hashsize - 1;
  w.neigh = iscr + (size_t)tid * (2 * (size_t)mn + p.hashsize);
  w.int_list = w.neigh + mn;
  w.hash = w.int_list + mn;
  w.Z = dscr + (size_t)tid * ((size_t)mn * (ntv + 1));
  w.col = w.Z + (size_t)mn * ntv;
  for (int i = 0; i < p.hashsize; ++i) w.hash[i] = 0;
  for (int inod = tid; inod < n; inod += nthr) {
    out_cnt[inod] = 0;
    c_mark[inod] = 0;
    status[inod] = 0;
    if (fc[inod] >= 0) continue;
    w.nneigh = 1;
    w.neigh[0] = inod;
    w.overflow = false;
    set_insert(w, inod);
    int b = 0, e = 1, distance = 0;
    while (distance < p.dist_min) {
      ++distance;
      d_add_ring(srp, sci, b, e, w);
      if (w.overflow || w.nneigh == e) break;
      b = e;
      e = w.nneigh;
    }
    const double bnorm = d_nrm2(ntv, TV + (size_t)inod * ntv);
    const double res_ass = p.eps * bnorm;
    double res_row = 0.0, row_nrm = 0.0;
    int rank = 0, cmark = 0;
    bool more = !w.overflow;
    while (more) {
      bool has_cand;
      rank = d_fit_row(p.mmax, p, inod, fc, TV, w, &res_row, &row_nrm, &has_cand);
      if (row_nrm < p.maxrownrm && (res_row < res_ass || rank == ntv)) {
        more = false;
      } else if (distance < p.dist_max) {
        ++distance;
        const int before = w.nneigh;
        d_add_ring(srp, sci, b, e, w);
        if (w.overflow) break;
        if (w.nneigh == before) {
          more = false;
          if (!has_cand) {
            cmark = 1;
          } else {
            if (row_nrm > kRelaxFacDev * p.maxrownrm)
              rank = d_reduce_set(kRelaxFacDev * p.maxrownrm, p, inod, rank, fc, TV, w, &row_nrm);
            res_row = rank == 0 ? bnorm : d_nrm2(ntv - rank, w.coef + rank);
            if (!(res_row < res_ass)) cmark = 1;
          }
        }
        b = e;
        e = w.nneigh;
      } else {
        more = false;
        if (row_nrm > kRelaxFacDev * p.maxrownrm)
          rank = d_reduce_set(kRelaxFacDev * p.maxrownrm, p, inod, rank, fc, TV, w, &row_nrm);
        res_row = rank == 0 ? bnorm : d_nrm2(ntv - rank, w.coef + rank);
        if (res_row > res_ass) cmark = 1;
      }
    }
    if (w.overflow) {
      status[inod] = 1;
    } else {
      int cnt = 0;
      for (int k = 0; k < rank; ++k) {
        if (w.coef[k] == 0.0) continue;             // explicit zeros are dropped
        out_col[(size_t)inod * ntv + cnt] = fc[w.int_list[k]];
        out_val[(size_t)inod * ntv + cnt] = w.coef[k];
        ++cnt;
      }
      out_cnt[inod] = cnt;
      c_mark[inod] = cmark;
    }
    set_clear(w);
  }
}

}  // namespace

HostCSR bamg_prolongation_device(const BamgParams &prm, const HostCSR &S,
                                 const std::vector<int> &fc, int nc, const double *TV, int ntv,
                                 std::vector<int> &c_mark, cudaStream_t st, int *host_rows,
                                 int max_neigh) {
  CHRONOS_REQUIRE(max_neigh == 0 || (max_neigh >= 16 && max_neigh <= 8192 &&
                                     (max_neigh & (max_neigh - 1)) == 0),
                  CHRONOS_EINVAL, "max_neigh must be 0 or a power of two in [16, 8192]");
  CHRONOS_REQUIRE(ntv >= 1 && ntv <= kBamgMaxTv && prm.mmax <= ntv, CHRONOS_ENOTSUP,
                  "BAMG on the GPU takes at most 16 test vectors");
  const int n = S.nrows;
  const bool verbose = std::getenv("CHRONOS_TUNE_VERBOSE") != nullptr;
  auto now = [] { return std::chrono::duration<double>(
                      std::chrono::steady_clock::now().time_since_epoch()).count(); };
  const double t0 = now();
  std::vector<int> srp_h(S.rp.begin(), S.rp.end());
  DBuf<int> srp, sci, dfc, out_cnt(n), out_col((size_t)n * ntv), cm(n), status(n);
  DBuf<double> dtv, out_val((size_t)n * ntv);
  srp.upload(srp_h, st);
  sci.upload(S.ci, st);
  dfc.upload(fc, st);
  dtv.upload(TV, (size_t)n * ntv, st);
  // Threads and the neighbourhood cap share a fixed scratch budget: a level
  // with many rows runs many threads with 512-node neighbourhoods; smaller
  // levels (coarse operators with wider rows and larger neighbourhoods)
  // fewer threads with up to 8192-node ones.
  const int blocks = (int)std::max<int64_t>(
      1, std::min<int64_t>(ceil_div(n, 16 * kBamgThreads), (int64_t)num_sms()));
  const int64_t nthr = (int64_t)blocks * kBamgThreads;
  int maxneigh = 512;
  while (maxneigh < 8192 &&
         nthr * (int64_t)(2 * maxneigh) * (int64_t)((ntv + 1) * 8 + 6 * 4) <=
             kBamgScratchBytes)
    maxneigh *= 2;
  if (max_neigh > 0) maxneigh = max_neigh;
  const int hashsize = 4 * maxneigh;
  DBuf<int> iscr((size_t)nthr * (2 * (size_t)maxneigh + hashsize));
  DBuf<double> dscr((size_t)nthr * maxneigh * (ntv + 1));
  const BamgDevParams p{prm.itmax_vol, prm.dist_min, prm.dist_max, prm.mmax, ntv,
                        prm.maxcond,   prm.maxrownrm, prm.tol_vol, prm.eps,
                        maxneigh,      hashsize};
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  const double t1 = now();
  k_bamg_rows<<<blocks, kBamgThreads, 0, st>>>(n, srp.get(), sci.get(), dfc.get(), dtv.get(), p,
                                               iscr.get(), dscr.get(), out_cnt.get(),
                                               out_col.get(), out_val.get(), cm.get(),
                                               status.get());
  CHRONOS_CHECK_LAUNCH();
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  const double t2 = now();
  std::vector<int> cnt(n), col((size_t)n * ntv), st_h(n);
  std::vector<double> val((size_t)n * ntv);
  c_mark.assign(n, 0);
  out_cnt.download(cnt.data(), n, st);
  out_col.download(col.data(), (size_t)n * ntv, st);
  out_val.download(val.data(), (size_t)n * ntv, st);
  cm.download(c_mark.data(), n, st);
  status.download(st_h.data(), n, st);
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  // rows that outgrew their scratch: the host restatement
  std::vector<int> rows;
  for (int i = 0; i < n; ++i)
    if (st_h[i]) rows.push_back(i);
  std::vector<std::vector<int>> rcols(n);
  std::vector<std::vector<double>> rvals(n);
  const double t3 = now();
  if (!rows.empty()) bamg_rows_host(prm, S, fc, TV, ntv, rows, rcols, rvals, c_mark);
  if (host_rows) *host_rows = (int)rows.size();
  if (verbose)
    std::fprintf(stderr, "chronos bamg: %d rows, uploads %.3f s, kernel %.3f s, downloads %.3f s, "
                 "%zu rows on the host %.3f s\n", n, t1 - t0, t2 - t1, t3 - t2, rows.size(),
                 now() - t3);
  HostCSR P;
  P.nrows = n;
  P.ncols = nc;
  P.rp.assign((size_t)n + 1, 0);
  for (int i = 0; i < n; ++i) {
    const int64_t len = fc[i] >= 0 ? 1 : st_h[i] ? (int64_t)rcols[i].size() : cnt[i];
    P.rp[i + 1] = P.rp[i] + len;
  }
  P.ci.resize(P.rp[n]);
  P.v.resize(P.rp[n]);
  for (int i = 0; i < n; ++i) {
    int64_t o = P.rp[i];
    if (fc[i] >= 0) {
      P.ci[o] = fc[i];
      P.v[o] = 1.0;
    } else if (st_h[i]) {
      std::copy(rcols[i].begin(), rcols[i].end(), P.ci.begin() + o);
      std::copy(rvals[i].begin(), rvals[i].end(), P.v.begin() + o);
    } else {
      for (int k = 0; k < cnt[i]; ++k) {
        P.ci[o + k] = col[(size_t)i * ntv + k];
        P.v[o + k] = val[(size_t)i * ntv + k];
      }
    }
  }
  return P;
}

}  // namespace chronos
