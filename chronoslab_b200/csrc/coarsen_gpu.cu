// Strength of connection (DOM or CLA) and the PMIS C/F splitting on the GPU.
//
// The same outputs as soc_matrix and pmis_split on the host
// (host/coarsen.cpp), bit for bit:
//  * cpt_SoC_dom.m:26-47 — s_ij = |a_ij| / sqrt(a_ii a_jj), entry (i, j) of S
//    when a_ij != 0 and s_ij > tau.  A warp per row compacts the strong
//    entries with ballots, so S keeps A's column order within each row;
//    the quotient and square root are IEEE-rounded as on the host.
//  * cpt_SoC_cla.m:109-159 — column statistics of the off-diagonal nonzeros
//    (the most negative value, counting the column's implicit zeros, and the
//    largest magnitude; a zero statistic reads as 1), then s_ij =
//    |a_ij| / max(maxabs_i, maxabs_j) when no off-diagonal entry is
//    negative, else a_ij / max(min_i, min_j); off-diagonal (i, j) is strong
//    when s_ij > tau, and every diagonal entry is in S (S + speye).  The
//    column statistics are exact: atomic max / min on integer keys that order
//    as the doubles do.
//  * mark_isolated_nodes.m — columns of A with a single nonzero are
//    Dirichlet nodes (fine from the start).
//  * cpt_PMIS.m — node weight = strong connections in the node's column of S
//    (diagonal excluded) plus a 53-bit uniform draw of the MT19937 stream
//    (drawn on the host, in node order).  An undecided node turns coarse
//    once no undecided neighbour in S + S' outweighs it, then every node it
//    strongly influences (its column of S) turns fine.  As the host
//    restatement shows, the outcome does not depend on the order of the
//    sweep, so rounds of simultaneous local maxima give it: a round picks
//    every undecided node heavier than all its undecided neighbours, marks
//    them coarse, then marks the nodes they influence fine.  The rounds only
//    read and write node states, so the order inside a round is irrelevant,
//    and neither is the order of the entries within a row of S', which is
//    built with atomics.
// Coarse and fine nodes are then numbered in node order as the reference
// numbers them (coarse k -> k, fine -> -k).
#include <cub/cub.cuh>

#include <algorithm>
#include <string>
#include <vector>

#include "host/host.h"
#include "internal.h"

namespace chronos {

namespace {

constexpr int kCoarsenThreads = 256;

inline int warp_grid(int64_t rows) {
  const int64_t want = (rows + kCoarsenThreads / 32 - 1) / (kCoarsenThreads / 32);
  return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)num_sms() * 32));
}

__global__ void k_row_diag(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                           const double *__restrict__ v, double *__restrict__ d) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    double di = 0.0;
    for (int k = rp[i] + lane; k < rp[i + 1]; k += 32)
      if (ci[k] == i) di = v[k];
    // rows are sorted without duplicates: at most one lane found the diagonal
    for (int o = 16; o > 0; o >>= 1) {
      const double t = __shfl_xor_sync(0xffffffffu, di, o);
      di = (di != 0.0) ? di : t;
    }
    if (lane == 0) d[i] = di;
  }
}

__device__ __forceinline__ bool dom_strong(double a, double di, double dj, double tau) {
  if (a == 0.0) return false;
  const double s = fabs(a) / sqrt(di * dj);
  return s > tau;
}

// Entry (i, j, a) of S, cpt_SoC_dom.m.
struct DomStrength {
  const double *d;
  double tau;
  __device__ bool operator()(int i, int j, double a) const { return dom_strong(a, d[i], d[j], tau); }
};

// Entry (i, j, a) of S + speye, cpt_SoC_cla.m (column statistics finished).
struct ClaStrength {
  const double *maxabs, *minc;
  const int *any_negative;
  double tau;
  __device__ bool operator()(int i, int j, double a) const {
    if (i == j) return true;
    if (a == 0.0) return false;
    const double s = *any_negative ? a / fmax(minc[i], minc[j])
                                   : fabs(a) / fmax(maxabs[i], maxabs[j]);
    return s > tau;
  }
};

// Integer keys that order as the doubles they encode (no NaN): the bits of
// a non-negative double, the complement of a negative one's, top bit set for
// the non-negative half.
__device__ __forceinline__ unsigned long long order_key(double x) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double order_value(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}

// cpt_SoC_cla.m's column statistics over the off-diagonal nonzeros of A:
// kmin[j] = key of min(0, smallest a_ij) (the column's implicit zeros make 0
// a candidate), kmax[j] = bits of the largest |a_ij|; any_negative set when
// some off-diagonal entry is negative.
__global__ void k_cla_colstats(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                               const double *__restrict__ v, unsigned long long *__restrict__ kmin,
                               unsigned long long *__restrict__ kmax, int *__restrict__ any_negative) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw)
    for (int k = rp[i] + lane; k < rp[i + 1]; k += 32) {
      const int j = ci[k];
      const double a = v[k];
      if (j == i || a == 0.0) continue;
      if (a < 0.0) {
        atomicMin(kmin + j, order_key(a));
        atomicExch(any_negative, 1);
      }
      atomicMax(kmax + j, (unsigned long long)__double_as_longlong(fabs(a)));
    }
}

// Statistics to values; a zero one reads as 1 (cpt_SoC_cla.m).
__global__ void k_cla_finish(int n, const unsigned long long *__restrict__ kmin,
                             const unsigned long long *__restrict__ kmax, double *__restrict__ minc,
                             double *__restrict__ maxabs) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const double mn = order_value(kmin[j]);
    const double mx = __longlong_as_double((long long)kmax[j]);
    minc[j] = mn == 0.0 ? 1.0 : mn;
    maxabs[j] = mx == 0.0 ? 1.0 : mx;
  }
}

__global__ void k_fill_u64(int n, unsigned long long *p, unsigned long long val) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) p[j] = val;
}

// Per row: strong entries (S), strong off-diagonal entries (S without its
// diagonal), and the nonzeros of each column of A.
template <typename Strong>
__global__ void k_strength_count(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                 const double *__restrict__ v, Strong strong,
                                 int *__restrict__ cnt_s, int *__restrict__ cnt_o,
                                 int *__restrict__ colcnt) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    int cs = 0, co = 0;
    for (int k = rp[i] + lane; k < rp[i + 1]; k += 32) {
      const int j = ci[k];
      const double a = v[k];
      if (a != 0.0) atomicAdd(colcnt + j, 1);
      if (strong(i, j, a)) {
        ++cs;
        co += (j != i);
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      cs += __shfl_xor_sync(0xffffffffu, cs, o);
      co += __shfl_xor_sync(0xffffffffu, co, o);
    }
    if (lane == 0) {
      cnt_s[i] = cs;
      cnt_o[i] = co;
    }
  }
}

// Ordered compaction of the strong entries of each row into S and of the
// strong off-diagonal ones into So.
template <typename Strong>
__global__ void k_strength_fill(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                const double *__restrict__ v, Strong pred,
                                const int *__restrict__ srp, int *__restrict__ sci,
                                const int *__restrict__ orp, int *__restrict__ oci) {
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    int ps = srp[i], po = orp[i];
    const int e = rp[i + 1];
    for (int k0 = rp[i]; k0 < e; k0 += 32) {
      const int k = k0 + lane;
      bool strong = false;
      int j = 0;
      if (k < e) {
        j = ci[k];
        strong = pred(i, j, v[k]);
      }
      const bool off = strong && j != i;
      const unsigned bs = __ballot_sync(0xffffffffu, strong);
      const unsigned bo = __ballot_sync(0xffffffffu, off);
      if (strong) sci[ps + __popc(bs & below)] = j;
      if (off) oci[po + __popc(bo & below)] = j;
      ps += __popc(bs);
      po += __popc(bo);
    }
  }
}

__global__ void k_col_count(int n, const int *__restrict__ orp, const int *__restrict__ oci,
                            int *__restrict__ tcnt) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw)
    for (int k = orp[i] + lane; k < orp[i + 1]; k += 32) atomicAdd(tcnt + oci[k], 1);
}

// Row j of St lists the rows i with So(i, j) != 0 (in no particular order).
__global__ void k_col_fill(int n, const int *__restrict__ orp, const int *__restrict__ oci,
                           int *__restrict__ cursor, int *__restrict__ tci) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw)
    for (int k = orp[i] + lane; k < orp[i + 1]; k += 32) tci[atomicAdd(cursor + oci[k], 1)] = i;
}

// Initial states: -1 fine (isolated), 0 undecided; weights and free weights.
__global__ void k_pmis_init(int n, const int *__restrict__ colcnt, const int *__restrict__ trp,
                            const double *__restrict__ rnd, int *__restrict__ state,
                            double *__restrict__ w, double *__restrict__ wfree) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const double wj = (double)(trp[j + 1] - trp[j]) + rnd[j];
    const int s = colcnt[j] == 1 ? -1 : 0;
    state[j] = s;
    w[j] = wj;
    wfree[j] = s == -1 ? -1.0 : wj;
  }
}

// A round's picks: undecided nodes that no undecided neighbour (row of So or
// row of St) outweighs.  counts[0] += picks, counts[1] += undecided nodes.
__global__ void k_pmis_pick(int n, const int *__restrict__ orp, const int *__restrict__ oci,
                            const int *__restrict__ trp, const int *__restrict__ tci,
                            const int *__restrict__ state, const double *__restrict__ w,
                            const double *__restrict__ wfree, unsigned char *__restrict__ pick,
                            unsigned *__restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  unsigned npick = 0, nund = 0;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    if (state[i] != 0) continue;                       // warp-uniform
    const double wi = w[i];
    bool heavier = false;
    for (int k = orp[i] + lane; k < orp[i + 1] && !heavier; k += 32) heavier = wfree[oci[k]] > wi;
    for (int k = trp[i] + lane; k < trp[i + 1] && !heavier; k += 32) heavier = wfree[tci[k]] > wi;
    const bool coarse = !__any_sync(0xffffffffu, heavier);
    if (lane == 0) {
      pick[i] = coarse ? 1 : 0;
      npick += coarse;
      ++nund;
    }
  }
  if (lane == 0 && (npick | nund)) {
    atomicAdd(counts, npick);
    atomicAdd(counts + 1, nund);
  }
}

__global__ void k_pmis_coarse(int n, unsigned char *__restrict__ pick, int *__restrict__ state,
                              double *__restrict__ wfree) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (pick[i]) {
      state[i] = 1;
      wfree[i] = -1.0;
    }
}

// The nodes a new coarse node strongly influences turn fine (a coarse one
// included, as in the reference's sweep); the picks are cleared.
__global__ void k_pmis_fine(int n, const int *__restrict__ trp, const int *__restrict__ tci,
                            unsigned char *__restrict__ pick, int *__restrict__ state,
                            double *__restrict__ wfree) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    if (!pick[i]) continue;                            // warp-uniform
    for (int k = trp[i] + lane; k < trp[i + 1]; k += 32) {
      const int j = tci[k];
      state[j] = -1;
      wfree[j] = -1.0;
    }
    __syncwarp();
    if (lane == 0) pick[i] = 0;
  }
}

void exclusive_scan(const int *in, int *out, int n, cudaStream_t st) {
  size_t bytes = 0;
  CHRONOS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, st));
  DBuf<unsigned char> tmp(std::max<size_t>(bytes, 1));
  CHRONOS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), bytes, in, out, n, st));
}

}  // namespace

void coarsen_device(int n, const int *rp, const int *ci, const double *v, const char *soc_type,
                    double tau, MT19937 &rng, HostCSR &S, std::vector<int> &fcnode, int *nc_out,
                    cudaStream_t st) {
  std::string t(soc_type);
  for (auto &c : t) c = (char)toupper(c);
  CHRONOS_REQUIRE(t == "DOM" || t == "CLA", CHRONOS_ENOTSUP,
                  "the GPU coarsening computes DOM or CLA strength (SoC type " + t + ")");
  CHRONOS_REQUIRE(tau >= 0, CHRONOS_ENOTSUP, t + " strength with tau < 0 is outside this path");
  const bool cla = t == "CLA";
  const int g = warp_grid(n);
  const int ge = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, kCoarsenThreads),
                                                             (int64_t)num_sms() * 16));
  DBuf<double> d(n), w(n), wfree(n), rnd(n);
  DBuf<int> cnt_s((size_t)n + 1), cnt_o((size_t)n + 1), colcnt(n), srp((size_t)n + 1),
      orp((size_t)n + 1), state(n);
  colcnt.zero(st);
  k_row_diag<<<g, kCoarsenThreads, 0, st>>>(n, rp, ci, v, d.get());
  CHRONOS_CHECK_LAUNCH();
  DBuf<double> minc, maxabs;
  DBuf<int> anyneg;
  if (cla) {
    // S + speye keeps every diagonal entry: rows must store a nonzero one
    // (an SPD operator always does; the host inserts a missing one)
    std::vector<double> dh(n);
    d.download(dh.data(), n, st);
    CHRONOS_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < n; ++i)
      CHRONOS_REQUIRE(dh[i] != 0.0, CHRONOS_ENOTSUP,
                      "CLA strength on the GPU needs a stored nonzero diagonal in every row");
    DBuf<unsigned long long> kmin(n), kmax(n);
    minc.alloc(n);
    maxabs.alloc(n);
    anyneg.alloc(1);
    anyneg.zero(st);
    kmax.zero(st);                                   // +0.0
    k_fill_u64<<<ge, kCoarsenThreads, 0, st>>>(n, kmin.get(), 0x8000000000000000ull);   // key(+0.0)
    CHRONOS_CHECK_LAUNCH();
    k_cla_colstats<<<g, kCoarsenThreads, 0, st>>>(n, rp, ci, v, kmin.get(), kmax.get(),
                                                  anyneg.get());
    CHRONOS_CHECK_LAUNCH();
    k_cla_finish<<<ge, kCoarsenThreads, 0, st>>>(n, kmin.get(), kmax.get(), minc.get(),
                                                 maxabs.get());
    CHRONOS_CHECK_LAUNCH();
    CHRONOS_CUDA(cudaStreamSynchronize(st));         // kmin, kmax released here
  }
  const DomStrength dom{d.get(), tau};
  const ClaStrength clas{maxabs.get(), minc.get(), anyneg.get(), tau};
  CHRONOS_CUDA(cudaMemsetAsync(cnt_s.get() + n, 0, sizeof(int), st));
  CHRONOS_CUDA(cudaMemsetAsync(cnt_o.get() + n, 0, sizeof(int), st));
  if (cla)
    k_strength_count<<<g, kCoarsenThreads, 0, st>>>(n, rp, ci, v, clas, cnt_s.get(), cnt_o.get(),
                                                    colcnt.get());
  else
    k_strength_count<<<g, kCoarsenThreads, 0, st>>>(n, rp, ci, v, dom, cnt_s.get(), cnt_o.get(),
                                                    colcnt.get());
  CHRONOS_CHECK_LAUNCH();
  exclusive_scan(cnt_s.get(), srp.get(), n + 1, st);
  exclusive_scan(cnt_o.get(), orp.get(), n + 1, st);
  int nnz_s = 0, nnz_o = 0;
  CHRONOS_CUDA(cudaMemcpyAsync(&nnz_s, srp.get() + n, sizeof(int), cudaMemcpyDeviceToHost, st));
  CHRONOS_CUDA(cudaMemcpyAsync(&nnz_o, orp.get() + n, sizeof(int), cudaMemcpyDeviceToHost, st));
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  DBuf<int> sci(std::max(nnz_s, 1)), oci(std::max(nnz_o, 1)), tci(std::max(nnz_o, 1));
  if (cla)
    k_strength_fill<<<g, kCoarsenThreads, 0, st>>>(n, rp, ci, v, clas, srp.get(), sci.get(),
                                                   orp.get(), oci.get());
  else
    k_strength_fill<<<g, kCoarsenThreads, 0, st>>>(n, rp, ci, v, dom, srp.get(), sci.get(),
                                                   orp.get(), oci.get());
  CHRONOS_CHECK_LAUNCH();
  // S' of the off-diagonal part: column counts, row pointers, unordered fill
  DBuf<int> tcnt((size_t)n + 1), trp((size_t)n + 1), cursor(n);
  tcnt.zero(st);
  k_col_count<<<g, kCoarsenThreads, 0, st>>>(n, orp.get(), oci.get(), tcnt.get());
  CHRONOS_CHECK_LAUNCH();
  exclusive_scan(tcnt.get(), trp.get(), n + 1, st);
  CHRONOS_CUDA(cudaMemcpyAsync(cursor.get(), trp.get(), sizeof(int) * n, cudaMemcpyDeviceToDevice,
                               st));
  k_col_fill<<<g, kCoarsenThreads, 0, st>>>(n, orp.get(), oci.get(), cursor.get(), tci.get());
  CHRONOS_CHECK_LAUNCH();
  // weights: column counts plus the stream's next n draws, in node order
  std::vector<double> r(n);
  for (int j = 0; j < n; ++j) r[j] = rng.next_res53();
  rnd.upload(r, st);
  k_pmis_init<<<ge, kCoarsenThreads, 0, st>>>(n, colcnt.get(), trp.get(), rnd.get(), state.get(),
                                              w.get(), wfree.get());
  CHRONOS_CHECK_LAUNCH();
  DBuf<unsigned char> pick(n);
  pick.zero(st);
  DBuf<unsigned> counts(2);
  unsigned ch[2] = {0, 0};
  for (int round = 0;; ++round) {
    CHRONOS_REQUIRE(round <= n, CHRONOS_EINVAL, "PMIS made no progress (equal node weights)");
    counts.zero(st);
    k_pmis_pick<<<g, kCoarsenThreads, 0, st>>>(n, orp.get(), oci.get(), trp.get(), tci.get(),
                                               state.get(), w.get(), wfree.get(), pick.get(),
                                               counts.get());
    CHRONOS_CHECK_LAUNCH();
    CHRONOS_CUDA(cudaMemcpyAsync(ch, counts.get(), sizeof(ch), cudaMemcpyDeviceToHost, st));
    CHRONOS_CUDA(cudaStreamSynchronize(st));
    if (ch[1] == 0) break;                             // no undecided node left
    CHRONOS_REQUIRE(ch[0] > 0, CHRONOS_EINVAL, "PMIS made no progress (equal node weights)");
    k_pmis_coarse<<<ge, kCoarsenThreads, 0, st>>>(n, pick.get(), state.get(), wfree.get());
    CHRONOS_CHECK_LAUNCH();
    k_pmis_fine<<<g, kCoarsenThreads, 0, st>>>(n, trp.get(), tci.get(), pick.get(), state.get(),
                                               wfree.get());
    CHRONOS_CHECK_LAUNCH();
  }
  // numbering and the strength pattern for the host prolongation
  std::vector<int> sh(n), srp_h((size_t)n + 1);
  S.nrows = S.ncols = n;
  S.ci.resize(nnz_s);
  S.v.clear();
  state.download(sh.data(), n, st);
  srp.download(srp_h.data(), (size_t)n + 1, st);
  sci.download(S.ci.data(), nnz_s, st);
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  S.rp.assign(srp_h.begin(), srp_h.end());
  fcnode.resize(n);
  int nc = 0, nf = 0;
  for (int j = 0; j < n; ++j) fcnode[j] = sh[j] > 0 ? ++nc : -(++nf);
  *nc_out = nc;
}

}  // namespace chronos
