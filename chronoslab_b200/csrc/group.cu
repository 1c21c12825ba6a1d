// Grouped solve of a batch of independent SPD problems: every problem keeps
// its own hierarchy (exactly what chronos_amg_setup builds for it), and one
// sequence of launches serves the whole batch.
//
//  * V-cycle: at each level l the operators of the problems that smooth there
//    are stacked block-diagonally (A_l, G_l, G_l' scaled by each problem's
//    omega, P_l, P_l'), so one apply per operator and level covers every
//    problem; the problems whose coarsest level is l get their dense solves
//    in one batched kernel at the bottom of the cycle.  The sweep is level
//    synchronous -- down through every level, the coarsest solves, up again --
//    which keeps each problem's own operations in the order of its single
//    V-cycle (AMG_Vcycle.m:1-54), with the same per-row arithmetic.
//  * PCG_CJ (PCG_CJ.m:34-66) per problem: the vector kernels give every
//    problem its own range of blocks, its own deterministic reductions and
//    scalars; a converged problem is frozen (its x and res stop changing),
//    and the loop -- one conditional CUDA graph -- ends when no problem is
//    active.  The outer product uses the FP64 operator.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <numeric>
#include <vector>

#include "group.h"
#include "spmv.cuh"

namespace chronos {

// ---------------------------------------------------------------------------
// per-problem deterministic reductions
// ---------------------------------------------------------------------------

// Problem of a block: bstart (np+1 entries) is ascending.
__device__ __forceinline__ int block_problem(const int *__restrict__ bstart, int np) {
  int lo = 0, hi = np - 1;
  const int b = blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(bstart + mid) <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// K sums over the blocks of problem p (blocks b0 .. b0+nbp-1): block partials
// in part[blockIdx.x*K + j], the last block of the problem to arrive (ticket
// per problem) adds them in block order and hands the totals to fin(p, t).
template <int K, typename Fin>
__device__ __forceinline__ void group_reduce(double (&v)[K], int p, int b0, int nbp,
                                             double *part, unsigned *tickets, Fin fin) {
  __shared__ double red[K][32];
  __shared__ double tot[K];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const double s = warp_sum(v[j]);
    if (lane == 0) red[j][wid] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < K; ++j) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += red[j][w];
      part[(size_t)blockIdx.x * K + j] = s;
    }
    __threadfence();
    last = atomicAdd(tickets + p, 1u) == (unsigned)(nbp - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double acc[K];
#pragma unroll
  for (int j = 0; j < K; ++j) acc[j] = 0.0;
  for (int b = threadIdx.x; b < nbp; b += blockDim.x)
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] += __ldcg(&part[(size_t)(b0 + b) * K + j]);
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const double s = warp_sum(acc[j]);
    if (lane == 0) red[j][wid] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < K; ++j) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += red[j][w];
      tot[j] = s;
    }
    tickets[p] = 0u;
    fin(p, tot);
  }
}

// Per-problem scalars: sc[p * GS_COUNT + GS_*].
enum GroupScalar {
  GS_BNORM = 0, GS_RR, GS_PTAP, GS_ALPHA, GS_PRES_AXP, GS_RESITER, GS_ITER, GS_ACTIVE,
  GS_BREAKDOWN, GS_COUNT = 10
};
// Global words: g[0] problems active at the start of the current x/res update,
// g[1] ticket of the problems' finalisers, g[2] active after it.
struct GroupCtl {
  double *sc;
  unsigned *g;
  double tol, itmax;
};

#define GROUP_BLOCK_SETUP                                                                    \
  const int p = block_problem(bstart, np);                                                   \
  const int b0 = __ldg(bstart + p), nbp = __ldg(bstart + p + 1) - b0;                        \
  const int r0 = __ldg(rstart + p), r1 = __ldg(rstart + p + 1);                              \
  const int lb = blockIdx.x - b0;

// ||b||^2 and ||res||^2 per problem (initial residual of PCG_CJ.m:18-30).
struct FinNorms {
  double *sc;
  __device__ void operator()(int p, const double *t) const {
    sc[p * GS_COUNT + GS_BNORM] = t[0];
    sc[p * GS_COUNT + GS_RR] = t[1];
  }
};

__global__ void __launch_bounds__(256)
k_group_norms(int np, const int *__restrict__ bstart, const int *__restrict__ rstart,
              const double *__restrict__ b, const double *__restrict__ res, double *part,
              unsigned *tickets, double *sc) {
  pdl_begin();
  GROUP_BLOCK_SETUP
  double v[2] = {0.0, 0.0};
  for (int i = r0 + lb * blockDim.x + threadIdx.x; i < r1; i += nbp * blockDim.x) {
    v[0] += b[i] * b[i];
    v[1] += res[i] * res[i];
  }
  group_reduce<2>(v, p, b0, nbp, part, tickets, FinNorms{sc});
}

__global__ void k_group_init(int np, double *sc, unsigned *g, double tol, double itmax) {
  __shared__ unsigned cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  for (int p = threadIdx.x; p < np; p += blockDim.x) {
    double *s = sc + p * GS_COUNT;
    const double bn = sqrt(s[GS_BNORM]);
    s[GS_BNORM] = bn;
    s[GS_RESITER] = bn > 0.0 ? sqrt(s[GS_RR]) / bn : 0.0;
    s[GS_ITER] = 0.0;
    s[GS_BREAKDOWN] = 0.0;
    const bool act = bn > 0.0 && itmax > 0.0;
    s[GS_ACTIVE] = act ? 1.0 : 0.0;
    if (act) atomicAdd(&cnt, 1u);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    g[0] = cnt;
    g[1] = 0u;
    g[2] = cnt;
  }
}

// pres'axp per problem (beta of PCG_CJ.m:40).
struct FinStore {
  double *sc;
  int which;
  __device__ void operator()(int p, const double *t) const { sc[p * GS_COUNT + which] = t[0]; }
};

__global__ void __launch_bounds__(256)
k_group_dot(int np, const int *__restrict__ bstart, const int *__restrict__ rstart,
            const double *__restrict__ a, const double *__restrict__ c, double *part,
            unsigned *tickets, double *sc) {
  pdl_begin();
  GROUP_BLOCK_SETUP
  if (sc[p * GS_COUNT + GS_ACTIVE] == 0.0) return;
  double v[1] = {0.0};
  for (int i = r0 + lb * blockDim.x + threadIdx.x; i < r1; i += nbp * blockDim.x)
    v[0] += a[i] * c[i];
  group_reduce<1>(v, p, b0, nbp, part, tickets, FinStore{sc, GS_PRES_AXP});
}

// p = pres (first iteration) or pres + beta p, beta = -(pres'axp)/ptap.
__global__ void __launch_bounds__(256)
k_group_p_update(int np, const int *__restrict__ bstart, const int *__restrict__ rstart,
                 const double *__restrict__ pres, double *__restrict__ pv,
                 const double *__restrict__ sc) {
  pdl_begin();
  GROUP_BLOCK_SETUP
  const double *s = sc + p * GS_COUNT;
  if (s[GS_ACTIVE] == 0.0) return;
  const bool first = s[GS_ITER] < 0.5;
  const double beta = first ? 0.0 : -s[GS_PRES_AXP] / s[GS_PTAP];
  for (int i = r0 + lb * blockDim.x + threadIdx.x; i < r1; i += nbp * blockDim.x)
    pv[i] = first ? pres[i] : pres[i] + beta * pv[i];
}

struct FinAlphaGroup {
  double *sc;
  __device__ void operator()(int p, const double *t) const {
    double *s = sc + p * GS_COUNT;
    s[GS_PTAP] = t[0];
    if (!(t[0] > 0.0) || !isfinite(t[1])) {
      s[GS_BREAKDOWN] = 1.0;
      s[GS_ALPHA] = 0.0;
    } else {
      s[GS_ALPHA] = t[1] / t[0];
    }
  }
};

// axp = A p on the problem's rows of the stacked FP64 operator, p'axp, p'res.
template <int L, bool I16>
__global__ void __launch_bounds__(256)
k_group_spmv(int np, const int *__restrict__ bstart, const int *__restrict__ rstart,
             const int *__restrict__ rp, const int *__restrict__ ci,
             const int *__restrict__ cbase, const uint16_t *__restrict__ c16,
             const double *__restrict__ v, const double *__restrict__ pv,
             const double *__restrict__ res, double *__restrict__ axp, double *part,
             unsigned *tickets, double *sc) {
  pdl_begin();
  GROUP_BLOCK_SETUP
  if (sc[p * GS_COUNT + GS_ACTIVE] == 0.0) return;
  constexpr int R = 32 / L;
  const int lane = threadIdx.x & 31, g = lane / L, gl = lane & (L - 1);
  const int warp = lb * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int nwarps = nbp * (blockDim.x >> 5);
  double d[2] = {0.0, 0.0};
  for (int base = r0 + warp * R; base < r1; base += nwarps * R) {   // warp-uniform trip count
    const int row = base + g;
    double a = 0.0;
    if (row < r1) {
      const int s0 = __ldg(rp + row), e = __ldg(rp + row + 1);
      a = csr_row_dot<double, double, double, L, I16>(s0 + gl, e, I16 ? __ldg(cbase + row) : 0,
                                                      ci, c16, v, pv);
    }
    a = group_sum<L>(a);
    if (row < r1 && gl == 0) {
      axp[row] = a;
      const double pi = pv[row];
      d[0] += pi * a;
      d[1] += pi * res[row];
    }
  }
  group_reduce<2>(d, p, b0, nbp, part, tickets, FinAlphaGroup{sc});
}

// x += alpha p; res -= alpha axp; ||res||^2; stop test per problem, and the
// loop condition once every active problem is done.
struct FinResidualGroup {
  GroupCtl c;
  cudaGraphConditionalHandle handle;
  int use_cond;
  __device__ void operator()(int p, const double *t) const {
    double *s = c.sc + p * GS_COUNT;
    // problems active when this update began; only the last of their
    // finalisers changes it, after every one of them has taken a ticket
    const unsigned nact = *(volatile unsigned *)c.g;
    const double resiter = sqrt(t[0]) / s[GS_BNORM];
    const double it = s[GS_ITER] + 1.0;
    s[GS_ITER] = it;
    s[GS_RESITER] = resiter;
    const bool stop = resiter < c.tol || it >= c.itmax || s[GS_BREAKDOWN] != 0.0 ||
                      !isfinite(resiter);
    if (stop) {
      s[GS_ACTIVE] = 0.0;
      atomicSub(c.g + 2, 1u);
    }
    __threadfence();
    if (atomicAdd(c.g + 1, 1u) == nact - 1) {     // the last active problem's finaliser
      __threadfence();
      const unsigned left = atomicAdd(c.g + 2, 0u);
      c.g[0] = left;
      c.g[1] = 0u;
      if (use_cond) cudaGraphSetConditional(handle, left > 0 ? 1u : 0u);
    }
  }
};

__global__ void __launch_bounds__(256)
k_group_xr_update(int np, const int *__restrict__ bstart, const int *__restrict__ rstart,
                  double *__restrict__ x, double *__restrict__ res,
                  const double *__restrict__ pv, const double *__restrict__ axp, double *part,
                  unsigned *tickets, GroupCtl c, cudaGraphConditionalHandle handle,
                  int use_cond) {
  pdl_begin();
  GROUP_BLOCK_SETUP
  const double *s = c.sc + p * GS_COUNT;
  if (s[GS_ACTIVE] == 0.0) return;
  const double alpha = s[GS_ALPHA];
  double v[1] = {0.0};
  for (int i = r0 + lb * blockDim.x + threadIdx.x; i < r1; i += nbp * blockDim.x) {
    x[i] += alpha * pv[i];
    const double ri = res[i] - alpha * axp[i];
    res[i] = ri;
    v[0] += ri * ri;
  }
  group_reduce<1>(v, p, b0, nbp, part, tickets, FinResidualGroup{c, handle, use_cond});
}

// Batched coarsest solves x = W b: a warp per row of every problem whose
// coarsest level this is (rows of all such problems listed back to back).
template <typename T>
__global__ void __launch_bounds__(256)
k_group_dense(int nrows, const int *__restrict__ row_prob, const int *__restrict__ row_local,
              const double *const *__restrict__ W, const int *__restrict__ n,
              const T *const *__restrict__ b, T *const *__restrict__ x) {
  pdl_begin();
  const int lane = threadIdx.x & 31;
  const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (r >= nrows) return;
  const int q = __ldg(row_prob + r), i = __ldg(row_local + r), m = __ldg(n + q);
  const double *w = W[q] + (size_t)i * m;
  const T *bq = b[q];
  double s = 0.0;
  for (int j = lane; j < m; j += 32) s += w[j] * (double)bq[j];
  s = warp_sum(s);
  if (lane == 0) x[q][i] = (T)s;
}

// ---------------------------------------------------------------------------
// host: stacking and the solve
// ---------------------------------------------------------------------------

// One block of a block-diagonal stack: a device matrix, the column offset
// of its block, and a scale applied to its values.
struct StackPart {
  const DMat *m;
  int coff;
  double scale;
};

// The blocks stacked row-wise into one host CSR of ncols columns: sizes
// summed first, every block downloaded straight into its slice, then the
// column shifts, scales and row pointers applied in one parallel pass.
static HostCSR stack_blocks(const std::vector<StackPart> &parts, int ncols, cudaStream_t st) {
  HostCSR S;
  S.ncols = ncols;
  S.nrows = 0;
  std::vector<int64_t> roff(parts.size() + 1, 0), koff(parts.size() + 1, 0);
  for (size_t b = 0; b < parts.size(); ++b) {
    roff[b + 1] = roff[b] + parts[b].m->nrows;
    koff[b + 1] = koff[b] + parts[b].m->nnz;
  }
  S.nrows = (int)roff.back();
  S.rp.assign((size_t)S.nrows + 1, 0);
  S.ci.resize(koff.back());
  S.v.resize(koff.back());
  for (size_t b = 0; b < parts.size(); ++b)
    if (parts[b].m->nnz) {
      parts[b].m->ci.download(S.ci.data() + koff[b], parts[b].m->nnz, st);
      parts[b].m->v64.download(S.v.data() + koff[b], parts[b].m->nnz, st);
    }
  CHRONOS_CUDA(cudaStreamSynchronize(st));
#pragma omp parallel for schedule(dynamic, 1)
  for (int b = 0; b < (int)parts.size(); ++b) {
    const StackPart &q = parts[b];
    for (int64_t k = koff[b]; k < koff[b + 1]; ++k) {
      S.ci[k] += q.coff;
      if (q.scale != 1.0) S.v[k] *= q.scale;
    }
    for (int i = 0; i < q.m->nrows; ++i) S.rp[roff[b] + i + 1] = koff[b] + q.m->rp_h[i + 1];
  }
  return S;
}

bool group_supported(const std::vector<std::unique_ptr<Hier>> &h) {
  if (h.empty()) return false;
  for (const auto &p : h)
    if (p->levels.size() < 2 || p->precision != h[0]->precision) return false;
  return true;
}

template <typename T> static T *gvec(DBuf<float> &f, DBuf<double> &d);
template <> float *gvec<float>(DBuf<float> &f, DBuf<double> &) { return f.get(); }
template <> double *gvec<double>(DBuf<float> &, DBuf<double> &d) { return d.get(); }

GroupSolve::~GroupSolve() {
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  if (st) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
}

std::unique_ptr<GroupSolve> group_build(const std::vector<std::unique_ptr<Hier>> &hs,
                                        const chronos_params &prm) {
  auto G = std::make_unique<GroupSolve>();
  GroupSolve &g = *G;
  CHRONOS_CUDA(cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking));
  cudaStream_t st = g.st;
  g.np = (int)hs.size();
  g.prm = prm;
  g.precision = hs[0]->precision;
  const bool fp32 = g.precision == CHRONOS_FP32;
  const int np = g.np;
  std::vector<int> depth(np);
  for (int p = 0; p < np; ++p) depth[p] = (int)hs[p]->levels.size() - 1;  // coarsest index
  const int lmax = *std::max_element(depth.begin(), depth.end());
  g.lev.resize(lmax + 1);
  // level 0: every problem smooths there (depth >= 1), in problem order
  {
    GroupLevel &L0 = g.lev[0];
    L0.off.assign(np, -1);
    int o = 0;
    for (int p = 0; p < np; ++p) {
      L0.S.push_back(p);
      L0.off[p] = o;
      o += hs[p]->levels[0].n;
    }
    L0.nS = L0.nV = o;
  }
  const bool verbose = std::getenv("CHRONOS_TUNE_VERBOSE") != nullptr;
  for (int l = 0; l < lmax; ++l) {
    const auto tl0 = std::chrono::steady_clock::now();
    GroupLevel &L = g.lev[l], &N = g.lev[l + 1];
    N.off.assign(np, -1);
    int o = 0;
    for (int p : L.S)
      if (depth[p] > l + 1) { N.S.push_back(p); N.off[p] = o; o += hs[p]->levels[l + 1].n; }
    N.nS = o;
    for (int p : L.S)
      if (depth[p] == l + 1) { N.C.push_back(p); N.off[p] = o; o += hs[p]->levels[l + 1].n; }
    N.nV = o;
    std::vector<StackPart> pa, pg, pgt, pp, ppt;
    for (int p : L.S) {
      const Level &lv = hs[p]->levels[l];
      pa.push_back({&lv.A, L.off[p], 1.0});
      pg.push_back({&lv.G, L.off[p], 1.0});
      pgt.push_back({&lv.Gt, L.off[p], lv.omega});
      pp.push_back({&lv.P, N.off[p], 1.0});
    }
    for (const auto *grp : {&N.S, &N.C})
      for (int p : *grp) ppt.push_back({&hs[p]->levels[l].Pt, L.off[p], 1.0});
    upload_csr(stack_blocks(pa, L.nS, st), L.A, fp32, st);
    upload_csr(stack_blocks(pg, L.nS, st), L.G, fp32, st);
    upload_csr(stack_blocks(pgt, L.nS, st), L.Gt, fp32, st);
    upload_csr(stack_blocks(pp, N.nV, st), L.P, fp32, st);
    upload_csr(stack_blocks(ppt, L.nS, st), L.Pt, fp32, st);
    CHRONOS_CUDA(cudaStreamSynchronize(st));
    const auto tl1 = std::chrono::steady_clock::now();
    for (DMat *m : {&L.A, &L.G, &L.Gt, &L.P, &L.Pt}) autotune_lanes(*m, fp32, st, prm.spmv_format);
    CHRONOS_CUDA(cudaStreamSynchronize(st));
    if (verbose)
      std::fprintf(stderr, "chronos group: level %d stacked in %.3f s, tuned in %.3f s\n", l,
                   std::chrono::duration<double>(tl1 - tl0).count(),
                   std::chrono::duration<double>(std::chrono::steady_clock::now() - tl1).count());
  }
  for (auto &L : g.lev) {
    const size_t m = (size_t)std::max(L.nV, 1);
    if (fp32) { L.b32.alloc(m); L.x32.alloc(m); L.r32.alloc(m); L.t32.alloc(m); }
    else { L.b64.alloc(m); L.x64.alloc(m); L.r64.alloc(m); L.t64.alloc(m); }
  }
  // coarsest solves of every level, listed row by row
  {
    std::vector<int> rprob, rloc, nq;
    std::vector<const double *> W;
    std::vector<void *> bq, xq;
    for (int l = 1; l <= lmax; ++l)
      for (int p : g.lev[l].C) {
        const Level &lv = hs[p]->levels[l];
        const int q = (int)W.size();
        W.push_back(lv.W.get());
        nq.push_back(lv.n);
        const size_t off = g.lev[l].off[p];
        if (fp32) {
          bq.push_back(g.lev[l].b32.get() + off);
          xq.push_back(g.lev[l].x32.get() + off);
        } else {
          bq.push_back(g.lev[l].b64.get() + off);
          xq.push_back(g.lev[l].x64.get() + off);
        }
        for (int i = 0; i < lv.n; ++i) { rprob.push_back(q); rloc.push_back(i); }
      }
    g.ncoarse_rows = (int)rprob.size();
    g.c_prob.upload(rprob, st);
    g.c_row.upload(rloc, st);
    g.c_n.upload(nq, st);
    g.c_W.upload(reinterpret_cast<const uintptr_t *>(W.data()), W.size(), st);
    g.c_b.upload(reinterpret_cast<const uintptr_t *>(bq.data()), bq.size(), st);
    g.c_x.upload(reinterpret_cast<const uintptr_t *>(xq.data()), xq.size(), st);
  }
  // finest operators of all problems for the outer product (FP64)
  {
    std::vector<StackPart> pa;
    for (int p = 0; p < np; ++p) pa.push_back({&hs[p]->levels[0].A, g.lev[0].off[p], 1.0});
    upload_csr(stack_blocks(pa, g.lev[0].nV, st), g.A0, false, st);
    autotune_lanes(g.A0, false, st, 1);
  }
  // per-problem rows and blocks of the vector kernels
  g.nrows = g.lev[0].nV;
  std::vector<int> rs(np + 1, 0), bs(np + 1, 0);
  for (int p = 0; p < np; ++p) {
    const int n = hs[p]->levels[0].n;
    rs[p + 1] = rs[p] + n;
    bs[p + 1] = bs[p] + std::max(1, std::min(256, (int)ceil_div(n, 2048)));
  }
  g.nblocks = bs[np];
  g.rstart.upload(rs, st);
  g.bstart.upload(bs, st);
  const size_t n0 = (size_t)g.nrows;
  g.x.alloc(n0); g.res.alloc(n0); g.p.alloc(n0); g.axp.alloc(n0); g.pres.alloc(n0); g.b.alloc(n0);
  g.sc.alloc((size_t)np * GS_COUNT);
  g.part.alloc((size_t)g.nblocks * 2);
  g.tickets.alloc(np);
  g.tickets.zero(st);
  g.ctl.alloc(4);
  g.ctl.zero(st);
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  return G;
}

// The level-synchronous V-cycle: res (FP64) -> pres (FP64) for every problem.
template <typename T>
static void group_vcycle(GroupSolve &g) {
  cudaStream_t st = g.st;
  const int lmax = (int)g.lev.size() - 1;
  const int npre = g.prm.nupre, npost = g.prm.nupost;
  // down
  for (int l = 0; l < lmax; ++l) {
    GroupLevel &L = g.lev[l];
    if (L.nS == 0) continue;
    T *x = gvec<T>(L.x32, L.x64), *r = gvec<T>(L.r32, L.r64), *t = gvec<T>(L.t32, L.t64);
    GroupLevel &N = g.lev[l + 1];
    T *bc = gvec<T>(N.b32, N.b64);
    if (l == 0) {
      const double *b = g.res.get();
      mat_apply<T, double, T, T, MODE_PLAIN, false>(st, L.G, vals<T>(L.G), b, nullptr, t, T(1));
      mat_apply<T, T, T, T, MODE_PLAIN, false>(st, L.Gt, vals<T>(L.Gt), t, nullptr, x, T(1));
      for (int k = 1; k < npre; ++k) {
        mat_apply<T, T, double, T, MODE_RESID, false>(st, L.A, vals<T>(L.A), x, b, r, T(1));
        mat_apply<T, T, T, T, MODE_PLAIN, false>(st, L.G, vals<T>(L.G), r, nullptr, t, T(1));
        mat_apply<T, T, T, T, MODE_AXPY, false>(st, L.Gt, vals<T>(L.Gt), t, x, x, T(1));
      }
      mat_apply<T, T, double, T, MODE_RESID, false>(st, L.A, vals<T>(L.A), x, b, r, T(1));
    } else {
      const T *b = gvec<T>(L.b32, L.b64);
      mat_apply<T, T, T, T, MODE_PLAIN, false>(st, L.G, vals<T>(L.G), b, nullptr, t, T(1));
      mat_apply<T, T, T, T, MODE_PLAIN, false>(st, L.Gt, vals<T>(L.Gt), t, nullptr, x, T(1));
      for (int k = 1; k < npre; ++k) {
        mat_apply<T, T, T, T, MODE_RESID, false>(st, L.A, vals<T>(L.A), x, b, r, T(1));
        mat_apply<T, T, T, T, MODE_PLAIN, false>(st, L.G, vals<T>(L.G), r, nullptr, t, T(1));
        mat_apply<T, T, T, T, MODE_AXPY, false>(st, L.Gt, vals<T>(L.Gt), t, x, x, T(1));
      }
      mat_apply<T, T, T, T, MODE_RESID, false>(st, L.A, vals<T>(L.A), x, b, r, T(1));
    }
    mat_apply<T, T, T, T, MODE_PLAIN, false>(st, L.Pt, vals<T>(L.Pt), r, nullptr, bc, T(1));
  }
  // coarsest solves of every problem
  if (g.ncoarse_rows > 0)
    launch_pdl(k_group_dense<T>, ceil_div((int64_t)g.ncoarse_rows * 32, 256), 256, st,
               g.ncoarse_rows, (const int *)g.c_prob.get(), (const int *)g.c_row.get(),
               reinterpret_cast<const double *const *>(g.c_W.get()), (const int *)g.c_n.get(),
               reinterpret_cast<const T *const *>(g.c_b.get()),
               reinterpret_cast<T *const *>(g.c_x.get()));
  // up
  for (int l = lmax - 1; l >= 0; --l) {
    GroupLevel &L = g.lev[l];
    if (L.nS == 0) continue;
    T *x = gvec<T>(L.x32, L.x64), *r = gvec<T>(L.r32, L.r64), *t = gvec<T>(L.t32, L.t64);
    GroupLevel &N = g.lev[l + 1];
    const T *xc = gvec<T>(N.x32, N.x64);
    mat_apply<T, T, T, T, MODE_AXPY, false>(st, L.P, vals<T>(L.P), xc, x, x, T(1));
    for (int k = 0; k < npost; ++k) {
      const bool lastk = k + 1 == npost;
      if (l == 0) {
        const double *b = g.res.get();
        mat_apply<T, T, double, T, MODE_RESID, false>(st, L.A, vals<T>(L.A), x, b, r, T(1));
        mat_apply<T, T, T, T, MODE_PLAIN, false>(st, L.G, vals<T>(L.G), r, nullptr, t, T(1));
        if (lastk)
          mat_apply<T, T, T, double, MODE_AXPY, false>(st, L.Gt, vals<T>(L.Gt), t, x,
                                                       g.pres.get(), T(1));
        else
          mat_apply<T, T, T, T, MODE_AXPY, false>(st, L.Gt, vals<T>(L.Gt), t, x, x, T(1));
      } else {
        const T *b = gvec<T>(L.b32, L.b64);
        mat_apply<T, T, T, T, MODE_RESID, false>(st, L.A, vals<T>(L.A), x, b, r, T(1));
        mat_apply<T, T, T, T, MODE_PLAIN, false>(st, L.G, vals<T>(L.G), r, nullptr, t, T(1));
        mat_apply<T, T, T, T, MODE_AXPY, false>(st, L.Gt, vals<T>(L.Gt), t, x, x, T(1));
      }
    }
    if (npost == 0 && l == 0)        // pres = x (through the same epilogue)
      mat_apply<T, T, T, double, MODE_AXPY, false>(st, L.Gt, vals<T>(L.Gt), t, x, g.pres.get(),
                                                   T(0));
  }
}

static void group_spmv(GroupSolve &g, const double *pv, const double *res, double *axp) {
  const DMat &A = g.A0;
  const int grid = g.nblocks;
#define CHRONOS_GS_CASE(LL)                                                                   \
  case LL:                                                                                    \
    if (A.idx16)                                                                              \
      launch_pdl(k_group_spmv<LL, true>, grid, 256, g.st, g.np, (const int *)g.bstart.get(),  \
                 (const int *)g.rstart.get(), (const int *)A.rp.get(), (const int *)A.ci.get(),\
                 (const int *)A.cbase.get(), (const uint16_t *)A.c16.get(),                   \
                 (const double *)A.v64.get(), pv, res, axp, g.part.get(), g.tickets.get(),    \
                 g.sc.get());                                                                 \
    else                                                                                      \
      launch_pdl(k_group_spmv<LL, false>, grid, 256, g.st, g.np, (const int *)g.bstart.get(), \
                 (const int *)g.rstart.get(), (const int *)A.rp.get(), (const int *)A.ci.get(),\
                 (const int *)A.cbase.get(), (const uint16_t *)A.c16.get(),                   \
                 (const double *)A.v64.get(), pv, res, axp, g.part.get(), g.tickets.get(),    \
                 g.sc.get());                                                                 \
    break;
  switch (A.lanes) {
    CHRONOS_GS_CASE(1)
    CHRONOS_GS_CASE(2)
    CHRONOS_GS_CASE(4)
    CHRONOS_GS_CASE(8)
    CHRONOS_GS_CASE(16)
    CHRONOS_GS_CASE(32)
    default: throw Error(CHRONOS_EINVAL, "bad lane count");
  }
#undef CHRONOS_GS_CASE
}

static void group_capture_iteration(GroupSolve &g, cudaGraphConditionalHandle handle,
                                    int use_cond, double tol, int itmax) {
  cudaStream_t st = g.st;
  if (g.precision == CHRONOS_FP32) group_vcycle<float>(g);
  else group_vcycle<double>(g);
  const int grid = g.nblocks;
  const int *bs = g.bstart.get(), *rs = g.rstart.get();
  launch_pdl(k_group_dot, grid, 256, st, g.np, bs, rs, (const double *)g.pres.get(),
             (const double *)g.axp.get(), g.part.get(), g.tickets.get(), g.sc.get());
  launch_pdl(k_group_p_update, grid, 256, st, g.np, bs, rs, (const double *)g.pres.get(),
             g.p.get(), (const double *)g.sc.get());
  group_spmv(g, g.p.get(), g.res.get(), g.axp.get());
  GroupCtl c{g.sc.get(), g.ctl.get(), tol, (double)itmax};
  launch_pdl(k_group_xr_update, grid, 256, st, g.np, bs, rs, g.x.get(), g.res.get(),
             (const double *)g.p.get(), (const double *)g.axp.get(), g.part.get(),
             g.tickets.get(), c, handle, use_cond);
}

void group_solve(GroupSolve &g, const std::vector<const double *> &b_h,
                 const std::vector<double *> &x_h, int itmax, double tol, int *iters, int *flags,
                 double *seconds) {
  cudaStream_t st = g.st;
  const int np = g.np;
  const GroupLevel &L0 = g.lev[0];
  for (int p = 0; p < np; ++p) {
    const int n = (p + 1 < np ? L0.off[p + 1] : L0.nV) - L0.off[p];
    CHRONOS_CUDA(cudaMemcpyAsync(g.b.get() + L0.off[p], b_h[p], sizeof(double) * n,
                                 cudaMemcpyHostToDevice, st));
    CHRONOS_CUDA(cudaMemcpyAsync(g.x.get() + L0.off[p], x_h[p], sizeof(double) * n,
                                 cudaMemcpyHostToDevice, st));
  }
  // the loop's scalars (tol, itmax) are baked into the graph: rebuild on change
  if (g.exec && (g.g_tol != tol || g.g_itmax != itmax)) {
    cudaGraphExecDestroy(g.exec);
    cudaGraphDestroy(g.graph);
    g.exec = nullptr;
    g.graph = nullptr;
  }
  cudaEvent_t e0, e1;
  CHRONOS_CUDA(cudaEventCreate(&e0));
  CHRONOS_CUDA(cudaEventCreate(&e1));
  CHRONOS_CUDA(cudaEventRecord(e0, st));
  // res = b - A x0, norms, per-problem initial state (PCG_CJ.m:11-30)
  mat_apply<double, double, double, double, MODE_RESID, false>(st, g.A0, g.A0.v64.get(),
                                                               g.x.get(), g.b.get(), g.res.get(),
                                                               1.0);
  const int grid = g.nblocks;
  launch_pdl(k_group_norms, grid, 256, st, np, (const int *)g.bstart.get(),
             (const int *)g.rstart.get(), (const double *)g.b.get(), (const double *)g.res.get(),
             g.part.get(), g.tickets.get(), g.sc.get());
  k_group_init<<<1, 256, 0, st>>>(np, g.sc.get(), g.ctl.get(), tol, (double)itmax);
  CHRONOS_CHECK_LAUNCH();
  unsigned active = 0;
  CHRONOS_CUDA(cudaMemcpyAsync(&active, g.ctl.get(), sizeof(unsigned), cudaMemcpyDeviceToHost,
                               st));
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  if (active > 0 && !g.prm.use_graph) {
    // one iteration per graph launch from a host loop (profilers cannot see
    // the kernel nodes of a graph holding a conditional node); same kernels
    if (!g.exec) {
      CHRONOS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      try {
        group_capture_iteration(g, 0, 0, tol, itmax);
      } catch (...) {
        cudaGraph_t dummy;
        cudaStreamEndCapture(st, &dummy);
        throw;
      }
      CHRONOS_CUDA(cudaStreamEndCapture(st, &g.graph));
      CHRONOS_CUDA(cudaGraphInstantiate(&g.exec, g.graph, 0));
      g.g_tol = tol;
      g.g_itmax = itmax;
    }
    for (int k = 0; k < itmax && active > 0; ++k) {
      CHRONOS_CUDA(cudaGraphLaunch(g.exec, st));
      CHRONOS_CUDA(cudaMemcpyAsync(&active, g.ctl.get(), sizeof(unsigned),
                                   cudaMemcpyDeviceToHost, st));
      CHRONOS_CUDA(cudaStreamSynchronize(st));
    }
  } else if (active > 0) {
    if (!g.exec) {
      CHRONOS_CUDA(cudaGraphCreate(&g.graph, 0));
      cudaGraphConditionalHandle handle;
      CHRONOS_CUDA(
          cudaGraphConditionalHandleCreate(&handle, g.graph, 1, cudaGraphCondAssignDefault));
      cudaGraphNodeParams np_{};
      np_.type = cudaGraphNodeTypeConditional;
      np_.conditional.handle = handle;
      np_.conditional.type = cudaGraphCondTypeWhile;
      np_.conditional.size = 1;
      cudaGraphNode_t node;
      CHRONOS_CUDA(cudaGraphAddNode(&node, g.graph, nullptr, 0, &np_));
      cudaGraph_t body = np_.conditional.phGraph_out[0];
      CHRONOS_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0,
                                                 cudaStreamCaptureModeThreadLocal));
      try {
        group_capture_iteration(g, handle, 1, tol, itmax);
      } catch (...) {
        cudaGraph_t dummy;
        cudaStreamEndCapture(st, &dummy);
        throw;
      }
      CHRONOS_CUDA(cudaStreamEndCapture(st, &body));
      CHRONOS_CUDA(cudaGraphInstantiate(&g.exec, g.graph, 0));
      g.g_tol = tol;
      g.g_itmax = itmax;
    }
    CHRONOS_CUDA(cudaGraphLaunch(g.exec, st));
  }
  CHRONOS_CUDA(cudaEventRecord(e1, st));
  std::vector<double> sc((size_t)np * GS_COUNT);
  g.sc.download(sc.data(), sc.size(), st);
  for (int p = 0; p < np; ++p) {
    const int n = (p + 1 < np ? L0.off[p + 1] : L0.nV) - L0.off[p];
    CHRONOS_CUDA(cudaMemcpyAsync(x_h[p], g.x.get() + L0.off[p], sizeof(double) * n,
                                 cudaMemcpyDeviceToHost, st));
  }
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  float ms = 0.f;
  CHRONOS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (seconds) *seconds = ms * 1e-3;
  for (int p = 0; p < np; ++p) {
    const double *s = sc.data() + (size_t)p * GS_COUNT;
    if (s[GS_BNORM] == 0.0) {              // PCG_CJ.m:12-16: x = 0, no iterations
      const int n = (p + 1 < np ? L0.off[p + 1] : L0.nV) - L0.off[p];
      std::fill(x_h[p], x_h[p] + n, 0.0);
      iters[p] = 0;
      flags[p] = 0;
      continue;
    }
    iters[p] = (int)(s[GS_ITER] + 0.5);
    const double r = s[GS_RESITER];
    flags[p] = (r > tol || !std::isfinite(r) || s[GS_BREAKDOWN] != 0.0) ? 1 : 0;
  }
}

}  // namespace chronos
