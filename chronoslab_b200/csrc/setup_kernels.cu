// Setup-phase kernels of the solve path (sm_100a):
//  * FSAI numeric phase: one warp per row gathers the local SPD system
//    A[P,P], -A[P,i] of its pattern, factors it in shared memory (FP64
//    Cholesky), solves, and scales the row by 1/sqrt(a_ii - A_iP A_PP^-1 A_Pi)
//    (cpt_afsai_coef.cpp:440-541).  Rows are bucketed by local size so each
//    bucket runs with the shared-memory tile that fits it.
//  * Galerkin product P'*(A*P) (cpt_aspAMG.m:277) as two row-wise sparse
//    products with per-row hash tables: symbolic count, then numeric
//    accumulation in Gustavson order (each output entry summed in the order
//    of the left factor's row, products and sums rounded separately), exact
//    zeros dropped, rows sorted.
//  * Coarsest level: dense FP64 Cholesky, inverse from the factor, dense
//    matvec apply (AMG_Vcycle.m:9-10).
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <numeric>
#include <string>

#include "internal.h"

namespace chronos {

// =============================================================================
// FSAI numeric
// =============================================================================

// Position of column c in the sorted row [k, ke) of aci, or -1.
__device__ __forceinline__ int find_col(const int *aci, int k, int ke, int c) {
  int lo = k, hi = ke - 1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    int v = aci[mid];
    if (v == c) return mid;
    if (v < c) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

// Row i of G by one warp (cpt_afsai_coef.cpp:440-541): gathers A[P,P] and
// -A[P,i] into the warp's shared-memory tile M (MMAX x MMAX, row-major lower,
// then rhs and y), factors and solves, and writes the scaled row.  Sets bit 0
// of *flags for a non-SPD local block or a non-positive Schur complement.
template <int MMAX>
__device__ __forceinline__ void fsai_row(int i, const int *__restrict__ arp,
                                         const int *__restrict__ aci, const double *__restrict__ av,
                                         const int *__restrict__ grp, const int *__restrict__ gci,
                                         double *__restrict__ gval, int *flags, double *M,
                                         int lane) {
  double *rhs = M + MMAX * MMAX;                // -A[i,P] (kept for the Schur term)
  double *y = rhs + MMAX;                       // solution
  const int gs = grp[i], ge = grp[i + 1];
  const int m = ge - gs - 1;                    // strictly-lower entries
  const int *P = gci + gs;
  const int ai = arp[i], aie = arp[i + 1];
  // Gather: column c (owned by lane c mod 32) from row P[c], entries P[j], j >= c.
  for (int c = lane; c < m; c += 32) {
    const int r = P[c];
    int k = arp[r];
    const int ke = arp[r + 1];
    // first entry with column >= r (binary search)
    int lo = k, hi = ke;
    while (lo < hi) { int mid = (lo + hi) >> 1; if (aci[mid] < r) lo = mid + 1; else hi = mid; }
    k = lo;
    for (int j = c; j < m; ++j) {
      const int pj = P[j];
      while (k < ke && aci[k] < pj) ++k;
      M[j * MMAX + c] = (k < ke && aci[k] == pj) ? av[k] : 0.0;
    }
    const int pos = find_col(aci, ai, aie, r);
    rhs[c] = pos >= 0 ? -av[pos] : 0.0;
  }
  double aii = 0.0;
  bool have_diag = false;
  {
    const int pos = find_col(aci, ai, aie, i);
    if (pos >= 0) { aii = av[pos]; have_diag = true; }
  }
  __syncwarp();
  bool spd = true;
  // Right-looking Cholesky; lane j owns rows j, j+32.
  for (int k = 0; k < m; ++k) {
    double d = M[k * MMAX + k];
    if (!(d > 0.0)) { spd = false; break; }     // warp-uniform (all lanes read the same d)
    d = sqrt(d);
    __syncwarp();
    for (int j = k + 1 + lane; j < m; j += 32) M[j * MMAX + k] /= d;
    if (lane == 0) M[k * MMAX + k] = d;
    __syncwarp();
    for (int j = k + 1 + lane; j < m; j += 32) {
      const double ljk = M[j * MMAX + k];
      for (int l = k + 1; l <= j; ++l) M[j * MMAX + l] -= ljk * M[l * MMAX + k];
    }
    __syncwarp();
  }
  double scal = 0.0;
  if (spd) {
    for (int j = lane; j < m; j += 32) y[j] = rhs[j];
    __syncwarp();
    for (int k = 0; k < m; ++k) {               // L z = rhs
      const double zk = y[k] / M[k * MMAX + k];
      __syncwarp();
      if (lane == 0) y[k] = zk;
      for (int j = k + 1 + lane; j < m; j += 32) y[j] -= M[j * MMAX + k] * zk;
      __syncwarp();
    }
    for (int k = m - 1; k >= 0; --k) {          // L^T y = z
      const double yk = y[k] / M[k * MMAX + k];
      __syncwarp();
      if (lane == 0) y[k] = yk;
      for (int j = lane; j < k; j += 32) y[j] -= M[k * MMAX + j] * yk;
      __syncwarp();
    }
    double part = 0.0;
    for (int j = lane; j < m; j += 32) part += rhs[j] * y[j];
    part = warp_sum(part);
    scal = aii - part;
  }
  bool ok = spd && have_diag && scal > 0.0;
  if (!ok) {
    if (lane == 0) atomicOr(flags, 1);
    scal = 1.0;
    if (!spd)                                    // keep a defined row: diagonal scaling only
      for (int j = lane; j < m; j += 32) y[j] = 0.0;
    __syncwarp();
  }
  const double s = 1.0 / sqrt(scal);
  for (int j = lane; j < m; j += 32) gval[gs + j] = s * y[j];
  if (lane == 0) gval[gs + m] = s;
}

template <int MMAX>
__global__ void k_fsai_numeric(int nb, const int *__restrict__ rows, const int *__restrict__ arp,
                               const int *__restrict__ aci, const double *__restrict__ av,
                               const int *__restrict__ grp, const int *__restrict__ gci,
                               double *__restrict__ gval, int *flags) {
  extern __shared__ double smem[];
  constexpr int STRIDE = MMAX * MMAX + 3 * MMAX;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int wglob = blockIdx.x * (blockDim.x >> 5) + wib;
  if (wglob >= nb) return;                      // warp-uniform exit
  fsai_row<MMAX>(rows[wglob], arp, aci, av, grp, gci, gval, flags, smem + (size_t)wib * STRIDE,
                 lane);
}

// One problem of a batched FSAI numeric launch (device pointers).
struct FsaiProblemDev {
  const int *arp, *aci;
  const double *av;
  const int *grp, *gci;
  double *gval;
};

// The rows of many problems in one launch: item k = (problem, row); flags
// per problem.
template <int MMAX>
__global__ void k_fsai_numeric_batched(int nb, const int2 *__restrict__ items,
                                       const FsaiProblemDev *__restrict__ tab, int *flags) {
  extern __shared__ double smem[];
  constexpr int STRIDE = MMAX * MMAX + 3 * MMAX;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int wglob = blockIdx.x * (blockDim.x >> 5) + wib;
  if (wglob >= nb) return;                      // warp-uniform exit
  const int2 it = items[wglob];
  const FsaiProblemDev pr = tab[it.x];
  fsai_row<MMAX>(it.y, pr.arp, pr.aci, pr.av, pr.grp, pr.gci, pr.gval, flags + it.x,
                 smem + (size_t)wib * STRIDE, lane);
}

int fsai_numeric_device(int n, const int *arp, const int *aci, const double *av, const int *grp,
                        const int *gci, double *gval, const std::vector<int> &rowlen_h,
                        cudaStream_t st) {
  // Bucket rows by local system size m = rowlen - 1.
  std::vector<int> b16, b32, b64;
  for (int i = 0; i < n; ++i) {
    const int m = rowlen_h[i] - 1;
    if (m <= 16) b16.push_back(i);
    else if (m <= 32) b32.push_back(i);
    else if (m <= 64) b64.push_back(i);
    else throw Error(CHRONOS_ENOTSUP, "FSAI local system larger than 64 (nstep*step_size)");
  }
  DBuf<int> flags(1);
  flags.zero(st);
  DBuf<int> d16, d32, d64;
  auto run = [&](auto kern, const std::vector<int> &rows, DBuf<int> &drows, int mmax, int warps) {
    if (rows.empty()) return;
    drows.upload(rows, st);
    const size_t sm = (size_t)warps * (mmax * mmax + 3 * mmax) * sizeof(double);
    CHRONOS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    const unsigned blocks = ceil_div((int64_t)rows.size(), warps);
    kern<<<blocks, warps * 32, sm, st>>>((int)rows.size(), drows.get(), arp, aci, av, grp, gci,
                                         gval, flags.get());
    CHRONOS_CHECK_LAUNCH();
  };
  run(k_fsai_numeric<16>, b16, d16, 16, 8);
  run(k_fsai_numeric<32>, b32, d32, 32, 4);
  run(k_fsai_numeric<64>, b64, d64, 64, 2);
  int fl = 0;
  CHRONOS_CUDA(cudaMemcpyAsync(&fl, flags.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  return fl;
}

// -----------------------------------------------------------------------------
// FSAI numeric phase of many problems at once (a batch's level): every row of
// every problem goes to the smallest shared-memory tile (MMAX) that holds its
// local system, and each tile size is one launch over all problems' rows.
// Which tile sizes exist -- the bucket edges -- is chosen per batch shape by
// timing the candidate sets below on the batch's own rows (CUDA events); a
// row's arithmetic does not depend on its tile, so every set gives the same
// values bit for bit and the timed runs may overwrite one another.
// -----------------------------------------------------------------------------

namespace {

const std::vector<std::vector<int>> &fsai_bucket_sets() {
  static const std::vector<std::vector<int>> sets = {
      {16, 32, 64}, {8, 16, 32, 64}, {16, 24, 32, 48, 64}, {8, 16, 24, 32, 48, 64}};
  return sets;
}

// warps per block of a tile size (shared memory: warps * (MMAX^2 + 3 MMAX) doubles)
int fsai_tile_warps(int mmax) { return mmax <= 24 ? 8 : mmax <= 32 ? 4 : 2; }

template <int MMAX>
void launch_fsai_batched(int cnt, const int2 *items, const FsaiProblemDev *tab, int *flags,
                         cudaStream_t st) {
  if (cnt == 0) return;
  const int warps = fsai_tile_warps(MMAX);
  const size_t sm = (size_t)warps * (MMAX * MMAX + 3 * MMAX) * sizeof(double);
  CHRONOS_CUDA(cudaFuncSetAttribute(k_fsai_numeric_batched<MMAX>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  k_fsai_numeric_batched<MMAX><<<ceil_div(cnt, warps), warps * 32, sm, st>>>(cnt, items, tab,
                                                                            flags);
  CHRONOS_CHECK_LAUNCH();
}

void launch_fsai_tile(int mmax, int cnt, const int2 *items, const FsaiProblemDev *tab, int *flags,
                      cudaStream_t st) {
  switch (mmax) {
    case 8: launch_fsai_batched<8>(cnt, items, tab, flags, st); break;
    case 16: launch_fsai_batched<16>(cnt, items, tab, flags, st); break;
    case 24: launch_fsai_batched<24>(cnt, items, tab, flags, st); break;
    case 32: launch_fsai_batched<32>(cnt, items, tab, flags, st); break;
    case 48: launch_fsai_batched<48>(cnt, items, tab, flags, st); break;
    case 64: launch_fsai_batched<64>(cnt, items, tab, flags, st); break;
    default: throw Error(CHRONOS_EINVAL, "no FSAI tile of this size");
  }
}

std::mutex g_fsai_tune_mu;
std::map<std::string, int> g_fsai_tune;       // batch shape -> index of the chosen set

}  // namespace

int fsai_bucket_set_count() { return (int)fsai_bucket_sets().size(); }

std::vector<int> fsai_numeric_batched(const std::vector<FsaiJob> &jobs, cudaStream_t st,
                                      int *chosen_set, int force_set) {
  CHRONOS_REQUIRE(force_set < (int)fsai_bucket_sets().size(), CHRONOS_EINVAL,
                  "no such FSAI tile set");
  const int nj = (int)jobs.size();
  std::vector<int> out(nj, 0);
  if (nj == 0) return out;
  // local sizes: histogram (the batch's shape) and the largest
  std::vector<int64_t> hist(65, 0);
  for (const auto &j : jobs)
    for (int i = 0; i < j.n; ++i) {
      const int m = (*j.rowlen)[i] - 1;
      CHRONOS_REQUIRE(m >= 0 && m <= 64, m > 64 ? CHRONOS_ENOTSUP : CHRONOS_EINVAL,
                      "FSAI local system larger than 64 (nstep*step_size) or an empty row");
      hist[m]++;
    }
  std::vector<FsaiProblemDev> tab_h(nj);
  for (int p = 0; p < nj; ++p)
    tab_h[p] = {jobs[p].arp, jobs[p].aci, jobs[p].av, jobs[p].grp, jobs[p].gci, jobs[p].gval};
  DBuf<FsaiProblemDev> tab;
  tab.upload(tab_h, st);
  DBuf<int> flags(nj);
  // items of one bucket set, bucket by bucket: (problem, row)
  const auto &sets = fsai_bucket_sets();
  auto build_items = [&](const std::vector<int> &set, std::vector<int2> &items,
                         std::vector<int> &start) {
    const int nb = (int)set.size();
    std::vector<int> bucket_of(65);
    for (int m = 0; m <= 64; ++m) {
      int b = 0;
      while (set[b] < m) ++b;
      bucket_of[m] = b;
    }
    start.assign(nb + 1, 0);
    for (int m = 0; m <= 64; ++m) start[bucket_of[m] + 1] += (int)hist[m];
    for (int b = 0; b < nb; ++b) start[b + 1] += start[b];
    items.resize(start[nb]);
    std::vector<int> cur(start.begin(), start.end() - 1);
    for (int p = 0; p < nj; ++p)
      for (int i = 0; i < jobs[p].n; ++i) items[cur[bucket_of[(*jobs[p].rowlen)[i] - 1]]++] = {p, i};
  };
  auto run = [&](const std::vector<int> &set, const DBuf<int2> &items, const std::vector<int> &start) {
    flags.zero(st);
    for (size_t b = 0; b < set.size(); ++b)
      launch_fsai_tile(set[b], start[b + 1] - start[b], items.get() + start[b], tab.get(),
                       flags.get(), st);
  };
  std::string key;
  for (int m = 0; m <= 64; ++m)
    if (hist[m]) key += std::to_string(m) + ":" + std::to_string(hist[m]) + ",";
  int choice = force_set >= 0 ? force_set : -1;
  if (choice < 0) {
    std::lock_guard<std::mutex> lk(g_fsai_tune_mu);
    auto it = g_fsai_tune.find(key);
    if (it != g_fsai_tune.end()) choice = it->second;
  }
  const int64_t rows = std::accumulate(hist.begin(), hist.end(), (int64_t)0);
  if (choice < 0 && rows < 20000) choice = 0;            // small batch: launch-bound either way
  std::vector<int2> items_h;
  std::vector<int> start;
  DBuf<int2> items;
  if (choice < 0) {
    const bool verbose = std::getenv("CHRONOS_TUNE_VERBOSE") != nullptr;
    cudaEvent_t e0, e1;
    CHRONOS_CUDA(cudaEventCreate(&e0));
    CHRONOS_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    for (int s = 0; s < (int)sets.size(); ++s) {
      build_items(sets[s], items_h, start);
      items.upload(items_h, st);
      run(sets[s], items, start);                         // warm-up (the attributes, caches)
      CHRONOS_CUDA(cudaEventRecord(e0, st));
      run(sets[s], items, start);
      CHRONOS_CUDA(cudaEventRecord(e1, st));
      CHRONOS_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      CHRONOS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (verbose) {
        std::string edges;
        for (int m : sets[s]) edges += std::to_string(m) + " ";
        std::fprintf(stderr, "chronos tune: fsai batch %lld rows, tiles %s %.4f ms\n",
                     (long long)rows, edges.c_str(), ms);
      }
      if (ms < best) { best = ms; choice = s; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::lock_guard<std::mutex> lk(g_fsai_tune_mu);
    g_fsai_tune[key] = choice;
  }
  build_items(sets[choice], items_h, start);
  items.upload(items_h, st);
  run(sets[choice], items, start);
  flags.download(out.data(), nj, st);
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  if (chosen_set) *chosen_set = choice;
  return out;
}

// =============================================================================
// Sparse product C = X * Y with per-row hash tables in global memory
// =============================================================================

__global__ void k_spgemm_products(int m, const int *xrp, const int *xci, const int *yrp,
                                  int64_t *prod) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  int64_t s = 0;
  for (int k = xrp[i]; k < xrp[i + 1]; ++k) {
    const int j = xci[k];
    s += yrp[j + 1] - yrp[j];
  }
  prod[i] = s;
}

__device__ __forceinline__ unsigned hash_slot(int key, unsigned mask) {
  return ((unsigned)key * 2654435761u) & mask;
}

// Inserts key into the open-addressing table (keys initialised to -1);
// returns the slot and whether this call created it.
__device__ __forceinline__ unsigned hash_insert(int *keys, unsigned mask, int key, bool *fresh) {
  unsigned s = hash_slot(key, mask);
  while (true) {
    int cur = keys[s];
    if (cur == key) { *fresh = false; return s; }
    if (cur == -1) {
      int prev = atomicCAS(keys + s, -1, key);
      if (prev == -1) { *fresh = true; return s; }
      if (prev == key) { *fresh = false; return s; }
    }
    s = (s + 1) & mask;
  }
}

// Symbolic: unique columns per row (warp per row, rows [r0, r1)).
__global__ void k_spgemm_symbolic(int r0, int r1, const int *rows, const int *xrp, const int *xci,
                                  const int *yrp, const int *yci, const int64_t *toff,
                                  const unsigned *tcap, int *keys, int *cnt) {
  const int lane = threadIdx.x & 31;
  const int t = r0 + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (t >= r1) return;
  const int i = rows[t];
  int *tk = keys + toff[t - r0];
  const unsigned cap = tcap[t - r0], mask = cap - 1;
  for (unsigned s = lane; s < cap; s += 32) tk[s] = -1;
  __syncwarp();
  int mine = 0;
  for (int k = xrp[i]; k < xrp[i + 1]; ++k) {
    const int j = xci[k];
    for (int kk = yrp[j] + lane; kk < yrp[j + 1]; kk += 32) {
      bool fresh;
      hash_insert(tk, mask, yci[kk], &fresh);
      mine += fresh;
    }
  }
  mine = warp_sum(mine);
  if (lane == 0) cnt[i] = mine;
}

// Numeric: accumulate in the order of row i of X (products rounded, then
// added), emit the nonzero entries unsorted into [crp_sym[i], ...); cnt_out[i]
// = number emitted.
__global__ void k_spgemm_numeric(int r0, int r1, const int *rows, const int *xrp, const int *xci,
                                 const double *xv, const int *yrp, const int *yci,
                                 const double *yv, const int64_t *toff, const unsigned *tcap,
                                 int *keys, double *vals, const int64_t *crp_sym, int *cci,
                                 double *cv, int *cnt_out) {
  const int lane = threadIdx.x & 31;
  const int t = r0 + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (t >= r1) return;
  const int i = rows[t];
  int *tk = keys + toff[t - r0];
  double *tv = vals + toff[t - r0];
  const unsigned cap = tcap[t - r0], mask = cap - 1;
  for (unsigned s = lane; s < cap; s += 32) { tk[s] = -1; tv[s] = 0.0; }
  __syncwarp();
  for (int k = xrp[i]; k < xrp[i + 1]; ++k) {
    const int j = xci[k];
    const double a = xv[k];
    for (int kk = yrp[j] + lane; kk < yrp[j + 1]; kk += 32) {
      bool fresh;
      const unsigned s = hash_insert(tk, mask, yci[kk], &fresh);
      tv[s] = __dadd_rn(tv[s], __dmul_rn(a, yv[kk]));
    }
    __syncwarp();
  }
  __syncwarp();
  int64_t base = crp_sym[i];
  int emitted = 0;
  for (unsigned s0 = 0; s0 < cap; s0 += 32) {
    const unsigned s = s0 + lane;
    bool keep = false;
    int key = -1;
    double val = 0.0;
    if (s < cap) {
      key = tk[s];
      val = tv[s];
      keep = key != -1 && val != 0.0;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    if (keep) {
      const int off = __popc(bal & ((1u << lane) - 1u));
      cci[base + emitted + off] = key;
      cv[base + emitted + off] = val;
    }
    emitted += __popc(bal);
  }
  if (lane == 0) cnt_out[i] = emitted;
}

// Shared-memory variants for rows whose distinct columns fit a warp's table
// of kSpgemmSmSlots: the same insertion order and sums as the global-table
// kernels (each output column gets its products in X's row order), so the
// results are bit-identical; only the table's place and size differ.
constexpr int kSpgemmSmSlots = 4096;
constexpr int kSpgemmSmWarps = 4;

__device__ __forceinline__ unsigned spgemm_cap(int64_t prod, int ncols) {
  const uint64_t want = (uint64_t)2 * (uint64_t)prod + 1, colcap = (uint64_t)2 * (uint64_t)max(ncols, 1);
  uint64_t p = 32, v = want < colcap ? want : colcap;
  while (p < v) p <<= 1;
  return (unsigned)p;
}

// Symbolic in shared memory: cnt[i] = distinct columns of row i, or -1 when
// they outgrow half the warp's table (the row then goes to the global table).
__global__ void __launch_bounds__(32 * kSpgemmSmWarps)
k_spgemm_symbolic_sm(int m, int ncols, const int *__restrict__ xrp, const int *__restrict__ xci,
                     const int *__restrict__ yrp, const int *__restrict__ yci,
                     const int64_t *__restrict__ prod, int *__restrict__ cnt) {
  extern __shared__ int spg_keys[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  int *tk = spg_keys + wib * kSpgemmSmSlots;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = gw; i < m; i += nw) {
    const unsigned cap = spgemm_cap(prod[i], ncols);
    const unsigned tsz = cap < (unsigned)kSpgemmSmSlots ? cap : (unsigned)kSpgemmSmSlots;
    const unsigned mask = tsz - 1;
    for (unsigned s = lane; s < tsz; s += 32) tk[s] = -1;
    __syncwarp();
    int count = 0;
    bool over = false;
    for (int k = xrp[i]; k < xrp[i + 1] && !over; ++k) {
      const int j = xci[k];
      for (int kk0 = yrp[j]; kk0 < yrp[j + 1]; kk0 += 32) {
        const int kk = kk0 + lane;
        int fresh_n = 0;
        if (kk < yrp[j + 1]) {
          bool fresh;
          hash_insert(tk, mask, yci[kk], &fresh);
          fresh_n = fresh;
        }
        count += warp_sum(fresh_n);
        if (2 * count > (int)tsz) {                    // the same for every lane
          over = true;
          break;
        }
      }
    }
    if (lane == 0) cnt[i] = over ? -1 : count;
    __syncwarp();
  }
}

// Numeric in shared memory for the rows with 0 <= cnt[i] <= kSpgemmSmSlots/2
// (others skipped): emits row i's nonzero entries unsorted at crp_sym[i].
__global__ void __launch_bounds__(32 * kSpgemmSmWarps)
k_spgemm_numeric_sm(int m, const int *__restrict__ xrp, const int *__restrict__ xci,
                    const double *__restrict__ xv, const int *__restrict__ yrp,
                    const int *__restrict__ yci, const double *__restrict__ yv,
                    const int *__restrict__ cnt, const int64_t *__restrict__ crp_sym,
                    int *__restrict__ cci, double *__restrict__ cv, int *__restrict__ cnt_out) {
  extern __shared__ double spg_vals[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double *tv = spg_vals + (size_t)wib * kSpgemmSmSlots;
  int *tk = reinterpret_cast<int *>(spg_vals + (size_t)kSpgemmSmWarps * kSpgemmSmSlots) +
            wib * kSpgemmSmSlots;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = gw; i < m; i += nw) {
    const int c = cnt[i];
    if (c < 0 || 2 * c > kSpgemmSmSlots) continue;
    unsigned tsz = 32;
    while (tsz < (unsigned)(2 * c + 1)) tsz <<= 1;
    const unsigned mask = tsz - 1;
    for (unsigned s = lane; s < tsz; s += 32) { tk[s] = -1; tv[s] = 0.0; }
    __syncwarp();
    for (int k = xrp[i]; k < xrp[i + 1]; ++k) {
      const int j = xci[k];
      const double a = xv[k];
      for (int kk = yrp[j] + lane; kk < yrp[j + 1]; kk += 32) {
        bool fresh;
        const unsigned s = hash_insert(tk, mask, yci[kk], &fresh);
        tv[s] = __dadd_rn(tv[s], __dmul_rn(a, yv[kk]));
      }
      __syncwarp();
    }
    const int64_t base = crp_sym[i];
    int emitted = 0;
    for (unsigned s0 = 0; s0 < tsz; s0 += 32) {
      const unsigned s = s0 + lane;
      bool keep = false;
      int key = -1;
      double val = 0.0;
      if (s < tsz) {
        key = tk[s];
        val = tv[s];
        keep = key != -1 && val != 0.0;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        const int off = __popc(bal & ((1u << lane) - 1u));
        cci[base + emitted + off] = key;
        cv[base + emitted + off] = val;
      }
      emitted += __popc(bal);
    }
    if (lane == 0) cnt_out[i] = emitted;
    __syncwarp();
  }
}

__global__ void k_compact_rows(int m, const int64_t *src_rp, const int *cnt, const int *crp,
                               const int *sci, const double *sv, int *dci, double *dv) {
  const int i = blockIdx.x;
  if (i >= m) return;
  const int64_t s = src_rp[i];
  const int d = crp[i], c = cnt[i];
  for (int k = threadIdx.x; k < c; k += blockDim.x) {
    dci[d + k] = sci[s + k];
    dv[d + k] = sv[s + k];
  }
}

static unsigned next_pow2(uint64_t v) {
  uint64_t p = 32;
  while (p < v) p <<= 1;
  return (unsigned)p;
}

void spgemm_device(int m, int ncols, const int *xrp, const int *xci, const double *xv,
                   const int *yrp, const int *yci, const double *yv, DBuf<int> &crp,
                   DBuf<int> &cci, DBuf<double> &cv, int64_t *nnz_c, cudaStream_t st) {
  crp.alloc((size_t)m + 1);
  if (m == 0) {
    crp.zero(st);
    *nnz_c = 0;
    return;
  }
  DBuf<int64_t> dprod(m);
  k_spgemm_products<<<ceil_div(m, 256), 256, 0, st>>>(m, xrp, xci, yrp, dprod.get());
  CHRONOS_CHECK_LAUNCH();
  // symbolic: in each warp's shared table first; rows whose distinct columns
  // outgrow it (cnt = -1) again in global tables sized from their products
  const size_t sym_smem = (size_t)kSpgemmSmWarps * kSpgemmSmSlots * sizeof(int);
  const size_t num_smem = (size_t)kSpgemmSmWarps * kSpgemmSmSlots * (sizeof(int) + sizeof(double));
  static const bool attrs = [&] {
    CHRONOS_CUDA(cudaFuncSetAttribute(k_spgemm_symbolic_sm,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sym_smem));
    CHRONOS_CUDA(cudaFuncSetAttribute(k_spgemm_numeric_sm,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)num_smem));
    return true;
  }();
  (void)attrs;
  const int sm_grid = (int)std::max<int64_t>(
      1, std::min<int64_t>(ceil_div(m, kSpgemmSmWarps), (int64_t)num_sms() * 8));
  DBuf<int> cnt(m);
  k_spgemm_symbolic_sm<<<sm_grid, 32 * kSpgemmSmWarps, sym_smem, st>>>(m, ncols, xrp, xci, yrp,
                                                                       yci, dprod.get(), cnt.get());
  CHRONOS_CHECK_LAUNCH();
  std::vector<int> cnt_h = cnt.to_host(st);
  std::vector<int> big;                                // rows for the global tables
  for (int i = 0; i < m; ++i)
    if (cnt_h[i] < 0) big.push_back(i);
  const int nbig = (int)big.size();
  DBuf<int> dbig;
  std::vector<int> bounds{0};
  DBuf<int> keys;
  DBuf<double> vals;
  DBuf<int64_t> toff;
  DBuf<unsigned> tcap;
  if (nbig > 0) {
    std::vector<int64_t> prod(m);
    dprod.download(prod.data(), m, st);
    CHRONOS_CUDA(cudaStreamSynchronize(st));
    std::vector<unsigned> cap(nbig);
    const uint64_t colcap = (uint64_t)2 * (uint64_t)std::max(ncols, 1);
    for (int t = 0; t < nbig; ++t)
      cap[t] = next_pow2(std::min<uint64_t>(2 * (uint64_t)prod[big[t]] + 1, colcap));
    // chunks of rows whose tables fit the slot budget
    const uint64_t budget = (uint64_t)1 << 24;     // 16M slots (192 MB with values)
    uint64_t acc = 0;
    for (int t = 0; t < nbig; ++t) {
      if (acc + cap[t] > budget && t > bounds.back()) { bounds.push_back(t); acc = 0; }
      acc += cap[t];
    }
    bounds.push_back(nbig);
    uint64_t maxchunk = 0;
    std::vector<int64_t> toff_h(nbig);
    for (size_t c = 0; c + 1 < bounds.size(); ++c) {
      int64_t a = 0;
      for (int t = bounds[c]; t < bounds[c + 1]; ++t) { toff_h[t] = a; a += cap[t]; }
      maxchunk = std::max<uint64_t>(maxchunk, (uint64_t)a);
    }
    keys.alloc(maxchunk);
    vals.alloc(maxchunk);
    toff.upload(toff_h, st);
    tcap.upload(cap.data(), nbig, st);
    dbig.upload(big, st);
    for (size_t c = 0; c + 1 < bounds.size(); ++c) {
      const int t0 = bounds[c], t1 = bounds[c + 1];
      k_spgemm_symbolic<<<ceil_div((int64_t)(t1 - t0) * 32, 256), 256, 0, st>>>(
          t0, t1, dbig.get(), xrp, xci, yrp, yci, toff.get() + t0, tcap.get() + t0, keys.get(),
          cnt.get());
      CHRONOS_CHECK_LAUNCH();
    }
    cnt_h = cnt.to_host(st);
  }
  std::vector<int64_t> rps(m + 1, 0);
  for (int i = 0; i < m; ++i) rps[i + 1] = rps[i] + cnt_h[i];
  DBuf<int64_t> drps(m + 1);
  drps.upload(rps, st);
  DBuf<int> sci(std::max<int64_t>(rps[m], 1));
  DBuf<double> sv(std::max<int64_t>(rps[m], 1));
  DBuf<int> cnt2(m);
  k_spgemm_numeric_sm<<<sm_grid, 32 * kSpgemmSmWarps, num_smem, st>>>(
      m, xrp, xci, xv, yrp, yci, yv, cnt.get(), drps.get(), sci.get(), sv.get(), cnt2.get());
  CHRONOS_CHECK_LAUNCH();
  for (size_t c = 0; c + 1 < bounds.size() && nbig > 0; ++c) {
    const int t0 = bounds[c], t1 = bounds[c + 1];
    k_spgemm_numeric<<<ceil_div((int64_t)(t1 - t0) * 32, 256), 256, 0, st>>>(
        t0, t1, dbig.get(), xrp, xci, xv, yrp, yci, yv, toff.get() + t0, tcap.get() + t0,
        keys.get(), vals.get(), drps.get(), sci.get(), sv.get(), cnt2.get());
    CHRONOS_CHECK_LAUNCH();
  }
  std::vector<int> cnt2_h = cnt2.to_host(st);
  // Sort every row segment [rps[i], rps[i]+cnt2[i]) by column.
  {
    DBuf<int64_t> seg_end(m);
    std::vector<int64_t> se(m);
    for (int i = 0; i < m; ++i) se[i] = rps[i] + cnt2_h[i];
    seg_end.upload(se, st);
    const int64_t total = rps[m];
    DBuf<int> sci2(std::max<int64_t>(total, 1));
    DBuf<double> sv2(std::max<int64_t>(total, 1));
    size_t tmp_bytes = 0;
    CHRONOS_CUDA(cub::DeviceSegmentedSort::SortPairs(nullptr, tmp_bytes, sci.get(), sci2.get(),
                                                     sv.get(), sv2.get(), total, m, drps.get(),
                                                     seg_end.get(), st));
    DBuf<unsigned char> tmp(std::max<size_t>(tmp_bytes, 1));
    CHRONOS_CUDA(cub::DeviceSegmentedSort::SortPairs(tmp.get(), tmp_bytes, sci.get(), sci2.get(),
                                                     sv.get(), sv2.get(), total, m, drps.get(),
                                                     seg_end.get(), st));
    sci = std::move(sci2);
    sv = std::move(sv2);
  }
  std::vector<int> crp_h(m + 1, 0);
  for (int i = 0; i < m; ++i) {
    const int64_t t = (int64_t)crp_h[i] + cnt2_h[i];
    CHRONOS_REQUIRE(t < INT32_MAX, CHRONOS_ENOTSUP, "sparse product exceeds 2^31 entries");
    crp_h[i + 1] = (int)t;
  }
  crp.upload(crp_h, st);
  const int64_t nnz = crp_h[m];
  cci.alloc(std::max<int64_t>(nnz, 1));
  cv.alloc(std::max<int64_t>(nnz, 1));
  k_compact_rows<<<m, 128, 0, st>>>(m, drps.get(), cnt2.get(), crp.get(), sci.get(), sv.get(),
                                    cci.get(), cv.get());
  CHRONOS_CHECK_LAUNCH();
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  *nnz_c = nnz;
}

// =============================================================================
// Dense coarse level
// =============================================================================

// Single-block right-looking Cholesky on an n x n column-major matrix.
__global__ void __launch_bounds__(1024) k_dense_cholesky(int n, double *A, int *info) {
  __shared__ int bad;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  if (tid == 0) { bad = 0; *info = 0; }
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    if (tid == 0) {
      const double d = A[(size_t)k * n + k];
      if (!(d > 0.0)) bad = k + 1;
      else A[(size_t)k * n + k] = sqrt(d);
    }
    __syncthreads();
    if (bad) break;
    const double dk = A[(size_t)k * n + k];
    for (int i = k + 1 + tid; i < n; i += blockDim.x) A[(size_t)k * n + i] /= dk;
    __syncthreads();
    for (int j = k + 1 + wid; j < n; j += nw) {
      const double ljk = A[(size_t)k * n + j];
      for (int i = j + lane; i < n; i += 32) A[(size_t)j * n + i] -= A[(size_t)k * n + i] * ljk;
    }
    __syncthreads();
  }
  if (tid == 0) *info = bad;
  // zero the strict upper triangle
  for (int j = 1 + wid; j < n; j += nw)
    for (int i = lane; i < j; i += 32) A[(size_t)j * n + i] = 0.0;
}

int dense_cholesky_device(int n, double *A, cudaStream_t st) {
  DBuf<int> info(1);
  k_dense_cholesky<<<1, 1024, 0, st>>>(n, A, info.get());
  CHRONOS_CHECK_LAUNCH();
  int h = 0;
  CHRONOS_CUDA(cudaMemcpyAsync(&h, info.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  return h;
}

// Column j of L^{-1} by forward substitution (one block per column).
__global__ void k_tri_inverse(int n, const double *L, double *X) {
  extern __shared__ double xs[];
  const int j = blockIdx.x;
  for (int i = threadIdx.x; i < n; i += blockDim.x) xs[i] = (i == j) ? 1.0 : 0.0;
  __syncthreads();
  for (int k = j; k < n; ++k) {
    const double xk = xs[k] / L[(size_t)k * n + k];
    __syncthreads();
    if (threadIdx.x == 0) xs[k] = xk;
    for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) xs[i] -= L[(size_t)k * n + i] * xk;
    __syncthreads();
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) X[(size_t)j * n + i] = xs[i];
}

// W = X^T X with X = L^{-1} lower (column-major); 16x16 tiles.
__global__ void k_gram(int n, const double *X, double *W) {
  __shared__ double a[16][17], b[16][17];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = blockIdx.y * 16 + ty, j = blockIdx.x * 16 + tx;
  double s = 0.0;
  const int kstart = max(blockIdx.y * 16, blockIdx.x * 16);
  for (int k0 = (kstart / 16) * 16; k0 < n; k0 += 16) {
    const int ka = k0 + tx, kb = k0 + ty;
    const int ci = blockIdx.y * 16 + ty, cj = blockIdx.x * 16 + tx;
    a[ty][tx] = (ci < n && ka < n) ? X[(size_t)ci * n + ka] : 0.0;   // X[ka][ci]
    b[ty][tx] = (cj < n && kb < n) ? X[(size_t)cj * n + kb] : 0.0;   // X[kb][cj]
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) s += a[ty][kk] * b[kk][tx];
    __syncthreads();
  }
  if (i < n && j < n) W[(size_t)i * n + j] = s;
}

void dense_inverse_from_chol(int n, const double *L, double *W, cudaStream_t st) {
  DBuf<double> X((size_t)n * n);
  const size_t sm = (size_t)n * sizeof(double);
  CHRONOS_REQUIRE(sm <= 200 * 1024, CHRONOS_ENOTSUP, "coarsest level too large for the dense solve");
  if (sm > 48 * 1024)
    CHRONOS_CUDA(cudaFuncSetAttribute(k_tri_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  k_tri_inverse<<<n, 256, sm, st>>>(n, L, X.get());
  CHRONOS_CHECK_LAUNCH();
  dim3 grid(ceil_div(n, 16), ceil_div(n, 16)), blk(16, 16);
  k_gram<<<grid, blk, 0, st>>>(n, X.get(), W);
  CHRONOS_CHECK_LAUNCH();
  CHRONOS_CUDA(cudaStreamSynchronize(st));
}

template <typename TI, typename TO>
__global__ void k_dense_matvec(int n, const double *__restrict__ W, const TI *__restrict__ b,
                               TO *__restrict__ x) {
  pdl_begin();
  const int lane = threadIdx.x & 31;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= n) return;
  const double *w = W + (size_t)row * n;
  double s = 0.0;
  for (int j = lane; j < n; j += 32) s += w[j] * (double)b[j];
  s = warp_sum(s);
  if (lane == 0) x[row] = (TO)s;
}

template <typename TI, typename TO>
void dense_matvec(int n, const double *W, const TI *b, TO *x, cudaStream_t st) {
  launch_pdl(k_dense_matvec<TI, TO>, ceil_div((int64_t)n * 32, 256), 256, st, n, W, b, x);
  CHRONOS_CHECK_LAUNCH();
}
template void dense_matvec<float, float>(int, const double *, const float *, float *, cudaStream_t);
template void dense_matvec<double, double>(int, const double *, const double *, double *, cudaStream_t);

// =============================================================================
// Vector helpers
// =============================================================================

__global__ void k_f64_to_f32(int64_t n, const double *s, float *d) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x)
    d[k] = (float)s[k];
}

void convert_f64_to_f32(int64_t n, const double *src, float *dst, cudaStream_t st) {
  if (n <= 0) return;
  k_f64_to_f32<<<std::min<int64_t>(ceil_div(n, 256), 4096), 256, 0, st>>>(n, src, dst);
  CHRONOS_CHECK_LAUNCH();
}

// =============================================================================
// CSR layouts on the device: transpose, 16-bit column offsets
// =============================================================================

__global__ void k_row_ids(int n, const int *__restrict__ rp, int *__restrict__ rid) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int k = rp[i]; k < rp[i + 1]; ++k) rid[k] = i;
}

__global__ void k_col_count(int nnz, const int *__restrict__ ci, int *__restrict__ cnt) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x)
    atomicAdd(cnt + ci[k], 1);
}

__global__ void k_iota(int n, int *__restrict__ a) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) a[k] = k;
}

__global__ void k_transpose_fill(int nnz, const int *__restrict__ perm, const int *__restrict__ rid,
                                 const double *__restrict__ v, int *__restrict__ tci,
                                 double *__restrict__ tv) {
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < nnz; d += gridDim.x * blockDim.x) {
    const int k = perm[d];
    tci[d] = rid[k];
    tv[d] = v[k];
  }
}

// Entry k of row i lands in row ci[k] of the transpose; a stable radix sort
// of the row-major entries by column keeps each transposed row in ascending
// order of i (then of k), which is the order the host transpose fills.
void csr_transpose_device(int nrows, int ncols, int64_t nnz64, const int *rp, const int *ci,
                          const double *v, DBuf<int> &trp, DBuf<int> &tci, DBuf<double> &tv,
                          cudaStream_t st) {
  CHRONOS_REQUIRE(nnz64 < INT32_MAX, CHRONOS_ENOTSUP, "matrix with 2^31 or more entries");
  const int nnz = (int)nnz64;
  trp.alloc((size_t)ncols + 1);
  tci.alloc(std::max(nnz, 1));
  tv.alloc(std::max(nnz, 1));
  DBuf<int> cnt((size_t)ncols + 1);
  cnt.zero(st);
  const int grid = std::max(1, std::min<int>(ceil_div(std::max(nnz, 1), 256), num_sms() * 16));
  if (nnz > 0) {
    k_col_count<<<grid, 256, 0, st>>>(nnz, ci, cnt.get());
    CHRONOS_CHECK_LAUNCH();
  }
  size_t bytes = 0;
  CHRONOS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, cnt.get(), trp.get(), ncols + 1, st));
  {
    DBuf<unsigned char> tmp(std::max<size_t>(bytes, 1));
    CHRONOS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), bytes, cnt.get(), trp.get(), ncols + 1,
                                               st));
    CHRONOS_CUDA(cudaStreamSynchronize(st));
  }
  if (nnz == 0) return;
  DBuf<int> rid(nnz), idx(nnz), perm(nnz), keys(nnz);
  k_row_ids<<<std::max(1, std::min<int>(ceil_div(std::max(nrows, 1), 256), num_sms() * 16)), 256,
              0, st>>>(nrows, rp, rid.get());
  CHRONOS_CHECK_LAUNCH();
  k_iota<<<grid, 256, 0, st>>>(nnz, idx.get());
  CHRONOS_CHECK_LAUNCH();
  int end_bit = 1;
  while (end_bit < 31 && (1LL << end_bit) < (long long)ncols) ++end_bit;
  bytes = 0;
  CHRONOS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, ci, keys.get(), idx.get(),
                                               perm.get(), nnz, 0, end_bit, st));
  {
    DBuf<unsigned char> tmp(std::max<size_t>(bytes, 1));
    CHRONOS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), bytes, ci, keys.get(), idx.get(),
                                                 perm.get(), nnz, 0, end_bit, st));
    k_transpose_fill<<<grid, 256, 0, st>>>(nnz, perm.get(), rid.get(), v, tci.get(), tv.get());
    CHRONOS_CHECK_LAUNCH();
    CHRONOS_CUDA(cudaStreamSynchronize(st));
  }
}

__global__ void k_row_span(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                           int *__restrict__ base, int *__restrict__ wide) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int s = rp[i], e = rp[i + 1];
    int lo = 0;
    if (e > s) {
      lo = ci[s];
      int hi = lo;
      for (int k = s + 1; k < e; ++k) {
        lo = min(lo, ci[k]);
        hi = max(hi, ci[k]);
      }
      if (hi - lo > 0xffff) atomicOr(wide, 1);
    }
    base[i] = lo;
  }
}

__global__ void k_col_offsets16(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                const int *__restrict__ base, uint16_t *__restrict__ off) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int k = rp[i]; k < rp[i + 1]; ++k) off[k] = (uint16_t)(ci[k] - base[i]);
}

bool csr_offsets16_device(int nrows, int64_t nnz, const int *rp, const int *ci, DBuf<int> &base,
                          DBuf<uint16_t> &off, cudaStream_t st) {
  if (nrows <= 0) return false;
  base.alloc(nrows);
  DBuf<int> wide(1);
  wide.zero(st);
  const int grid = std::max(1, std::min<int>(ceil_div(nrows, 256), num_sms() * 16));
  k_row_span<<<grid, 256, 0, st>>>(nrows, rp, ci, base.get(), wide.get());
  CHRONOS_CHECK_LAUNCH();
  int w = 0;
  CHRONOS_CUDA(cudaMemcpyAsync(&w, wide.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  if (w) {
    base.release();
    return false;
  }
  off.alloc(std::max<int64_t>(nnz, 1));
  k_col_offsets16<<<grid, 256, 0, st>>>(nrows, rp, ci, base.get(), off.get());
  CHRONOS_CHECK_LAUNCH();
  return true;
}

__global__ void k_dot_partial(int n, const double *a, const double *b, double *part) {
  __shared__ double red[32];
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s += a[i] * b[i];
  s = block_sum(s, red);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

double device_dot(int n, const double *a, const double *b, double *scratch, cudaStream_t st) {
  const int blocks = 256;
  k_dot_partial<<<blocks, 256, 0, st>>>(n, a, b, scratch);
  CHRONOS_CHECK_LAUNCH();
  double h[256];
  CHRONOS_CUDA(cudaMemcpyAsync(h, scratch, sizeof(h), cudaMemcpyDeviceToHost, st));
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  double s = 0.0;
  for (int i = 0; i < blocks; ++i) s += h[i];
  return s;
}

__global__ void k_axpby(int n, double a, const double *x, double b, double *y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = a * x[i] + b * y[i];
}

void device_axpby(int n, double a, const double *x, double b, double *y, cudaStream_t st) {
  k_axpby<<<std::min<int64_t>(ceil_div(n, 256), 4096), 256, 0, st>>>(n, a, x, b, y);
  CHRONOS_CHECK_LAUNCH();
}

__global__ void k_scale_copy(int n, double a, const double *x, double *y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = a * x[i];
}

void device_scale_copy(int n, double a, const double *x, double *y, cudaStream_t st) {
  k_scale_copy<<<std::min<int64_t>(ceil_div(n, 256), 4096), 256, 0, st>>>(n, a, x, y);
  CHRONOS_CHECK_LAUNCH();
}

__global__ void k_diag_mul(int n, const double *d, const double *x, double *y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = d[i] * x[i];
}

void device_diag_mul(int n, const double *d, const double *x, double *y, cudaStream_t st) {
  k_diag_mul<<<std::min<int64_t>(ceil_div(n, 256), 4096), 256, 0, st>>>(n, d, x, y);
  CHRONOS_CHECK_LAUNCH();
}

// One warp per row: grad[k] = -lambda_i * u_{col(k)} over the row's entries.
__global__ void k_adjoint_scatter(int n, const int *rp, const int *ci, const double *lam,
                                  const double *u, double *grad) {
  const int lane = threadIdx.x & 31;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= n) return;
  const double li = -lam[row];
  for (int k = rp[row] + lane; k < rp[row + 1]; k += 32) grad[k] = li * u[ci[k]];
}

void adjoint_scatter(int n, const int *rp, const int *ci, const double *lambda, const double *u,
                     double *grad, cudaStream_t st) {
  if (n <= 0) return;
  k_adjoint_scatter<<<ceil_div((int64_t)n * 32, 256), 256, 0, st>>>(n, rp, ci, lambda, u, grad);
  CHRONOS_CHECK_LAUNCH();
}

// =============================================================================
// FSAI numeric phase without allocation (chronos_fsai_numeric_noalloc)
// =============================================================================
//
// Same kernels as fsai_numeric_device, but the scratch they need -- the three
// row-bucket lists and the flag word -- lives in one file-scope device array
// instead of cudaMalloc'd buffers.  The array is a fixed 12 MiB + 256 B per
// device that loads the library, held until the process exits.  Every call
// shares it: calls that overlap on the GPU (two streams, two host threads)
// race on it and must be serialised by the caller.

constexpr int kNoAllocMaxRows = 1 << 20;
constexpr int kNoAllocHeader = 64;            // ints: [0..2] bucket counts, [3] flags
static __device__ __align__(256) int g_fsai_noalloc_scratch[kNoAllocHeader + 3 * kNoAllocMaxRows];

// In host code g_fsai_noalloc_scratch names a host-side stand-in, not a device
// address: the device address is looked up once per device with
// cudaGetSymbolAddress (with that device current) and cached here.
static int *g_noalloc_addr[64] = {nullptr};
static std::mutex g_noalloc_mu;

static int *noalloc_scratch_address() {
  int dev = 0;
  CHRONOS_CUDA(cudaGetDevice(&dev));
  CHRONOS_REQUIRE(dev >= 0 && dev < 64, CHRONOS_EINVAL, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    CHRONOS_CUDA(cudaGetSymbolAddress(&p, g_fsai_noalloc_scratch));
    g_noalloc_addr[dev] = static_cast<int *>(p);
  }
  return g_noalloc_addr[dev];
}

// Checks row i of both patterns and sorts it into the 16 / 32 / 64 buckets of
// fsai_numeric_device.  The numeric kernel indexes A's rows by G's columns and
// writes G's row at gval[grp[i] .. grp[i+1]-1] with the diagonal last, so a
// malformed row sets flag bit 2 (and is not bucketed): a G row without
// entries, a last column other than i, strictly-lower columns not ascending
// or outside [0, i); an A row whose pointers decrease or whose columns are not
// ascending inside [0, n); row pointers of either that do not start at 0.
// A row longer than 64 strictly-lower entries sets flag bit 1.
__global__ void k_fsai_bucket_rows(int n, const int *__restrict__ arp, const int *__restrict__ aci,
                                   const int *__restrict__ grp, const int *__restrict__ gci,
                                   int *scratch) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int gs = grp[i], ge = grp[i + 1];
  bool bad = ge <= gs || (i == 0 && (gs != 0 || arp[0] != 0));
  if (!bad) {
    bad = gci[ge - 1] != i;
    for (int k = gs, prev = -1; !bad && k < ge - 1; ++k) {
      const int c = gci[k];
      bad = c <= prev || c >= i;
      prev = c;
    }
  }
  const int as = arp[i], ae = arp[i + 1];
  bad = bad || ae < as;
  for (int k = as, prev = -1; !bad && k < ae; ++k) {
    const int c = aci[k];
    bad = c <= prev || c >= n;
    prev = c;
  }
  if (bad) { atomicOr(scratch + 3, 4); return; }
  const int m = ge - gs - 1;
  int b;
  if (m <= 16) b = 0;
  else if (m <= 32) b = 1;
  else if (m <= 64) b = 2;
  else { atomicOr(scratch + 3, 2); return; }
  const int pos = atomicAdd(scratch + b, 1);
  scratch[kNoAllocHeader + b * kNoAllocMaxRows + pos] = i;
}

int fsai_numeric_noalloc(int n, const int *arp, const int *aci, const double *av, const int *grp,
                         const int *gci, double *gval, cudaStream_t st) {
  CHRONOS_REQUIRE(n > 0 && n <= kNoAllocMaxRows, CHRONOS_EINVAL,
                  "chronos_fsai_numeric_noalloc: n must be in [1, 1048576] (its static scratch "
                  "holds 1048576 rows)");
  int *scr = noalloc_scratch_address();
  // the previous call's contents remain: clear the counts and the flag word
  CHRONOS_CUDA(cudaMemsetAsync(scr, 0, kNoAllocHeader * sizeof(int), st));
  k_fsai_bucket_rows<<<ceil_div(n, 256), 256, 0, st>>>(n, arp, aci, grp, gci, scr);
  CHRONOS_CHECK_LAUNCH();
  int hdr[4] = {0, 0, 0, 0};
  CHRONOS_CUDA(cudaMemcpyAsync(hdr, scr, sizeof(hdr), cudaMemcpyDeviceToHost, st));
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  // no numeric kernel runs on a malformed pattern: it would read A and write
  // G's values outside the rows the caller's buffers hold
  CHRONOS_REQUIRE(!(hdr[3] & 4), CHRONOS_EINVAL,
                  "malformed CSR: a G row is empty, does not end with its diagonal or has "
                  "strictly-lower columns not ascending in [0, i); or A's row pointers / "
                  "columns are not a sorted 0-based CSR");
  CHRONOS_REQUIRE(!(hdr[3] & 2), CHRONOS_ENOTSUP,
                  "FSAI local system larger than 64 (nstep*step_size)");
  auto run = [&](auto kern, int cnt, int bucket, int mmax, int warps) {
    if (cnt == 0) return;
    const size_t sm = (size_t)warps * (mmax * mmax + 3 * mmax) * sizeof(double);
    CHRONOS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    kern<<<ceil_div(cnt, warps), warps * 32, sm, st>>>(
        cnt, scr + kNoAllocHeader + bucket * kNoAllocMaxRows, arp, aci, av, grp, gci, gval, scr + 3);
    CHRONOS_CHECK_LAUNCH();
  };
  run(k_fsai_numeric<16>, hdr[0], 0, 16, 8);
  run(k_fsai_numeric<32>, hdr[1], 1, 32, 4);
  run(k_fsai_numeric<64>, hdr[2], 2, 64, 2);
  int fl = 0;
  CHRONOS_CUDA(cudaMemcpyAsync(&fl, scr + 3, sizeof(int), cudaMemcpyDeviceToHost, st));
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  return fl;
}

}  // namespace chronos

extern "C" int chronos_fsai_numeric_noalloc(int n, const int *iat_A_d, const int *ja_A_d,
                                            const double *val_A_d, const int *iat_G_d,
                                            const int *ja_G_d, double *val_G_d, int *is_posdef,
                                            void *stream) {
  try {
    CHRONOS_REQUIRE(iat_A_d && ja_A_d && val_A_d && iat_G_d && ja_G_d && val_G_d && is_posdef,
                    CHRONOS_EINVAL, "null argument");
    const int fl = chronos::fsai_numeric_noalloc(n, iat_A_d, ja_A_d, val_A_d, iat_G_d, ja_G_d,
                                                 val_G_d, static_cast<cudaStream_t>(stream));
    *is_posdef = (fl & 1) ? 0 : 1;
    return CHRONOS_OK;
  } catch (const chronos::Error &e) {
    chronos::set_last_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    chronos::set_last_error(e.what());
    return CHRONOS_EINVAL;
  }
}
