// Block of K right-hand sides solved together: SpMM V-cycles and K independent
// PCG_CJ recurrences (PCG_CJ.m:34-66 per column) in one CUDA graph.
//
// Vectors are row-major n x K (X[i*K + j]).  In the SpMM kernel K consecutive
// lanes own one row, lane j its column j: every stored value and column index
// is fetched once (a broadcast to the K lanes) and reused K times, and the
// gathers X[c*K + 0..K-1] are K-wide coalesced loads.  Each column keeps its
// own scalars, iteration count and stopping test; a converged column is frozen
// (its x, res and p no longer change), so every column returns exactly what a
// single-column PCG_CJ returns.  The block dot products are K-wide
// deterministic grid reductions.
#include <algorithm>
#include <cmath>

#include "hier.h"
#include "spmv.cuh"

namespace chronos {

template <int K> struct StoreK {
  double *dst;
  __device__ void operator()(const double *t) const {
    for (int q = 0; q < K; ++q) dst[q] = t[q];
  }
};

// VEC consecutive elements as one 8- or 16-byte access (aligned: K is a
// multiple of VEC and every block starts on a 256-byte boundary).
template <typename T, int VEC> struct Vec;
template <> struct Vec<float, 4> {
  __device__ static void ld(const float *p, float (&o)[4]) {
    const float4 t = __ldg(reinterpret_cast<const float4 *>(p));
    o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
  }
  __device__ static void st(float *p, const float (&o)[4]) {
    *reinterpret_cast<float4 *>(p) = make_float4(o[0], o[1], o[2], o[3]);
  }
};
template <> struct Vec<float, 2> {
  __device__ static void ld(const float *p, float (&o)[2]) {
    const float2 t = __ldg(reinterpret_cast<const float2 *>(p));
    o[0] = t.x; o[1] = t.y;
  }
  __device__ static void st(float *p, const float (&o)[2]) {
    *reinterpret_cast<float2 *>(p) = make_float2(o[0], o[1]);
  }
};
template <> struct Vec<double, 2> {
  __device__ static void ld(const double *p, double (&o)[2]) {
    const double2 t = __ldg(reinterpret_cast<const double2 *>(p));
    o[0] = t.x; o[1] = t.y;
  }
  __device__ static void st(double *p, const double (&o)[2]) {
    *reinterpret_cast<double2 *>(p) = make_double2(o[0], o[1]);
  }
};

// Lanes own VEC consecutive right-hand-side columns of one row: K/VEC lanes
// per row, 32*VEC/K rows per warp; each stored value and column index is
// fetched once per row group and applied to K columns.
template <typename VT, typename XT, typename ZT, typename YT, int K, int VEC, int MODE, bool DOT>
__global__ void __launch_bounds__(kApplyThreads)
k_csr_spmm(int n, const int *__restrict__ rp, const int *__restrict__ ci,
           const VT *__restrict__ v, const XT *__restrict__ X, const ZT *Z, YT *Y, VT alpha,
           const double *__restrict__ DW, double *part, unsigned *ticket, double *dot_out) {
  constexpr int LPR = K / VEC;
  constexpr int R = 32 / LPR;
  const int lane = threadIdx.x & 31, g = lane / LPR, j0 = (lane % LPR) * VEC;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double dacc[VEC];
#pragma unroll
  for (int e = 0; e < VEC; ++e) dacc[e] = 0.0;
  for (int base = warp * R; base < n; base += nwarps * R) {
    const int row = base + g;
    if (row < n) {
      VT s[VEC];
#pragma unroll
      for (int e = 0; e < VEC; ++e) s[e] = VT(0);
      const int e1 = __ldg(rp + row + 1);
      int k = __ldg(rp + row);
      for (; k + 3 < e1; k += 4) {            // four entries' loads in flight
        int c[4];
        VT a[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) { c[u] = __ldg(ci + k + u); a[u] = __ldg(v + k + u); }
        XT xv[4][VEC];
#pragma unroll
        for (int u = 0; u < 4; ++u) Vec<XT, VEC>::ld(X + (size_t)c[u] * K + j0, xv[u]);
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int e = 0; e < VEC; ++e) s[e] += a[u] * (VT)xv[u][e];
      }
      for (; k < e1; ++k) {
        const VT a = __ldg(v + k);
        XT xv[VEC];
        Vec<XT, VEC>::ld(X + (size_t)__ldg(ci + k) * K + j0, xv);
#pragma unroll
        for (int e = 0; e < VEC; ++e) s[e] += a * (VT)xv[e];
      }
      const size_t o = (size_t)row * K + j0;
      ZT zv[VEC];
      if (MODE == MODE_RESID || MODE == MODE_AXPY) Vec<ZT, VEC>::ld(Z + o, zv);
      YT out[VEC];
#pragma unroll
      for (int e = 0; e < VEC; ++e) {
        VT r;
        if (MODE == MODE_PLAIN) r = s[e];
        else if (MODE == MODE_SCALE) r = alpha * s[e];
        else if (MODE == MODE_RESID) r = (VT)zv[e] - s[e];
        else r = (VT)zv[e] + alpha * s[e];
        out[e] = (YT)r;
        if (DOT) dacc[e] += (double)out[e] * DW[o + e];
      }
      Vec<YT, VEC>::st(Y + o, out);
    }
  }
  if (DOT) {
    double vals[1][VEC];
#pragma unroll
    for (int e = 0; e < VEC; ++e) vals[0][e] = dacc[e];
    grid_reduce_cols<K, VEC, 1>(vals, part, ticket, StoreK<K>{dot_out});
  }
}

// 16-byte accesses when every operand is FP32 (VEC 4), else VEC 2.
template <typename XT, typename ZT, typename YT, int K>
struct SpmmVec {
  static constexpr int v4 = (sizeof(XT) == 4 && sizeof(YT) == 4 && sizeof(ZT) == 4) ? 4 : 2;
  static constexpr int value = v4 > K ? K : v4;
};

template <typename VT, typename XT, typename ZT, typename YT, int K, int MODE, bool DOT>
static void spmm(cudaStream_t st, const DMat &M, const VT *vals, const XT *X, const ZT *Z, YT *Y,
                 VT alpha, const double *DW = nullptr, double *part = nullptr,
                 unsigned *tick = nullptr, double *dot_out = nullptr) {
  constexpr int VEC = SpmmVec<XT, ZT, YT, K>::value;
  const int n = M.nrows;
  if (n <= 0) return;
  const int rows_per_block = kApplyThreads * VEC / K;
  int blocks = (int)ceil_div(n, rows_per_block);
  blocks = std::min(blocks, num_sms() * 8);
  k_csr_spmm<VT, XT, ZT, YT, K, VEC, MODE, DOT><<<blocks, kApplyThreads, 0, st>>>(
      n, M.rp, M.ci, vals, X, Z, Y, alpha, DW, part, tick, dot_out);
  CHRONOS_CHECK_LAUNCH();
}

// Y = W B on the coarsest level (W FP64 n x n row-major, B n x K row-major).
template <typename TI, typename TO, int K>
__global__ void k_dense_matmat(int n, const double *__restrict__ W, const TI *__restrict__ B,
                               TO *__restrict__ Y) {
  const int row = blockIdx.x, j = threadIdx.x % K, g = threadIdx.x / K, G = blockDim.x / K;
  __shared__ double red[256];
  double s = 0.0;
  for (int c = g; c < n; c += G) s += W[(size_t)row * n + c] * (double)B[(size_t)c * K + j];
  red[threadIdx.x] = s;
  __syncthreads();
  if (g == 0) {
    double t = 0.0;
    for (int q = 0; q < G; ++q) t += red[q * K + j];
    Y[(size_t)row * K + j] = (TO)t;
  }
}

// ---------------------------------------------------------------------------

struct BlockState {
  int K = 0, n = 0;
  std::vector<DBuf<float>> b32, x32, r32, t32;
  std::vector<DBuf<double>> b64, x64, r64, t64;
  DBuf<double> x, res, p, axp, pres;
  DBuf<double> sc;              // per-column scalars, see BS_* below
  DBuf<double> part;
  DBuf<unsigned> tickets;
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  ~BlockState() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
};

// per-column scalar arrays (each K wide) inside sc
enum { BS_BNORM = 0, BS_PTAP, BS_ALPHA, BS_PRES_AXP, BS_RESITER, BS_ITER, BS_ACTIVE, BS_FLAG,
       BS_PRES, BS_COUNT };
// after the K-wide arrays: tol, itmax
__host__ __device__ constexpr int bs_off(int which, int K) { return which * K; }

template <typename T, typename BT, typename OT, int K>
static void vcycle_block(Hier &h, BlockState &s, int l, const BT *b, OT *out, const double *dw,
                         double *dot_out);

template <typename T> static T *blk(std::vector<DBuf<float>> &f, std::vector<DBuf<double>> &d, int l);
template <> float *blk<float>(std::vector<DBuf<float>> &f, std::vector<DBuf<double>> &, int l) { return f[l].get(); }
template <> double *blk<double>(std::vector<DBuf<float>> &, std::vector<DBuf<double>> &d, int l) { return d[l].get(); }

template <typename T, typename BT, typename OT, int K>
static void vcycle_block(Hier &h, BlockState &s, int l, const BT *b, OT *out, const double *dw,
                         double *dot_out) {
  Level &L = h.levels[l];
  cudaStream_t st = h.st;
  const int n = L.n;
  double *part = s.part.get();
  unsigned *tick = s.tickets.get();
  if (L.coarsest) {
    k_dense_matmat<BT, OT, K><<<n, 256, 0, st>>>(n, L.W.get(), b, out);
    CHRONOS_CHECK_LAUNCH();
    return;
  }
  T *x = blk<T>(s.x32, s.x64, l), *r = blk<T>(s.r32, s.r64, l), *t = blk<T>(s.t32, s.t64, l);
  const T w = (T)L.omega;
  spmm<T, BT, T, T, K, MODE_PLAIN, false>(st, L.G, vals<T>(L.G), b, (const T *)nullptr, t, T(1));
  spmm<T, T, T, T, K, MODE_SCALE, false>(st, L.Gt, vals<T>(L.Gt), t, (const T *)nullptr, x, w);
  for (int k = 1; k < h.prm.nupre; ++k) {
    spmm<T, T, BT, T, K, MODE_RESID, false>(st, L.A, vals<T>(L.A), x, b, r, T(1));
    spmm<T, T, T, T, K, MODE_PLAIN, false>(st, L.G, vals<T>(L.G), r, (const T *)nullptr, t, T(1));
    spmm<T, T, T, T, K, MODE_AXPY, false>(st, L.Gt, vals<T>(L.Gt), t, x, x, w);
  }
  spmm<T, T, BT, T, K, MODE_RESID, false>(st, L.A, vals<T>(L.A), x, b, r, T(1));
  T *bc = blk<T>(s.b32, s.b64, l + 1), *xc = blk<T>(s.x32, s.x64, l + 1);
  spmm<T, T, T, T, K, MODE_PLAIN, false>(st, L.Pt, vals<T>(L.Pt), r, (const T *)nullptr, bc, T(1));
  vcycle_block<T, T, T, K>(h, s, l + 1, bc, xc, nullptr, nullptr);
  spmm<T, T, T, T, K, MODE_AXPY, false>(st, L.P, vals<T>(L.P), xc, x, x, T(1));
  const int npost = h.prm.nupost;
  for (int k = 0; k < npost; ++k) {
    spmm<T, T, BT, T, K, MODE_RESID, false>(st, L.A, vals<T>(L.A), x, b, r, T(1));
    spmm<T, T, T, T, K, MODE_PLAIN, false>(st, L.G, vals<T>(L.G), r, (const T *)nullptr, t, T(1));
    if (k + 1 < npost)
      spmm<T, T, T, T, K, MODE_AXPY, false>(st, L.Gt, vals<T>(L.Gt), t, x, x, w);
    else if (dw)
      spmm<T, T, T, OT, K, MODE_AXPY, true>(st, L.Gt, vals<T>(L.Gt), t, x, out, w, dw, part, tick,
                                            dot_out);
    else
      spmm<T, T, T, OT, K, MODE_AXPY, false>(st, L.Gt, vals<T>(L.Gt), t, x, out, w);
  }
  if (npost == 0) {
    if (dw)
      spmm<T, T, T, OT, K, MODE_AXPY, true>(st, L.Gt, vals<T>(L.Gt), t, x, out, T(0), dw, part,
                                            tick, dot_out);
    else
      spmm<T, T, T, OT, K, MODE_AXPY, false>(st, L.Gt, vals<T>(L.Gt), t, x, out, T(0));
  }
}

// ---- block PCG kernels ------------------------------------------------------

template <int K>
__global__ void k_bpcg_p_update(int n, const double *__restrict__ pres, double *__restrict__ p,
                                const double *__restrict__ sc) {
  const double *ptap = sc + bs_off(BS_PTAP, K), *pa = sc + bs_off(BS_PRES_AXP, K);
  const double *it = sc + bs_off(BS_ITER, K), *act = sc + bs_off(BS_ACTIVE, K);
  const size_t total = (size_t)n * K;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < total;
       o += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(o % K);
    if (act[j] == 0.0) continue;
    if (it[j] < 0.5) p[o] = pres[o];
    else p[o] = pres[o] + (-pa[j] / ptap[j]) * p[o];
  }
}

template <int K> struct FinAlphaBlock {
  double *sc;
  __device__ void operator()(const double *t) const {
    for (int j = 0; j < K; ++j) {
      if (sc[bs_off(BS_ACTIVE, K) + j] == 0.0) continue;
      const double ptap = t[j], pr = t[K + j];
      sc[bs_off(BS_PTAP, K) + j] = ptap;
      if (!(ptap > 0.0) || !isfinite(pr)) {
        sc[bs_off(BS_ALPHA, K) + j] = 0.0;
        sc[bs_off(BS_FLAG, K) + j] = 2.0;          // breakdown
      } else {
        sc[bs_off(BS_ALPHA, K) + j] = pr / ptap;
      }
    }
  }
};

// axp = A p (FP64, block) with p'axp and p'res per column.
template <int K>
__global__ void __launch_bounds__(kApplyThreads)
k_bpcg_spmm(int n, const int *__restrict__ rp, const int *__restrict__ ci,
            const double *__restrict__ v, const double *__restrict__ p,
            const double *__restrict__ res, double *__restrict__ axp, double *part,
            unsigned *ticket, double *sc) {
  constexpr int LPR = K / 2;                      // two columns per lane (double2)
  constexpr int R = 32 / LPR;
  const int lane = threadIdx.x & 31, g = lane / LPR, j0 = (lane % LPR) * 2;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double d0[2] = {0.0, 0.0}, d1[2] = {0.0, 0.0};
  for (int base = warp * R; base < n; base += nwarps * R) {
    const int row = base + g;
    if (row < n) {
      double s[2] = {0.0, 0.0};
      const int e1 = __ldg(rp + row + 1);
      int k = __ldg(rp + row);
      for (; k + 3 < e1; k += 4) {            // four entries' loads in flight
        int c[4];
        double a[4], pv[4][2];
#pragma unroll
        for (int u = 0; u < 4; ++u) { c[u] = __ldg(ci + k + u); a[u] = __ldg(v + k + u); }
#pragma unroll
        for (int u = 0; u < 4; ++u) Vec<double, 2>::ld(p + (size_t)c[u] * K + j0, pv[u]);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          s[0] += a[u] * pv[u][0];
          s[1] += a[u] * pv[u][1];
        }
      }
      if (k < e1) {                            // the last 1..3 entries, loads predicated
        int c[3];
        double a[3], pv[3][2];
#pragma unroll
        for (int u = 0; u < 3; ++u) {
          c[u] = -1;
          a[u] = 0.0;
          if (k + u < e1) { c[u] = __ldg(ci + k + u); a[u] = __ldg(v + k + u); }
        }
#pragma unroll
        for (int u = 0; u < 3; ++u)
          if (c[u] >= 0) Vec<double, 2>::ld(p + (size_t)c[u] * K + j0, pv[u]);
#pragma unroll
        for (int u = 0; u < 3; ++u)
          if (c[u] >= 0) {
            s[0] += a[u] * pv[u][0];
            s[1] += a[u] * pv[u][1];
          }
      }
      const size_t o = (size_t)row * K + j0;
      Vec<double, 2>::st(axp + o, s);
      double po[2], ro[2];
      Vec<double, 2>::ld(p + o, po);
      Vec<double, 2>::ld(res + o, ro);
      for (int e = 0; e < 2; ++e) {
        d0[e] += po[e] * s[e];
        d1[e] += po[e] * ro[e];
      }
    }
  }
  double vals[2][2] = {{d0[0], d0[1]}, {d1[0], d1[1]}};
  grid_reduce_cols<K, 2, 2>(vals, part, ticket, FinAlphaBlock<K>{sc});
}

template <int K> struct FinResidualBlock {
  double *sc;
  cudaGraphConditionalHandle handle;
  int use_cond;
  __device__ void operator()(const double *t) const {
    const double tol = sc[BS_COUNT * K], itmax = sc[BS_COUNT * K + 1];
    bool any = false;
    for (int j = 0; j < K; ++j) {
      if (sc[bs_off(BS_ACTIVE, K) + j] == 0.0) continue;
      const double it = sc[bs_off(BS_ITER, K) + j] + 1.0;
      sc[bs_off(BS_ITER, K) + j] = it;
      const double r = sqrt(t[j]) / sc[bs_off(BS_BNORM, K) + j];
      sc[bs_off(BS_RESITER, K) + j] = r;
      const bool stop = r < tol || it >= itmax || sc[bs_off(BS_FLAG, K) + j] != 0.0 ||
                        !isfinite(r);
      if (stop) sc[bs_off(BS_ACTIVE, K) + j] = 0.0;
      else any = true;
    }
    sc[BS_COUNT * K + 2] = any ? 1.0 : 0.0;
    if (use_cond) cudaGraphSetConditional(handle, any ? 1u : 0u);
  }
};

template <int K>
__global__ void __launch_bounds__(256)
k_bpcg_xr_update(int n, double *__restrict__ x, double *__restrict__ res,
                 const double *__restrict__ p, const double *__restrict__ axp, double *part,
                 unsigned *ticket, double *sc, cudaGraphConditionalHandle handle, int use_cond) {
  // K threads of a group of K walk the K columns of consecutive rows
  const int j = threadIdx.x % K;
  const bool act = sc[bs_off(BS_ACTIVE, K) + j] != 0.0;
  const double alpha = sc[bs_off(BS_ALPHA, K) + j];
  double rr = 0.0;
  const size_t total = (size_t)n * K;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < total;
       o += (size_t)gridDim.x * blockDim.x) {
    double ri = res[o];
    if (act) {
      x[o] += alpha * p[o];
      ri -= alpha * axp[o];
      res[o] = ri;
    }
    rr += ri * ri;
  }
  double vals[1][1] = {{rr}};
  grid_reduce_cols<K, 1, 1>(vals, part, ticket, FinResidualBlock<K>{sc, handle, use_cond});
}

// ||B(:,j)||^2 and ||R(:,j)||^2 into sc (BNORM, RESITER hold squares until init)
template <int K>
__global__ void __launch_bounds__(256)
k_bnorm2(int n, const double *__restrict__ B, double *part, unsigned *ticket, double *dst) {
  const int j = threadIdx.x % K;
  double s = 0.0;
  const size_t total = (size_t)n * K;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < total;
       o += (size_t)gridDim.x * blockDim.x)
    s += B[o] * B[o];
  double vals[1][1] = {{s}};
  grid_reduce_cols<K, 1, 1>(vals, part, ticket, StoreK<K>{dst});
}

template <int K>
__global__ void k_bpcg_init(double *sc, const double *b2, const double *r2, double tol,
                            double itmax) {
  for (int j = 0; j < K; ++j) {
    const double bn = sqrt(b2[j]);
    sc[bs_off(BS_BNORM, K) + j] = bn;
    sc[bs_off(BS_RESITER, K) + j] = bn > 0.0 ? sqrt(r2[j]) / bn : 0.0;
    sc[bs_off(BS_ITER, K) + j] = 0.0;
    sc[bs_off(BS_FLAG, K) + j] = 0.0;
    sc[bs_off(BS_ACTIVE, K) + j] = (bn > 0.0 && itmax > 0.0) ? 1.0 : 0.0;
  }
  sc[BS_COUNT * K] = tol;
  sc[BS_COUNT * K + 1] = itmax;
}

// zero columns with b = 0 (PCG_CJ.m:12-16)
template <int K>
__global__ void k_zero_null_columns(int n, double *x, const double *sc) {
  const size_t total = (size_t)n * K;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < total;
       o += (size_t)gridDim.x * blockDim.x)
    if (sc[bs_off(BS_BNORM, K) + (int)(o % K)] == 0.0) x[o] = 0.0;
}

template <int K>
static void capture_block_iteration(Hier &h, BlockState &s, cudaGraphConditionalHandle handle,
                                    int use_cond) {
  cudaStream_t st = h.st;
  const int n = s.n;
  double *sc = s.sc.get();
  unsigned *tk = s.tickets.get();
  const int nb = std::max(1, std::min(num_sms() * 8, (int)ceil_div((int64_t)n * K, 256)));
  if (h.precision == CHRONOS_FP32)
    vcycle_block<float, double, double, K>(h, s, 0, s.res.get(), s.pres.get(), s.axp.get(),
                                           sc + bs_off(BS_PRES_AXP, K));
  else
    vcycle_block<double, double, double, K>(h, s, 0, s.res.get(), s.pres.get(), s.axp.get(),
                                            sc + bs_off(BS_PRES_AXP, K));
  k_bpcg_p_update<K><<<nb, 256, 0, st>>>(n, s.pres.get(), s.p.get(), sc);
  CHRONOS_CHECK_LAUNCH();
  const DMat &A = h.levels[0].A;
  const int blocks = std::min(num_sms() * 8, (int)ceil_div(n, kApplyThreads * 2 / K));
  k_bpcg_spmm<K><<<blocks, kApplyThreads, 0, st>>>(n, A.rp, A.ci, A.v64, s.p.get(), s.res.get(),
                                                   s.axp.get(), s.part.get() + 2 * K * 2048,
                                                   tk + 1, sc);
  CHRONOS_CHECK_LAUNCH();
  k_bpcg_xr_update<K><<<nb, 256, 0, st>>>(n, s.x.get(), s.res.get(), s.p.get(), s.axp.get(),
                                          s.part.get() + 4 * K * 2048, tk + 2, sc, handle,
                                          use_cond);
  CHRONOS_CHECK_LAUNCH();
}

template <int K>
static void block_solve(Hier &h, const double *B_h, double *X_h, int itmax, double tol,
                        int *iters, int *flags, double *seconds) {
  cudaStream_t st = h.st;
  auto &sp = h.block;
  if (!sp || sp->K != K) {
    sp = std::make_shared<BlockState>();
    BlockState &s = *sp;
    s.K = K;
    s.n = h.levels[0].n;
    const bool fp32 = h.precision == CHRONOS_FP32;
    const int nl = (int)h.levels.size();
    s.b32.resize(nl); s.x32.resize(nl); s.r32.resize(nl); s.t32.resize(nl);
    s.b64.resize(nl); s.x64.resize(nl); s.r64.resize(nl); s.t64.resize(nl);
    for (int l = 0; l < nl; ++l) {
      const size_t m = (size_t)std::max(h.levels[l].n, 1) * K;
      if (fp32) { s.b32[l].alloc(m); s.x32[l].alloc(m); s.r32[l].alloc(m); s.t32[l].alloc(m); }
      else { s.b64[l].alloc(m); s.x64[l].alloc(m); s.r64[l].alloc(m); s.t64[l].alloc(m); }
    }
    const size_t m0 = (size_t)s.n * K;
    s.x.alloc(m0); s.res.alloc(m0); s.p.alloc(m0); s.axp.alloc(m0); s.pres.alloc(m0);
    s.p.zero(st);
    s.axp.zero(st);
    s.sc.alloc((size_t)BS_COUNT * K + 8);
    s.part.alloc((size_t)6 * K * 2048);
    s.tickets.alloc(8);
    s.tickets.zero(st);
  }
  BlockState &s = *sp;
  const int n = s.n;
  const size_t m0 = (size_t)n * K;
  DBuf<double> b(m0), r2(K), b2(K);
  // column-major host blocks -> row-major device blocks
  {
    std::vector<double> tmp(m0), tx(m0);
    for (int j = 0; j < K; ++j)
      for (int i = 0; i < n; ++i) {
        tmp[(size_t)i * K + j] = B_h[(size_t)j * n + i];
        tx[(size_t)i * K + j] = X_h[(size_t)j * n + i];
      }
    b.upload(tmp, st);
    s.x.upload(tx, st);
  }
  cudaEvent_t e0, e1;
  CHRONOS_CUDA(cudaEventCreate(&e0));
  CHRONOS_CUDA(cudaEventCreate(&e1));
  CHRONOS_CUDA(cudaEventRecord(e0, st));
  const DMat &A = h.levels[0].A;
  spmm<double, double, double, double, K, MODE_RESID, false>(st, A, A.v64.get(), s.x.get(), b.get(),
                                                             s.res.get(), 1.0);
  const int nb = std::max(1, std::min(num_sms() * 8, (int)ceil_div((int64_t)n * K, 256)));
  k_bnorm2<K><<<nb, 256, 0, st>>>(n, b.get(), s.part.get(), s.tickets.get() + 3, b2.get());
  CHRONOS_CHECK_LAUNCH();
  k_bnorm2<K><<<nb, 256, 0, st>>>(n, s.res.get(), s.part.get(), s.tickets.get() + 3, r2.get());
  CHRONOS_CHECK_LAUNCH();
  k_bpcg_init<K><<<1, 1, 0, st>>>(s.sc.get(), b2.get(), r2.get(), tol, (double)itmax);
  CHRONOS_CHECK_LAUNCH();
  if (itmax > 0 && !h.prm.use_graph) {
    // one iteration per graph launch from a host loop (profilers cannot see
    // the kernel nodes of a graph holding a conditional node); same kernels
    if (!s.exec) {
      CHRONOS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      try {
        capture_block_iteration<K>(h, s, 0, 0);
      } catch (...) {
        cudaGraph_t dummy;
        cudaStreamEndCapture(st, &dummy);
        throw;
      }
      CHRONOS_CUDA(cudaStreamEndCapture(st, &s.graph));
      CHRONOS_CUDA(cudaGraphInstantiate(&s.exec, s.graph, 0));
    }
    double act_h[K];
    for (int k = 0; k < itmax; ++k) {
      CHRONOS_CUDA(cudaMemcpyAsync(act_h, s.sc.get() + bs_off(BS_ACTIVE, K), sizeof(act_h),
                                   cudaMemcpyDeviceToHost, st));
      CHRONOS_CUDA(cudaStreamSynchronize(st));
      bool any = false;
      for (int j = 0; j < K; ++j) any |= act_h[j] != 0.0;
      if (!any) break;
      CHRONOS_CUDA(cudaGraphLaunch(s.exec, st));
    }
  } else if (itmax > 0) {
    if (!s.exec) {
      CHRONOS_CUDA(cudaGraphCreate(&s.graph, 0));
      cudaGraphConditionalHandle handle;
      CHRONOS_CUDA(cudaGraphConditionalHandleCreate(&handle, s.graph, 1, cudaGraphCondAssignDefault));
      cudaGraphNodeParams np{};
      np.type = cudaGraphNodeTypeConditional;
      np.conditional.handle = handle;
      np.conditional.type = cudaGraphCondTypeWhile;
      np.conditional.size = 1;
      cudaGraphNode_t node;
      CHRONOS_CUDA(cudaGraphAddNode(&node, s.graph, nullptr, 0, &np));
      cudaGraph_t body = np.conditional.phGraph_out[0];
      CHRONOS_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0,
                                                 cudaStreamCaptureModeThreadLocal));
      try {
        capture_block_iteration<K>(h, s, handle, 1);
      } catch (...) {
        cudaGraph_t dummy;
        cudaStreamEndCapture(st, &dummy);
        throw;
      }
      CHRONOS_CUDA(cudaStreamEndCapture(st, &body));
      CHRONOS_CUDA(cudaGraphInstantiate(&s.exec, s.graph, 0));
    }
    // the while loop runs its body once before testing: skip it when no
    // column is active (all b = 0)
    double act_h[K];
    CHRONOS_CUDA(cudaMemcpyAsync(act_h, s.sc.get() + bs_off(BS_ACTIVE, K), sizeof(act_h),
                                 cudaMemcpyDeviceToHost, st));
    CHRONOS_CUDA(cudaStreamSynchronize(st));
    bool any = false;
    for (int j = 0; j < K; ++j) any |= act_h[j] != 0.0;
    if (any) CHRONOS_CUDA(cudaGraphLaunch(s.exec, st));
  }
  k_zero_null_columns<K><<<nb, 256, 0, st>>>(n, s.x.get(), s.sc.get());
  CHRONOS_CHECK_LAUNCH();
  CHRONOS_CUDA(cudaEventRecord(e1, st));
  std::vector<double> sc_h((size_t)BS_COUNT * K + 8), xr(m0);
  s.sc.download(sc_h.data(), sc_h.size(), st);
  s.x.download(xr.data(), m0, st);
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  float ms = 0.f;
  CHRONOS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (seconds) *seconds = ms * 1e-3;
  for (int j = 0; j < K; ++j) {
    for (int i = 0; i < n; ++i) X_h[(size_t)j * n + i] = xr[(size_t)i * K + j];
    iters[j] = (int)(sc_h[bs_off(BS_ITER, K) + j] + 0.5);
    const double r = sc_h[bs_off(BS_RESITER, K) + j];
    flags[j] = (sc_h[bs_off(BS_BNORM, K) + j] == 0.0) ? 0
               : (r > tol || !std::isfinite(r) || sc_h[bs_off(BS_FLAG, K) + j] != 0.0) ? 1 : 0;
  }
}

void Hier::pcg_block(int nrhs, const double *B_h, double *X_h, int itmax, double tol,
                     int *iters, int *flags, double *seconds) {
  CHRONOS_REQUIRE(nrhs >= 1 && nrhs <= 16, CHRONOS_EINVAL, "block solve: 1 <= nrhs <= 16");
  const int n = levels[0].n;
  int K = 1;
  while (K < nrhs) K <<= 1;
  if (K < 2) K = 2;
  // pad to K columns with zero right-hand sides (they stay at x = 0)
  std::vector<double> B((size_t)n * K, 0.0), X((size_t)n * K, 0.0);
  std::copy(B_h, B_h + (size_t)n * nrhs, B.begin());
  std::copy(X_h, X_h + (size_t)n * nrhs, X.begin());
  std::vector<int> it(K), fl(K);
  switch (K) {
    case 2: block_solve<2>(*this, B.data(), X.data(), itmax, tol, it.data(), fl.data(), seconds); break;
    case 4: block_solve<4>(*this, B.data(), X.data(), itmax, tol, it.data(), fl.data(), seconds); break;
    case 8: block_solve<8>(*this, B.data(), X.data(), itmax, tol, it.data(), fl.data(), seconds); break;
    default: block_solve<16>(*this, B.data(), X.data(), itmax, tol, it.data(), fl.data(), seconds); break;
  }
  std::copy(X.begin(), X.begin() + (size_t)n * nrhs, X_h);
  std::copy(it.begin(), it.begin() + nrhs, iters);
  std::copy(fl.begin(), fl.begin() + nrhs, flags);
}

}  // namespace chronos
