// CSR apply kernels of the V-cycle and the outer PCG (sm_100a).
//
// Row-group CSR: L consecutive lanes (L in {2,4,8,16,32}) share one row, load
// its values and column indices with coalesced accesses, gather x, and reduce
// with warp shuffles.  Grids are persistent (a multiple of the SM count);
// every warp walks rows in warp-uniform steps so the shuffles always see full
// warps.  The row result goes through one of the fused epilogues
//   PLAIN  y = A x             SCALE  y = alpha A x
//   RESID  y = z - A x         AXPY   y = z + alpha A x
// and, optionally, a dot product sum_i y_i w_i reduced deterministically
// (fixed-order block partials, finished by the last block to arrive).
//
// Storage and accumulation precision follow the matrix value type VT (float
// for the FP32 hierarchy, double for the FP64 one); the vector types XT (x),
// ZT (z) and YT (y) may differ from VT, which fuses the FP64<->FP32
// conversions at the ends of the V-cycle into its first and last kernels.
#pragma once

#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "internal.h"

namespace chronos {

enum ApplyMode { MODE_PLAIN = 0, MODE_SCALE = 1, MODE_RESID = 2, MODE_AXPY = 3 };

constexpr int kApplyThreads = 256;

// Deterministic K-value reduction across the grid.  Each block writes its
// partials to part[blk*K + j]; the last block to finish (atomic ticket) sums
// them in block order and hands the K totals to fin(totals) in thread 0.
template <int K, typename Fin>
__device__ __forceinline__ void grid_reduce(double (&v)[K], double *part, unsigned *ticket,
                                            Fin fin) {
  __shared__ double red[K][32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    double s = warp_sum(v[j]);
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
    unsigned t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double acc[K];
#pragma unroll
  for (int j = 0; j < K; ++j) acc[j] = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] += __ldcg(&part[(size_t)b * K + j]);
#pragma unroll
  for (int j = 0; j < K; ++j) {
    double s = warp_sum(acc[j]);
    if (lane == 0) red[j][wid] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += red[j][w];
      tot[j] = s;
    }
    *ticket = 0u;
    fin(tot);
  }
}

// Deterministic grid reduction of NQ quantities of K columns (block
// right-hand sides).  Lane l owns columns (l % (K/VEC))*VEC .. +VEC-1 and
// v[q][e] is its partial of quantity q for the e-th of them; lanes owning the
// same columns are combined by shuffles, warps through shared memory, blocks
// by the last block to arrive (fixed orders throughout).  fin receives the
// NQ*K totals, quantity-major (t[q*K + j]).  K*NQ <= 32, K/VEC <= 32.
template <int K, int VEC, int NQ, typename Fin>
__device__ __forceinline__ void grid_reduce_cols(double (&v)[NQ][VEC], double *part,
                                                 unsigned *ticket, Fin fin) {
  constexpr int LPR = K / VEC;       // lanes per column set
  constexpr int NC = NQ * K;
  static_assert(NC <= 32 && LPR <= 32, "grid_reduce_cols: K*NQ <= 32");
  __shared__ double red[32][NC];
  __shared__ double tot[NC];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q)
#pragma unroll
    for (int e = 0; e < VEC; ++e)
#pragma unroll
      for (int o = LPR; o < 32; o <<= 1) v[q][e] += __shfl_xor_sync(0xffffffffu, v[q][e], o);
  if (lane < LPR)
#pragma unroll
    for (int q = 0; q < NQ; ++q)
#pragma unroll
      for (int e = 0; e < VEC; ++e) red[wid][q * K + lane * VEC + e] = v[q][e];
  __syncthreads();
  if ((int)threadIdx.x < NC) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += red[w][threadIdx.x];
    part[(size_t)blockIdx.x * NC + threadIdx.x] = s;
    __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  const int stripes = min((int)blockDim.x / NC, 32);
  const int c = threadIdx.x % NC, sidx = threadIdx.x / NC;
  if (sidx < stripes) {
    double acc = 0.0;
    for (int b = sidx; b < (int)gridDim.x; b += stripes) acc += __ldcg(&part[(size_t)b * NC + c]);
    red[sidx][c] = acc;
  }
  __syncthreads();
  if ((int)threadIdx.x < NC) {
    double s2 = 0.0;
    for (int w = 0; w < stripes; ++w) s2 += red[w][threadIdx.x];
    tot[threadIdx.x] = s2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *ticket = 0u;
    fin(tot);
  }
}

struct StoreScalar {
  double *dst;
  __device__ void operator()(const double *t) const { *dst = t[0]; }
};

template <typename VT, int MODE, typename ZT>
__device__ __forceinline__ VT apply_epilogue(VT sum, VT alpha, const ZT *z, int row) {
  if (MODE == MODE_PLAIN) return sum;
  if (MODE == MODE_SCALE) return alpha * sum;
  if (MODE == MODE_RESID) return (VT)z[row] - sum;
  return (VT)z[row] + alpha * sum;
}

template <typename VT, typename XT, typename ZT, typename YT, int L, int MODE, bool DOT>
__global__ void __launch_bounds__(kApplyThreads)
k_csr_apply(int n, const int *__restrict__ rp, const int *__restrict__ ci,
            const VT *__restrict__ v, const XT *__restrict__ x, const ZT *z, YT *y, VT alpha,
            const double *__restrict__ dw, double *part, unsigned *ticket, double *dot_out) {
  // Each lane group holds two rows in flight (rows base+g and base+R+g) so
  // short rows, whose cost is the dependent chain row pointer -> column ->
  // x gather, overlap two chains per thread.
  constexpr int R = 32 / L;                       // groups per warp
  const int lane = threadIdx.x & 31;
  const int g = lane / L, gl = lane & (L - 1);
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double dacc = 0.0;
  for (int base = warp * 2 * R; base < n; base += nwarps * 2 * R) {
    const int r0 = base + g, r1 = base + R + g;
    int k0 = 0, e0 = 0, k1 = 0, e1 = 0;
    if (r0 < n) { k0 = __ldg(rp + r0) + gl; e0 = __ldg(rp + r0 + 1); }
    if (r1 < n) { k1 = __ldg(rp + r1) + gl; e1 = __ldg(rp + r1 + 1); }
    VT a0 = VT(0), a1 = VT(0);
    while (k0 < e0 || k1 < e1) {
      if (k0 < e0) { a0 += __ldg(v + k0) * (VT)__ldg(x + __ldg(ci + k0)); k0 += L; }
      if (k1 < e1) { a1 += __ldg(v + k1) * (VT)__ldg(x + __ldg(ci + k1)); k1 += L; }
    }
    a0 = group_sum<L>(a0);
    a1 = group_sum<L>(a1);
    if (gl == 0) {
      if (r0 < n) {
        const YT out = (YT)apply_epilogue<VT, MODE>(a0, alpha, z, r0);
        y[r0] = out;
        if (DOT) dacc += (double)out * dw[r0];
      }
      if (r1 < n) {
        const YT out = (YT)apply_epilogue<VT, MODE>(a1, alpha, z, r1);
        y[r1] = out;
        if (DOT) dacc += (double)out * dw[r1];
      }
    }
  }
  if (DOT) {
    double vals[1] = {dacc};
    grid_reduce<1>(vals, part, ticket, StoreScalar{dot_out});
  }
}

// Sliced 3x3 block apply (SELL-32 over 3x3 blocks) for operators assembled
// from 3x3 node blocks (3 DOF per node).  Block rows are grouped in chunks of
// 32; chunk c is padded to its longest block row w_c and stored slot-major:
// slot j of the chunk's 32 rows is contiguous, so thread `lane` of the warp
// owning the chunk reads block (row 32c+lane, slot j) with every load of the
// warp coalesced.  Values are plane-major (V[e * nslots + k], e = 3*r + c):
// nine coalesced 4- or 8-byte loads per block, one 4-byte column index per
// nine values (0.44 index bytes per entry), no cross-lane reduction; padding
// slots hold zeros and column 0.  The three row results go through the same
// fused epilogues as the CSR kernel.
// T threads share a block row (T = 1, 2, 4): a chunk holds C = 32/T block
// rows and slot j of row l sits at off_c + (j/T)*32 + (j%T)*C + l, so lane
// p*C + l walks slots j = p, p+T, ... with the same coalesced warp loads, and
// the T partial sums meet through warp shuffles.  chw holds w_c / T.
template <int T, typename VT>
__device__ __forceinline__ VT slot_sum(VT v) {
  constexpr int C = 32 / T;
#pragma unroll
  for (int o = C; o < 32; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename VT, typename XT, typename ZT, typename YT, int T, int MODE, bool DOT>
__global__ void __launch_bounds__(kApplyThreads)
k_sell3_apply(int nb, int nchunk, const int *__restrict__ choff, const int *__restrict__ chw,
              const int *__restrict__ sci, const VT *__restrict__ V, int64_t nslots,
              const XT *__restrict__ x, const ZT *z, YT *y, VT alpha,
              const double *__restrict__ dw, double *part, unsigned *ticket, double *dot_out) {
  pdl_begin();
  constexpr int C = 32 / T;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double dacc = 0.0;
  for (int c = warp; c < nchunk; c += nwarps) {
    const int off = __ldg(choff + c) + lane, w = __ldg(chw + c);
    VT s0 = VT(0), s1 = VT(0), s2 = VT(0);
#pragma unroll 2
    for (int j = 0; j < w; ++j) {
      const int k = off + 32 * j;
      const int col = 3 * __ldg(sci + k);
      const VT xa = (VT)__ldg(x + col), xb = (VT)__ldg(x + col + 1), xc = (VT)__ldg(x + col + 2);
      s0 += __ldg(V + k) * xa + __ldg(V + nslots + k) * xb + __ldg(V + 2 * nslots + k) * xc;
      s1 += __ldg(V + 3 * nslots + k) * xa + __ldg(V + 4 * nslots + k) * xb +
            __ldg(V + 5 * nslots + k) * xc;
      s2 += __ldg(V + 6 * nslots + k) * xa + __ldg(V + 7 * nslots + k) * xb +
            __ldg(V + 8 * nslots + k) * xc;
    }
    if (T > 1) {
      s0 = slot_sum<T>(s0);
      s1 = slot_sum<T>(s1);
      s2 = slot_sum<T>(s2);
    }
    const int br = C * c + (lane & (C - 1));
    if (lane < C && br < nb) {
      const VT s[3] = {s0, s1, s2};
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const int row = 3 * br + r;
        const YT out = (YT)apply_epilogue<VT, MODE>(s[r], alpha, z, row);
        y[row] = out;
        if (DOT) dacc += (double)out * dw[row];
      }
    }
  }
  if (DOT) {
    double vals[1] = {dacc};
    grid_reduce<1>(vals, part, ticket, StoreScalar{dot_out});
  }
}

template <typename VT, typename XT, typename ZT, typename YT, int MODE, bool DOT>
void sell3_apply(cudaStream_t st, int T, int nb, int nchunk, const int *choff, const int *chw,
                 const int *sci, const VT *V, int64_t nslots, const XT *x, const ZT *z, YT *y,
                 VT alpha, const double *dw = nullptr, double *part = nullptr,
                 unsigned *ticket = nullptr, double *dot_out = nullptr) {
  if (nb <= 0) return;
  int blocks = (int)ceil_div(nchunk, kApplyThreads / 32);
  const int cap = num_sms() * 8;
  if (blocks > cap) blocks = cap;
#define CHRONOS_SELL_CASE(TT)                                                                  \
  case TT:                                                                                     \
    launch_pdl(k_sell3_apply<VT, XT, ZT, YT, TT, MODE, DOT>, blocks, kApplyThreads, st, nb,    \
               nchunk, choff, chw, sci, V, nslots, x, z, y, alpha, dw, part, ticket, dot_out); \
    break;
  switch (T) {
    CHRONOS_SELL_CASE(1)
    CHRONOS_SELL_CASE(2)
    CHRONOS_SELL_CASE(4)
    default:
      throw Error(CHRONOS_EINVAL, "sell3_apply: threads per block row must be 1, 2 or 4");
  }
#undef CHRONOS_SELL_CASE
  CHRONOS_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// Hybrid CSR apply of the V-cycle operators (G, G', P, P' and the CSR levels
// of A).  Differences from k_csr_apply:
//  * each lane issues the loads of up to kRowUnroll entries (values, column
//    indices, then the x gathers) before it uses any of them, so the
//    dependent chain row pointer -> column -> x is paid once per kRowUnroll
//    entries instead of once per entry;
//  * rows longer than lthresh (listed in longrows) are skipped by the
//    L-lane groups and applied by whole warps in a second range of blocks of
//    the same launch, so a few long rows (the transposed FSAI factor's
//    popular columns) no longer serialise a short-row warp;
//  * optional 16-bit column offsets from a per-row base.
// Each row's entries are summed in a fixed order (lane-strided partial sums,
// then a shuffle tree), so results are deterministic.
constexpr int kRowUnroll = 4;

// Partial sum of lane entries k, k+L, ... < e of one row, accumulated in AT.
template <typename AT, typename VT, typename XT, int L, bool I16>
__device__ __forceinline__ AT csr_row_dot(int k, int e, int cb, const int *__restrict__ ci,
                                          const uint16_t *__restrict__ c16,
                                          const VT *__restrict__ v, const XT *__restrict__ x) {
  constexpr int U = kRowUnroll;
  AT acc = AT(0);
  for (; k + (U - 1) * L < e; k += U * L) {
    int c[U];
    VT a[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      c[u] = I16 ? cb + (int)__ldg(c16 + k + u * L) : __ldg(ci + k + u * L);
      a[u] = __ldg(v + k + u * L);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) acc += (AT)a[u] * (AT)__ldg(x + c[u]);
  }
  // the fewer than U entries left to this lane
  int c[U - 1];
  VT a[U - 1];
#pragma unroll
  for (int u = 0; u < U - 1; ++u) {
    const int kk = k + u * L;
    c[u] = -1;
    a[u] = VT(0);
    if (kk < e) {
      c[u] = I16 ? cb + (int)__ldg(c16 + kk) : __ldg(ci + kk);
      a[u] = __ldg(v + kk);
    }
  }
#pragma unroll
  for (int u = 0; u < U - 1; ++u)
    if (c[u] >= 0) acc += (AT)a[u] * (AT)__ldg(x + c[u]);
  return acc;
}

template <typename VT, typename XT, typename ZT, typename YT, int L, int MODE, bool DOT, bool I16>
__global__ void __launch_bounds__(kApplyThreads)
k_csrh_apply(int n, const int *__restrict__ rp, const int *__restrict__ ci,
             const int *__restrict__ cbase, const uint16_t *__restrict__ c16,
             const VT *__restrict__ v, const XT *__restrict__ x, const ZT *z, YT *y, VT alpha,
             int short_blocks, int lthresh, const int *__restrict__ longrows, int nlong,
             const double *__restrict__ dw, double *part, unsigned *ticket, double *dot_out) {
  pdl_begin();
  const int lane = threadIdx.x & 31;
  double dacc = 0.0;
  if ((int)blockIdx.x < short_blocks) {
    constexpr int R = 32 / L;                      // row groups per warp
    const int g = lane / L, gl = lane & (L - 1);
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (short_blocks * blockDim.x) >> 5;
    for (int base = warp * R; base < n; base += nwarps * R) {   // warp-uniform trip count
      const int row = base + g;
      VT a = VT(0);
      bool live = false;
      if (row < n) {
        const int s = __ldg(rp + row), e = __ldg(rp + row + 1);
        if (e - s <= lthresh) {
          live = true;
          a = csr_row_dot<VT, VT, XT, L, I16>(s + gl, e, I16 ? __ldg(cbase + row) : 0, ci, c16, v,
                                              x);
        }
      }
      a = group_sum<L>(a);
      if (live && gl == 0) {
        const YT out = (YT)apply_epilogue<VT, MODE>(a, alpha, z, row);
        y[row] = out;
        if (DOT) dacc += (double)out * dw[row];
      }
    }
  } else {
    const int warp = ((blockIdx.x - short_blocks) * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = ((gridDim.x - short_blocks) * blockDim.x) >> 5;
    for (int i = warp; i < nlong; i += nwarps) {
      const int row = __ldg(longrows + i);
      const int s = __ldg(rp + row), e = __ldg(rp + row + 1);
      VT a = csr_row_dot<VT, VT, XT, 32, I16>(s + lane, e, I16 ? __ldg(cbase + row) : 0, ci, c16,
                                              v, x);
      a = warp_sum(a);
      if (lane == 0) {
        const YT out = (YT)apply_epilogue<VT, MODE>(a, alpha, z, row);
        y[row] = out;
        if (DOT) dacc += (double)out * dw[row];
      }
    }
  }
  if (DOT) {
    double vals[1] = {dacc};
    grid_reduce<1>(vals, part, ticket, StoreScalar{dot_out});
  }
}

// Sliced ELL apply (see DMat::use_sell): a warp per chunk of 32 rows, lane l
// owns chunk row l and walks its slots with coalesced 128-byte (values) and
// 64-byte (16-bit offsets) warp loads, four slots' loads in flight before
// the gathers; each row's entries are summed in CSR order.  Rows longer than
// the threshold are applied by whole warps from the CSR arrays in a second
// range of blocks.
template <typename VT, typename XT, typename ZT, typename YT, int MODE, bool DOT, bool I16>
__global__ void __launch_bounds__(kApplyThreads)
k_sell_apply(int nchunk, const int *__restrict__ choff, const int *__restrict__ chw,
             const int *__restrict__ cbase, const int *__restrict__ perm,
             const int *__restrict__ sci, const uint16_t *__restrict__ sc16,
             const VT *__restrict__ sv, const int *__restrict__ rp, const int *__restrict__ ci,
             const VT *__restrict__ v, const XT *__restrict__ x, const ZT *z, YT *y, VT alpha,
             int short_blocks, const int *__restrict__ longrows, int nlong,
             const double *__restrict__ dw, double *part, unsigned *ticket, double *dot_out) {
  pdl_begin();
  const int lane = threadIdx.x & 31;
  double dacc = 0.0;
  if ((int)blockIdx.x < short_blocks) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (short_blocks * blockDim.x) >> 5;
    for (int c = warp; c < nchunk; c += nwarps) {
      const int off = __ldg(choff + c) + lane, w = __ldg(chw + c);
      const int cb = I16 ? __ldg(cbase + c) : 0;
      const int row = __ldg(perm + 32 * c + lane);
      VT acc = VT(0);
      int j = 0;
      for (; j + 3 < w; j += 4) {
        int col[4];
        VT a[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int k = off + 32 * (j + u);
          col[u] = I16 ? cb + (int)__ldg(sc16 + k) : __ldg(sci + k);
          a[u] = __ldg(sv + k);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) acc += a[u] * (VT)__ldg(x + col[u]);
      }
      {
        int col[3];
        VT a[3];
#pragma unroll
        for (int u = 0; u < 3; ++u) {
          col[u] = -1;
          a[u] = VT(0);
          if (j + u < w) {
            const int k = off + 32 * (j + u);
            col[u] = I16 ? cb + (int)__ldg(sc16 + k) : __ldg(sci + k);
            a[u] = __ldg(sv + k);
          }
        }
#pragma unroll
        for (int u = 0; u < 3; ++u)
          if (col[u] >= 0) acc += a[u] * (VT)__ldg(x + col[u]);
      }
      if (row >= 0) {
        const YT out = (YT)apply_epilogue<VT, MODE>(acc, alpha, z, row);
        y[row] = out;
        if (DOT) dacc += (double)out * dw[row];
      }
    }
  } else {
    const int warp = ((blockIdx.x - short_blocks) * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = ((gridDim.x - short_blocks) * blockDim.x) >> 5;
    for (int i = warp; i < nlong; i += nwarps) {
      const int row = __ldg(longrows + i);
      const int s = __ldg(rp + row), e = __ldg(rp + row + 1);
      VT a = csr_row_dot<VT, VT, XT, 32, false>(s + lane, e, 0, ci, nullptr, v, x);
      a = warp_sum(a);
      if (lane == 0) {
        const YT out = (YT)apply_epilogue<VT, MODE>(a, alpha, z, row);
        y[row] = out;
        if (DOT) dacc += (double)out * dw[row];
      }
    }
  }
  if (DOT) {
    double vals[1] = {dacc};
    grid_reduce<1>(vals, part, ticket, StoreScalar{dot_out});
  }
}

template <typename VT> inline const VT *sell_vals(const DMat &m);
template <> inline const float *sell_vals<float>(const DMat &m) { return m.s_v32.get(); }
template <> inline const double *sell_vals<double>(const DMat &m) { return m.s_v64.get(); }
template <typename VT> inline const VT *csr_vals(const DMat &m);
template <> inline const float *csr_vals<float>(const DMat &m) { return m.v32.get(); }
template <> inline const double *csr_vals<double>(const DMat &m) { return m.v64.get(); }

// Long-row threshold for `lanes`-lane groups: rows longer than 32 entries per
// lane go to whole warps.
inline int long_row_threshold(int lanes) { return lanes >= 32 ? 0x7fffffff : 32 * lanes; }

// Blocks of a grid of `cap` given to the long rows: their share of the
// entries (at least one warp per 8 long rows' worth, at most half the grid,
// never more than one warp per long row).
inline int long_blocks(const DMat &M, int cap) {
  if (M.nlong <= 0) return 0;
  const int wpb = kApplyThreads / 32;
  const double share = M.nnz > 0 ? (double)M.nnz_long / (double)M.nnz : 0.0;
  int lb = (int)std::ceil(share * cap);
  lb = std::max(lb, (int)std::min<int64_t>(ceil_div(M.nlong, 8 * wpb), cap / 4));
  lb = std::min(lb, cap / 2);
  lb = std::min<int64_t>(lb, ceil_div(M.nlong, wpb));
  return std::max(lb, 1);
}

// Apply of a device matrix through k_csrh_apply with its tuned lanes, long-row
// list and index width.  At most num_sms()*8 blocks (the reduction partial
// buffers hold 2048 per slot).
template <typename VT, typename XT, typename ZT, typename YT, int MODE, bool DOT>
void mat_apply(cudaStream_t st, const DMat &M, const VT *v, const XT *x, const ZT *z, YT *y,
               VT alpha, const double *dw = nullptr, double *part = nullptr,
               unsigned *ticket = nullptr, double *dot_out = nullptr) {
  const int n = M.nrows;
  if (n <= 0) return;
  const int L = M.lanes;
  const int cap = num_sms() * 8;
  const int wpb = kApplyThreads / 32;
  const int lb = long_blocks(M, cap);
  if (M.use_sell) {
    const int sb = (int)std::min<int64_t>(ceil_div(M.s_nchunk, wpb), cap - lb);
    const VT *sv = sell_vals<VT>(M), *cv = csr_vals<VT>(M);
    if (M.sell16)
      launch_pdl(k_sell_apply<VT, XT, ZT, YT, MODE, DOT, true>, sb + lb, kApplyThreads, st,
                 M.s_nchunk, M.s_choff.get(), M.s_chw.get(), M.s_cbase.get(), M.s_perm.get(),
                 M.s_ci.get(), M.s_c16.get(), sv, M.rp.get(), M.ci.get(), cv, x, z, y, alpha, sb,
                 M.longrows.get(), M.nlong, dw, part, ticket, dot_out);
    else
      launch_pdl(k_sell_apply<VT, XT, ZT, YT, MODE, DOT, false>, sb + lb, kApplyThreads, st,
                 M.s_nchunk, M.s_choff.get(), M.s_chw.get(), M.s_cbase.get(), M.s_perm.get(),
                 M.s_ci.get(), M.s_c16.get(), sv, M.rp.get(), M.ci.get(), cv, x, z, y, alpha, sb,
                 M.longrows.get(), M.nlong, dw, part, ticket, dot_out);
    return;
  }
  int sb = (int)std::min<int64_t>(ceil_div(n, kApplyThreads / L), cap - lb);
  const int grid = sb + lb;
#define CHRONOS_H_CASE(LL)                                                                    \
  case LL:                                                                                    \
    if (M.idx16)                                                                              \
      launch_pdl(k_csrh_apply<VT, XT, ZT, YT, LL, MODE, DOT, true>, grid, kApplyThreads, st, \
                 n, M.rp.get(), M.ci.get(), M.cbase.get(), M.c16.get(), v, x, z, y, alpha, sb, \
                 M.lthresh, M.longrows.get(), M.nlong, dw, part, ticket, dot_out);             \
    else                                                                                      \
      launch_pdl(k_csrh_apply<VT, XT, ZT, YT, LL, MODE, DOT, false>, grid, kApplyThreads, st,\
                 n, M.rp.get(), M.ci.get(), M.cbase.get(), M.c16.get(), v, x, z, y, alpha, sb, \
                 M.lthresh, M.longrows.get(), M.nlong, dw, part, ticket, dot_out);             \
    break;
  switch (L) {
    CHRONOS_H_CASE(1)
    CHRONOS_H_CASE(2)
    CHRONOS_H_CASE(4)
    CHRONOS_H_CASE(8)
    CHRONOS_H_CASE(16)
    CHRONOS_H_CASE(32)
    default:
      throw Error(CHRONOS_EINVAL, "mat_apply: lanes per row must be 1,2,4,8,16 or 32");
  }
#undef CHRONOS_H_CASE
  CHRONOS_CHECK_LAUNCH();
}

// Launch helper: persistent grid of blocks_per_sm * #SMs blocks (or fewer
// when the matrix is small).
template <typename VT, typename XT, typename ZT, typename YT, int MODE, bool DOT>
void csr_apply(cudaStream_t st, int L, int n, const int *rp, const int *ci, const VT *v,
               const XT *x, const ZT *z, YT *y, VT alpha, const double *dw = nullptr,
               double *part = nullptr, unsigned *ticket = nullptr, double *dot_out = nullptr,
               int max_blocks = 0) {
  if (n <= 0) return;
  const int rows_per_block = 2 * kApplyThreads / L;
  int blocks = (int)ceil_div(n, rows_per_block);
  const int cap = max_blocks > 0 ? max_blocks : num_sms() * 8;
  if (blocks > cap) blocks = cap;
#define CHRONOS_APPLY_CASE(LL)                                                            \
  case LL:                                                                                \
    k_csr_apply<VT, XT, ZT, YT, LL, MODE, DOT><<<blocks, kApplyThreads, 0, st>>>(         \
        n, rp, ci, v, x, z, y, alpha, dw, part, ticket, dot_out);                         \
    break;
  switch (L) {
    CHRONOS_APPLY_CASE(1)
    CHRONOS_APPLY_CASE(2)
    CHRONOS_APPLY_CASE(4)
    CHRONOS_APPLY_CASE(8)
    CHRONOS_APPLY_CASE(16)
    CHRONOS_APPLY_CASE(32)
    default:
      throw Error(CHRONOS_EINVAL, "csr_apply: lanes per row must be 1,2,4,8,16 or 32");
  }
#undef CHRONOS_APPLY_CASE
  CHRONOS_CHECK_LAUNCH();
}

}  // namespace chronos
