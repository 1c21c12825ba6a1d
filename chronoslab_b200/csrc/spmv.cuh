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

#include "common.cuh"

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

struct StoreScalar {
  double *dst;
  __device__ void operator()(const double *t) const { *dst = t[0]; }
};

template <typename VT, typename XT, typename ZT, typename YT, int L, int MODE, bool DOT>
__global__ void __launch_bounds__(kApplyThreads)
k_csr_apply(int n, const int *__restrict__ rp, const int *__restrict__ ci,
            const VT *__restrict__ v, const XT *__restrict__ x, const ZT *z, YT *y, VT alpha,
            const double *__restrict__ dw, double *part, unsigned *ticket, double *dot_out) {
  constexpr int R = 32 / L;                       // rows per warp step
  const int lane = threadIdx.x & 31;
  const int g = lane / L, gl = lane & (L - 1);
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double dacc = 0.0;
  for (int base = warp * R; base < n; base += nwarps * R) {
    const int row = base + g;
    VT sum = VT(0);
    if (row < n) {
      const int s = __ldg(rp + row), e = __ldg(rp + row + 1);
      int k = s + gl;
      // two independent accumulators keep more loads in flight
      VT s2 = VT(0);
      for (; k + L < e; k += 2 * L) {
        sum += __ldg(v + k) * (VT)__ldg(x + __ldg(ci + k));
        s2 += __ldg(v + k + L) * (VT)__ldg(x + __ldg(ci + k + L));
      }
      if (k < e) sum += __ldg(v + k) * (VT)__ldg(x + __ldg(ci + k));
      sum += s2;
    }
    sum = group_sum<L>(sum);
    if (row < n && gl == 0) {
      VT r;
      if (MODE == MODE_PLAIN) r = sum;
      else if (MODE == MODE_SCALE) r = alpha * sum;
      else if (MODE == MODE_RESID) r = (VT)z[row] - sum;
      else r = (VT)z[row] + alpha * sum;
      const YT out = (YT)r;
      y[row] = out;
      if (DOT) dacc += (double)out * dw[row];
    }
  }
  if (DOT) {
    double vals[1] = {dacc};
    grid_reduce<1>(vals, part, ticket, StoreScalar{dot_out});
  }
}

// Launch helper: persistent grid of blocks_per_sm * #SMs blocks (or fewer
// when the matrix is small).
template <typename VT, typename XT, typename ZT, typename YT, int MODE, bool DOT>
void csr_apply(cudaStream_t st, int L, int n, const int *rp, const int *ci, const VT *v,
               const XT *x, const ZT *z, YT *y, VT alpha, const double *dw = nullptr,
               double *part = nullptr, unsigned *ticket = nullptr, double *dot_out = nullptr,
               int max_blocks = 0) {
  if (n <= 0) return;
  const int rows_per_block = kApplyThreads / L;
  int blocks = (int)ceil_div(n, rows_per_block);
  const int cap = max_blocks > 0 ? max_blocks : num_sms() * 8;
  if (blocks > cap) blocks = cap;
#define CHRONOS_APPLY_CASE(LL)                                                            \
  case LL:                                                                                \
    k_csr_apply<VT, XT, ZT, YT, LL, MODE, DOT><<<blocks, kApplyThreads, 0, st>>>(         \
        n, rp, ci, v, x, z, y, alpha, dw, part, ticket, dot_out);                         \
    break;
  switch (L) {
    CHRONOS_APPLY_CASE(2)
    CHRONOS_APPLY_CASE(4)
    CHRONOS_APPLY_CASE(8)
    CHRONOS_APPLY_CASE(16)
    CHRONOS_APPLY_CASE(32)
    default:
      throw Error(CHRONOS_EINVAL, "csr_apply: lanes per row must be 2,4,8,16 or 32");
  }
#undef CHRONOS_APPLY_CASE
  CHRONOS_CHECK_LAUNCH();
}

}  // namespace chronos
