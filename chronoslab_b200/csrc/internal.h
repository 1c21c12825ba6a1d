// Host-callable launchers shared between the translation units of the
// library.  Device pointers unless named *_h.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

#include "common.cuh"

namespace chronos {

// Device CSR, 0-based, int32 row pointers and columns; values in FP64 and,
// for the FP32 hierarchy, an FP32 copy sharing the pattern.
struct DMat {
  int nrows = 0, ncols = 0;
  int64_t nnz = 0;
  DBuf<int> rp, ci;
  DBuf<double> v64;
  DBuf<float> v32;
  int lanes = 8;            // SpMV lanes per row (autotuned)
  std::vector<int> rp_h;    // host copy of the row pointers (long-row lists)
  // 16-bit column offsets from a per-row base (the row's smallest column),
  // present when every row spans fewer than 65536 columns: 2 index bytes per
  // entry plus 4 per row instead of 4 per entry.
  bool idx16 = false;
  DBuf<int> cbase;
  DBuf<uint16_t> c16;
  // Rows longer than lthresh are applied by whole warps (listed in
  // longrows); the others by groups of `lanes` lanes.
  int lthresh = 0x7fffffff, nlong = 0;
  int64_t nnz_long = 0;     // entries in the long rows
  DBuf<int> longrows;
  // Sliced ELL form for short rows (use_sell; chosen by the autotuner):
  // chunks of 32 rows taken in the order s_perm (row order, the long rows
  // left out; -1 pads the last chunk), slot-major
  // (slot j of chunk row l at s_choff[c] + 32 j + l), chunk widths s_chw;
  // columns as 16-bit offsets from the chunk's smallest column (s_cbase) when
  // every chunk spans fewer than 65536 columns (sell16), else int32 (s_ci);
  // padding slots hold value 0 and offset 0.  Rows longer than lthresh stay
  // on the warp path (longrows).
  bool use_sell = false, sell16 = false;
  int s_nchunk = 0;
  DBuf<int> s_choff, s_chw, s_cbase, s_perm, s_ci;
  DBuf<uint16_t> s_c16;
  DBuf<double> s_v64;
  DBuf<float> s_v32;
  // Optional sliced 3x3 block form of the same matrix (chunks of 32 block
  // rows, slot-major, plane-major values), used when every row triple shares
  // a pattern of whole aligned 3x3 blocks.
  int nb = 0;               // block rows (0: no block form)
  int sell_T = 1;           // threads per block row (1, 2, 4; autotuned)
  int nchunk = 0;
  int64_t nnzb = 0;         // true blocks
  int64_t nslots = 0;       // stored slots (blocks + padding)
  DBuf<int> choff, chw, sci;
  DBuf<double> bv64;
  DBuf<float> bv32;
};

// ---- FSAI numeric (setup_kernels.cu) ------------------------------------------
// G values on the pattern grp/gci (rows: strictly-lower ascending, diagonal
// last).  A: 0-based CSR, sorted rows.  Returns the flags word: bit 0 =
// non-SPD local block or non-positive Schur complement somewhere.
int fsai_numeric_device(int n, const int *arp, const int *aci, const double *av, const int *grp,
                        const int *gci, double *gval, const std::vector<int> &rowlen_h,
                        cudaStream_t st);

// One problem of fsai_numeric_batched: device CSR of A, G's pattern and the
// buffer of G's values; rowlen: the host row lengths of G.
struct FsaiJob {
  int n = 0;
  const int *arp = nullptr, *aci = nullptr;
  const double *av = nullptr;
  const int *grp = nullptr, *gci = nullptr;
  double *gval = nullptr;
  const std::vector<int> *rowlen = nullptr;
};
// The FSAI numeric phase of all jobs at once: one launch per tile size over
// every job's rows, the tile sizes (bucket edges) chosen by timing candidate
// sets on the batch (cached per batch shape).  Returns each job's flags word
// (bit 0: non-SPD local block); chosen_set (may be null) receives the index of
// the set used.  Values are those of fsai_numeric_device, bit for bit.
// force_set >= 0 uses that candidate set instead of the tuned one.
std::vector<int> fsai_numeric_batched(const std::vector<FsaiJob> &jobs, cudaStream_t st,
                                      int *chosen_set = nullptr, int force_set = -1);
int fsai_bucket_set_count();

// ---- Galerkin (setup_kernels.cu) ---------------------------------------------
// C = X * Y (X: m x k, Y: k x ncols), Gustavson accumulation order, exact
// zeros dropped, columns sorted.  Output arrays allocated here.
void spgemm_device(int m, int ncols, const int *xrp, const int *xci, const double *xv,
                   const int *yrp, const int *yci, const double *yv, DBuf<int> &crp,
                   DBuf<int> &cci, DBuf<double> &cv, int64_t *nnz_c, cudaStream_t st);

// ---- dense coarse level (setup_kernels.cu) ----------------------------------
// In-place lower Cholesky of the n x n column-major A (device); returns 0 or
// the 1-based index of the first non-positive pivot.
int dense_cholesky_device(int n, double *A, cudaStream_t st);
// W = A^{-1} = L^{-T} L^{-1} from the lower factor L (column-major).  W is
// symmetric (row- and column-major alike).
void dense_inverse_from_chol(int n, const double *L, double *W, cudaStream_t st);
// x = W b (W FP64 row-major n x n).
template <typename TI, typename TO>
void dense_matvec(int n, const double *W, const TI *b, TO *x, cudaStream_t st);

// ---- vector helpers (setup_kernels.cu) ---------------------------------------
void convert_f64_to_f32(int64_t n, const double *src, float *dst, cudaStream_t st);
// Transpose (ncols x nrows) of a device CSR: its row pointers, columns and
// values as the host transpose orders them (rows of the transpose in
// ascending order of the original row).  Synchronises st.
void csr_transpose_device(int nrows, int ncols, int64_t nnz, const int *rp, const int *ci,
                          const double *v, DBuf<int> &trp, DBuf<int> &tci, DBuf<double> &tv,
                          cudaStream_t st);
// 16-bit column offsets from each row's smallest column (rows without
// entries: base 0), when every row spans fewer than 65536 columns; returns
// false (nothing kept) otherwise.
bool csr_offsets16_device(int nrows, int64_t nnz, const int *rp, const int *ci, DBuf<int> &base,
                          DBuf<uint16_t> &off, cudaStream_t st);
double device_dot(int n, const double *a, const double *b, double *scratch, cudaStream_t st);
void device_axpby(int n, double a, const double *x, double b, double *y, cudaStream_t st);
void device_scale_copy(int n, double a, const double *x, double *y, cudaStream_t st);
// y = d .* x
void device_diag_mul(int n, const double *d, const double *x, double *y, cudaStream_t st);
// grad[k] = -lambda[row(k)] * u[col(k)]
void adjoint_scatter(int n, const int *rp, const int *ci, const double *lambda, const double *u,
                     double *grad, cudaStream_t st);

}  // namespace chronos
