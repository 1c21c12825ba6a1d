// Host-side setup code of the solve path: the parts the reference keeps on the
// host (coarsening, C/F splitting, BAMG prolongation, the adaptive FSAI pattern
// search) restated in C++ with OpenMP.  All CSR here is 0-based with int32
// columns and sorted rows unless stated.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../../include/chronos_b200.h"

namespace chronos {

struct HostCSR {
  int nrows = 0, ncols = 0;
  std::vector<int64_t> rp;   // nrows + 1
  std::vector<int> ci;
  std::vector<double> v;
  int64_t nnz() const { return rp.empty() ? 0 : rp.back(); }
};

// MT19937 (Matsumoto & Nishimura 1998): init_genrand seeding and the 53-bit
// genrand_res53 doubles that MATLAB's rand draws after rng(0) (seed 5489).
class MT19937 {
 public:
  explicit MT19937(uint32_t seed = 5489u) { seed_(seed); }
  uint32_t next_u32();
  double next_res53() {
    uint32_t a = next_u32() >> 5, b = next_u32() >> 6;
    return (a * 67108864.0 + b) * (1.0 / 9007199254740992.0);
  }

 private:
  void seed_(uint32_t s);
  uint32_t mt_[624];
  int mti_ = 625;
};

// ---- coarsening (coarsen.m) ------------------------------------------------
// Strength-of-connection matrix (pattern + values), DOM (cpt_SoC_dom.m) or CLA
// (cpt_SoC_cla.m, with the unit diagonal added).
HostCSR soc_matrix(const HostCSR &A, const char *soc_type, double tau);
// mark_isolated_nodes.m + cpt_PMIS.m on S.  Returns fcnode numbered as the
// reference: coarse k -> k (1..nc), fine -> -(1..nf).  rng is advanced by
// exactly n draws (rand(nn,1)).
std::vector<int> pmis_split(const HostCSR &A, const HostCSR &S, MT19937 &rng, int *nc_out);

// ---- BAMG prolongation (cpt_ProlMEX_BAMG.m + BAMG.cpp) ----------------------
struct BamgParams {
  int itmax_vol, dist_min, dist_max, mmax, nthreads;
  double maxcond, maxrownrm, tol_vol, eps;
};
// fc: coarse index (0-based) or -1.  TV row-major [n x ntv].  Returns P
// (n x nc) with exact zeros dropped; c_mark[i] = 1 for rows not interpolated
// to the requested accuracy.
HostCSR bamg_prolongation(const BamgParams &prm, const HostCSR &S, const std::vector<int> &fc,
                          int nc, const double *TV, int ntv, std::vector<int> &c_mark);
// The rows `rows` of the same prolongation: rcols[i], rvals[i] and c_mark[i]
// (sized n by the caller) for each listed row i.
void bamg_rows_host(const BamgParams &prm, const HostCSR &S, const std::vector<int> &fc,
                    const double *TV, int ntv, const std::vector<int> &rows,
                    std::vector<std::vector<int>> &rcols, std::vector<std::vector<double>> &rvals,
                    std::vector<int> &c_mark);

// A CSR borrowed from its owner: int32 row pointers, v may be null.
struct CsrRef {
  int nrows = 0, ncols = 0;
  const int *rp = nullptr;
  const int *ci = nullptr;
  const double *v = nullptr;
  int64_t nnz() const { return rp ? rp[nrows] : 0; }
};

// ---- EMIN prolongation pattern (MEX_cptProlPatt.cpp) -------------------------
// One row of a power step of the EMIN pattern (MEX_cptProlPatt.cpp:356-443):
// the columns of (S * Pc)(i, :) that are not in P0's row i, summed in S's row
// order and Pc's, the nonzero ones only; beyond the budget nnzr - |P0(i,:)|
// the budget's worth of largest magnitude (ties: lower column first); then
// P0's own columns with value 1; by column.  S with values, rows of P0 and
// Pc with ascending columns.  The GPU pattern kernel hands rows whose
// candidate lists outgrow its per-warp table to this function.
void emin_pattern_row(int i, const CsrRef &S, const CsrRef &Pc, const CsrRef &P0, int nnzr,
                      std::vector<int> &cols, std::vector<double> &vals);

// ---- adaptive FSAI pattern search (cpt_afsai_coef.cpp) ----------------------
// Rows of G hold their strictly-lower columns ascending, then the diagonal.
// vals receives the host FP64 values of the final per-row solve (the GPU
// numeric phase recomputes them).  ref_abs = true reproduces the reference's
// magnitude comparisons through C's int abs (see fsai_pattern.cpp).
struct FsaiResult {
  HostCSR G;
  bool posdef = true;
};
FsaiResult fsai_adaptive(const HostCSR &A, int nstep, int step_size, double eps, int nthreads,
                         bool ref_abs);

// Thin QR (Householder) of an n x k column-major matrix: Q overwrites X.
void qr_orthonormalize(int n, int k, double *X);

// On-disk formats of the reference (formats.cpp): example_cpp binary CSR,
// Chronos .Ext_bin matrix and test space (column-major n x ntv in memory).
HostCSR read_matrix_bin(const std::string &path);
HostCSR read_ext_bin(const std::string &path);
void write_ext_bin(const std::string &path, const HostCSR &A);
void read_tv_ext_bin(const std::string &path, int *nrows, int *ntv, std::vector<double> &tv);
void write_tv_ext_bin(const std::string &path, int nrows, int ntv, const double *tv_colmajor);

// CSR utilities
HostCSR csr_transpose(const HostCSR &A);

}  // namespace chronos
