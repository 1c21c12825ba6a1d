// C entry points over the reference's own, unmodified EMIN C++ sources, built
// into oracle/_ref/ by oracle/Makefile straight from the reference sources.
//
// ORACLE TEST INFRASTRUCTURE.  Only tests/ and the CPU baseline / reference
// arm of bench.py load the library this file is part of; the chronoslab_b200
// package never does.
//
//   ref_emin_pattern -> the mexFunction of MEX_EMIN/MEX_cptProlPatt.cpp:234-490,
//                       run through the MEX stand-in in oracle/mex_shim with the
//                       arguments prolong.m:222 passes (kpow = patt_pow,
//                       S_emin, P, fcnode, nnzr_max, nnzr_min = ntv, np).
//   ref_emin         -> EMIN_ImpProl (Cpp_EMIN/EMIN_ImpProl.cpp:84-410),
//                       called as the gateway EMIN_Prolong_compute.cpp:150-172
//                       does, with the arrays prepared as
//                       MEX_EMIN_enhance_prol.m:29-98 prepares them (0-based
//                       CSR with ascending columns, fcnode coarse index >= 0 and
//                       fine < 0, TV as row pointers into a row-major array).
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mex.h"                  // oracle/mex_shim
#include "EMIN_ImpProl.h"         // reference: Cpp_EMIN/include

namespace {

// 0-based CSR (ascending columns) -> MATLAB CSC sparse array.
mxArray *csr_to_mx(int m, int n, const int *rp, const int *ci, const double *v) {
  const int nnz = rp[m];
  mxArray *a = mxCreateSparse(m, n, nnz > 0 ? nnz : 1, mxREAL);
  std::vector<mwIndex> cnt(n + 1, 0);
  for (int k = 0; k < nnz; ++k) cnt[ci[k] + 1]++;
  for (int c = 0; c < n; ++c) cnt[c + 1] += cnt[c];
  a->jc = cnt;
  std::vector<mwIndex> next(cnt.begin(), cnt.end() - 1);
  for (int i = 0; i < m; ++i)
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const mwIndex d = next[ci[k]]++;
      a->ir[d] = i;
      a->pr[d] = v ? v[k] : 1.0;
    }
  return a;
}

mxArray *scalar(double x) {
  mxArray *a = new mxArray;
  a->m = a->n = 1;
  a->pr.assign(1, x);
  return a;
}

}  // namespace

extern "C" {

struct RefCsr {
  int nrows, ncols, nnz;
  int *rp;
  int *ci;
  double *v;
};

void ref_csr_free(RefCsr *c) {
  free(c->rp);
  free(c->ci);
  free(c->v);
  c->rp = c->ci = nullptr;
  c->v = nullptr;
}

// The reference's EMIN prolongation pattern.  S: n x n strength matrix with
// values (0-based CSR), P: n x nc prolongation, fcnode in the C convention
// (coarse index >= 0, fine -1; converted here to MATLAB's, coarse index + 1).
// Returns 0 and the n x nc pattern (values as the MEX returns them) in *out,
// or -1 when the MEX raised an error.
int ref_emin_pattern(int kpow, int n, int nc, const int *rp_S, const int *ci_S,
                     const double *v_S, const int *rp_P, const int *ci_P, const double *v_P,
                     const int *fcnode, int nnzr, int nnzr_min, int np, RefCsr *out) {
  std::vector<mxArray *> in;
  in.push_back(scalar(kpow));
  in.push_back(csr_to_mx(n, n, rp_S, ci_S, v_S));
  in.push_back(csr_to_mx(n, nc, rp_P, ci_P, v_P));
  mxArray *fc = new mxArray;
  fc->m = n;
  fc->n = 1;
  fc->pr.resize(n);
  for (int i = 0; i < n; ++i) fc->pr[i] = fcnode[i] >= 0 ? fcnode[i] + 1.0 : -1.0;
  in.push_back(fc);
  in.push_back(scalar(nnzr));
  in.push_back(scalar(nnzr_min));
  in.push_back(scalar(np));
  mxArray *res = nullptr;
  int rc = 0;
  try {
    mexFunction(1, &res, (int)in.size(), const_cast<const mxArray **>(in.data()));
  } catch (const MexError &) {
    rc = -1;
  }
  for (mxArray *a : in) delete a;
  if (rc != 0 || res == nullptr) { delete res; return -1; }
  // CSC -> CSR (rows ascending within a column, so columns come out ascending)
  const int m = (int)res->m, ncol = (int)res->n, nnz = (int)res->jc[ncol];
  out->nrows = m;
  out->ncols = ncol;
  out->nnz = nnz;
  out->rp = (int *)calloc(m + 1, sizeof(int));
  out->ci = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
  out->v = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
  for (int k = 0; k < nnz; ++k) out->rp[res->ir[k] + 1]++;
  for (int i = 0; i < m; ++i) out->rp[i + 1] += out->rp[i];
  std::vector<int> next(out->rp, out->rp + m);
  for (int c = 0; c < ncol; ++c)
    for (mwIndex k = res->jc[c]; k < res->jc[c + 1]; ++k) {
      const int d = next[res->ir[k]]++;
      out->ci[d] = c;
      out->v[d] = res->pr[k];
    }
  delete res;
  return 0;
}

// The reference's energy minimisation of P on the pattern.  A: n x n, Pin and
// patt: n x nc (0-based CSR, ascending columns; patt without coarse rows),
// fcnode in the C convention, TV row-major n x ntv.  Returns EMIN_ImpProl's
// error code; on success *out holds P (malloc'd, free with ref_csr_free) and
// info[0..11] the reference's info array.
int ref_emin(int np, int itmax, double en_tol, double condmax, int prec_type, int sol_type,
             int n, int nc, int ntv, const int *fcnode, int spd, const int *rp_A,
             const int *ci_A, const double *v_A, const int *rp_Pin, const int *ci_Pin,
             const double *v_Pin, const int *rp_patt, const int *ci_patt,
             const double *tv_rowmajor, RefCsr *out, double *info) {
  std::vector<const double *> tv(n);
  for (int i = 0; i < n; ++i) tv[i] = tv_rowmajor + (size_t)i * ntv;
  int *iat = nullptr, *ja = nullptr;
  double *coef = nullptr;
  double inf[EMIN_INFO_SZ] = {};
  const int ierr = EMIN_ImpProl(np, itmax, en_tol, condmax, prec_type, sol_type, n, nc, ntv,
                                rp_patt[n], fcnode, spd != 0, rp_A, ci_A, v_A, rp_Pin, ci_Pin,
                                v_Pin, rp_patt, ci_patt, tv.data(), iat, ja, coef, inf, false);
  if (info)
    for (int k = 0; k < EMIN_INFO_SZ; ++k) info[k] = inf[k];
  if (ierr != 0) {
    free(iat);
    free(ja);
    free(coef);
    return ierr;
  }
  out->nrows = n;
  out->ncols = nc;
  out->nnz = iat[n];
  out->rp = iat;
  out->ci = ja;
  out->v = coef;
  return 0;
}

}  // extern "C"
