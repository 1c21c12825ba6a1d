// C entry points over the reference's own, unmodified C++ kernels, built into
// oracle/_ref/ by oracle/Makefile straight from the reference sources.
//
// ORACLE TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and the CPU
// baseline / reference arm of bench.py load the library this file is part of;
// the chronoslab_b200 package never does.
//
//   ref_fsai  -> compute_local_fsai  (MEX_SYM_AFSAI/compute_local_fsai.cpp:6-116),
//                called exactly as the MEX gateway does (SYM_aFSAI_compute.cpp:100-149)
//                with tau = 0 as forced by afsai_cpp.m:46.
//   ref_bamg  -> BAMG                (MEX_BAMG_Prol/BAMG.cpp:19-311),
//                called as cpt_Prolongation_BAMG.cpp:82-84 does (nn_L = 0,
//                nn_C = nn_S), with the TV transposed to row-major as there (:43-52).
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "BAMG.h"                 // reference: MEX_BAMG_Prol/include

extern "C" {

struct RefBamgResult {
  int nt;
  int *iat;
  int *ja;
  double *coef;
  int *c_mark;
};

// BAMG prolongation of the reference on the strength pattern (0-based CSR),
// fcnodes as prepared by cpt_ProlMEX_BAMG.m:48-51 (coarse index >= 0, fine -1),
// TV row-major [nn_S x ntv].  The result arrays are malloc'd; free them with
// ref_bamg_free.  Returns BAMG's error code (0 = ok).
int ref_bamg(int np, int itmax_vol, int dist_min, int dist_max, int mmax,
             double maxcond, double maxrownrm, double tol_vol, double eps_prol,
             int nn_S, const int *iat_S, const int *ja_S, int ntv,
             const int *fcnodes, const double *tv_rowmajor, RefBamgResult *out) {
  std::vector<const double *> tv_ptr(nn_S);
  for (int i = 0; i < nn_S; ++i) tv_ptr[i] = tv_rowmajor + (size_t)i * ntv;
  BAMG_params params;
  params.verbosity = 0;
  params.itmax_vol = itmax_vol;
  params.dist_min = dist_min;
  params.dist_max = dist_max;
  params.mmax = mmax;
  params.maxcond = maxcond;
  params.maxrownrm = maxrownrm;
  params.tol_vol = tol_vol;
  params.eps = eps_prol;
  int nt_I = 0;
  std::vector<int> iat, ja, c_mark;
  std::vector<double> coef;
  int ierr = BAMG(params, np, 0, nn_S, nn_S, iat_S, ja_S, ntv, fcnodes,
                  tv_ptr.data(), nt_I, iat, ja, coef, c_mark);
  if (ierr != 0) return ierr;
  out->nt = nt_I;
  out->iat = (int *)malloc(sizeof(int) * (nn_S + 1));
  out->ja = (int *)malloc(sizeof(int) * (nt_I > 0 ? nt_I : 1));
  out->coef = (double *)malloc(sizeof(double) * (nt_I > 0 ? nt_I : 1));
  out->c_mark = (int *)malloc(sizeof(int) * (nn_S > 0 ? nn_S : 1));
  memcpy(out->iat, iat.data(), sizeof(int) * (nn_S + 1));
  if (nt_I > 0) {
    memcpy(out->ja, ja.data(), sizeof(int) * nt_I);
    memcpy(out->coef, coef.data(), sizeof(double) * nt_I);
  }
  if (nn_S > 0) memcpy(out->c_mark, c_mark.data(), sizeof(int) * nn_S);
  return 0;
}

void ref_bamg_free(RefBamgResult *r) {
  free(r->iat);
  free(r->ja);
  free(r->coef);
  free(r->c_mark);
  r->iat = nullptr;
  r->ja = nullptr;
  r->coef = nullptr;
  r->c_mark = nullptr;
}

}  // extern "C"
