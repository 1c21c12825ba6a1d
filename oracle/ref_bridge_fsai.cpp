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

#include "compute_local_fsai.h"   // reference: MEX_SYM_AFSAI

extern "C" {

// Adaptive symmetric FSAI of the reference.  Inputs use the reference's 1-based
// CSR with int64 row pointers and int32 columns (afsai_cpp.m:26-39).
// Outputs: iat_G[n+1] (1-based), ja_G / coef_G sized n*(1+nstep*step_size)
// by the caller.  Returns 0.
int ref_fsai(int nthread, int n_step, int step_size, double eps, int nrows,
             int64_t nterm_M, const int64_t *iat_M, const int *ja_M,
             const double *coef_M, int64_t *nterm_G, int64_t *iat_G, int *ja_G,
             double *coef_G, int *is_posdef) {
  bool posdef = true;
  compute_local_fsai(nthread, n_step, step_size, 0.0, eps, nrows, nrows, nterm_M,
                     iat_M, ja_M, coef_M, nterm_G, iat_G, ja_G, coef_G, &posdef);
  *is_posdef = posdef ? 1 : 0;
  return 0;
}

}  // extern "C"
