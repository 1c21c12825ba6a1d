/* CPU oracle of the solve path in C (FP64, OpenMP).
 *
 * ORACLE TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and the CPU
 * baseline / reference arm of bench.py load liboracle.so, and only as the
 * checker or the timed CPU baseline.  The chronoslab_b200 package never does.
 *
 * Restates, line by line:
 *   oracle_pcg_cj   sources/LinearSolver/PCG_CJ.m:1-73
 *   oracle_vcycle   sources/Preconditioner/AMG/aspAMG/AMG_Vcycle.m:1-54
 *                   (smoother handle Minv = omega*F'*(F*x), cpt_aspAMG.m:301-302;
 *                    coarsest x = L'\(L\b), AMG_Vcycle.m:9-10)
 *   oracle_pmis     sources/Preconditioner/AMG/coarsen/cpt_PMIS.m:1-102
 *   oracle_spmv     y = A*x (MATLAB sparse product), row-parallel CSR
 */
#ifndef CHRONOS_ORACLE_H
#define CHRONOS_ORACLE_H
#include <stdint.h>

typedef struct {
  int nrows, ncols;
  const int64_t *rp;   /* 0-based */
  const int *ci;
  const double *v;
} ocsr;

typedef struct {
  int n;
  ocsr A, G, Gt, P, Pt; /* G, Gt, P, Pt unused on the coarsest level */
  double omega;
  const double *L;      /* coarsest level: lower Cholesky factor, column-major n x n */
  int nupre, nupost;
} olevel;

void oracle_set_threads(int nthreads);
void oracle_spmv(const ocsr *A, const double *x, double *y);
void oracle_vcycle(int nlev, const olevel *lv, const double *b, double *x);
/* Returns the flag of PCG_CJ (0 converged, 1 not); iters and resvec
 * (itmax + 1 entries) as the reference returns them. */
int oracle_pcg_cj(int nlev, const olevel *lv, const ocsr *A, const double *b, double *x,
                  int itmax, double tol, int *iters, double *resvec);
/* fcnode on entry: 0 free, -2 Dirichlet; S: strength pattern (diagonal
 * ignored); rnd: the nn random draws rand(nn,1).  On exit fcnode numbered as
 * the reference (coarse 1..nc, fine -(1..nf)); returns nc. */
int oracle_pmis(int n, const int64_t *S_rp, const int *S_ci, const double *rnd, int *fcnode);

#endif
