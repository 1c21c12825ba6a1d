/*
 * chronos_b200.h -- C ABI of the B200 (sm_100a) AMG-preconditioned SPD solve path.
 *
 * Drop-in boundary for ChronosLab's solve path.  Every entry point returns an
 * int status: 0 = ok, negative = error (CHRONOS_E*); the message of the last
 * error on the calling thread is available from chronos_last_error().  No C++
 * exception crosses this boundary.
 *
 * Ownership: input pointers are borrowed and never freed by the library; the
 * library owns everything a handle (chronos_hier, chronos_galerkin_plan) holds
 * until the matching *_free call.  One handle is used by one host thread at a
 * time; the solve calls order their device work on the caller's stream
 * argument (see "Streams of the solve entry points").  Pointers named *_h are
 * host memory; *_d are device memory of the current device.
 *
 * Reference interfaces replaced (paths inside the ChronosLab project):
 *   chronos_fsai_compute   <- SYM_aFSAI_compute MEX
 *                             (sources/Preconditioner/AMG/smoother/MEX_SYM_AFSAI/
 *                              SYM_aFSAI_compute.cpp:15-20,57-149; compute_local_fsai.h:8-11)
 *   chronos_fsai_numeric   <- numeric half of the same MEX (cpt_afsai_coef.cpp:440-541)
 *   chronos_amg_setup      <- cpt_aspAMG(param,A,TV0)   (aspAMG/cpt_aspAMG.m:1,54; called at
 *                             Drivers/driver_AMG/aspAMG_main.m:175, utils/computeAMG.m:46)
 *   chronos_vcycle(_dev)   <- AMG_Vcycle(hrc,A,b)       (aspAMG/AMG_Vcycle.m:1-54)
 *   chronos_pcg            <- PCG_CJ(prodM,prodA,b,x0,itmax,tol) (LinearSolver/PCG_CJ.m:1-73;
 *                             called at aspAMG_main.m:199-202)
 *   chronos_sqmr           <- SQMR(Afun,rhs,tol,itmax,lprec,rprec) (LinearSolver/SQMR.m:1-108;
 *                             called at Tests/CubeBAMG_NONE.m:28)
 *   chronos_galerkin_*     <- Anext = Pf'*(A*Pf)        (aspAMG/cpt_aspAMG.m:277)
 *   chronos_dense_chol     <- [L,p,S] = chol(A,'lower') (aspAMG/cpt_aspAMG.m:109) and the
 *                             coarsest solve S*(L'\(L\(S'*b))) (AMG_Vcycle.m:9-10)
 *   chronos_params_read    <- readDefaultParams.m / aspAMG_main.m:17-59 and read_*.m
 *   chronos_emin_pattern   <- MEX_cptProlPatt          (prolong/EMIN/MEX_EMIN/MEX_cptProlPatt.cpp)
 *   chronos_emin           <- EMIN_Prolong_compute / EMIN_ImpProl (prolong/EMIN/Cpp_EMIN/
 *                             EMIN_ImpProl.cpp:84-410; called from prolong.m:224-225)
 */
#ifndef CHRONOS_B200_H
#define CHRONOS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define CHRONOS_OK            0
#define CHRONOS_EINVAL       -1   /* bad argument, malformed CSR, size limit */
#define CHRONOS_ECUDA        -2   /* CUDA runtime error */
#define CHRONOS_ENOMEM       -3   /* host or device allocation failed */
#define CHRONOS_ENOTSPD      -4   /* non-SPD block / Cholesky breakdown */
#define CHRONOS_EBREAKDOWN   -5   /* Krylov breakdown (p'Ap <= 0, NaN) */
#define CHRONOS_EIO          -6   /* parameter or data file error */
#define CHRONOS_ENOTSUP      -7   /* option outside this solve path */

/* ---- precision of the stored hierarchy -------------------------------- */
#define CHRONOS_FP64 0            /* all-FP64 GPU path */
#define CHRONOS_FP32 1            /* FP32 hierarchy, FP32 accumulate; FP64 outer solve */

/* ---- parameters: the positional parm_* files of the reference ----------- */
typedef struct chronos_params {
  /* parm_AMG (read_amg.m) */
  int nLevMax, maxCoarseSZ;
  /* parm_SMOOTH (read_smoother.m:73-79) */
  int nthread, nupre, nupost, nstep, step_size;
  double epsilon;
  char smoother_method[32];       /* AFSAI_SYM on this path */
  /* parm_TSPACE (read_tspace.m) */
  int ntv, tspace_itmax;
  double tspace_tol;
  char tspace_method[32];         /* NONE on this path */
  int init_approx;
  /* parm_COARSEN (read_coarsen.m:177-179) */
  char SoC_type[16];              /* DOM or CLA */
  double soc_tau;
  int nl_agg;
  /* parm_PROLONG (read_prolong.m; the BAMG lines) */
  char proltype[16];              /* BAMG */
  char prol_emin[16];             /* NONE, SMOOTH or EMIN */
  int prol_np, itmax_vol;
  double tol_vol;
  int dist_min, dist_max;
  double maxcond, maxrownrm, eps_prol;
  int updateCF;
  /* parm_PROLONG, the EMIN lines (prol_emin = EMIN, prolong.m:207-235) */
  int patt_pow;                   /* power steps of the EMIN pattern (2) */
  double patt_tau;                /* DOM threshold of its strength matrix (0.01) */
  int nnzr_max, itmax_emin;       /* entries per pattern row (30); CG steps (10) */
  double energ_tol, condmax_emin; /* energy-decrease exit (1e-3); constraint blocks' condition (1e10) */
  int prec_emin, solv_emin;       /* 1 (Jacobi); 4 (products with A) */
  /* parm_FILTER (read_filter.m) */
  int filt_np;
  double filt_wgt, filt_tol, filt_tau;
  int min_patt;
  /* parm_GENERAL (read_general.m:4-11) */
  int ascii_input;
  char rhs_build[16];
  int symmetric;
  char solv_method[16];
  int itmax;
  double tol;
  int restart;
  /* build options (no counterpart in the parameter files) */
  int precision;                  /* CHRONOS_FP32 or CHRONOS_FP64 */
  int use_graph;                  /* 1: whole solve as one CUDA graph with a device-side loop */
  uint64_t seed;                  /* MT19937 seed of MATLAB's rng(0) stream: 5489 */
  int fsai_fabs;                  /* 0 (default): FSAI candidate ranking and exit test compare
                                     magnitudes as the reference's g++ build does, through C's
                                     int abs (truncation toward zero); 1: through fabs */
  int use_bsr;                    /* 1 (default): apply the level-1 operator in 3x3 block form
                                     when its pattern is made of whole aligned 3x3 blocks */
  int exact_outer;                /* 1: the outer PCG applies the level-1 operator with its FP64
                                     values (PCG_CJ's arithmetic exactly).  0 (default): with
                                     the hierarchy's stored values (FP32 for CHRONOS_FP32)
                                     accumulated in FP64, the recursive residual being replaced
                                     by the FP64 true residual b - A x whenever it has fallen
                                     by replace_ratio since the last replacement and before
                                     every stop; the returned relative residual is then the
                                     true one.  No effect for CHRONOS_FP64 hierarchies. */
  double replace_ratio;           /* 0.01 (default), in (0, 1) */
  int spmv_format;                /* storage of the V-cycle's CSR operators: 0 (default) the
                                     autotuner's choice per operator; 1 row-grouped CSR only;
                                     2 sliced ELL for every operator averaging at most 16
                                     entries per row */
  int batch_grouped;              /* chronos_batch_*: 1 (default) one launch sequence for the
                                     whole batch (stacked level operators, per-problem PCG
                                     scalars); 0 one graph per problem on its own stream */
} chronos_params;

/* Reference regression-test parameters (Tests/parm_*): DOM 0.01, BAMG/NONE,
 * AFSAI_SYM 15/1/1e-3, ntv 6, V(1,1), nLevMax 10, maxCoarseSZ 1000. */
void chronos_params_default(chronos_params *p);
/* Reads an aspAMG.fnames file (first 7 lines name parm_AMG, parm_SMOOTH,
 * parm_TSPACE, parm_COARSEN, parm_PROLONG, parm_FILTER, parm_GENERAL, relative
 * to the fnames file) into p; fields not in the files keep their value. */
int chronos_params_read(const char *fnames_path, chronos_params *p);

/* Copies the last error message of this thread into buf (NUL-terminated). */
int chronos_last_error(char *buf, int len);
/* Library version string. */
const char *chronos_version(void);

/* ---- FSAI ------------------------------------------------------------- */
/* Drop-in for SYM_aFSAI_compute: same argument meaning (1-based CSR, int64 row
 * pointers, int32 columns, nrows_M - nrows = trailing-block shift).  Pattern by
 * the adaptive Kaporin search on the host; values by the GPU numeric kernel
 * (FP64).  ja_G/coef_G must hold nrows*(1+n_step*step_size) entries.  Each row
 * lists its strictly-lower entries ascending, then the diagonal.  Non-SPD is a
 * flag (is_posdef = 0), not an error, as in the MEX. */
int chronos_fsai_compute(int nthread, int n_step, int step_size, double tau, double eps,
                         int nrows, int nrows_M, int64_t nterm_M,
                         const int64_t *iat_M_h, const int *ja_M_h, const double *coef_M_h,
                         int64_t *nterm_G, int64_t *iat_G_h, int *ja_G_h, double *coef_G_h,
                         int *is_posdef);
/* Numeric phase only: G values on a given pattern (CSR of G, each row
 * strictly-lower ascending then the diagonal).  A and G are CSR with int64
 * row pointers and int32 columns, 0-based (base = 0) or 1-based as the MEX
 * passes them (base = 1).  One dense SPD solve per row on the GPU in FP64;
 * val_G_h receives double values (out_precision = CHRONOS_FP64) or float
 * values rounded from them (CHRONOS_FP32).  The work is ordered on `stream`
 * (a cudaStream_t; NULL: the legacy default stream) and the call returns
 * after it completes. */
int chronos_fsai_numeric(int n, int base, const int64_t *iat_A_h, const int *ja_A_h,
                         const double *val_A_h, const int64_t *iat_G_h, const int *ja_G_h,
                         int out_precision, void *val_G_h, int *is_posdef, void *stream);

/* The FSAI numeric phase of many problems at once (no counterpart call in the
 * reference, which runs the MEX once per matrix): one launch per
 * shared-memory tile size over every problem's rows, each row in the
 * smallest tile that holds its local system.  The tile sizes -- the bucket
 * edges -- are candidate sets {16,32,64}, {8,16,32,64}, {16,24,32,48,64},
 * {8,16,24,32,48,64} (tile_set 0..3); tile_set = -1 picks the fastest by
 * timing them on these rows (remembered per shape of the batch, in-process).
 * The values do not depend on the set: per problem they are those of
 * chronos_fsai_numeric bit for bit.  0-based CSR (int32) per problem; rows of
 * G strictly-lower ascending, then the diagonal; is_posdef[p] as the MEX's
 * flag; tile_set_used (may be NULL) receives the set run.  The batch setup
 * (chronos_batch_setup) runs each level's FSAI this way. */
int chronos_fsai_numeric_batch(int nprob, const int *n, const int *const *iat_A_h,
                               const int *const *ja_A_h, const double *const *val_A_h,
                               const int *const *iat_G_h, const int *const *ja_G_h,
                               double *const *val_G_h, int *is_posdef, int tile_set,
                               int *tile_set_used);

/* FSAI numeric phase that allocates nothing.  This entry point has no
 * counterpart in the reference.  It is for callers that cannot let a library
 * call cudaMalloc or cudaFree: hosts that own all device memory through their
 * own pool (a framework's caching allocator, a MATLAB gpuArray host, an
 * embedded or real-time host that reserves memory up front) and callers whose
 * other streams must not be stalled by the device-wide synchronisation that
 * cudaFree implies.  Same result as chronos_fsai_numeric, but every pointer is
 * device memory the caller owns: A and the pattern of G as 0-based CSR with
 * int32 row pointers and columns (G rows: strictly-lower columns ascending,
 * then the diagonal), val_G_d receives the values; is_posdef is host memory.
 * Work is queued on `stream` (a cudaStream_t; NULL for the legacy default
 * stream) and the call returns after it completes.
 * Scratch: a fixed 12 MiB + 256 B array in device memory, part of the
 * library's module, held on every GPU that loads the library until the
 * process exits; n is limited to 1048576 rows (larger n returns
 * CHRONOS_EINVAL).  The first call on a device looks up the array's device
 * address for that device.  All calls share the array: calls that overlap on
 * the GPU race on it and must be serialised by the caller.
 * Both patterns are checked on the device before any value is computed: an
 * empty G row, a G row not ending with its diagonal or with strictly-lower
 * columns not ascending in [0, i), or A row pointers / columns that are not a
 * sorted 0-based CSR return CHRONOS_EINVAL with val_G_d untouched. */
int chronos_fsai_numeric_noalloc(int n, const int *iat_A_d, const int *ja_A_d,
                                 const double *val_A_d, const int *iat_G_d, const int *ja_G_d,
                                 double *val_G_d, int *is_posdef, void *stream);

/* ---- host-side setup pieces (no GPU) ------------------------------------ */
/* Result handle for a CSR produced by the library (0-based, FP64). */
typedef struct chronos_csr chronos_csr;
int chronos_csr_info(const chronos_csr *m, int *nrows, int *ncols, int64_t *nnz);
int chronos_csr_fetch(const chronos_csr *m, int *iat_h, int *ja_h, double *val_h);
int chronos_csr_free(chronos_csr *m);

/* ---- on-disk formats of the reference ------------------------------------- */
/* example_cpp binary CSR, replaces readBinaryMatrix (Cpp_EMIN/readMat.cpp:27-80):
 * int32 rows and entries, then {int32 row, int32 column, double value} records,
 * 1-based, grouped by row.  Returns a 0-based CSR (columns ascending). */
int chronos_read_matrix_bin(const char *path, chronos_csr **A);
/* Chronos .Ext_bin matrix as DumpChronos writes it (debug_stuff/dump_chronos/
 * DumpChronos.cpp:27-36): int64 rows and entries, then {int64 row, int64 column,
 * double value} records, 1-based.  Read returns a 0-based CSR; write takes one. */
int chronos_read_ext_bin(const char *path, chronos_csr **A);
int chronos_write_ext_bin(const char *path, int n, int ncols, const int *iat_h, const int *ja_h,
                          const double *val_h);
/* Chronos .Ext_bin test space (DumpChronos.cpp:38-45): int64 rows and columns,
 * then the values row by row.  TV_h is n x ntv column-major; read with TV_h =
 * NULL returns the sizes.  A file that ends after its header (the reference's
 * dumper writes the values to the closed matrix file) reads as ntv = 0. */
int chronos_read_tv_ext_bin(const char *path, int *n, int *ntv, double *TV_h);
int chronos_write_tv_ext_bin(const char *path, int n, int ntv, const double *TV_h);

/* Symbolic half of SYM_aFSAI_compute on the host (cpt_afsai_coef.cpp:316-543):
 * the adaptive pattern with the host FP64 values of the final local solves.
 * A: 0-based CSR, sorted rows.  G rows: strictly-lower ascending, then the
 * diagonal.  fsai_fabs as in chronos_params. */
int chronos_fsai_pattern(int n, const int *iat_h, const int *ja_h, const double *val_h,
                         int nstep, int step_size, double eps, int nthread, int fsai_fabs,
                         int *is_posdef, chronos_csr **G);
/* coarsen.m on the host: strength of connection (prm->SoC_type, prm->soc_tau)
 * and the PMIS C/F splitting with the MT19937 stream of prm->seed advanced by
 * rng_skip draws first.  fcnode_h[n]: coarse k -> k (1..nc), fine -> -(1..nf),
 * as the reference numbers them.  S (may be NULL) receives the strength matrix. */
int chronos_coarsen(const chronos_params *prm, int n, const int *iat_h, const int *ja_h,
                    const double *val_h, uint64_t rng_skip, int *fcnode_h, int *nc,
                    chronos_csr **S);
/* The same on the GPU for DOM strength (cpt_SoC_dom.m:26-47) or CLA strength
 * (cpt_SoC_cla.m:109-159; every row must store a nonzero diagonal), with
 * cpt_PMIS.m and mark_isolated_nodes.m: identical fcnode and nc, and S with
 * the strength pattern (values 1).  CHRONOS_ENOTSUP for another SoC type.
 * The hierarchy setup coarsens this way unless CHRONOS_GPU_COARSEN=0. */
int chronos_coarsen_device(const chronos_params *prm, int n, const int *iat_h, const int *ja_h,
                           const double *val_h, uint64_t rng_skip, int *fcnode_h, int *nc,
                           chronos_csr **S);
/* cpt_ProlMEX_BAMG on the host: BAMG prolongation (n x nc) from the strength
 * pattern S, fcnode as returned by chronos_coarsen, and the test space TV
 * (n x ntv, column-major).  c_mark_h[n] (may be NULL) flags rows not
 * interpolated to eps_prol. */
int chronos_bamg(const chronos_params *prm, int n, const int *iat_S_h, const int *ja_S_h,
                 const int *fcnode_h, int ntv, const double *TV_h, int *c_mark_h,
                 chronos_csr **P);
/* The same prolongation with the per-row work on the GPU (one thread per fine
 * row: neighbourhood rings, maximum-volume selection, least-squares fit, set
 * reduction; MEX_BAMG_Prol/BAMG.cpp:119-225): P and c_mark equal chronos_bamg's
 * bit for bit (at most 16 test vectors).  Each thread's scratch holds up to
 * max_neigh neighbourhood nodes (a power of two in [16, 8192]; 0: 512 to 8192,
 * from a 2 GiB budget and the number of rows); a row whose neighbourhood
 * outgrows it is computed on the host, their count going to host_rows (may
 * be NULL).  The hierarchy setup builds BAMG prolongations this way when
 * CHRONOS_GPU_BAMG=1. */
int chronos_bamg_device(const chronos_params *prm, int n, const int *iat_S_h, const int *ja_S_h,
                        const int *fcnode_h, int ntv, const double *TV_h, int *c_mark_h,
                        int max_neigh, chronos_csr **P, int *host_rows);
/* EMIN prolongation pattern on the GPU, replaces MEX_cptProlPatt
 * (MEX_EMIN/MEX_cptProlPatt.cpp:234-490) as prolong.m:222 calls it:
 * Ppatt = MEX_cptProlPatt(kpow, S, P, fcnode, nnzr, nnzr_min, np).  S (n x n,
 * strength values), P (n x nc) 0-based CSR with ascending columns, fcnode as
 * chronos_coarsen returns it.  The n x nc pattern (coarse rows empty; values
 * as the MEX returns them: 1 on P's own entries, those of S*P on the added
 * ones) is bit-identical to the reference's.  *host_rows (may be NULL):
 * rows computed on the host because their candidates outgrew a GPU warp's
 * table. */
int chronos_emin_pattern(int kpow, int n, int nc, const int *iat_S_h, const int *ja_S_h,
                         const double *coef_S_h, const int *iat_P_h, const int *ja_P_h,
                         const double *coef_P_h, const int *fcnode_h, int nnzr_max, int nnzr_min,
                         chronos_csr **patt, int *host_rows);
/* Energy minimisation of a prolongation on the GPU, replaces
 * EMIN_Prolong_compute / EMIN_ImpProl (Cpp_EMIN/EMIN_ImpProl.cpp:84-410,
 * MEX_EMIN/EMIN_Prolong_compute.cpp:73-209) with prm->solv_emin 3 or 4
 * (products with A, EMIN_matfree.cpp:69-308), prm->prec_emin 1 (Jacobi) and
 * spd != 0 (DEFL_PCG_matfree.cpp; the GMRES variant for a nonsymmetric A is
 * outside this path: CHRONOS_ENOTSUP).  A (n x n), P (n x nc) and the pattern
 * (n x nc, no coarse rows, e.g. from chronos_emin_pattern) as 0-based CSR with
 * ascending columns; fcnode as chronos_coarsen returns it; TV_h n x ntv
 * column-major (ntv <= 16).  Returns P with unit coarse rows and exact zeros
 * dropped (as sparse() does in MEX_EMIN_enhance_prol.m:102) and info[12] (may
 * be NULL) as the reference's info array: [2] constraint setup s, [3] CG s,
 * [5] total s, [6] rows whose constraint block took the SVD branch, [7] CG
 * iterations, [10] pattern entries, [11] entries of Q. */
int chronos_emin(const chronos_params *prm, int n, const int *iat_A_h, const int *ja_A_h,
                 const double *coef_A_h, int nc, const int *iat_P_h, const int *ja_P_h,
                 const double *coef_P_h, const int *iat_patt_h, const int *ja_patt_h,
                 const int *fcnode_h, int ntv, const double *TV_h, int spd, chronos_csr **P,
                 double *info);

/* ---- Galerkin product P'*(A*P) on the GPU (0-based CSR, FP64) --------- */
typedef struct chronos_galerkin_plan chronos_galerkin_plan;
/* Symbolic + numeric phase; returns the nnz of Ac (exact zeros dropped, as
 * MATLAB's sparse product does).  Each output entry is accumulated in the same
 * order as a row-wise Gustavson product, so values and pattern are bitwise
 * reproducible. */
int chronos_galerkin_compute(int n, int nc,
                             const int *iat_A_h, const int *ja_A_h, const double *val_A_h,
                             const int *iat_P_h, const int *ja_P_h, const double *val_P_h,
                             int64_t *nnz_Ac, chronos_galerkin_plan **plan);
/* Copies Ac (row pointers nc+1, sorted columns, values) to host buffers. */
int chronos_galerkin_fetch(chronos_galerkin_plan *plan, int *iat_Ac_h, int *ja_Ac_h,
                           double *val_Ac_h);
int chronos_galerkin_free(chronos_galerkin_plan *plan);

/* ---- Dense Cholesky of the coarsest level (FP64, GPU) ------------------- */
/* A_h: n x n column-major SPD.  On success L_h (n x n column-major) holds the
 * lower factor with zeros above the diagonal.  Returns CHRONOS_ENOTSPD on a
 * non-positive pivot. */
int chronos_dense_chol(int n, const double *A_h, double *L_h);

/* ---- CSR SpMV on the GPU (parity helper) ------------------------------- */
/* y = A x, 0-based CSR, values stored in `precision` and accumulated in it,
 * through the V-cycle's apply kernels.  format as chronos_params.spmv_format
 * (0 tuned, 1 row-grouped CSR, 2 sliced ELL); lanes > 0 forces the CSR path's
 * lanes per row (1, 2, 4, 8, 16 or 32; rows longer than 32 per lane go to
 * whole warps). */
int chronos_spmv(int n, int ncols, const int *iat_h, const int *ja_h, const double *val_h,
                 const double *x_h, double *y_h, int precision, int format, int lanes);

/* ---- AMG hierarchy ------------------------------------------------------ */
typedef struct chronos_hier chronos_hier;

typedef struct chronos_level_info {
  int n;                /* rows */
  int64_t nnz_A, nnz_G, nnz_P;
  int nc;               /* columns of P (0 on the coarsest level) */
  double omega, lambda; /* smoother damping and lambda_max(G A G') */
  int threads_per_row;  /* SpMV lanes per row chosen by the autotuner for A */
  int block_rows;       /* > 0: A is applied in 3x3 block form with this many block rows */
  int sell_mask;        /* bits 0-4: A, G, G', P, P' applied in sliced ELL form */
} chronos_level_info;

/* Builds the hierarchy of A (0-based CSR, FP64, in host or device memory)
 * with the test space TV0 (n x ntv0, column-major, host or device; may be NULL
 * with ntv0 = 0).  Coarsening
 * (SoC + PMIS), C/F splitting and the BAMG prolongation run on the host as in
 * the reference; FSAI values, lambda_max, the Galerkin products and the
 * coarse Cholesky run on the GPU.  prm->precision selects the stored
 * precision.  A diagonal entry equal to 1 is NOT rewritten here (the
 * computeAMG.m:5-10 Dirichlet fix is the caller's, see chronos_diag_fix). */
int chronos_amg_setup(const chronos_params *prm, int n, const int *iat_h, const int *ja_h,
                      const double *val_h, int ntv0, const double *TV0_h, chronos_hier **out);

/* A level's prolongation as the caller's host code computed it: P is n x nc,
 * 0-based CSR, columns ascending in each row.  The arrays belong to the
 * caller and must stay valid until the callback is called again or the
 * setup returns; the library copies them. */
typedef struct chronos_prolongation {
  int nc;                   /* coarse size, 0 < nc < n */
  const int *iat_P_h;       /* n + 1 row pointers, iat_P_h[0] = 0 */
  const int *ja_P_h;        /* iat_P_h[n] coarse columns */
  const double *val_P_h;    /* iat_P_h[n] values */
} chronos_prolongation;
/* Called once per level that is not the coarsest, with the 1-based level
 * number and that level's operator (host FP64 0-based CSR, sorted rows; the
 * GPU Galerkin product from level 2 on).  Returns 0 after filling *P, or a
 * nonzero value to abort the setup (chronos_amg_setup_prolong then returns
 * CHRONOS_EINVAL). */
typedef int (*chronos_prolong_fn)(void *ctx, int level, int n, const int *iat_A_h,
                                  const int *ja_A_h, const double *val_A_h,
                                  chronos_prolongation *P);
/* cpt_aspAMG with the prolongation from the caller (aspAMG/cpt_aspAMG.m:224-225
 * calls prolong(...), and :277 forms Anext = Pf'*(A*Pf)): coarsening, C/F
 * splitting, the test space and the prolongation -- P's pattern and values,
 * any post-process included -- stay on the caller's host code, level by level,
 * while the library computes everything else as chronos_amg_setup does: FSAI
 * pattern and values, lambda_max and omega, the Galerkin product on the GPU
 * (pattern and values reproducible bit for bit), the coarse factor.  The
 * stopping rule is the reference's (n <= maxCoarseSZ or nLevMax levels); the
 * test-space, prolongation and coarsening fields of prm are not used. */
int chronos_amg_setup_prolong(const chronos_params *prm, int n, const int *iat_h,
                              const int *ja_h, const double *val_h, chronos_prolong_fn prolong,
                              void *ctx, chronos_hier **out);
int chronos_hier_free(chronos_hier *h);
/* Hierarchy files (no counterpart in the reference, whose hierarchy lives in
 * the MATLAB workspace): save writes every level's operator, smoother factor
 * and prolongation (FP64), omega, lambda_max, the coarsest inverse and the
 * parameters; load rebuilds a handle from such a file without the setup --
 * same V-cycle bit for bit -- or returns CHRONOS_EIO for a file it cannot
 * use (wrong magic, version, parameter layout, truncated or inconsistent). */
int chronos_hier_save(const chronos_hier *h, const char *path);
/* Device memory the library holds in this process (bytes; no counterpart in
 * the reference).  The environment variable CHRONOS_DEVICE_ALLOC_CAP (bytes)
 * caps it: an allocation beyond the cap fails with CHRONOS_ENOMEM as a failed
 * cudaMalloc does, and the call that met it frees what it had allocated. */
int chronos_device_bytes(int64_t *bytes);
int chronos_hier_load(const char *path, chronos_hier **out);
int chronos_hier_nlevels(const chronos_hier *h, int *nlev);
int chronos_hier_level_info(const chronos_hier *h, int level, chronos_level_info *info);
/* Exports level `level` (0-based) matrix `which` ('A', 'G' or 'P') as 0-based
 * CSR in FP64.  Call with null arrays to get the sizes in *nrows / *nnz. */
int chronos_hier_export(const chronos_hier *h, int level, char which, int *nrows, int *ncols,
                        int64_t *nnz, int *iat_h, int *ja_h, double *val_h);
/* Setup timings in seconds: [fsai_pattern, fsai_numeric, omega, coarsen, prolong,
 * galerkin, coarse_factor, total]. */
int chronos_hier_setup_times(const chronos_hier *h, double *t8);
/* All setup phases (no counterpart in the reference): the first n of [the
 * eight above, uploads (operators and their 3x3 block form), layouts
 * (transposes and FP32 copies of G and P), autotune, other (total minus the
 * named phases)], n <= 12. */
int chronos_hier_setup_phases(const chronos_hier *h, double *t, int n);
/* Writes operator which ('A', 'G' or 'P') of a level in the .Ext_bin format
 * (FP64 values), e.g. to feed a level to the reference's own tools. */
int chronos_hier_dump_ext_bin(const chronos_hier *h, int level, char which, const char *path);

/* Kernel timings of a built hierarchy (CUDA events on its stream, `reps`
 * launches each after one warm-up) and the algorithmic bytes each moves:
 * values + column indices + row pointers once, every vector read or written
 * once (the compulsory traffic of a CSR apply). */
typedef struct chronos_profile {
  double vcycle_ms, vcycle_bytes;          /* one V-cycle, FP64 in/out */
  double top_apply_ms, top_apply_bytes;    /* level-1 residual b - A x in the stored precision */
  double outer_spmv_ms, outer_spmv_bytes;  /* the PCG's A p (FP64 accumulation) with its two dots */
  double iteration_bytes;                  /* one PCG_CJ iteration in total */
  int kernels_per_iteration;               /* kernel launches of one PCG iteration */
  int kernels_per_solve;                   /* launches outside the loop, per solve */
} chronos_profile;
int chronos_hier_profile(chronos_hier *h, int reps, chronos_profile *out);

/* computeAMG.m:5-10: diagonal entries equal to 1 become lambda_max(A)/10
 * (lambda_max by a GPU Lanczos run).  Updates val_h in place. */
int chronos_diag_fix(int n, const int *iat_h, const int *ja_h, double *val_h);

/* Streams of the solve entry points: `stream` is a cudaStream_t (NULL: the
 * legacy default stream).  The call's device work starts after the work the
 * stream has queued before the call, and work queued on the stream after the
 * call starts after the call's device work; the ordering uses events, with no
 * device-wide synchronisation.  Calls that return host results (iterations,
 * flags, host vectors) wait for their own work before returning.  Handles are
 * independent: two handles used from two host threads on two streams run
 * concurrently. */

/* One V(nupre,nupost) cycle x = M^{-1} b (x0 absent), host vectors, FP64 in/out.
 * nrhs columns, column-major (leading dimension n). */
int chronos_vcycle(chronos_hier *h, const double *b_h, double *x_h, int nrhs, void *stream);
/* The same V-cycle on device vectors (column-major n x nrhs): io_precision
 * CHRONOS_FP64 (double) or CHRONOS_FP32 (float).  An FP32 hierarchy reads and
 * writes float vectors directly (AMG_Vcycle.m:1-54 in FP32 end to end, the
 * coarsest solve in FP64 as always); an FP64 hierarchy runs on FP64 copies.
 * Work is ordered on stream with no host synchronisation. */
int chronos_vcycle_dev(chronos_hier *h, int io_precision, const void *b_d, void *x_d, int nrhs,
                       void *stream);

/* PCG_CJ with the V-cycle preconditioner, x0 = x_h on input.  The operator is
 * PCG_CJ's prodA (PCG_CJ.m:1; aspAMG_main.m:199-202 passes @(x)A*x): the
 * 0-based FP64 CSR (iat_h, ja_h, val_h) of the hierarchy's level-1 size,
 * copied to the device on every call that passes it, or the hierarchy's
 * level-1 operator when iat_h is NULL.  resvec_h (itmax+1 entries, may be NULL)
 * receives ||r_k||/||b||.  flag = 1 when not converged (PCG_CJ.m:69-71).
 * seconds (may be NULL) receives the device time of the solve (CUDA events,
 * copies excluded). */
int chronos_pcg(chronos_hier *h, const int *iat_h, const int *ja_h, const double *val_h,
                const double *b_h, double *x_h, int itmax, double tol, int *iters,
                double *resvec_h, int *flag, double *seconds, void *stream);
/* Same on device vectors (b_d, x_d: n FP64) with the hierarchy's level-1
 * operator, the hot path without copies. */
int chronos_pcg_dev(chronos_hier *h, const double *b_d, double *x_d, int itmax, double tol,
                    int *iters, double *resvec_h, int *flag, double *seconds, void *stream);
/* Block of nrhs independent right-hand sides (column-major n x nrhs) solved
 * together: one SpMM V-cycle per iteration, per-column PCG_CJ recurrences and
 * stopping tests.  iters_h[nrhs], flags_h[nrhs]. */
int chronos_pcg_block(chronos_hier *h, int nrhs, const double *B_h, double *X_h, int itmax,
                      double tol, int *iters_h, int *flags_h, double *seconds, void *stream);

/* ---- Batch of independent problems of uneven sizes ---------------------- */
/* One hierarchy per problem (each what chronos_amg_setup builds for it with
 * the constant vector as TV0, padded to ntv columns as the reference does).  No
 * counterpart call in the reference, which solves one system per driver run
 * (aspAMG_main.m:175,199-202); each problem of the batch is that run. */
typedef struct chronos_batch chronos_batch;
int chronos_batch_setup(const chronos_params *prm, int nprob, const int *n,
                        const int *const *iat_h, const int *const *ja_h,
                        const double *const *val_h, chronos_batch **out);
/* PCG_CJ on every problem (x0 = x_h[p] on input), all queued before any
 * result is read: per problem one conditional-graph launch on its own stream,
 * largest first.  iters[p], flags[p] as chronos_pcg; seconds = device time
 * from the first launch to the last problem's completion. */
int chronos_batch_solve(chronos_batch *b, const double *const *b_h, double *const *x_h,
                        int itmax, double tol, int *iters, int *flags, double *seconds);
int chronos_batch_info(const chronos_batch *b, int p, int *nlevels, int *n0);
/* The setup phases of chronos_hier_setup_phases summed over the batch's
 * problems (thread time: problems are built several at once). */
int chronos_batch_setup_phases(const chronos_batch *b, double *t, int n);
/* The batch setup's wall clock in seconds: [first levels begun (operators,
 * FSAI patterns), batched FSAI numeric phase of the first levels, the rest of
 * the hierarchies, tuning and grouping, total]. */
int chronos_batch_setup_wall(const chronos_batch *b, double *t5);
int chronos_batch_free(chronos_batch *b);

/* SQMR (SQMR.m) with the V-cycle as left preconditioner and identity right.
 * The operator is the 0-based FP64 CSR (iat_h, ja_h, val_h) of the hierarchy's
 * size, or the level-1 operator when iat_h is NULL (the reference's tests
 * apply the unmodified A while the preconditioner was built from the
 * Dirichlet-fixed one, Tests/CubeBAMG_NONE.m:19,28). */
int chronos_sqmr(chronos_hier *h, const int *iat_h, const int *ja_h, const double *val_h,
                 const double *b_h, double *x_h, int itmax, double tol, int *iters,
                 double *relres, int *info);
/* gmres_RIGHT.m (LinearSolver/GMRES_CJ/gmres_RIGHT.m:7-650), as
 * Tests/CubeBAMG_EMIN.m:30 calls it: right-preconditioned GMRES(restart) with
 * the hierarchy's V-cycle as M, at most maxit restart cycles, operator A from
 * (iat_h, ja_h, val_h) (0-based CSR) or, when iat_h is NULL, the hierarchy's
 * level-1 operator.  x_h holds x0 on entry.  flag: 0 converged (explicit
 * residual <= tol ||b||), 1 maxit cycles, 2 non-finite preconditioned vector,
 * 3 stagnation; iter_outer / iter_inner as the reference's iter(1:2) (the
 * total is (outer-1)*restart + inner).  resvec_h (may be NULL) receives
 * *nresvec <= restart*maxit+1 residual norms. */
int chronos_gmres(chronos_hier *h, const int *iat_h, const int *ja_h, const double *val_h,
                  const double *b_h, double *x_h, int restart, double tol, int maxit,
                  int *iter_outer, int *iter_inner, double *relres, int *flag,
                  double *resvec_h, int *nresvec);

/* ---- Adjoint ------------------------------------------------------------ */
/* For J(u) with u = A^{-1} b and dJ/du = g: solves A lambda = g with the same
 * hierarchy (A is SPD so A^T = A) and returns dJ/dA on A's pattern,
 * grad_h[k] = -lambda[row(k)] * u[col(k)] (nnz_A entries), plus lambda_h. */
int chronos_adjoint_grad(chronos_hier *h, const double *u_h, const double *g_h, int itmax,
                         double tol, double *lambda_h, double *grad_h, int *iters);

#ifdef __cplusplus
}
#endif
#endif /* CHRONOS_B200_H */
