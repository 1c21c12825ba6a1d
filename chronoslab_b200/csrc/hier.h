// The AMG hierarchy handle behind chronos_hier: per-level device matrices,
// work vectors, the PCG state and its CUDA graph.
#pragma once

#include <array>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "host/host.h"
#include "internal.h"

namespace chronos {

// DOM or CLA strength of connection and PMIS C/F splitting on the GPU
// (coarsen_gpu.cu) for the device CSR (rp, ci, v) of an n x n level:
// fcnode numbered as the reference numbers it, nc coarse nodes, and S the
// strength pattern (values left empty) for the host prolongation.  Draws n
// numbers from rng, as pmis_split does; bit-identical to soc_matrix(soc_type)
// + pmis_split.
void coarsen_device(int n, const int *rp, const int *ci, const double *v, const char *soc_type,
                    double tau, MT19937 &rng, HostCSR &S, std::vector<int> &fcnode, int *nc_out,
                    cudaStream_t st);

// Outcome of gmres_right_device, as gmres_RIGHT.m returns it.
struct GmresResult {
  int flag = 1, outer = 0, inner = 0;
  double relres = 0.0;
  std::vector<double> resvec;
};

struct Hier;
// Right-preconditioned restarted GMRES (gmres.cu) on device vectors b, x (x0
// on entry), the hierarchy's V-cycle as the preconditioner and apply_op as
// the operator.
void gmres_right_device(Hier &h, const std::function<void(const double *, double *)> &apply_op,
                        const double *b, double *x, int restart, double tol, int maxit,
                        GmresResult &res);

// Square, sorted, in-range, finite CSR, or CHRONOS_EINVAL.
void validate_csr(const HostCSR &A);

// Whether the setup coarsens on the GPU: DOM or CLA strength and
// CHRONOS_GPU_COARSEN not set to 0.
bool gpu_coarsening(const char *soc_type);

struct Level {
  int n = 0, nc = 0;
  bool coarsest = false;
  DMat A, G, Gt, P, Pt;
  DBuf<double> W;                  // coarsest: A^{-1} from the Cholesky factor
  double omega = 1.0, lambda = 0.0;
  // work vectors (one set per precision in use)
  DBuf<float> b32, x32, r32, t32;
  DBuf<double> b64, x64, r64, t64;
  template <typename T> T *b();
  template <typename T> T *x();
  template <typename T> T *r();
  template <typename T> T *t();
};

template <> inline float *Level::b<float>() { return b32.get(); }
template <> inline float *Level::x<float>() { return x32.get(); }
template <> inline float *Level::r<float>() { return r32.get(); }
template <> inline float *Level::t<float>() { return t32.get(); }
template <> inline double *Level::b<double>() { return b64.get(); }
template <> inline double *Level::x<double>() { return x64.get(); }
template <> inline double *Level::r<double>() { return r64.get(); }
template <> inline double *Level::t<double>() { return t64.get(); }

template <typename T> inline const T *vals(const DMat &m);
template <> inline const float *vals<float>(const DMat &m) { return m.v32.get(); }
template <> inline const double *vals<double>(const DMat &m) { return m.v64.get(); }

// Device scalars of the PCG recurrence.
enum PcgScalar {
  SC_BNORM = 0, SC_PTAP, SC_ALPHA, SC_PRES_AXP, SC_RR, SC_RESITER, SC_ITER, SC_TOL, SC_ITMAX,
  SC_BREAKDOWN, SC_PRES, SC_RMAX, SC_REPLACE, SC_RATIO, SC_COUNT = 16
};

struct PcgState {
  int n = 0;
  DBuf<double> x, res, p, axp, pres, resvec;
  DBuf<double> b;                   // copy of the right-hand side (true-residual replacement)
  DBuf<double> sc;                  // SC_COUNT scalars
  DBuf<double> part;                // block partials (3 per block, several slots)
  DBuf<unsigned> tickets;           // one ticket per reducing kernel
  cudaGraphExec_t exec = nullptr;   // the whole solve (device-side loop) or one iteration
  cudaGraph_t graph = nullptr;
  bool conditional = false;
  int resvec_cap = 0;
  double *sc_pinned = nullptr;      // pinned copy of the scalars for queued solves
  ~PcgState();
};

struct BlockState;   // block-of-right-hand-sides solve state (block.cu)

struct Hier {
  chronos_params prm{};
  int precision = CHRONOS_FP32;
  std::vector<Level> levels;
  cudaStream_t st = nullptr;
  // setup timings (s): fsai_pattern, fsai_numeric, omega, coarsen (with the
  // test space), prolong, galerkin, coarse_factor, total, uploads (operators
  // and their block form), layouts (transposes and FP32 copies of G and P),
  // autotune, other (the rest of total)
  std::array<double, 12> times{};
  PcgState pcg;
  // Operator of the outer PCG when the caller passes one (PCG_CJ's prodA,
  // PCG_CJ.m:1): FP64 CSR of the level-1 size; otherwise levels[0].A.
  DMat user_op;
  bool use_user_op = false;
  // events that order st after a caller's stream and the caller's stream after st
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  ~Hier();

  const DMat &outer_A() const { return use_user_op ? user_op : levels[0].A; }
  // Sets (A != nullptr) or clears the outer operator; the PCG graph is
  // rebuilt when the operator in use changes.
  void set_outer_operator(const HostCSR *A);

  // one V-cycle: out = M^{-1} b on device FP64 vectors of length n0;
  // when dw != nullptr also *dot_out = out . dw (deterministic).
  void vcycle(const double *b, double *out, const double *dw, double *dot_out);
  // the same on FP32 device vectors (an FP32 hierarchy reads and writes them
  // directly; an FP64 one through FP64 copies)
  void vcycle_f32(const float *b, float *out);
  // PCG_CJ to tolerance on device vectors; returns iterations, flag.
  void pcg_solve(const double *b, double *x, int itmax, double tol, int *iters, int *flag,
                 std::vector<double> *resvec, double *seconds);
  // the same solve queued on st without host synchronisation (b != 0), and
  // its outcome once st has drained
  void pcg_enqueue(const double *b, double *x, int itmax, double tol);
  void pcg_collect(double tol, int *iters, int *flag) const;
  // y = A x with the level-0 FP64 operator.
  void apply_A(const double *x, double *y);
  // timings and algorithmic bytes of the hot kernels
  void profile(int reps, chronos_profile *out);
  // nrhs <= 16 columns (column-major host blocks) solved together
  void pcg_block(int nrhs, const double *B_h, double *X_h, int itmax, double tol, int *iters,
                 int *flags, double *seconds);
  std::shared_ptr<BlockState> block;
  DBuf<double> stage_b, stage_x;    // host-buffer entry points' device staging
};

// BAMG prolongation with the GPU doing the per-row work (bamg_gpu.cu): the
// result of bamg_prolongation bit for bit; rows whose neighbourhood outgrows
// the GPU's per-thread scratch (max_neigh nodes, 0: chosen by the level's
// size) are computed on the host (their count in *host_rows, may be null).
HostCSR bamg_prolongation_device(const BamgParams &prm, const HostCSR &S,
                                 const std::vector<int> &fc, int nc, const double *TV, int ntv,
                                 std::vector<int> &c_mark, cudaStream_t st,
                                 int *host_rows = nullptr, int max_neigh = 0);
// Whether the setup runs BAMG on the GPU: when CHRONOS_GPU_BAMG=1.
bool gpu_bamg();

// Strength rows for the EMIN pattern (emin_gpu.cu): an explicit S with values
// (S != nullptr, host), or DOM strength with threshold tau computed on the
// fly from the device CSR (arp, aci, av) of an n x n A with nnz entries and
// rows of at most max_row entries (cpt_SoC_dom.m:26-47, prolong.m:213-217).
struct EminStrength {
  const CsrRef *S = nullptr;
  const int *arp = nullptr, *aci = nullptr;
  const double *av = nullptr;
  int n = 0, max_row = 0;
  int64_t nnz = 0;
  double tau = 0.0;
};
// An n x nc EMIN pattern in device memory (values kept when asked for), with
// its row pointers on the host.
struct DevPattern {
  int n = 0, nc = 0, mmax = 0;
  int64_t nnz = 0;
  DBuf<int> rp, ci;
  DBuf<double> v;
  std::vector<int> rp_h;
  HostCSR to_host(cudaStream_t st) const;
};
// MEX_cptProlPatt (MEX_EMIN/MEX_cptProlPatt.cpp:234-490) on the GPU: the
// n x nc EMIN pattern (values as the MEX returns them) from P0 (n x nc,
// ascending columns), fc0 (coarse index or -1) and kpow power steps, with at
// most max(nnzr_max, nnzr_min) entries per row beyond P0's own.  Bit-identical
// to the reference; rows whose candidates outgrow a warp's table are computed
// by emin_pattern_row on the host (their count in *host_rows, may be null).
void emin_pattern_device(int kpow, int n, int nc, const EminStrength &str, const CsrRef &P0,
                         const std::vector<int> &fc0, int nnzr_max, int nnzr_min, bool values,
                         DevPattern &out, cudaStream_t st, int *host_rows = nullptr);
// EMIN parameters of parm_PROLONG (read_prolong.m): itmax_emin, energ_tol,
// condmax_emin, prec_emin, solv_emin, and whether A is symmetric.
struct EminParams {
  int itmax = 10;
  double energ_tol = 1e-3, condmax = 1e10;
  int prec = 1, solv = 4;
  bool spd = true;
};
// EMIN_ImpProl (Cpp_EMIN/EMIN_ImpProl.cpp:84-410) with the matrix-free path
// of EMIN_matfree.cpp on the GPU: P (n x nc) improved on the pattern patt
// (no coarse rows) for the device CSR A (FP64), TVr row-major n x ntv.
// Returns P with unit coarse rows and exact zeros dropped; info[12] as the
// reference's info array (info[6]: rows whose constraint block took the SVD
// branch; info[7]: iterations).
HostCSR emin_device(const EminParams &prm, int n, int nc, const int *arp, const int *aci,
                    const double *av, const CsrRef &Pin, const DevPattern &patt,
                    const std::vector<int> &fc0, const double *TVr, int ntv, cudaStream_t st,
                    double *info);
// Row pointers, columns ascending in [0, ncols) and (when coarse is given)
// no entries in coarse rows, or CHRONOS_EINVAL naming what; rows checked in
// parallel.
void validate_ref(const CsrRef &M, const char *what, const std::vector<int> *coarse = nullptr);
// int32 row pointers of a HostCSR, for a CsrRef over it.
std::vector<int> rp32(const HostCSR &M);

// Source of a level's prolongation outside the library: given the 1-based
// level number and the level's operator (FP64, from the GPU Galerkin product
// on levels > 1), returns P (n x nc, 0-based CSR, sorted rows).
using ProlongFn = std::function<HostCSR(int level, const HostCSR &A)>;

// Orders a handle's work on a caller's CUDA stream: on construction the
// handle's stream waits for what the caller's stream has queued so far; on
// destruction the caller's stream waits for what the handle queued.  Event
// joins only: no device-wide synchronisation.  A null caller stream means
// the legacy default stream.
class CallerStream {
 public:
  CallerStream(Hier &h, void *stream);
  ~CallerStream();
  CallerStream(const CallerStream &) = delete;
  CallerStream &operator=(const CallerStream &) = delete;

 private:
  Hier &h_;
  cudaStream_t caller_;
};

// tune = false leaves the apply kernels' lane counts and formats at their
// defaults; tune_hierarchy then chooses them (timed on a quiet GPU).
// prolong != nullptr takes every level's P from it (coarsening, C/F splitting
// and the prolongation stay with the caller; TV0 is unused); otherwise the
// library's own coarsening and BAMG build P from the test space.
std::unique_ptr<Hier> build_hierarchy(const chronos_params &prm, HostCSR A,
                                      int ntv0, const double *TV0, bool tune = true,
                                      const ProlongFn *prolong = nullptr);
void tune_hierarchy(Hier &h);

// One hierarchy built level by level (what build_hierarchy runs): a level is
// begun (its operator uploaded; the coarsest factored, begin_level then
// returning false; otherwise its FSAI pattern computed on the host and
// uploaded), its FSAI numeric phase run -- alone (fsai_numeric_single) or,
// by a batch setup, together with other builders' (fsai_job) -- and ended
// (omega, coarsening, prolongation, Galerkin product of the next level).
class HierBuilder {
 public:
  HierBuilder(const chronos_params &prm, HostCSR A0, int ntv0, const double *TV0,
              const ProlongFn *prolong = nullptr);
  ~HierBuilder();
  bool begin_level();
  FsaiJob fsai_job() const;
  int fsai_numeric_single();             // returns the flags word
  void add_numeric_time(double seconds); // a batched numeric phase's share
  void end_level(int fsai_flags);
  std::unique_ptr<Hier> finish(bool tune);

 private:
  // time spent inside this builder's calls (its total; waits between calls
  // of a batch setup are not part of it)
  double active_ = 0.0;
  struct Active;
  chronos_params prm_;
  const ProlongFn *prolong_;
  MT19937 rng_;
  std::unique_ptr<Hier> h_;
  bool fp32_ = false;
  int nth_ = 1, ntv_ = 1, level_ = 0;
  std::string pemin_;
  std::vector<double> TV_;
  HostCSR Al_, Gh_;
  std::vector<int> rowlen_;
};

// Serialisation of a built hierarchy (every level's operator, smoother
// factor and prolongation in FP64, omega, lambda_max, the coarsest inverse
// and the parameters), so a later run skips the setup: load rebuilds the
// device layouts (FP32 copies, block form, transposes, autotuned lanes) from
// the stored matrices and gives the same V-cycle bit for bit.
void save_hierarchy(const Hier &h, const char *path);
std::unique_ptr<Hier> load_hierarchy(const char *path);

void params_default(chronos_params *p);
void params_read(const char *fnames_path, chronos_params *p);

// Upload a host CSR (FP64) to a device matrix, with FP32 values when fp32.
void upload_csr(const HostCSR &h, DMat &d, bool fp32, cudaStream_t st);
// T = M' built on the device from M's device arrays (as upload_csr of the
// host transpose would give); Mh: the same matrix on the host, if at hand.
void upload_transpose(const DMat &M, DMat &T, bool fp32, cudaStream_t st,
                      const HostCSR *Mh = nullptr);
// SpMV lane count by timing the candidates (cached per shape).
// format: 0 tuned (row-grouped CSR or sliced ELL), 1 CSR only, 2 sliced ELL
// whenever the rows average at most 16 entries.
void autotune_lanes(DMat &m, bool fp32, cudaStream_t st, int format = 0);
// Lanes per row from the mean row length; setting the lanes also rebuilds the
// matrix's long-row list.
int heuristic_lanes(const DMat &m);
void set_lanes(DMat &m, int L, cudaStream_t st);
// Largest eigenvalue of the symmetric operator given as a device FP64 matvec,
// by Lanczos with a unit start vector; relative tolerance tol.
double lanczos_lmax(int n, const std::function<void(const double *, double *)> &mv, double tol,
                    int maxit, cudaStream_t st);

}  // namespace chronos
