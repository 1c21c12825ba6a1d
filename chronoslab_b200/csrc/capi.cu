// extern "C" boundary of the library (include/chronos_b200.h).  Every entry
// point converts C++ errors into a status code and records the message for
// chronos_last_error(); no exception crosses the boundary.
#include <cstring>
#include <new>
#include <string>

#include "hier.h"
#include "spmv.cuh"
#include <nvtx3/nvToolsExt.h>

namespace {
// NVTX range over one C ABI call (shown by nsys and usable with ncu --nvtx).
struct CallRange {
  explicit CallRange(const char *name) { nvtxRangePushA(name); }
  ~CallRange() { nvtxRangePop(); }
  CallRange(const CallRange &) = delete;
  CallRange &operator=(const CallRange &) = delete;
};
}  // namespace

namespace chronos {

static thread_local std::string g_last_error;
void set_last_error(const std::string &msg) { g_last_error = msg; }

template <typename F>
static int guard(F &&f) {
  try {
    f();
    return CHRONOS_OK;
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc &) {
    set_last_error("host allocation failed");
    return CHRONOS_ENOMEM;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return CHRONOS_EINVAL;
  } catch (...) {
    set_last_error("unknown error");
    return CHRONOS_EINVAL;
  }
}

// 1-based CSR with int64 row pointers (the MEX layout, afsai_cpp.m:26-39) -> HostCSR.
static HostCSR from_mex_csr(int n, int ncols, const int64_t *iat, const int *ja, const double *v) {
  CHRONOS_REQUIRE(n > 0 && iat && ja && v, CHRONOS_EINVAL, "null CSR input");
  CHRONOS_REQUIRE(iat[0] == 1, CHRONOS_EINVAL, "1-based CSR expected (iat[0] == 1)");
  HostCSR h;
  h.nrows = n;
  h.ncols = ncols;
  h.rp.resize((size_t)n + 1);
  for (int i = 0; i <= n; ++i) {
    h.rp[i] = iat[i] - 1;
    CHRONOS_REQUIRE(i == 0 || h.rp[i] >= h.rp[i - 1], CHRONOS_EINVAL, "decreasing row pointers");
  }
  const int64_t nnz = h.rp[n];
  h.ci.resize(nnz);
  h.v.assign(v, v + nnz);
  for (int64_t k = 0; k < nnz; ++k) {
    h.ci[k] = ja[k] - 1;
    CHRONOS_REQUIRE(h.ci[k] >= 0 && h.ci[k] < ncols, CHRONOS_EINVAL, "column index out of range");
  }
  for (int i = 0; i < n; ++i)
    for (int64_t k = h.rp[i] + 1; k < h.rp[i + 1]; ++k)
      CHRONOS_REQUIRE(h.ci[k] > h.ci[k - 1], CHRONOS_EINVAL, "columns must increase within a row");
  return h;
}

static HostCSR from_csr0(int n, int ncols, const int *iat, const int *ja, const double *v) {
  CHRONOS_REQUIRE(n > 0 && iat && (iat[n] == 0 || (ja && v)), CHRONOS_EINVAL, "null CSR input");
  CHRONOS_REQUIRE(iat[0] == 0, CHRONOS_EINVAL, "0-based CSR expected (iat[0] == 0)");
  HostCSR h;
  h.nrows = n;
  h.ncols = ncols;
  h.rp.assign(iat, iat + n + 1);
  const int64_t nnz = h.rp[n];
  for (int i = 0; i < n; ++i)
    CHRONOS_REQUIRE(h.rp[i + 1] >= h.rp[i], CHRONOS_EINVAL, "decreasing row pointers");
  h.ci.assign(ja, ja + nnz);
  h.v.assign(v, v + nnz);
  for (int64_t k = 0; k < nnz; ++k)
    CHRONOS_REQUIRE(h.ci[k] >= 0 && h.ci[k] < ncols, CHRONOS_EINVAL, "column index out of range");
  for (int i = 0; i < n; ++i)
    for (int64_t k = h.rp[i] + 1; k < h.rp[i + 1]; ++k)
      CHRONOS_REQUIRE(h.ci[k] > h.ci[k - 1], CHRONOS_EINVAL,
                      "CSR columns must be strictly increasing within a row");
  return h;
}

// True for memory the device owns (cudaMalloc'd or managed); host memory,
// registered or not, and any pointer when no GPU is present are host memory.
static bool is_device_pointer(const void *p) {
  if (!p) return false;
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice;
}

// from_csr0 for arrays in host or device memory (chronos_amg_setup takes A
// from either, as a MEX caller may hold it on the host or in a gpuArray).
static HostCSR from_csr0_any(int n, int ncols, const int *iat, const int *ja, const double *v) {
  if (!is_device_pointer(iat)) return from_csr0(n, ncols, iat, ja, v);
  CHRONOS_REQUIRE(n > 0, CHRONOS_EINVAL, "n must be positive");
  std::vector<int> rp((size_t)n + 1);
  CHRONOS_CUDA(cudaMemcpy(rp.data(), iat, sizeof(int) * rp.size(), cudaMemcpyDeviceToHost));
  CHRONOS_REQUIRE(rp[0] == 0 && rp[n] >= 0, CHRONOS_EINVAL, "0-based CSR expected (iat[0] == 0)");
  std::vector<int> ci(std::max(rp[n], 1));
  std::vector<double> vv(std::max(rp[n], 1));
  if (rp[n] > 0) {
    CHRONOS_REQUIRE(ja && v, CHRONOS_EINVAL, "null CSR input");
    CHRONOS_CUDA(cudaMemcpy(ci.data(), ja, sizeof(int) * (size_t)rp[n], cudaMemcpyDeviceToHost));
    CHRONOS_CUDA(cudaMemcpy(vv.data(), v, sizeof(double) * (size_t)rp[n], cudaMemcpyDeviceToHost));
  }
  return from_csr0(n, ncols, rp.data(), ci.data(), vv.data());
}

struct ScopedStream {
  cudaStream_t st = nullptr;
  ScopedStream() { CHRONOS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)); }
  ~ScopedStream() { if (st) { cudaStreamSynchronize(st); cudaStreamDestroy(st); } }
};

// Records an event on `from` and makes `to` wait for it.
static void stream_wait(cudaStream_t to, cudaStream_t from) {
  cudaEvent_t e;
  CHRONOS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaError_t r = cudaEventRecord(e, from);
  if (r == cudaSuccess) r = cudaStreamWaitEvent(to, e, 0);
  cudaEventDestroy(e);
  CHRONOS_CUDA(r);
}

// Device-side FSAI numeric phase on a host pattern; vals out in G's order.
// join: the work starts after what the caller's stream (null: the legacy
// default stream) has queued, and that stream waits for the work.
static int fsai_values(const HostCSR &A, const HostCSR &G, std::vector<double> &gval,
                       cudaStream_t caller = nullptr, bool join = false) {
  ScopedStream s;
  if (join) stream_wait(s.st, caller);
  DMat dA, dG;
  upload_csr(A, dA, false, s.st);
  upload_csr(G, dG, false, s.st);
  std::vector<int> rowlen(G.nrows);
  for (int i = 0; i < G.nrows; ++i) {
    rowlen[i] = (int)(G.rp[i + 1] - G.rp[i]);
    CHRONOS_REQUIRE(rowlen[i] >= 1 && G.ci[G.rp[i + 1] - 1] == i, CHRONOS_EINVAL,
                    "FSAI pattern rows must end with their diagonal");
    for (int64_t k = G.rp[i]; k + 1 < G.rp[i + 1]; ++k)
      CHRONOS_REQUIRE(G.ci[k] < i && (k == G.rp[i] || G.ci[k] > G.ci[k - 1]), CHRONOS_EINVAL,
                      "FSAI pattern rows must list strictly-lower columns ascending");
  }
  const int fl = fsai_numeric_device(A.nrows, dA.rp, dA.ci, dA.v64, dG.rp, dG.ci, dG.v64,
                                     rowlen, s.st);
  gval.resize(G.nnz());
  dG.v64.download(gval.data(), G.nnz(), s.st);
  CHRONOS_CUDA(cudaStreamSynchronize(s.st));
  if (join) stream_wait(caller, s.st);
  return fl;
}

}  // namespace chronos

using namespace chronos;

struct chronos_hier {
  std::unique_ptr<Hier> h;
};

struct chronos_galerkin_plan {
  int nc = 0;
  int64_t nnz = 0;
  DBuf<int> rp, ci;
  DBuf<double> v;
};

struct chronos_csr {
  HostCSR m;
};

static chronos_csr *wrap_csr(HostCSR &&m) {
  auto *r = new chronos_csr();
  r->m = std::move(m);
  return r;
}

extern "C" {

int chronos_csr_info(const chronos_csr *m, int *nrows, int *ncols, int64_t *nnz) {
  return guard([&] {
    CHRONOS_REQUIRE(m && nrows && ncols && nnz, CHRONOS_EINVAL, "null argument");
    *nrows = m->m.nrows;
    *ncols = m->m.ncols;
    *nnz = m->m.nnz();
  });
}

int chronos_csr_fetch(const chronos_csr *m, int *iat_h, int *ja_h, double *val_h) {
  return guard([&] {
    CHRONOS_REQUIRE(m && iat_h && ja_h && val_h, CHRONOS_EINVAL, "null argument");
    for (int i = 0; i <= m->m.nrows; ++i) iat_h[i] = (int)m->m.rp[i];
    std::memcpy(ja_h, m->m.ci.data(), sizeof(int) * m->m.ci.size());
    std::memcpy(val_h, m->m.v.data(), sizeof(double) * m->m.v.size());
  });
}

int chronos_csr_free(chronos_csr *m) {
  return guard([&] { delete m; });
}

int chronos_read_matrix_bin(const char *path, chronos_csr **A) {
  return guard([&] {
    CHRONOS_REQUIRE(path && A, CHRONOS_EINVAL, "null argument");
    *A = wrap_csr(read_matrix_bin(path));
  });
}

int chronos_read_ext_bin(const char *path, chronos_csr **A) {
  return guard([&] {
    CHRONOS_REQUIRE(path && A, CHRONOS_EINVAL, "null argument");
    *A = wrap_csr(read_ext_bin(path));
  });
}

int chronos_write_ext_bin(const char *path, int n, int ncols, const int *iat_h, const int *ja_h,
                          const double *val_h) {
  return guard([&] {
    CHRONOS_REQUIRE(path && iat_h && ja_h && val_h && n >= 0 && ncols >= 0, CHRONOS_EINVAL,
                    "bad argument");
    write_ext_bin(path, from_csr0(n, ncols, iat_h, ja_h, val_h));
  });
}

int chronos_read_tv_ext_bin(const char *path, int *n, int *ntv, double *TV_h) {
  return guard([&] {
    CHRONOS_REQUIRE(path && n && ntv, CHRONOS_EINVAL, "null argument");
    std::vector<double> tv;
    read_tv_ext_bin(path, n, ntv, tv);
    if (TV_h && !tv.empty()) std::memcpy(TV_h, tv.data(), sizeof(double) * tv.size());
  });
}

int chronos_write_tv_ext_bin(const char *path, int n, int ntv, const double *TV_h) {
  return guard([&] {
    CHRONOS_REQUIRE(path && (TV_h || (size_t)n * ntv == 0) && n >= 0 && ntv >= 0,
                    CHRONOS_EINVAL, "bad argument");
    write_tv_ext_bin(path, n, ntv, TV_h);
  });
}

int chronos_fsai_pattern(int n, const int *iat_h, const int *ja_h, const double *val_h, int nstep,
                         int step_size, double eps, int nthread, int fsai_fabs, int *is_posdef,
                         chronos_csr **G) {
  return guard([&] {
    CHRONOS_REQUIRE(is_posdef && G, CHRONOS_EINVAL, "null argument");
    CHRONOS_REQUIRE(nstep >= 0 && step_size >= 1 && nstep * step_size <= 64, CHRONOS_EINVAL,
                    "nstep*step_size must be <= 64");
    HostCSR A = from_csr0(n, n, iat_h, ja_h, val_h);
    FsaiResult fr = fsai_adaptive(A, nstep, step_size, eps, nthread > 0 ? nthread : 1,
                                  fsai_fabs == 0);
    *is_posdef = fr.posdef ? 1 : 0;
    *G = wrap_csr(std::move(fr.G));
  });
}

int chronos_coarsen(const chronos_params *prm, int n, const int *iat_h, const int *ja_h,
                    const double *val_h, uint64_t rng_skip, int *fcnode_h, int *nc,
                    chronos_csr **S) {
  return guard([&] {
    CHRONOS_REQUIRE(prm && fcnode_h && nc, CHRONOS_EINVAL, "null argument");
    HostCSR A = from_csr0(n, n, iat_h, ja_h, val_h);
    MT19937 rng((uint32_t)(prm->seed ? prm->seed : 5489));
    for (uint64_t k = 0; k < rng_skip; ++k) rng.next_res53();
    HostCSR Sm = soc_matrix(A, prm->SoC_type, prm->soc_tau);
    std::vector<int> fc = pmis_split(A, Sm, rng, nc);
    std::memcpy(fcnode_h, fc.data(), sizeof(int) * n);
    if (S) *S = wrap_csr(std::move(Sm));
  });
}

int chronos_coarsen_device(const chronos_params *prm, int n, const int *iat_h, const int *ja_h,
                           const double *val_h, uint64_t rng_skip, int *fcnode_h, int *nc,
                           chronos_csr **S) {
  return guard([&] {
    CallRange range_("chronos_coarsen_device");
    CHRONOS_REQUIRE(prm && fcnode_h && nc && n > 0, CHRONOS_EINVAL, "bad argument");
    HostCSR A = from_csr0(n, n, iat_h, ja_h, val_h);
    validate_csr(A);
    MT19937 rng((uint32_t)(prm->seed ? prm->seed : 5489));
    for (uint64_t k = 0; k < rng_skip; ++k) rng.next_res53();
    cudaStream_t st;
    CHRONOS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    try {
      DMat d;
      upload_csr(A, d, false, st);
      HostCSR Sm;
      std::vector<int> fc;
      coarsen_device(n, d.rp, d.ci, d.v64, prm->SoC_type, prm->soc_tau, rng, Sm, fc, nc, st);
      CHRONOS_CUDA(cudaStreamSynchronize(st));
      std::memcpy(fcnode_h, fc.data(), sizeof(int) * n);
      if (S) {
        Sm.v.assign(Sm.ci.size(), 1.0);
        *S = wrap_csr(std::move(Sm));
      }
    } catch (...) {
      cudaStreamDestroy(st);
      throw;
    }
    cudaStreamDestroy(st);
  });
}

static int bamg_entry(const chronos_params *prm, int n, const int *iat_S_h, const int *ja_S_h,
                      const int *fcnode_h, int ntv, const double *TV_h, int *c_mark_h,
                      chronos_csr **P, bool device, int *host_rows, int max_neigh) {
  return guard([&] {
    CHRONOS_REQUIRE(prm && iat_S_h && ja_S_h && fcnode_h && TV_h && P && ntv >= 1 && n > 0,
                    CHRONOS_EINVAL, "bad argument");
    HostCSR S;
    S.nrows = S.ncols = n;
    S.rp.assign(iat_S_h, iat_S_h + n + 1);
    S.ci.assign(ja_S_h, ja_S_h + S.rp[n]);
    S.v.assign(S.rp[n], 1.0);
    std::vector<int> fc0(n);
    int nc = 0;
    for (int i = 0; i < n; ++i) {
      fc0[i] = fcnode_h[i] > 0 ? fcnode_h[i] - 1 : -1;
      if (fcnode_h[i] > 0) ++nc;
    }
    std::vector<double> TVr((size_t)n * ntv);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < ntv; ++j) TVr[(size_t)i * ntv + j] = TV_h[(size_t)j * n + i];
    int nth = prm->prol_np;
    if (nth <= 0) nth = 1;
    BamgParams bp{prm->itmax_vol, prm->dist_min, prm->dist_max, ntv, nth, prm->maxcond,
                  prm->maxrownrm, prm->tol_vol, prm->eps_prol};
    std::vector<int> cm;
    HostCSR Pm;
    if (device) {
      ScopedStream ss;
      Pm = bamg_prolongation_device(bp, S, fc0, nc, TVr.data(), ntv, cm, ss.st, host_rows,
                                    max_neigh);
    } else {
      Pm = bamg_prolongation(bp, S, fc0, nc, TVr.data(), ntv, cm);
    }
    if (c_mark_h) std::memcpy(c_mark_h, cm.data(), sizeof(int) * n);
    *P = wrap_csr(std::move(Pm));
  });
}

int chronos_bamg(const chronos_params *prm, int n, const int *iat_S_h, const int *ja_S_h,
                 const int *fcnode_h, int ntv, const double *TV_h, int *c_mark_h,
                 chronos_csr **P) {
  return bamg_entry(prm, n, iat_S_h, ja_S_h, fcnode_h, ntv, TV_h, c_mark_h, P, false, nullptr, 0);
}

int chronos_bamg_device(const chronos_params *prm, int n, const int *iat_S_h, const int *ja_S_h,
                        const int *fcnode_h, int ntv, const double *TV_h, int *c_mark_h,
                        int max_neigh, chronos_csr **P, int *host_rows) {
  return bamg_entry(prm, n, iat_S_h, ja_S_h, fcnode_h, ntv, TV_h, c_mark_h, P, true, host_rows,
                    max_neigh);
}

// fcnode as chronos_coarsen numbers it (coarse k -> k in 1..nc, fine < 0)
// -> coarse index or -1; nc counted.
static std::vector<int> coarse_index(int n, const int *fcnode_h, int *nc) {
  std::vector<int> fc0(n);
  *nc = 0;
  for (int i = 0; i < n; ++i) {
    fc0[i] = fcnode_h[i] > 0 ? fcnode_h[i] - 1 : -1;
    if (fcnode_h[i] > 0) ++*nc;
  }
  return fc0;
}

int chronos_emin_pattern(int kpow, int n, int nc, const int *iat_S_h, const int *ja_S_h,
                         const double *coef_S_h, const int *iat_P_h, const int *ja_P_h,
                         const double *coef_P_h, const int *fcnode_h, int nnzr_max, int nnzr_min,
                         chronos_csr **patt, int *host_rows) {
  return guard([&] {
    CallRange range_("chronos_emin_pattern");
    CHRONOS_REQUIRE(n > 0 && nc > 0 && nc <= n && fcnode_h && coef_S_h && coef_P_h && patt,
                    CHRONOS_EINVAL, "bad argument");
    const CsrRef S{n, n, iat_S_h, ja_S_h, coef_S_h};
    const CsrRef P{n, nc, iat_P_h, ja_P_h, coef_P_h};
    validate_ref(S, "S");
    validate_ref(P, "P");
    int ncf = 0;
    std::vector<int> fc0 = coarse_index(n, fcnode_h, &ncf);
    CHRONOS_REQUIRE(ncf == nc, CHRONOS_EINVAL, "fcnode must mark exactly nc coarse nodes");
    EminStrength str;
    str.S = &S;
    ScopedStream ss;
    DevPattern dp;
    emin_pattern_device(kpow, n, nc, str, P, fc0, nnzr_max, nnzr_min, true, dp, ss.st,
                        host_rows);
    *patt = wrap_csr(dp.to_host(ss.st));
  });
}

int chronos_emin(const chronos_params *prm, int n, const int *iat_A_h, const int *ja_A_h,
                 const double *coef_A_h, int nc, const int *iat_P_h, const int *ja_P_h,
                 const double *coef_P_h, const int *iat_patt_h, const int *ja_patt_h,
                 const int *fcnode_h, int ntv, const double *TV_h, int spd, chronos_csr **P,
                 double *info) {
  return guard([&] {
    CallRange range_("chronos_emin");
    CHRONOS_REQUIRE(prm && n > 0 && nc > 0 && nc <= n && coef_A_h && coef_P_h && fcnode_h &&
                        TV_h && P && ntv >= 1,
                    CHRONOS_EINVAL, "bad argument");
    const CsrRef A{n, n, iat_A_h, ja_A_h, coef_A_h};
    const CsrRef Pin{n, nc, iat_P_h, ja_P_h, coef_P_h};
    const CsrRef T{n, nc, iat_patt_h, ja_patt_h, nullptr};
    validate_ref(A, "A");
    validate_ref(Pin, "P");
    int ncf = 0;
    std::vector<int> fc0 = coarse_index(n, fcnode_h, &ncf);
    CHRONOS_REQUIRE(ncf == nc, CHRONOS_EINVAL, "fcnode must mark exactly nc coarse nodes");
    validate_ref(T, "pattern", &fc0);
    std::vector<double> TVr((size_t)n * ntv);
#pragma omp parallel for schedule(static, 8192)
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < ntv; ++j) TVr[(size_t)i * ntv + j] = TV_h[(size_t)j * n + i];
    EminParams ep;
    ep.itmax = prm->itmax_emin;
    ep.energ_tol = prm->energ_tol;
    ep.condmax = prm->condmax_emin;
    ep.prec = prm->prec_emin;
    ep.solv = prm->solv_emin;
    ep.spd = spd != 0;
    ScopedStream ss;
    DBuf<int> arp, aci;
    DBuf<double> av;
    arp.upload(iat_A_h, (size_t)n + 1, ss.st);
    aci.upload(ja_A_h, (size_t)A.nnz(), ss.st);
    av.upload(coef_A_h, (size_t)A.nnz(), ss.st);
    DevPattern dp;
    dp.n = n;
    dp.nc = nc;
    dp.rp_h.assign(iat_patt_h, iat_patt_h + n + 1);
    dp.nnz = T.nnz();
    dp.mmax = 0;
    for (int i = 0; i < n; ++i) dp.mmax = std::max(dp.mmax, dp.rp_h[i + 1] - dp.rp_h[i]);
    dp.rp.upload(dp.rp_h, ss.st);
    dp.ci.alloc(std::max<int64_t>(dp.nnz, 1));
    if (dp.nnz)
      CHRONOS_CUDA(cudaMemcpyAsync(dp.ci.get(), ja_patt_h, sizeof(int) * dp.nnz,
                                   cudaMemcpyHostToDevice, ss.st));
    *P = wrap_csr(emin_device(ep, n, nc, arp.get(), aci.get(), av.get(), Pin, dp, fc0,
                              TVr.data(), ntv, ss.st, info));
  });
}

void chronos_params_default(chronos_params *p) {
  if (p) params_default(p);
}

int chronos_params_read(const char *fnames_path, chronos_params *p) {
  return guard([&] {
    CHRONOS_REQUIRE(fnames_path && p, CHRONOS_EINVAL, "null argument");
    params_read(fnames_path, p);
  });
}

int chronos_last_error(char *buf, int len) {
  if (!buf || len <= 0) return CHRONOS_EINVAL;
  std::snprintf(buf, (size_t)len, "%s", g_last_error.c_str());
  return CHRONOS_OK;
}

const char *chronos_version(void) { return "chronos_b200 1.0 (sm_100a)"; }

int chronos_fsai_compute(int nthread, int n_step, int step_size, double tau, double eps,
                         int nrows, int nrows_M, int64_t nterm_M, const int64_t *iat_M_h,
                         const int *ja_M_h, const double *coef_M_h, int64_t *nterm_G,
                         int64_t *iat_G_h, int *ja_G_h, double *coef_G_h, int *is_posdef) {
  return guard([&] {
    CallRange range_("chronos_fsai_compute");
    CHRONOS_REQUIRE(nterm_G && iat_G_h && ja_G_h && coef_G_h && is_posdef, CHRONOS_EINVAL,
                    "null output");
    CHRONOS_REQUIRE(nrows == nrows_M, CHRONOS_ENOTSUP,
                    "trailing-block FSAI (nrows_M > nrows) is outside this path");
    CHRONOS_REQUIRE(tau == 0.0, CHRONOS_ENOTSUP, "FSAI dropping (tau > 0) is outside this path");
    CHRONOS_REQUIRE(n_step >= 0 && step_size >= 1 && n_step * step_size <= 64, CHRONOS_EINVAL,
                    "n_step*step_size must be <= 64");
    HostCSR A = from_mex_csr(nrows, nrows, iat_M_h, ja_M_h, coef_M_h);
    CHRONOS_REQUIRE(A.nnz() == nterm_M, CHRONOS_EINVAL, "nterm_M does not match iat_M");
    FsaiResult fr = fsai_adaptive(A, n_step, step_size, eps, nthread, true);
    std::vector<double> gval;
    const int fl = fsai_values(A, fr.G, gval);
    const HostCSR &G = fr.G;
    for (int i = 0; i <= nrows; ++i) iat_G_h[i] = G.rp[i] + 1;
    for (int64_t k = 0; k < G.nnz(); ++k) {
      ja_G_h[k] = G.ci[k] + 1;
      coef_G_h[k] = gval[k];
    }
    *nterm_G = G.nnz();
    *is_posdef = (fr.posdef && fl == 0) ? 1 : 0;
  });
}

int chronos_fsai_numeric(int n, int base, const int64_t *iat_A_h, const int *ja_A_h,
                         const double *val_A_h, const int64_t *iat_G_h, const int *ja_G_h,
                         int out_precision, void *val_G_h, int *is_posdef, void *stream) {
  return guard([&] {
    CallRange range_("chronos_fsai_numeric");
    CHRONOS_REQUIRE(val_G_h && is_posdef && iat_G_h && ja_G_h && iat_A_h, CHRONOS_EINVAL,
                    "null argument");
    CHRONOS_REQUIRE(base == 0 || base == 1, CHRONOS_EINVAL, "base must be 0 or 1");
    CHRONOS_REQUIRE(out_precision == CHRONOS_FP64 || out_precision == CHRONOS_FP32,
                    CHRONOS_EINVAL, "out_precision must be CHRONOS_FP64 or CHRONOS_FP32");
    CHRONOS_REQUIRE(n > 0 && iat_A_h[0] == base && iat_G_h[0] == base, CHRONOS_EINVAL,
                    "row pointers must start at the given base");
    // the MEX layout shifted to 1-based when the caller's arrays are 0-based
    std::vector<int64_t> ia;
    std::vector<int> ja;
    const int64_t *iat = iat_A_h;
    const int *jat = ja_A_h;
    if (base == 0) {
      ia.assign(iat_A_h, iat_A_h + n + 1);
      for (auto &v : ia) v += 1;
      CHRONOS_REQUIRE(ia[n] >= 1, CHRONOS_EINVAL, "decreasing row pointers");
      ja.assign(ja_A_h, ja_A_h + (ia[n] - 1));
      for (auto &v : ja) v += 1;
      iat = ia.data();
      jat = ja.data();
    }
    HostCSR A = from_mex_csr(n, n, iat, jat, val_A_h);
    HostCSR G;
    G.nrows = G.ncols = n;
    G.rp.resize((size_t)n + 1);
    for (int i = 0; i <= n; ++i) {
      G.rp[i] = iat_G_h[i] - base;
      CHRONOS_REQUIRE(i == 0 || G.rp[i] >= G.rp[i - 1], CHRONOS_EINVAL,
                      "decreasing G row pointers");
    }
    G.ci.resize(G.rp[n]);
    for (int64_t k = 0; k < G.rp[n]; ++k) {
      G.ci[k] = ja_G_h[k] - base;
      CHRONOS_REQUIRE(G.ci[k] >= 0 && G.ci[k] < n, CHRONOS_EINVAL, "G column out of range");
    }
    G.v.assign(G.rp[n], 0.0);
    std::vector<double> gval;
    const int fl = fsai_values(A, G, gval, static_cast<cudaStream_t>(stream), true);
    if (out_precision == CHRONOS_FP64) {
      std::memcpy(val_G_h, gval.data(), sizeof(double) * gval.size());
    } else {
      float *o = static_cast<float *>(val_G_h);
      for (size_t k = 0; k < gval.size(); ++k) o[k] = (float)gval[k];
    }
    *is_posdef = fl == 0 ? 1 : 0;
  });
}

int chronos_fsai_numeric_batch(int nprob, const int *n, const int *const *iat_A_h,
                               const int *const *ja_A_h, const double *const *val_A_h,
                               const int *const *iat_G_h, const int *const *ja_G_h,
                               double *const *val_G_h, int *is_posdef, int tile_set,
                               int *tile_set_used) {
  return guard([&] {
    CallRange range_("chronos_fsai_numeric_batch");
    CHRONOS_REQUIRE(nprob > 0 && n && iat_A_h && ja_A_h && val_A_h && iat_G_h && ja_G_h &&
                        val_G_h && is_posdef, CHRONOS_EINVAL, "null argument");
    CHRONOS_REQUIRE(tile_set >= -1 && tile_set < fsai_bucket_set_count(), CHRONOS_EINVAL,
                    "tile_set must be -1 (tuned) or a candidate index");
    ScopedStream s;
    std::vector<DMat> dA(nprob), dG(nprob);
    std::vector<std::vector<int>> rowlen(nprob);
    std::vector<FsaiJob> jobs(nprob);
    for (int p = 0; p < nprob; ++p) {
      const HostCSR A = from_csr0(n[p], n[p], iat_A_h[p], ja_A_h[p], val_A_h[p]);
      HostCSR G;
      G.nrows = G.ncols = n[p];
      G.rp.assign(iat_G_h[p], iat_G_h[p] + n[p] + 1);
      CHRONOS_REQUIRE(G.rp[0] == 0, CHRONOS_EINVAL, "0-based G pattern expected");
      rowlen[p].resize(n[p]);
      for (int i = 0; i < n[p]; ++i) {
        CHRONOS_REQUIRE(G.rp[i + 1] > G.rp[i], CHRONOS_EINVAL, "a G row without entries");
        rowlen[p][i] = (int)(G.rp[i + 1] - G.rp[i]);
      }
      G.ci.assign(ja_G_h[p], ja_G_h[p] + G.rp[n[p]]);
      G.v.assign(G.ci.size(), 0.0);
      for (int i = 0; i < n[p]; ++i) {
        CHRONOS_REQUIRE(G.ci[G.rp[i + 1] - 1] == i, CHRONOS_EINVAL,
                        "FSAI pattern rows must end with their diagonal");
        for (int64_t k = G.rp[i]; k + 1 < G.rp[i + 1]; ++k)
          CHRONOS_REQUIRE(G.ci[k] >= 0 && G.ci[k] < i && (k == G.rp[i] || G.ci[k] > G.ci[k - 1]),
                          CHRONOS_EINVAL,
                          "FSAI pattern rows must list strictly-lower columns ascending");
      }
      upload_csr(A, dA[p], false, s.st);
      upload_csr(G, dG[p], false, s.st);
      jobs[p] = FsaiJob{n[p], dA[p].rp.get(), dA[p].ci.get(), dA[p].v64.get(), dG[p].rp.get(),
                        dG[p].ci.get(), dG[p].v64.get(), &rowlen[p]};
    }
    int used = -1;
    const std::vector<int> fl = fsai_numeric_batched(jobs, s.st, &used, tile_set);
    for (int p = 0; p < nprob; ++p) {
      dG[p].v64.download(val_G_h[p], dG[p].nnz, s.st);
      is_posdef[p] = fl[p] == 0 ? 1 : 0;
    }
    CHRONOS_CUDA(cudaStreamSynchronize(s.st));
    if (tile_set_used) *tile_set_used = used;
  });
}

int chronos_galerkin_compute(int n, int nc, const int *iat_A_h, const int *ja_A_h,
                             const double *val_A_h, const int *iat_P_h, const int *ja_P_h,
                             const double *val_P_h, int64_t *nnz_Ac, chronos_galerkin_plan **plan) {
  return guard([&] {
    CHRONOS_REQUIRE(plan && nnz_Ac && nc > 0, CHRONOS_EINVAL, "bad argument");
    HostCSR A = from_csr0(n, n, iat_A_h, ja_A_h, val_A_h);
    HostCSR P = from_csr0(n, nc, iat_P_h, ja_P_h, val_P_h);
    for (int i = 0; i < n; ++i)
      for (int64_t k = A.rp[i] + 1; k < A.rp[i + 1]; ++k)
        CHRONOS_REQUIRE(A.ci[k] > A.ci[k - 1], CHRONOS_EINVAL, "A rows must be sorted");
    ScopedStream s;
    DMat dA, dP, dPt;
    upload_csr(A, dA, false, s.st);
    upload_csr(P, dP, false, s.st);
    upload_transpose(dP, dPt, false, s.st, &P);
    DBuf<int> aprp, apci;
    DBuf<double> apv;
    int64_t nnz_ap = 0;
    spgemm_device(n, nc, dA.rp, dA.ci, dA.v64, dP.rp, dP.ci, dP.v64, aprp, apci, apv, &nnz_ap, s.st);
    auto *pl = new chronos_galerkin_plan();
    try {
      pl->nc = nc;
      spgemm_device(nc, nc, dPt.rp, dPt.ci, dPt.v64, aprp, apci, apv, pl->rp, pl->ci, pl->v,
                    &pl->nnz, s.st);
    } catch (...) {
      delete pl;
      throw;
    }
    *nnz_Ac = pl->nnz;
    *plan = pl;
  });
}

int chronos_galerkin_fetch(chronos_galerkin_plan *plan, int *iat_Ac_h, int *ja_Ac_h,
                           double *val_Ac_h) {
  return guard([&] {
    CHRONOS_REQUIRE(plan && iat_Ac_h && ja_Ac_h && val_Ac_h, CHRONOS_EINVAL, "null argument");
    plan->rp.download(iat_Ac_h, (size_t)plan->nc + 1);
    plan->ci.download(ja_Ac_h, plan->nnz);
    plan->v.download(val_Ac_h, plan->nnz);
    CHRONOS_CUDA(cudaDeviceSynchronize());
  });
}

int chronos_galerkin_free(chronos_galerkin_plan *plan) {
  return guard([&] { delete plan; });
}

int chronos_dense_chol(int n, const double *A_h, double *L_h) {
  return guard([&] {
    CHRONOS_REQUIRE(n > 0 && n <= 8192 && A_h && L_h, CHRONOS_EINVAL, "bad argument (n <= 8192)");
    ScopedStream s;
    DBuf<double> d;
    d.upload(A_h, (size_t)n * n, s.st);
    const int info = dense_cholesky_device(n, d.get(), s.st);
    CHRONOS_REQUIRE(info == 0, CHRONOS_ENOTSPD, "non-positive pivot " + std::to_string(info));
    d.download(L_h, (size_t)n * n, s.st);
    CHRONOS_CUDA(cudaStreamSynchronize(s.st));
  });
}

int chronos_spmv(int n, int ncols, const int *iat_h, const int *ja_h, const double *val_h,
                 const double *x_h, double *y_h, int precision, int format, int lanes) {
  return guard([&] {
    CHRONOS_REQUIRE(x_h && y_h, CHRONOS_EINVAL, "null vector");
    CHRONOS_REQUIRE(format >= 0 && format <= 2, CHRONOS_EINVAL, "format must be 0, 1 or 2");
    CHRONOS_REQUIRE(lanes == 0 || lanes == 1 || lanes == 2 || lanes == 4 || lanes == 8 ||
                        lanes == 16 || lanes == 32, CHRONOS_EINVAL,
                    "lanes must be 0, 1, 2, 4, 8, 16 or 32");
    HostCSR A = from_csr0(n, ncols, iat_h, ja_h, val_h);
    ScopedStream s;
    DMat d;
    const bool fp32 = precision == CHRONOS_FP32;
    upload_csr(A, d, fp32, s.st);
    if (lanes > 0 && format != 2) set_lanes(d, lanes, s.st);
    else autotune_lanes(d, fp32, s.st, format);
    if (fp32) {
      std::vector<float> xf(x_h, x_h + ncols), yf(n);
      DBuf<float> x, y(n);
      x.upload(xf, s.st);
      mat_apply<float, float, float, float, MODE_PLAIN, false>(s.st, d, d.v32.get(), x.get(),
                                                              (const float *)nullptr, y.get(),
                                                              1.0f);
      y.download(yf.data(), n, s.st);
      CHRONOS_CUDA(cudaStreamSynchronize(s.st));
      for (int i = 0; i < n; ++i) y_h[i] = yf[i];
    } else {
      DBuf<double> x, y(n);
      x.upload(x_h, ncols, s.st);
      mat_apply<double, double, double, double, MODE_PLAIN, false>(
          s.st, d, d.v64.get(), x.get(), (const double *)nullptr, y.get(), 1.0);
      y.download(y_h, n, s.st);
      CHRONOS_CUDA(cudaStreamSynchronize(s.st));
    }
  });
}

int chronos_amg_setup(const chronos_params *prm, int n, const int *iat_h, const int *ja_h,
                      const double *val_h, int ntv0, const double *TV0_h, chronos_hier **out) {
  return guard([&] {
    CallRange range_("chronos_amg_setup");
    CHRONOS_REQUIRE(prm && out, CHRONOS_EINVAL, "null argument");
    CHRONOS_REQUIRE(ntv0 == 0 || TV0_h, CHRONOS_EINVAL, "TV0 missing");
    HostCSR A = from_csr0_any(n, n, iat_h, ja_h, val_h);
    std::vector<double> tv;
    if (ntv0 > 0 && is_device_pointer(TV0_h)) {
      tv.resize((size_t)n * ntv0);
      CHRONOS_CUDA(cudaMemcpy(tv.data(), TV0_h, sizeof(double) * tv.size(), cudaMemcpyDeviceToHost));
      TV0_h = tv.data();
    }
    auto *hh = new chronos_hier();
    try {
      hh->h = build_hierarchy(*prm, std::move(A), ntv0, TV0_h);
    } catch (...) {
      delete hh;
      throw;
    }
    *out = hh;
  });
}

int chronos_amg_setup_prolong(const chronos_params *prm, int n, const int *iat_h,
                              const int *ja_h, const double *val_h, chronos_prolong_fn prolong,
                              void *ctx, chronos_hier **out) {
  return guard([&] {
    CallRange range_("chronos_amg_setup_prolong");
    CHRONOS_REQUIRE(prm && out && prolong, CHRONOS_EINVAL, "null argument");
    HostCSR A = from_csr0_any(n, n, iat_h, ja_h, val_h);
    const ProlongFn fn = [&](int level, const HostCSR &Al) {
      const int nl = Al.nrows;
      std::vector<int> rp(Al.rp.begin(), Al.rp.end());
      chronos_prolongation P{};
      const int rc = prolong(ctx, level, nl, rp.data(), Al.ci.data(), Al.v.data(), &P);
      CHRONOS_REQUIRE(rc == 0, CHRONOS_EINVAL,
                      "prolongation callback failed at level " + std::to_string(level) +
                          " (returned " + std::to_string(rc) + ")");
      CHRONOS_REQUIRE(P.iat_P_h && P.nc > 0 && P.nc < nl && P.iat_P_h[0] == 0 &&
                          P.iat_P_h[nl] >= 0 && (P.iat_P_h[nl] == 0 || (P.ja_P_h && P.val_P_h)),
                      CHRONOS_EINVAL,
                      "prolongation callback returned no usable P at level " +
                          std::to_string(level) + " (0 < nc < n, 0-based row pointers)");
      return from_csr0(nl, P.nc, P.iat_P_h, P.ja_P_h, P.val_P_h);
    };
    auto *hh = new chronos_hier();
    try {
      hh->h = build_hierarchy(*prm, A, 0, nullptr, true, &fn);
    } catch (...) {
      delete hh;
      throw;
    }
    *out = hh;
  });
}

int chronos_hier_free(chronos_hier *h) {
  return guard([&] { delete h; });
}

int chronos_device_bytes(int64_t *bytes) {
  return guard([&] {
    CHRONOS_REQUIRE(bytes, CHRONOS_EINVAL, "null argument");
    *bytes = device_bytes_live().load();
  });
}

int chronos_hier_save(const chronos_hier *h, const char *path) {
  return guard([&] {
    CHRONOS_REQUIRE(h && path, CHRONOS_EINVAL, "null argument");
    save_hierarchy(*h->h, path);
  });
}

int chronos_hier_load(const char *path, chronos_hier **out) {
  return guard([&] {
    CallRange range_("chronos_hier_load");
    CHRONOS_REQUIRE(path && out, CHRONOS_EINVAL, "null argument");
    auto *hh = new chronos_hier();
    try {
      hh->h = load_hierarchy(path);
    } catch (...) {
      delete hh;
      throw;
    }
    *out = hh;
  });
}

int chronos_hier_nlevels(const chronos_hier *h, int *nlev) {
  return guard([&] {
    CHRONOS_REQUIRE(h && nlev, CHRONOS_EINVAL, "null argument");
    *nlev = (int)h->h->levels.size();
  });
}

int chronos_hier_level_info(const chronos_hier *h, int level, chronos_level_info *info) {
  return guard([&] {
    CHRONOS_REQUIRE(h && info && level >= 0 && level < (int)h->h->levels.size(), CHRONOS_EINVAL,
                    "bad level");
    const Level &L = h->h->levels[level];
    info->n = L.n;
    info->nnz_A = L.A.nnz;
    info->nnz_G = L.coarsest ? 0 : L.G.nnz;
    info->nnz_P = L.coarsest ? 0 : L.P.nnz;
    info->nc = L.coarsest ? 0 : L.nc;
    info->omega = L.omega;
    info->lambda = L.lambda;
    info->threads_per_row = L.A.nb > 0 ? 1 : L.A.lanes;   // block form: a thread per block row
    info->block_rows = L.A.nb;
    info->sell_mask = (L.A.use_sell ? 1 : 0) | (L.G.use_sell ? 2 : 0) | (L.Gt.use_sell ? 4 : 0) |
                      (L.P.use_sell ? 8 : 0) | (L.Pt.use_sell ? 16 : 0);
  });
}

int chronos_hier_dump_ext_bin(const chronos_hier *h, int level, char which, const char *path) {
  int nr = 0, nc = 0;
  int64_t nnz = 0;
  int rc = chronos_hier_export(h, level, which, &nr, &nc, &nnz, nullptr, nullptr, nullptr);
  if (rc != CHRONOS_OK) return rc;
  return guard([&] {
    CHRONOS_REQUIRE(path, CHRONOS_EINVAL, "null path");
    std::vector<int> iat((size_t)nr + 1), ja(std::max<int64_t>(nnz, 1));
    std::vector<double> v(std::max<int64_t>(nnz, 1));
    const int rc2 = chronos_hier_export(h, level, which, &nr, &nc, &nnz, iat.data(), ja.data(),
                                        v.data());
    CHRONOS_REQUIRE(rc2 == CHRONOS_OK, rc2, "export failed");
    write_ext_bin(path, from_csr0(nr, nc, iat.data(), ja.data(), v.data()));
  });
}

int chronos_hier_export(const chronos_hier *h, int level, char which, int *nrows, int *ncols,
                        int64_t *nnz, int *iat_h, int *ja_h, double *val_h) {
  return guard([&] {
    CHRONOS_REQUIRE(h && nrows && ncols && nnz && level >= 0 &&
                        level < (int)h->h->levels.size(), CHRONOS_EINVAL, "bad argument");
    const Level &L = h->h->levels[level];
    const DMat *m = nullptr;
    if (which == 'A') m = &L.A;
    else if (which == 'G' && !L.coarsest) m = &L.G;
    else if (which == 'P' && !L.coarsest) m = &L.P;
    CHRONOS_REQUIRE(m, CHRONOS_EINVAL, "matrix not available on this level");
    *nrows = m->nrows;
    *ncols = m->ncols;
    *nnz = m->nnz;
    if (!iat_h || !ja_h || !val_h) return;
    m->rp.download(iat_h, (size_t)m->nrows + 1, h->h->st);
    m->ci.download(ja_h, m->nnz, h->h->st);
    m->v64.download(val_h, m->nnz, h->h->st);
    CHRONOS_CUDA(cudaStreamSynchronize(h->h->st));
  });
}

int chronos_hier_setup_phases(const chronos_hier *h, double *t, int n) {
  return guard([&] {
    CHRONOS_REQUIRE(h && t && n >= 0, CHRONOS_EINVAL, "bad argument");
    for (int i = 0; i < n && i < (int)h->h->times.size(); ++i) t[i] = h->h->times[i];
  });
}

int chronos_hier_setup_times(const chronos_hier *h, double *t8) {
  return guard([&] {
    CHRONOS_REQUIRE(h && t8, CHRONOS_EINVAL, "null argument");
    for (int i = 0; i < 8; ++i) t8[i] = h->h->times[i];
  });
}

int chronos_hier_profile(chronos_hier *hh, int reps, chronos_profile *out) {
  return guard([&] {
    CHRONOS_REQUIRE(hh && out, CHRONOS_EINVAL, "null argument");
    hh->h->profile(reps, out);
  });
}

int chronos_diag_fix(int n, const int *iat_h, const int *ja_h, double *val_h) {
  return guard([&] {
    HostCSR A = from_csr0(n, n, iat_h, ja_h, val_h);
    ScopedStream s;
    DMat d;
    upload_csr(A, d, false, s.st);
    auto mv = [&](const double *x, double *y) {
      csr_apply<double, double, double, double, MODE_PLAIN, false>(s.st, 8, n, d.rp, d.ci, d.v64, x,
                                                                  nullptr, y, 1.0);
    };
    // |lambda|_max of A (eigs(A,1,'lm'), A SPD: the largest eigenvalue)
    const double lmax = lanczos_lmax(n, mv, 1e-3, 300, s.st);
    for (int i = 0; i < n; ++i)
      for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
        if (A.ci[k] == i && val_h[k] == 1.0) val_h[k] = lmax / 10.0;
  });
}

int chronos_vcycle(chronos_hier *hh, const double *b_h, double *x_h, int nrhs, void *stream) {
  return guard([&] {
    CallRange range_("chronos_vcycle");
    CHRONOS_REQUIRE(hh && b_h && x_h && nrhs >= 1, CHRONOS_EINVAL, "bad argument");
    Hier &h = *hh->h;
    const int n = h.levels[0].n;
    if (h.stage_b.size() < (size_t)n) { h.stage_b.alloc(n); h.stage_x.alloc(n); }
    CallerStream order(h, stream);
    for (int c = 0; c < nrhs; ++c) {
      h.stage_b.upload(b_h + (size_t)c * n, n, h.st);
      h.vcycle(h.stage_b.get(), h.stage_x.get(), nullptr, nullptr);
      h.stage_x.download(x_h + (size_t)c * n, n, h.st);
    }
    CHRONOS_CUDA(cudaStreamSynchronize(h.st));
  });
}

int chronos_vcycle_dev(chronos_hier *hh, int io_precision, const void *b_d, void *x_d, int nrhs,
                       void *stream) {
  return guard([&] {
    CallRange range_("chronos_vcycle_dev");
    CHRONOS_REQUIRE(hh && b_d && x_d && nrhs >= 1, CHRONOS_EINVAL, "bad argument");
    CHRONOS_REQUIRE(io_precision == CHRONOS_FP64 || io_precision == CHRONOS_FP32, CHRONOS_EINVAL,
                    "io_precision must be CHRONOS_FP64 or CHRONOS_FP32");
    Hier &h = *hh->h;
    const size_t n = (size_t)h.levels[0].n;
    CallerStream order(h, stream);
    for (int c = 0; c < nrhs; ++c) {
      if (io_precision == CHRONOS_FP64)
        h.vcycle(static_cast<const double *>(b_d) + c * n, static_cast<double *>(x_d) + c * n,
                 nullptr, nullptr);
      else
        h.vcycle_f32(static_cast<const float *>(b_d) + c * n, static_cast<float *>(x_d) + c * n);
    }
  });
}

int chronos_pcg_dev(chronos_hier *hh, const double *b_d, double *x_d, int itmax, double tol,
                    int *iters, double *resvec_h, int *flag, double *seconds, void *stream) {
  return guard([&] {
    CallRange range_("chronos_pcg_dev");
    CHRONOS_REQUIRE(hh && b_d && x_d && iters && flag, CHRONOS_EINVAL, "null argument");
    std::vector<double> rv;
    int it = 0, fl = 0;
    CallerStream order(*hh->h, stream);
    try {
      hh->h->pcg_solve(b_d, x_d, itmax, tol, &it, &fl, resvec_h ? &rv : nullptr, seconds);
    } catch (const Error &e) {
      *iters = it;
      *flag = 1;
      throw;
    }
    *iters = it;
    *flag = fl;
    if (resvec_h) std::memcpy(resvec_h, rv.data(), sizeof(double) * rv.size());
  });
}

int chronos_pcg(chronos_hier *hh, const int *iat_h, const int *ja_h, const double *val_h,
                const double *b_h, double *x_h, int itmax, double tol, int *iters,
                double *resvec_h, int *flag, double *seconds, void *stream) {
  return guard([&] {
    CallRange range_("chronos_pcg");
    CHRONOS_REQUIRE(hh && b_h && x_h && iters && flag, CHRONOS_EINVAL, "null argument");
    Hier &h = *hh->h;
    const int n = h.levels[0].n;
    // the caller's operator serves this call only: later calls (and the
    // other entry points) apply the hierarchy's level-1 operator again
    struct OperatorScope {
      Hier &h;
      ~OperatorScope() {
        try { h.set_outer_operator(nullptr); } catch (...) {}
      }
    } op_scope{h};
    if (iat_h) {
      const HostCSR op = from_csr0(n, n, iat_h, ja_h, val_h);
      h.set_outer_operator(&op);
    }
    // staging buffers live with the handle: no allocation per call
    if (h.stage_b.size() < (size_t)n) { h.stage_b.alloc(n); h.stage_x.alloc(n); }
    CallerStream order(h, stream);
    DBuf<double> &b = h.stage_b, &x = h.stage_x;
    b.upload(b_h, n, h.st);
    x.upload(x_h, n, h.st);
    std::vector<double> rv;
    int it = 0, fl = 0;
    h.pcg_solve(b.get(), x.get(), itmax, tol, &it, &fl, resvec_h ? &rv : nullptr, seconds);
    x.download(x_h, n, h.st);
    CHRONOS_CUDA(cudaStreamSynchronize(h.st));
    *iters = it;
    *flag = fl;
    if (resvec_h) std::memcpy(resvec_h, rv.data(), sizeof(double) * rv.size());
  });
}

int chronos_pcg_block(chronos_hier *hh, int nrhs, const double *B_h, double *X_h, int itmax,
                      double tol, int *iters_h, int *flags_h, double *seconds, void *stream) {
  return guard([&] {
    CallRange range_("chronos_pcg_block");
    CHRONOS_REQUIRE(hh && B_h && X_h && iters_h && flags_h && nrhs >= 1, CHRONOS_EINVAL,
                    "bad argument");
    Hier &h = *hh->h;
    const int n = h.levels[0].n;
    CallerStream order(h, stream);
    double total = 0.0;
    // chunks of at most 16 columns, each one SpMM block solve
    for (int c0 = 0; c0 < nrhs; c0 += 16) {
      const int m = std::min(16, nrhs - c0);
      double sec = 0.0;
      h.pcg_block(m, B_h + (size_t)c0 * n, X_h + (size_t)c0 * n, itmax, tol, iters_h + c0,
                  flags_h + c0, &sec);
      total += sec;
    }
    if (seconds) *seconds = total;
  });
}

int chronos_sqmr(chronos_hier *hh, const int *iat_h, const int *ja_h, const double *val_h,
                 const double *b_h, double *x_h, int itmax, double tol, int *iters,
                 double *relres, int *info) {
  return guard([&] {
    CallRange range_("chronos_sqmr");
    CHRONOS_REQUIRE(hh && b_h && x_h && iters && relres && info, CHRONOS_EINVAL, "null argument");
    Hier &h = *hh->h;
    cudaStream_t st = h.st;
    const int n = h.levels[0].n;
    DMat op;
    if (iat_h) {
      upload_csr(from_csr0(n, n, iat_h, ja_h, val_h), op, false, st);
      autotune_lanes(op, false, st);
    }
    auto apply_op = [&](const double *x, double *y) {
      if (!iat_h) { h.apply_A(x, y); return; }
      csr_apply<double, double, double, double, MODE_PLAIN, false>(st, op.lanes, n, op.rp, op.ci,
                                                                  op.v64, x, nullptr, y, 1.0);
    };
    DBuf<double> rhs, pnew, r(n), q(n), d(n), vscr(n), u(n), tmp(n), scratch(256);
    rhs.upload(b_h, n, st);
    pnew.upload(x_h, n, st);
    d.zero(st);
    auto dot = [&](const double *a, const double *b) { return device_dot(n, a, b, scratch.get(), st); };
    auto lprec = [&](const double *in, double *out) { h.vcycle(in, out, nullptr, nullptr); };
    // SQMR.m:24-36
    const double bnorm = std::sqrt(dot(rhs.get(), rhs.get()));
    apply_op(pnew.get(), tmp.get());
    device_scale_copy(n, 1.0, rhs.get(), r.get(), st);
    device_axpby(n, -1.0, tmp.get(), 1.0, r.get(), st);
    lprec(r.get(), vscr.get());
    device_scale_copy(n, 1.0, vscr.get(), q.get(), st);
    double tau = std::sqrt(dot(vscr.get(), vscr.get()));
    double rho0 = dot(r.get(), q.get());
    double theta0 = 0.0;
    int niter = 0, inf = 0;
    bool exit_test = false;
    while (!exit_test && niter < itmax) {
      ++niter;
      apply_op(q.get(), vscr.get());
      const double sigma = dot(q.get(), vscr.get());
      if (std::fabs(sigma) < 1e-20 * rho0) { inf = 10; break; }
      const double alpha = rho0 / sigma;
      device_axpby(n, -alpha, vscr.get(), 1.0, r.get(), st);
      lprec(r.get(), vscr.get());
      const double theta1 = std::sqrt(dot(vscr.get(), vscr.get())) / tau;
      const double gamma = 1.0 / std::sqrt(1.0 + theta1 * theta1);
      tau = tau * theta1 * gamma;
      // d = d*gamma^2*theta0^2 + gamma^2*alpha*q
      device_axpby(n, gamma * gamma * alpha, q.get(), gamma * gamma * theta0 * theta0, d.get(), st);
      theta0 = theta1;
      device_axpby(n, 1.0, d.get(), 1.0, pnew.get(), st);
      const double resnorm = std::sqrt(dot(r.get(), r.get())) / bnorm;
      if (resnorm < tol) {
        exit_test = true;
      } else {
        device_scale_copy(n, 1.0, vscr.get(), u.get(), st);
        const double rho1 = dot(r.get(), u.get());
        if (std::fabs(rho0) < 1e-20 * rho1) { inf = 20; break; }
        const double beta = rho1 / rho0;
        rho0 = rho1;
        device_axpby(n, 1.0, u.get(), beta, q.get(), st);
      }
    }
    if (niter >= itmax) inf = 1;
    apply_op(pnew.get(), tmp.get());
    device_axpby(n, 1.0, rhs.get(), -1.0, tmp.get(), st);
    *relres = std::sqrt(dot(tmp.get(), tmp.get())) / bnorm;
    *iters = niter;
    *info = inf;
    pnew.download(x_h, n, st);
    CHRONOS_CUDA(cudaStreamSynchronize(st));
  });
}

int chronos_gmres(chronos_hier *hh, const int *iat_h, const int *ja_h, const double *val_h,
                  const double *b_h, double *x_h, int restart, double tol, int maxit,
                  int *iter_outer, int *iter_inner, double *relres, int *flag,
                  double *resvec_h, int *nresvec) {
  return guard([&] {
    CallRange range_("chronos_gmres");
    CHRONOS_REQUIRE(hh && b_h && x_h && iter_outer && iter_inner && relres && flag,
                    CHRONOS_EINVAL, "null argument");
    CHRONOS_REQUIRE(restart >= 0 && maxit >= 0, CHRONOS_EINVAL, "restart and maxit must be >= 0");
    Hier &h = *hh->h;
    cudaStream_t st = h.st;
    const int n = h.levels[0].n;
    DMat op;
    if (iat_h) {
      upload_csr(from_csr0(n, n, iat_h, ja_h, val_h), op, false, st);
      autotune_lanes(op, false, st);
    }
    auto apply_op = [&](const double *x, double *y) {
      if (!iat_h) { h.apply_A(x, y); return; }
      csr_apply<double, double, double, double, MODE_PLAIN, false>(st, op.lanes, n, op.rp, op.ci,
                                                                  op.v64, x, nullptr, y, 1.0);
    };
    DBuf<double> b, x;
    b.upload(b_h, n, st);
    x.upload(x_h, n, st);
    GmresResult r;
    gmres_right_device(h, apply_op, b.get(), x.get(), restart, tol, maxit, r);
    x.download(x_h, n, st);
    CHRONOS_CUDA(cudaStreamSynchronize(st));
    *iter_outer = r.outer;
    *iter_inner = r.inner;
    *relres = r.relres;
    *flag = r.flag;
    if (nresvec) *nresvec = (int)r.resvec.size();
    if (resvec_h) std::memcpy(resvec_h, r.resvec.data(), sizeof(double) * r.resvec.size());
  });
}

int chronos_adjoint_grad(chronos_hier *hh, const double *u_h, const double *g_h, int itmax,
                         double tol, double *lambda_h, double *grad_h, int *iters) {
  return guard([&] {
    CallRange range_("chronos_adjoint_grad");
    CHRONOS_REQUIRE(hh && u_h && g_h && lambda_h && grad_h && iters, CHRONOS_EINVAL, "null argument");
    Hier &h = *hh->h;
    const int n = h.levels[0].n;
    const DMat &A = h.levels[0].A;
    DBuf<double> u, g, lam(n), grad(std::max<int64_t>(A.nnz, 1));
    u.upload(u_h, n, h.st);
    g.upload(g_h, n, h.st);
    lam.zero(h.st);
    int it = 0, fl = 0;
    h.pcg_solve(g.get(), lam.get(), itmax, tol, &it, &fl, nullptr, nullptr);
    adjoint_scatter(n, A.rp, A.ci, lam.get(), u.get(), grad.get(), h.st);
    lam.download(lambda_h, n, h.st);
    grad.download(grad_h, A.nnz, h.st);
    CHRONOS_CUDA(cudaStreamSynchronize(h.st));
    *iters = it;
    CHRONOS_REQUIRE(fl == 0, CHRONOS_EBREAKDOWN, "adjoint solve did not converge");
  });
}

}  // extern "C"
