// AMG hierarchy on the GPU: setup orchestration (cpt_aspAMG.m), the V-cycle
// (AMG_Vcycle.m) and the outer PCG_CJ loop (PCG_CJ.m) as one CUDA graph.
//
// Setup per level (cpt_aspAMG.m:87-347, filters off):
//   host  adaptive FSAI pattern search          smoother.m:35 -> afsai_cpp
//   GPU   FSAI numeric phase (FP64 local solves) cpt_afsai_coef.cpp:440-541
//   GPU   lambda_max(G A G') by Lanczos -> omega = min(1, 1.9/lambda)   smoother.m:73-81
//   host  test space qr (tspace NONE), SoC + PMIS, BAMG prolongation
//   GPU   Galerkin Ac = P'(A P) (FP64, Gustavson order)                   cpt_aspAMG.m:277
//   GPU   coarsest: dense FP64 Cholesky and inverse                      cpt_aspAMG.m:107-116
// The stored hierarchy is FP32 (values of A_l, G_l, G_l', P_l, P_l' with FP32
// accumulation) or FP64; the outer PCG, its dot products, the level-1 operator
// used by PCG and the coarsest solve stay FP64.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <cstdio>
#include <cstdlib>
#include <sys/stat.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include <nvtx3/nvToolsExt.h>

#include "hier.h"
#include "spmv.cuh"

namespace chronos {

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// One phase of the setup: adds its wall time to *acc and marks an NVTX range
// of the same name, so timeline tools (nsys, ncu --nvtx) show the phases.
class SetupPhase {
 public:
  SetupPhase(const char *name, double *acc) : t0_(now_s()), acc_(acc) { nvtxRangePushA(name); }
  SetupPhase(const SetupPhase &) = delete;
  SetupPhase &operator=(const SetupPhase &) = delete;
  ~SetupPhase() { end(); }
  void end() {
    if (!acc_) return;
    *acc_ += now_s() - t0_;
    acc_ = nullptr;
    nvtxRangePop();
  }

 private:
  double t0_;
  double *acc_;
};

PcgState::~PcgState() {
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  if (sc_pinned) cudaFreeHost(sc_pinned);
}

Hier::~Hier() {
  if (st) cudaStreamSynchronize(st);
  levels.clear();
  if (pcg.exec) { cudaGraphExecDestroy(pcg.exec); pcg.exec = nullptr; }
  if (pcg.graph) { cudaGraphDestroy(pcg.graph); pcg.graph = nullptr; }
  if (ev_in) cudaEventDestroy(ev_in);
  if (ev_out) cudaEventDestroy(ev_out);
  if (st) cudaStreamDestroy(st);
}

CallerStream::CallerStream(Hier &h, void *stream)
    : h_(h), caller_(static_cast<cudaStream_t>(stream)) {
  if (!h_.ev_in) CHRONOS_CUDA(cudaEventCreateWithFlags(&h_.ev_in, cudaEventDisableTiming));
  if (!h_.ev_out) CHRONOS_CUDA(cudaEventCreateWithFlags(&h_.ev_out, cudaEventDisableTiming));
  CHRONOS_CUDA(cudaEventRecord(h_.ev_in, caller_));
  CHRONOS_CUDA(cudaStreamWaitEvent(h_.st, h_.ev_in, 0));
}

CallerStream::~CallerStream() {
  // runs on normal return and on error: the caller's stream never overtakes
  // work the handle queued
  if (cudaEventRecord(h_.ev_out, h_.st) == cudaSuccess)
    cudaStreamWaitEvent(caller_, h_.ev_out, 0);
}

// ---------------------------------------------------------------------------
// Device matrices
// ---------------------------------------------------------------------------

// Matrices of at least this many entries get their 16-bit column offsets and
// their transposes built on the device; smaller ones on the host, where the
// device path's temporary allocations and synchronisations cost more (the
// batch setup builds many small levels from several host threads).
constexpr int64_t kDeviceLayoutNnz = 1 << 20;

// 16-bit column offsets on the host (rows without entries: base 0); false
// when a row spans 65536 columns or more.
static bool offsets16_host(const HostCSR &h, std::vector<int> &base, std::vector<uint16_t> &off) {
  base.assign(std::max(h.nrows, 1), 0);
  int fits = h.nrows > 0;
#pragma omp parallel for schedule(static, 4096) reduction(&& : fits)
  for (int i = 0; i < h.nrows; ++i) {
    if (h.rp[i] == h.rp[i + 1]) continue;
    int lo = h.ci[h.rp[i]], hi = lo;
    for (int64_t k = h.rp[i] + 1; k < h.rp[i + 1]; ++k) {
      lo = std::min(lo, h.ci[k]);
      hi = std::max(hi, h.ci[k]);
    }
    base[i] = lo;
    fits = fits && hi - lo <= 0xffff;
  }
  if (!fits) return false;
  off.assign(std::max<int64_t>(h.nnz(), 1), 0);
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < h.nrows; ++i)
    for (int64_t k = h.rp[i]; k < h.rp[i + 1]; ++k) off[k] = (uint16_t)(h.ci[k] - base[i]);
  return true;
}

// FP32 copy, 16-bit column offsets (every row spanning fewer than 65536
// columns: 2 index bytes per entry plus a 4-byte base per row; from the host
// arrays h when given, else on the device) and the lane heuristic of a CSR
// whose arrays are on the device and whose row pointers are in rp_h.
static void finish_csr(DMat &d, const HostCSR *h, bool fp32, cudaStream_t st) {
  if (fp32) {
    d.v32.alloc(std::max<int64_t>(d.nnz, 1));
    convert_f64_to_f32(d.nnz, d.v64.get(), d.v32.get(), st);
  }
  if (h) {
    std::vector<int> base;
    std::vector<uint16_t> off;
    d.idx16 = offsets16_host(*h, base, off);
    if (d.idx16) {
      d.cbase.upload(base, st);
      d.c16.upload(off, st);
    }
  } else {
    d.idx16 = csr_offsets16_device(d.nrows, d.nnz, d.rp.get(), d.ci.get(), d.cbase, d.c16, st);
  }
  if (!d.idx16) {
    d.cbase.release();
    d.c16.release();
  }
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  set_lanes(d, heuristic_lanes(d), st);
}

void upload_csr(const HostCSR &h, DMat &d, bool fp32, cudaStream_t st) {
  CHRONOS_REQUIRE(h.nnz() < INT32_MAX, CHRONOS_ENOTSUP, "matrix with 2^31 or more entries");
  d.nrows = h.nrows;
  d.ncols = h.ncols;
  d.nnz = h.nnz();
  d.rp_h.assign(h.rp.begin(), h.rp.end());
  d.rp.upload(d.rp_h, st);
  d.ci.upload(h.ci, st);
  d.v64.upload(h.v, st);
  finish_csr(d, d.nnz >= kDeviceLayoutNnz ? nullptr : &h, fp32, st);
}

static HostCSR download_csr(int nrows, int ncols, const DBuf<int> &rp, const DBuf<int> &ci,
                            const DBuf<double> &v, int64_t nnz, cudaStream_t st);

// M' of a device CSR: the pattern and values that uploading csr_transpose of
// the host matrix gives (built on the device for large matrices).  Mh, when
// given, is the same matrix on the host (values included), which spares a
// small matrix its download.
void upload_transpose(const DMat &M, DMat &T, bool fp32, cudaStream_t st, const HostCSR *Mh) {
  if (M.nnz < kDeviceLayoutNnz) {
    if (Mh)
      upload_csr(csr_transpose(*Mh), T, fp32, st);
    else
      upload_csr(csr_transpose(download_csr(M.nrows, M.ncols, M.rp, M.ci, M.v64, M.nnz, st)), T,
                 fp32, st);
    return;
  }
  T.nrows = M.ncols;
  T.ncols = M.nrows;
  T.nnz = M.nnz;
  csr_transpose_device(M.nrows, M.ncols, M.nnz, M.rp.get(), M.ci.get(), M.v64.get(), T.rp, T.ci,
                       T.v64, st);
  T.rp_h.resize((size_t)T.nrows + 1);
  T.rp.download(T.rp_h.data(), (size_t)T.nrows + 1, st);
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  finish_csr(T, nullptr, fp32, st);
}

int heuristic_lanes(const DMat &m) {
  const double avg = m.nrows ? (double)m.nnz / m.nrows : 1.0;
  int L = 2;
  while (L < 32 && L < avg * 0.75) L <<= 1;
  return L;
}

// Rows longer than thresh go to the warp path (both apply forms read the list).
static void set_long_rows(DMat &m, int thresh, cudaStream_t st) {
  m.lthresh = thresh;
  std::vector<int> rows;
  m.nnz_long = 0;
  if (thresh < 0x7fffffff)
    for (int i = 0; i < m.nrows; ++i)
      if (m.rp_h[i + 1] - m.rp_h[i] > thresh) {
        rows.push_back(i);
        m.nnz_long += m.rp_h[i + 1] - m.rp_h[i];
      }
  m.nlong = (int)rows.size();
  if (m.nlong) {
    m.longrows.upload(rows, st);
    CHRONOS_CUDA(cudaStreamSynchronize(st));
  }
}

void set_lanes(DMat &m, int L, cudaStream_t st) {
  m.lanes = L;
  set_long_rows(m, long_row_threshold(L), st);
}

// Bytes written between timed launches of the autotuners (more than L2).
constexpr size_t kL2FlushBytes = 256u << 20;

// Rows longer than this are left out of the sliced ELL chunks.
constexpr int kSellLongRow = 32;

// Builds the sliced ELL form (DMat::use_sell) from the matrix's final values.
// Returns false (nothing attached) when the slot count does not fit int32.
static bool build_sell(DMat &m, bool fp32, cudaStream_t st) {
  const int n = m.nrows;
  const std::vector<int> ci = m.ci.to_host(st);
  const std::vector<double> v = m.v64.to_host(st);
  auto len = [&](int i) { return m.rp_h[i + 1] - m.rp_h[i]; };
  // chunks in row order (output accesses stay coalesced); the padding to each
  // chunk's longest row is part of what the autotuner times
  std::vector<int> order;
  order.reserve(n);
  for (int i = 0; i < n; ++i)
    if (len(i) <= kSellLongRow) order.push_back(i);
  const int nch = (int)((order.size() + 31) / 32);
  std::vector<int> choff(nch + 1, 0), chw(nch, 0), cbase(nch, 0), perm((size_t)nch * 32, -1);
  int64_t tot = 0;
  bool fits16 = true;
  for (int c = 0; c < nch; ++c) {
    int w = 0, lo = 0x7fffffff, hi = -1;
    for (int l = 0; l < 32 && 32 * (size_t)c + l < order.size(); ++l) {
      const int row = order[32 * (size_t)c + l];
      perm[32 * (size_t)c + l] = row;
      w = std::max(w, len(row));
      for (int k = m.rp_h[row]; k < m.rp_h[row + 1]; ++k) {
        lo = std::min(lo, ci[k]);
        hi = std::max(hi, ci[k]);
      }
    }
    cbase[c] = hi >= 0 ? lo : 0;
    if (hi >= 0 && hi - lo > 0xffff) fits16 = false;
    choff[c] = (int)tot;
    chw[c] = w;
    tot += 32LL * w;
    if (tot >= INT32_MAX) return false;
  }
  choff[nch] = (int)tot;
  std::vector<double> sv(std::max<int64_t>(tot, 1), 0.0);
  std::vector<int> sci;
  std::vector<uint16_t> s16;
  if (fits16) s16.assign(std::max<int64_t>(tot, 1), 0);
  else sci.assign(std::max<int64_t>(tot, 1), 0);
  for (int c = 0; c < nch; ++c)
    for (int l = 0; l < 32; ++l) {
      const int row = perm[32 * (size_t)c + l];
      if (row < 0) continue;
      for (int j = 0; j < len(row); ++j) {
        const int64_t k = choff[c] + 32LL * j + l;
        const int e = m.rp_h[row] + j;
        sv[k] = v[e];
        if (fits16) s16[k] = (uint16_t)(ci[e] - cbase[c]);
        else sci[k] = ci[e];
      }
    }
  m.s_nchunk = nch;
  m.sell16 = fits16;
  m.s_choff.upload(choff, st);
  m.s_chw.upload(chw, st);
  m.s_cbase.upload(cbase, st);
  m.s_perm.upload(perm, st);
  if (fits16) { m.s_c16.upload(s16, st); m.s_ci.release(); }
  else { m.s_ci.upload(sci, st); m.s_c16.release(); }
  m.s_v64.upload(sv, st);
  if (fp32) {
    m.s_v32.alloc(sv.size());
    convert_f64_to_f32((int64_t)sv.size(), m.s_v64.get(), m.s_v32.get(), st);
  }
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  return true;
}

static void drop_sell(DMat &m) {
  m.use_sell = false;
  m.s_nchunk = 0;
  for (auto *b : {&m.s_choff, &m.s_chw, &m.s_cbase, &m.s_perm, &m.s_ci}) b->release();
  m.s_c16.release();
  m.s_v64.release();
  m.s_v32.release();
}


// Autotuner of the lanes per row (CSR) or per block row (BSR3): times each
// candidate on the matrix itself and keeps the fastest.  Decisions are cached
// per matrix signature (format, rows, entries, columns, precision, longest
// row -- G and G' share the first five but not their row lengths) in memory
// and in a text file (CHRONOS_TUNE_CACHE, default ~/.cache/chronos_b200_tune.txt;
// lines "v2 kind rows entries columns fp32 longest decision", other lines
// ignored) so later processes on the machine -- a profiler run included --
// reuse them.
namespace {
using TuneKey = std::tuple<char, int, int64_t, int, bool, int>;
std::mutex g_tune_mu;
std::map<TuneKey, int> g_tune;
bool g_tune_loaded = false;

std::string tune_path() {
  if (const char *p = std::getenv("CHRONOS_TUNE_CACHE")) return p;
  const char *home = std::getenv("HOME");
  return std::string(home ? home : "/tmp") + "/.cache/chronos_b200_tune.txt";
}

void tune_load_locked() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  FILE *f = std::fopen(tune_path().c_str(), "r");
  if (!f) return;
  char line[256];
  while (std::fgets(line, sizeof(line), f)) {
    char kind;
    int nr, nc, fp, mx, L;
    long long nnz;
    if (std::sscanf(line, "v2 %c %d %lld %d %d %d %d", &kind, &nr, &nnz, &nc, &fp, &mx, &L) == 7)
      g_tune[TuneKey(kind, nr, (int64_t)nnz, nc, fp != 0, mx)] = L;
  }
  std::fclose(f);
}

void tune_store_locked(const TuneKey &k, int L) {
  g_tune[k] = L;
  const std::string path = tune_path();
  const auto slash = path.find_last_of('/');
  if (slash != std::string::npos) {
    const std::string dir = path.substr(0, slash);
    // create the directory without a shell
    for (size_t i = 1; i <= dir.size(); ++i)
      if (i == dir.size() || dir[i] == '/') mkdir(dir.substr(0, i).c_str(), 0755);
  }
  if (FILE *f = std::fopen(path.c_str(), "a")) {
    std::fprintf(f, "v2 %c %d %lld %d %d %d %d\n", std::get<0>(k), std::get<1>(k),
                 (long long)std::get<2>(k), std::get<3>(k), std::get<4>(k) ? 1 : 0,
                 std::get<5>(k), L);
    std::fclose(f);
  }
}

}  // namespace

void autotune_lanes(DMat &m, bool fp32, cudaStream_t st, int format) {
  if (m.nrows <= 0) return;
  // 'H': the hybrid CSR kernel (k_csrh_apply); the index width is part of the
  // shape.  A cached value is lanes + 100 * form (decoded at the end).
  int maxrow = 0;
  for (int i = 0; i < m.nrows; ++i) maxrow = std::max(maxrow, m.rp_h[i + 1] - m.rp_h[i]);
  const TuneKey key(m.idx16 ? 'h' : 'H', m.nrows, m.nnz, m.ncols, fp32, maxrow);
  int L = -1;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load_locked();
    auto it = g_tune.find(key);
    if (it != g_tune.end()) L = it->second;
  }
  const bool verbose = std::getenv("CHRONOS_TUNE_VERBOSE") != nullptr;
  if (L < 0) {
    L = heuristic_lanes(m);
    if (m.nnz >= 4096) {                    // below: launch-latency bound, keep the heuristic
      DBuf<double> x64(m.ncols), y64(m.nrows);
      DBuf<float> x32(m.ncols), y32(m.nrows);
      x64.zero(st);
      x32.zero(st);
      cudaEvent_t e0, e1;
      CHRONOS_CUDA(cudaEventCreate(&e0));
      CHRONOS_CUDA(cudaEventCreate(&e1));
      auto launch = [&] {
        if (fp32)
          mat_apply<float, float, float, float, MODE_PLAIN, false>(st, m, m.v32.get(), x32.get(),
                                                                  (const float *)nullptr,
                                                                  y32.get(), 1.0f);
        else
          mat_apply<double, double, double, double, MODE_PLAIN, false>(
              st, m, m.v64.get(), x64.get(), (const double *)nullptr, y64.get(), 1.0);
      };
      // In the V-cycle an operator is read after larger ones have passed
      // through L2, so each timed launch starts from a flushed L2.
      DBuf<char> flush(kL2FlushBytes);
      auto time_it = [&] {
        launch();
        float tmin = 1e30f;
        for (int r = 0; r < 5; ++r) {
          CHRONOS_CUDA(cudaMemsetAsync(flush.get(), r, kL2FlushBytes, st));
          CHRONOS_CUDA(cudaEventRecord(e0, st));
          launch();
          CHRONOS_CUDA(cudaEventRecord(e1, st));
          CHRONOS_CUDA(cudaEventSynchronize(e1));
          float ms = 0;
          CHRONOS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
          tmin = std::min(tmin, ms);
        }
        return tmin * 4;          // per four launches, as reported below
      };
      float best = 1e30f;
      for (int cand : {1, 2, 4, 8, 16, 32}) {
        set_lanes(m, cand, st);
        const float t = time_it();
        if (verbose)
          std::fprintf(stderr, "chronos tune: csr %d x %d (%lld) lanes %d  %.4f ms\n", m.nrows,
                       m.ncols, (long long)m.nnz, cand, t / 4);
        if (t < best) { best = t; L = cand; }
      }
      if (format == 0 && (double)m.nnz <= 16.0 * m.nrows && build_sell(m, fp32, st)) {
        m.use_sell = true;
        set_long_rows(m, kSellLongRow, st);
        const float t = time_it();
        if (verbose)
          std::fprintf(stderr, "chronos tune: csr %d x %d (%lld) sliced ELL  %.4f ms\n",
                       m.nrows, m.ncols, (long long)m.nnz, t / 4);
        if (t < best) L += 100;
        drop_sell(m);
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_store_locked(key, L);
  }
  // L = lanes + 100 * form: 0 row-grouped CSR, 1 sliced ELL
  int form = L / 100;
  const int lanes = L % 100;
  if (format == 1) form = 0;
  if (format == 2 && form == 0 && (double)m.nnz <= 16.0 * m.nrows) form = 1;
  if (form == 1 && build_sell(m, fp32, st)) {
    m.use_sell = true;
    m.lanes = lanes;
    set_long_rows(m, kSellLongRow, st);
  } else {
    set_lanes(m, lanes, st);
  }
}

// Sliced 3x3 block form of a CSR matrix whose row triples share a pattern of
// whole, aligned 3x3 blocks (structural zeros included); layout as
// k_sell3_apply reads it.
// Block lengths of the 3x3 block form, or empty when A has none.
static std::vector<int> block_row_lengths(const HostCSR &A) {
  if (A.nrows % 3 != 0 || A.ncols % 3 != 0 || A.nrows == 0) return {};
  const int nb = A.nrows / 3;
  std::vector<int> blen(nb);
  int ok = 1;
#pragma omp parallel for schedule(static, 4096) reduction(&& : ok)
  for (int I = 0; I < nb; ++I) {
    const int64_t len = A.rp[3 * I + 1] - A.rp[3 * I];
    bool good = len % 3 == 0;
    for (int r = 1; r < 3 && good; ++r) good = A.rp[3 * I + r + 1] - A.rp[3 * I + r] == len;
    const int64_t s0 = A.rp[3 * I];
    for (int64_t k = 0; k < len && good; k += 3) {
      const int c = A.ci[s0 + k];
      good = c % 3 == 0;
      for (int r = 0; r < 3 && good; ++r)
        for (int cc = 0; cc < 3 && good; ++cc) good = A.ci[A.rp[3 * I + r] + k + cc] == c + cc;
    }
    blen[I] = good ? (int)(len / 3) : 0;
    ok = ok && good;
  }
  if (!ok) return {};
  return blen;
}

// Layout for T threads per block row: chunks of C = 32/T block rows, each
// padded to its longest row rounded up to a multiple of T; slot j of row l
// at off_c + (j/T)*32 + (j%T)*C + l; chw = padded width / T.  Returns false
// when the slot count does not fit int32.
static bool sell3_offsets(const std::vector<int> &blen, int T, std::vector<int> &choff,
                          std::vector<int> &chw) {
  const int nb = (int)blen.size();
  const int C = 32 / T;
  const int nchunk = (nb + C - 1) / C;
  choff.assign((size_t)nchunk + 1, 0);
  chw.assign(nchunk, 0);
  for (int c = 0; c < nchunk; ++c) {
    int w = 0;
    for (int l = 0; l < C && C * c + l < nb; ++l) w = std::max(w, blen[C * c + l]);
    w = (w + T - 1) / T;
    chw[c] = w;
    const int64_t next = (int64_t)choff[c] + 32LL * w;
    if (next >= INT32_MAX) return false;
    choff[c + 1] = (int)next;
  }
  return true;
}

// Block row I's blocks into their slots (a thread per block row): the block
// column and the nine values, plane-major, from the device CSR whose row
// triples share one pattern of aligned 3x3 blocks.  Padding slots stay as
// set before (zero values, block column 0).
__global__ void k_fill_sell3(int nb, int T, const int *__restrict__ blen,
                             const int *__restrict__ choff, const int *__restrict__ rp,
                             const int *__restrict__ ci, const double *__restrict__ v,
                             int64_t nslots, int *__restrict__ sci, double *__restrict__ planes) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= nb) return;
  const int C = 32 / T;
  const int c = I / C, l = I % C;
  const int r0 = rp[3 * I], r1 = rp[3 * I + 1], r2 = rp[3 * I + 2];
  const int64_t base = choff[c];
  for (int j = 0; j < blen[I]; ++j) {
    const int64_t slot = base + 32LL * (j / T) + (int64_t)(j % T) * C + l;
    sci[slot] = ci[r0 + 3 * j] / 3;
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) {
      planes[(int64_t)cc * nslots + slot] = v[r0 + 3 * j + cc];
      planes[(int64_t)(3 + cc) * nslots + slot] = v[r1 + 3 * j + cc];
      planes[(int64_t)(6 + cc) * nslots + slot] = v[r2 + 3 * j + cc];
    }
  }
}

// Builds d's sliced 3x3 block form for T threads per block row on the
// device, from src's device CSR (src and d may be the same matrix).
static void upload_sell3(const DMat &src, const std::vector<int> &blen, int T, DMat &d,
                         bool fp32, cudaStream_t st) {
  std::vector<int> choff, chw;
  if (!sell3_offsets(blen, T, choff, chw)) return;
  const int nb = (int)blen.size();
  const int64_t nslots = choff.back();
  DBuf<int> blen_d;
  blen_d.upload(blen, st);
  d.nb = nb;
  d.sell_T = T;
  d.nchunk = (int)chw.size();
  d.nnzb = 0;
  for (int l : blen) d.nnzb += l;
  d.nslots = nslots;
  d.choff.upload(choff, st);
  d.chw.upload(chw, st);
  d.sci.alloc(std::max<int64_t>(nslots, 1));
  d.bv64.alloc(std::max<int64_t>(9 * nslots, 1));
  CHRONOS_CUDA(cudaMemsetAsync(d.sci.get(), 0, sizeof(int) * std::max<int64_t>(nslots, 1), st));
  CHRONOS_CUDA(cudaMemsetAsync(d.bv64.get(), 0,
                               sizeof(double) * std::max<int64_t>(9 * nslots, 1), st));
  k_fill_sell3<<<ceil_div(nb, 256), 256, 0, st>>>(nb, T, blen_d.get(), d.choff.get(), src.rp.get(),
                                                  src.ci.get(), src.v64.get(), nslots,
                                                  d.sci.get(), d.bv64.get());
  CHRONOS_CHECK_LAUNCH();
  if (fp32) {
    d.bv32.alloc(std::max<int64_t>(9 * nslots, 1));
    convert_f64_to_f32(9 * nslots, d.bv64.get(), d.bv32.get(), st);
  }
  CHRONOS_CUDA(cudaStreamSynchronize(st));
}

static void launch_pcg_spmv(cudaStream_t st, const DMat &A, bool fp32vals, const double *p,
                            const double *res, double *axp, double *part, unsigned *tick,
                            double *sc);

// Attaches the sliced block form with the fastest threads-per-block-row.
// The layout serves the V-cycle's residuals (two per cycle, hierarchy
// precision) and the outer PCG's A p (FP64 accumulation, stored FP32 values
// in FP32 hierarchies), so a candidate is timed on that mix: two residual
// applies and one outer product.  Cached like the CSR lanes.
static void attach_sell3(const HostCSR &A, DMat &d, bool fp32, cudaStream_t st) {
  const std::vector<int> blen = block_row_lengths(A);
  if (blen.empty()) return;
  const TuneKey key('B', (int)blen.size(), A.nnz(), A.ncols, fp32,
                    *std::max_element(blen.begin(), blen.end()));
  int T = -1;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load_locked();
    auto it = g_tune.find(key);
    if (it != g_tune.end()) T = it->second;
  }
  if (T < 0) {
    DBuf<double> x64(A.ncols), y64(A.nrows), p64(A.ncols), q64(A.nrows), part(3 * 2048),
        sc(SC_COUNT);
    DBuf<float> x32(A.ncols), y32(A.nrows);
    DBuf<unsigned> tick(1);
    DBuf<char> flush(kL2FlushBytes);
    x64.zero(st);
    x32.zero(st);
    p64.zero(st);
    tick.zero(st);
    float best = 1e30f;
    cudaEvent_t e0, e1;
    CHRONOS_CUDA(cudaEventCreate(&e0));
    CHRONOS_CUDA(cudaEventCreate(&e1));
    DMat winner;                                    // the fastest layout, kept for d
    for (int t : {1, 2, 4}) {
      DMat probe;
      upload_sell3(d, blen, t, probe, fp32, st);
      auto launch = [&] {
        for (int k = 0; k < 2; ++k) {
          if (fp32)
            sell3_apply<float, float, float, float, MODE_PLAIN, false>(
                st, t, probe.nb, probe.nchunk, probe.choff, probe.chw, probe.sci,
                probe.bv32.get(), probe.nslots, x32.get(), (const float *)nullptr, y32.get(),
                1.0f);
          else
            sell3_apply<double, double, double, double, MODE_PLAIN, false>(
                st, t, probe.nb, probe.nchunk, probe.choff, probe.chw, probe.sci,
                probe.bv64.get(), probe.nslots, x64.get(), (const double *)nullptr, y64.get(),
                1.0);
        }
        launch_pcg_spmv(st, probe, fp32, p64.get(), p64.get(), q64.get(), part.get(),
                        tick.get(), sc.get());
      };
      launch();
      float tmin = 1e30f;
      for (int r = 0; r < 3; ++r) {
        CHRONOS_CUDA(cudaMemsetAsync(flush.get(), r, kL2FlushBytes, st));
        CHRONOS_CUDA(cudaEventRecord(e0, st));
        launch();
        CHRONOS_CUDA(cudaEventRecord(e1, st));
        CHRONOS_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        CHRONOS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        tmin = std::min(tmin, 4 * ms);
      }
      if (std::getenv("CHRONOS_TUNE_VERBOSE")) {
        // the two parts alone, for the record
        auto part_time = [&](bool outer) {
          float m = 1e30f;
          for (int r = 0; r < 3; ++r) {
            CHRONOS_CUDA(cudaMemsetAsync(flush.get(), r, kL2FlushBytes, st));
            CHRONOS_CUDA(cudaEventRecord(e0, st));
            if (outer)
              launch_pcg_spmv(st, probe, fp32, p64.get(), p64.get(), q64.get(), part.get(),
                              tick.get(), sc.get());
            else if (fp32)
              sell3_apply<float, float, float, float, MODE_PLAIN, false>(
                  st, t, probe.nb, probe.nchunk, probe.choff, probe.chw, probe.sci,
                  probe.bv32.get(), probe.nslots, x32.get(), (const float *)nullptr, y32.get(),
                  1.0f);
            else
              sell3_apply<double, double, double, double, MODE_PLAIN, false>(
                  st, t, probe.nb, probe.nchunk, probe.choff, probe.chw, probe.sci,
                  probe.bv64.get(), probe.nslots, x64.get(), (const double *)nullptr,
                  y64.get(), 1.0);
            CHRONOS_CUDA(cudaEventRecord(e1, st));
            CHRONOS_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            CHRONOS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            m = std::min(m, ms);
          }
          return m;
        };
        const float tr = part_time(false), to = part_time(true);
        std::fprintf(stderr,
                     "chronos tune: block form T=%d  %.4f ms per residual pair + outer "
                     "(residual %.4f, outer %.4f ms alone)\n",
                     t, tmin / 4, tr, to);
      }
      if (tmin < best) {
        best = tmin;
        T = t;
        winner = std::move(probe);
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      tune_store_locked(key, T);
    }
    // the timed layout becomes d's block form (no second build and upload)
    d.nb = winner.nb;
    d.sell_T = winner.sell_T;
    d.nchunk = winner.nchunk;
    d.nnzb = winner.nnzb;
    d.nslots = winner.nslots;
    d.choff = std::move(winner.choff);
    d.chw = std::move(winner.chw);
    d.sci = std::move(winner.sci);
    d.bv64 = std::move(winner.bv64);
    d.bv32 = std::move(winner.bv32);
    return;
  }
  upload_sell3(d, blen, T, d, fp32, st);
}

template <typename T> inline const T *bvals(const DMat &m);
template <> inline const float *bvals<float>(const DMat &m) { return m.bv32.get(); }
template <> inline const double *bvals<double>(const DMat &m) { return m.bv64.get(); }

// Operator apply through the block form when the matrix has one.
template <typename T, typename XT, typename ZT, typename YT, int MODE, bool DOT>
static void op_apply(cudaStream_t st, const DMat &A, const XT *x, const ZT *z, YT *y, T alpha,
                     const double *dw = nullptr, double *part = nullptr, unsigned *tick = nullptr,
                     double *dot_out = nullptr) {
  if (A.nb > 0)
    sell3_apply<T, XT, ZT, YT, MODE, DOT>(st, A.sell_T, A.nb, A.nchunk, A.choff, A.chw, A.sci,
                                          bvals<T>(A), A.nslots, x, z, y, alpha, dw, part, tick,
                                          dot_out);
  else
    mat_apply<T, XT, ZT, YT, MODE, DOT>(st, A, vals<T>(A), x, z, y, alpha, dw, part, tick,
                                        dot_out);
}

// ---------------------------------------------------------------------------
// Lanczos estimate of lambda_max (replaces eigs(...,'la', tol) / 'lm')
// ---------------------------------------------------------------------------

// Largest eigenvalue of the symmetric tridiagonal (a, b) by Sturm bisection.
static double tridiag_lmax(const std::vector<double> &a, const std::vector<double> &b) {
  const int m = (int)a.size();
  double lo = 1e300, hi = -1e300;
  for (int i = 0; i < m; ++i) {
    double r = (i > 0 ? std::fabs(b[i - 1]) : 0.0) + (i + 1 < m ? std::fabs(b[i]) : 0.0);
    lo = std::min(lo, a[i] - r);
    hi = std::max(hi, a[i] + r);
  }
  auto count_below = [&](double x) {   // eigenvalues < x
    int c = 0;
    double d = 1.0;
    for (int i = 0; i < m; ++i) {
      double bb = i > 0 ? b[i - 1] * b[i - 1] : 0.0;
      d = a[i] - x - (i > 0 ? bb / d : 0.0);
      if (d == 0.0) d = -1e-300;
      if (d < 0) ++c;
    }
    return c;
  };
  for (int it = 0; it < 200 && hi - lo > 1e-15 * std::max(std::fabs(hi), 1e-300); ++it) {
    double mid = 0.5 * (lo + hi);
    if (count_below(mid) >= m) hi = mid; else lo = mid;
  }
  return hi;
}

// |last component| of the unit eigenvector of the symmetric tridiagonal (a, b)
// for its largest eigenvalue theta: inverse iteration with the shift
// theta + delta, which leaves T - shift negative definite, so the LDL'
// recurrence of each solve needs no pivoting.
static double tridiag_last_component(const std::vector<double> &a, const std::vector<double> &b,
                                     double theta) {
  const int m = (int)a.size();
  if (m == 1) return 1.0;
  double scale = 0.0;
  for (int i = 0; i < m; ++i) scale = std::max(scale, std::fabs(a[i]));
  const double shift = theta + 1e-10 * std::max(scale, std::fabs(theta)) + 1e-300;
  std::vector<double> y(m, 1.0 / std::sqrt((double)m)), d(m), l(m);
  for (int i = 0; i < m; ++i) {           // LDL' of T - shift
    d[i] = a[i] - shift - (i > 0 ? l[i - 1] * l[i - 1] * d[i - 1] : 0.0);
    if (d[i] == 0.0) d[i] = -1e-300;
    if (i + 1 < m) l[i] = b[i] / d[i];
  }
  for (int it = 0; it < 3; ++it) {
    for (int i = 1; i < m; ++i) y[i] -= l[i - 1] * y[i - 1];
    for (int i = 0; i < m; ++i) y[i] /= d[i];
    for (int i = m - 2; i >= 0; --i) y[i] -= l[i] * y[i + 1];
    double nrm = 0.0;
    for (int i = 0; i < m; ++i) nrm += y[i] * y[i];
    nrm = std::sqrt(nrm);
    if (!(nrm > 0.0) || !std::isfinite(nrm)) return 1.0;
    for (int i = 0; i < m; ++i) y[i] /= nrm;
  }
  return std::fabs(y[m - 1]);
}

// Largest eigenvalue of the operator mv by Lanczos.  The start vector is
// random, as eigs' default is (here uniform in [-1/2, 1/2) from MT19937
// seeded 5489, normalised, so the value is reproducible): a structured start
// such as the ones vector can be nearly orthogonal to the top eigenvector --
// on Cubo_4820's operator it first converges to an eigenvalue 15 % below the
// largest.  Stops as ARPACK's dsaupd does for eigs(...,opts.tol): once the
// Ritz pair's residual norm beta_j |s_j| (s the unit eigenvector of the
// tridiagonal for theta) is at most tol |theta|.
double lanczos_lmax(int n, const std::function<void(const double *, double *)> &mv, double tol,
                    int maxit, cudaStream_t st) {
  DBuf<double> v(n), vp(n), w(n), scratch(256);
  std::vector<double> v0(n);
  {
    MT19937 r(5489u);
    double nrm = 0.0;
    for (int i = 0; i < n; ++i) {
      v0[i] = r.next_res53() - 0.5;
      nrm += v0[i] * v0[i];
    }
    nrm = std::sqrt(nrm);
    for (int i = 0; i < n; ++i) v0[i] /= nrm;
  }
  v.upload(v0, st);
  vp.zero(st);
  std::vector<double> a, b;
  double theta = 0.0, beta = 0.0;
  for (int j = 0; j < maxit; ++j) {
    mv(v.get(), w.get());
    const double alpha = device_dot(n, w.get(), v.get(), scratch.get(), st);
    device_axpby(n, -alpha, v.get(), 1.0, w.get(), st);
    if (j > 0) device_axpby(n, -beta, vp.get(), 1.0, w.get(), st);
    a.push_back(alpha);
    beta = std::sqrt(std::max(device_dot(n, w.get(), w.get(), scratch.get(), st), 0.0));
    const double th = tridiag_lmax(a, b);
    const bool conv = beta * tridiag_last_component(a, b, th) <= tol * std::fabs(th);
    theta = th;
    if (conv || beta <= 1e-300 * std::fabs(theta)) break;
    b.push_back(beta);
    std::swap(vp, v);                     // vp <- v
    device_scale_copy(n, 1.0 / beta, w.get(), v.get(), st);
  }
  return theta;
}

// ---------------------------------------------------------------------------
// Setup
// ---------------------------------------------------------------------------

static void alloc_vectors(Level &L, int precision, cudaStream_t st) {
  const size_t n = std::max(L.n, 1);
  if (precision == CHRONOS_FP32) {
    L.b32.alloc(n); L.x32.alloc(n); L.r32.alloc(n); L.t32.alloc(n);
    L.b32.zero(st); L.x32.zero(st); L.r32.zero(st); L.t32.zero(st);
  } else {
    L.b64.alloc(n); L.x64.alloc(n); L.r64.alloc(n); L.t64.alloc(n);
    L.b64.zero(st); L.x64.zero(st); L.r64.zero(st); L.t64.zero(st);
  }
}

static HostCSR download_csr(int nrows, int ncols, const DBuf<int> &rp, const DBuf<int> &ci,
                            const DBuf<double> &v, int64_t nnz, cudaStream_t st) {
  HostCSR h;
  h.nrows = nrows;
  h.ncols = ncols;
  std::vector<int> r(nrows + 1);
  rp.download(r.data(), nrows + 1, st);
  h.ci.resize(nnz);
  h.v.resize(nnz);
  ci.download(h.ci.data(), nnz, st);
  v.download(h.v.data(), nnz, st);
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  h.rp.assign(r.begin(), r.end());
  return h;
}

void validate_csr(const HostCSR &A) {
  CHRONOS_REQUIRE(A.nrows > 0 && A.ncols == A.nrows, CHRONOS_EINVAL, "matrix must be square, n > 0");
  CHRONOS_REQUIRE((int64_t)A.rp.size() == (int64_t)A.nrows + 1 && A.rp[0] == 0, CHRONOS_EINVAL,
                  "malformed CSR row pointers");
  CHRONOS_REQUIRE((int64_t)A.ci.size() >= A.rp[A.nrows] && (int64_t)A.v.size() >= A.rp[A.nrows],
                  CHRONOS_EINVAL, "malformed CSR row pointers");
  // rows checked in parallel; the first failure kind found is reported
  int bad = 0;
#pragma omp parallel for schedule(static, 4096) reduction(| : bad)
  for (int i = 0; i < A.nrows; ++i) {
    if (A.rp[i + 1] < A.rp[i]) { bad |= 1; continue; }
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      if (A.ci[k] < 0 || A.ci[k] >= A.ncols) bad |= 2;
      else if (k > A.rp[i] && A.ci[k] <= A.ci[k - 1]) bad |= 4;
      if (!std::isfinite(A.v[k])) bad |= 8;
    }
  }
  CHRONOS_REQUIRE(!(bad & 1), CHRONOS_EINVAL, "CSR row pointers must not decrease");
  CHRONOS_REQUIRE(!(bad & 2), CHRONOS_EINVAL, "CSR column out of range");
  CHRONOS_REQUIRE(!(bad & 4), CHRONOS_EINVAL, "CSR columns must be strictly increasing within a row");
  CHRONOS_REQUIRE(!(bad & 8), CHRONOS_EINVAL, "non-finite matrix entry");
}

// Jacobi-smoothed prolongation (prolong.m:180-196, prol_emin = SMOOTH):
// P - omega*DA*P with DA = diag(diag(A))\A, omega = 1.9/lambda_max(DA).
// lambda_max by Lanczos on D^{-1/2} A D^{-1/2} (the spectrum of DA; eigs'
// tolerance 1e-3); (omega*DA)*P -- DA's entries a_ik/a_ii scaled by omega, as
// MATLAB evaluates the expression left to right -- by the GPU SpGEMM; the
// difference, with exact zeros dropped, on the host.
static HostCSR smooth_prolongation(const HostCSR &A, const DMat &dA, const HostCSR &P,
                                   cudaStream_t st) {
  const int n = A.nrows;
  std::vector<double> d(n, 0.0), dm(n);
  for (int i = 0; i < n; ++i)
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] == i) d[i] = A.v[k];
  for (int i = 0; i < n; ++i) {
    CHRONOS_REQUIRE(d[i] > 0.0, CHRONOS_ENOTSPD,
                    "prolongation smoothing: non-positive diagonal entry at row " +
                        std::to_string(i + 1));
    dm[i] = 1.0 / std::sqrt(d[i]);
  }
  DBuf<double> ddm, t1(n), t2(n);
  ddm.upload(dm, st);
  auto mv = [&](const double *v, double *w) {
    device_diag_mul(n, ddm.get(), v, t1.get(), st);
    csr_apply<double, double, double, double, MODE_PLAIN, false>(
        st, 8, n, dA.rp, dA.ci, dA.v64, t1.get(), (const double *)nullptr, t2.get(), 1.0);
    device_diag_mul(n, ddm.get(), t2.get(), w, st);
  };
  const double lam = lanczos_lmax(n, mv, 1e-3, 300, st);
  const double omega = 1.9 / lam;
  HostCSR W = A;
  for (int i = 0; i < n; ++i)
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) W.v[k] = omega * (A.v[k] / d[i]);
  DMat dW, dP;
  upload_csr(W, dW, false, st);
  upload_csr(P, dP, false, st);
  DBuf<int> wrp, wci;
  DBuf<double> wv;
  int64_t nnz = 0;
  spgemm_device(n, P.ncols, dW.rp, dW.ci, dW.v64, dP.rp, dP.ci, dP.v64, wrp, wci, wv, &nnz, st);
  const HostCSR WP = download_csr(n, P.ncols, wrp, wci, wv, nnz, st);
  HostCSR Ps;
  Ps.nrows = n;
  Ps.ncols = P.ncols;
  Ps.rp.assign(1, 0);
  std::vector<std::pair<int, double>> row;
  for (int i = 0; i < n; ++i) {
    row.clear();
    for (int64_t k = P.rp[i]; k < P.rp[i + 1]; ++k) row.emplace_back(P.ci[k], P.v[k]);
    std::sort(row.begin(), row.end(),
              [](const std::pair<int, double> &a, const std::pair<int, double> &b) {
                return a.first < b.first;
              });
    size_t a = 0;
    int64_t b = WP.rp[i];
    const int64_t be = WP.rp[i + 1];
    while (a < row.size() || b < be) {
      int c;
      double v;
      if (b >= be || (a < row.size() && row[a].first < WP.ci[b])) {
        c = row[a].first; v = row[a].second; ++a;
      } else if (a >= row.size() || WP.ci[b] < row[a].first) {
        c = WP.ci[b]; v = -WP.v[b]; ++b;
      } else {
        c = row[a].first; v = row[a].second - WP.v[b]; ++a; ++b;
      }
      if (v != 0.0) {
        Ps.ci.push_back(c);
        Ps.v.push_back(v);
      }
    }
    Ps.rp.push_back((int64_t)Ps.ci.size());
  }
  return Ps;
}

// Off by default: on C2 (elasticity 80^3) the host restatement on the box's
// host threads builds the three prolongations in 0.56 s, the GPU in 0.70 s
// (kernels 0.21, 0.17 and 0.07 s; coarse levels have few rows and large
// neighbourhoods).
bool gpu_bamg() {
  static const bool on = [] {
    const char *e = std::getenv("CHRONOS_GPU_BAMG");
    return e && e[0] == '1';
  }();
  return on;
}

bool gpu_coarsening(const char *soc_type) {
  static const bool on = [] {
    const char *e = std::getenv("CHRONOS_GPU_COARSEN");
    return !(e && e[0] == '0');
  }();
  std::string t(soc_type);
  for (auto &c : t) c = (char)toupper(c);
  return on && (t == "DOM" || t == "CLA");
}

// Adds the duration of a builder call to its active time.
struct HierBuilder::Active {
  double &acc;
  double t0;
  explicit Active(double &a) : acc(a), t0(now_s()) {}
  ~Active() { acc += now_s() - t0; }
};

HierBuilder::HierBuilder(const chronos_params &prm_in, HostCSR A0, int ntv0,
                         const double *TV0, const ProlongFn *prolong)
    : prm_(prm_in), prolong_(prolong),
      rng_((uint32_t)(prm_in.seed ? prm_in.seed : 5489)) {
  Active act(active_);
  const chronos_params &prm = prm_;
  validate_csr(A0);
  std::string smeth(prm.smoother_method), tmeth(prm.tspace_method), ptype(prm.proltype),
      pemin(prm.prol_emin);
  for (auto *s : {&smeth, &tmeth, &ptype, &pemin})
    for (auto &c : *s) c = (char)toupper(c);
  pemin_ = pemin;
  CHRONOS_REQUIRE(smeth == "AFSAI_SYM", CHRONOS_ENOTSUP, "smoother " + smeth + " is outside this path");
  if (!prolong) {   // with a caller-supplied P these choices are the caller's
    CHRONOS_REQUIRE(tmeth == "NONE", CHRONOS_ENOTSUP, "test-space method " + tmeth + " is outside this path");
    CHRONOS_REQUIRE(ptype == "BAMG", CHRONOS_ENOTSUP, "prolongation " + ptype + " is outside this path");
    CHRONOS_REQUIRE(pemin == "NONE" || pemin == "SMOOTH" || pemin == "EMIN", CHRONOS_ENOTSUP,
                    "prolongation post-process " + pemin + " is outside this path");
    if (pemin == "EMIN") {
      CHRONOS_REQUIRE(prm.symmetric, CHRONOS_ENOTSUP,
                      "EMIN for a nonsymmetric problem (DEFL_GMRES_matfree) is outside this path");
      CHRONOS_REQUIRE(prm.prec_emin == 1 && (prm.solv_emin == 3 || prm.solv_emin == 4),
                      CHRONOS_ENOTSUP,
                      "EMIN is on this path with prec_emin 1 (Jacobi) and solv_emin 3 or 4");
      CHRONOS_REQUIRE(prm.ntv <= 16, CHRONOS_ENOTSUP, "EMIN takes at most 16 test vectors");
    }
    CHRONOS_REQUIRE(prm.nl_agg == 0, CHRONOS_ENOTSUP, "aggressive coarsening is outside this path");
    CHRONOS_REQUIRE(prm.updateCF == 0, CHRONOS_ENOTSUP, "updateCF != 0 is outside this path");
  }
  CHRONOS_REQUIRE(prm.filt_wgt >= 100 && prm.filt_tau <= 0, CHRONOS_ENOTSUP,
                  "prolongation / coarse-operator filtering is outside this path");
  CHRONOS_REQUIRE(prm.ntv >= 1 && prm.nstep >= 0 && prm.step_size >= 1 &&
                      prm.nstep * prm.step_size <= 64, CHRONOS_EINVAL,
                  "bad smoother / test-space sizes (nstep*step_size <= 64)");
  CHRONOS_REQUIRE(prm.precision == CHRONOS_FP32 || prm.precision == CHRONOS_FP64, CHRONOS_EINVAL,
                  "precision must be CHRONOS_FP32 or CHRONOS_FP64");

  h_ = std::make_unique<Hier>();
  h_->prm = prm;
  h_->precision = prm.precision;
  fp32_ = prm.precision == CHRONOS_FP32;
  CHRONOS_CUDA(cudaStreamCreateWithFlags(&h_->st, cudaStreamNonBlocking));
  nth_ = prm.nthread > 0 ? prm.nthread : 0;
  if (nth_ <= 0) {
#ifdef _OPENMP
    nth_ = omp_get_max_threads();
#else
    nth_ = 1;
#endif
  }
  const int n = A0.nrows;
  ntv_ = prm.ntv;
  if (!prolong) {
    TV_.assign((size_t)n * ntv_, 0.0);                    // column-major n x ntv
    const int ncopy = std::min(std::max(ntv0, 0), ntv_);
    for (int j = 0; j < ncopy; ++j)
      std::copy(TV0 + (size_t)j * n, TV0 + (size_t)(j + 1) * n, TV_.begin() + (size_t)j * n);
    for (int j = std::max(ntv0, 0); j < ntv_; ++j)        // rand(n, ntv-ntv0), column-major
      for (int i = 0; i < n; ++i) TV_[(size_t)j * n + i] = rng_.next_res53();
    SetupPhase ph3("chronos setup: coarsening", &h_->times[3]);
    qr_orthonormalize(n, ntv_, TV_.data());
  }
  Al_ = std::move(A0);
}

HierBuilder::~HierBuilder() = default;

bool HierBuilder::begin_level() {
  Active act(active_);
  const chronos_params &prm = prm_;
  ++level_;
  Hier &H = *h_;
  cudaStream_t st = H.st;
  std::array<double, 12> &T = H.times;
  H.levels.emplace_back();
  Level &L = H.levels.back();
  const int n = Al_.nrows;
  L.n = n;
  {
    SetupPhase ph8("chronos setup: uploads", &T[8]);
    upload_csr(Al_, L.A, fp32_, st);
    if (prm.use_bsr) attach_sell3(Al_, L.A, fp32_, st);
    CHRONOS_CUDA(cudaStreamSynchronize(st));
  }
  if (n <= prm.maxCoarseSZ || level_ >= prm.nLevMax) {
    SetupPhase ph6("chronos setup: coarse factor", &T[6]);
    CHRONOS_REQUIRE(n <= 8192, CHRONOS_ENOTSUP, "coarsest level larger than 8192 rows");
    std::vector<double> dense((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i)
      for (int64_t k = Al_.rp[i]; k < Al_.rp[i + 1]; ++k) dense[(size_t)Al_.ci[k] * n + i] = Al_.v[k];
    DBuf<double> Ld;
    Ld.upload(dense, st);
    const int info = dense_cholesky_device(n, Ld.get(), st);
    CHRONOS_REQUIRE(info == 0, CHRONOS_ENOTSPD,
                    "coarsest-level Cholesky failed at pivot " + std::to_string(info));
    L.W.alloc((size_t)n * n);
    dense_inverse_from_chol(n, Ld.get(), L.W.get(), st);
    L.coarsest = true;
    alloc_vectors(L, H.precision, st);
    CHRONOS_CUDA(cudaStreamSynchronize(st));
    return false;
  }
  // ---- smoother: adaptive FSAI (host pattern, GPU values) ----------------
  SetupPhase ph0("chronos setup: fsai pattern", &T[0]);
  FsaiResult fr = fsai_adaptive(Al_, prm.nstep, prm.step_size, prm.epsilon, nth_,
                                prm.fsai_fabs == 0);
  CHRONOS_REQUIRE(fr.posdef, CHRONOS_ENOTSPD,
                  "matrix deemed indefinite during FSAI (the nonsymmetric fallback is outside this path)");
  Gh_ = std::move(fr.G);
  rowlen_.resize(n);
  for (int i = 0; i < n; ++i) rowlen_[i] = (int)(Gh_.rp[i + 1] - Gh_.rp[i]);
  upload_csr(Gh_, L.G, false, st);       // pattern (+ host values, overwritten)
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  return true;
}

FsaiJob HierBuilder::fsai_job() const {
  const Level &L = h_->levels.back();
  FsaiJob j;
  j.n = L.n;
  j.arp = L.A.rp.get();
  j.aci = L.A.ci.get();
  j.av = L.A.v64.get();
  j.grp = L.G.rp.get();
  j.gci = L.G.ci.get();
  j.gval = L.G.v64.get();
  j.rowlen = &rowlen_;
  return j;
}

int HierBuilder::fsai_numeric_single() {
  Active act(active_);
  Level &L = h_->levels.back();
  SetupPhase ph1("chronos setup: fsai numeric", &h_->times[1]);
  return fsai_numeric_device(L.n, L.A.rp, L.A.ci, L.A.v64, L.G.rp, L.G.ci, L.G.v64, rowlen_,
                             h_->st);
}

void HierBuilder::add_numeric_time(double seconds) {
  h_->times[1] += seconds;
  active_ += seconds;
}

void HierBuilder::end_level(int fl) {
  Active act(active_);
  const chronos_params &prm = prm_;
  Hier &H = *h_;
  cudaStream_t st = H.st;
  std::array<double, 12> &T = H.times;
  Level &L = H.levels.back();
  const int n = L.n;
  const int level = level_;
  const ProlongFn *prolong = prolong_;
  const int ntv = ntv_;
  const int nth = nth_;
  const bool fp32 = fp32_;
  HostCSR &Al = Al_;
  std::vector<double> &TV = TV_;
  MT19937 &rng = rng_;
  const std::string &pemin = pemin_;
  CHRONOS_REQUIRE(fl == 0, CHRONOS_ENOTSPD, "FSAI numeric phase met a non-SPD local system");
  SetupPhase ph1("chronos setup: fsai numeric", &T[1]);
  {
    HostCSR &Gh = Gh_;
    // NaN-diagonal repair (smoother.m:61-71): row -> 1/sqrt(a_ii) e_i
    std::vector<double> gv(L.G.nnz);
    L.G.v64.download(gv.data(), L.G.nnz, st);
    CHRONOS_CUDA(cudaStreamSynchronize(st));
    bool fixed = false;
    for (int i = 0; i < n; ++i) {
      const int64_t dpos = Gh.rp[i + 1] - 1;
      if (std::isnan(gv[dpos])) {
        double aii = 0;
        for (int64_t k = Al.rp[i]; k < Al.rp[i + 1]; ++k) if (Al.ci[k] == i) aii = Al.v[k];
        for (int64_t k = Gh.rp[i]; k < dpos; ++k) gv[k] = 0.0;
        gv[dpos] = 1.0 / std::sqrt(aii);
        fixed = true;
      }
    }
    if (fixed) L.G.v64.upload(gv, st);
    ph1.end();
    SetupPhase ph9("chronos setup: layouts", &T[9]);
    upload_transpose(L.G, L.Gt, false, st);
    if (fp32) {
      L.G.v32.alloc(std::max<int64_t>(L.G.nnz, 1));
      L.Gt.v32.alloc(std::max<int64_t>(L.Gt.nnz, 1));
      convert_f64_to_f32(L.G.nnz, L.G.v64.get(), L.G.v32.get(), st);
      convert_f64_to_f32(L.Gt.nnz, L.Gt.v64.get(), L.Gt.v32.get(), st);
    }
    CHRONOS_CUDA(cudaStreamSynchronize(st));
  }
  ph1.end();
  // ---- omega = min(1, 1.9 / lambda_max(G A G')) ----------------------------
  SetupPhase ph2("chronos setup: omega", &T[2]);
  {
    DBuf<double> t1(n), t2(n);
    Level *Lp = &L;
    auto mv = [&](const double *v, double *w) {
      csr_apply<double, double, double, double, MODE_PLAIN, false>(
          st, 8, n, Lp->Gt.rp, Lp->Gt.ci, Lp->Gt.v64, v, nullptr, t1.get(), 1.0);
      csr_apply<double, double, double, double, MODE_PLAIN, false>(
          st, 8, n, Lp->A.rp, Lp->A.ci, Lp->A.v64, t1.get(), nullptr, t2.get(), 1.0);
      csr_apply<double, double, double, double, MODE_PLAIN, false>(
          st, 8, n, Lp->G.rp, Lp->G.ci, Lp->G.v64, t2.get(), nullptr, w, 1.0);
    };
    L.lambda = lanczos_lmax(n, mv, 5e-4, 200, st);
    L.omega = std::min(1.0, 1.9 / L.lambda);
  }
  ph2.end();
  HostCSR Ph;
  int nc = 0;
  if (prolong) {
    // ---- prolongation from the caller (coarsening, C/F split, P pattern and
    // values are the caller's host code, as cpt_aspAMG.m:224-225 calls prolong)
    SetupPhase ph4("chronos setup: prolongation (caller)", &T[4]);
    Ph = (*prolong)(level, Al);
    nc = Ph.ncols;
    CHRONOS_REQUIRE(Ph.nrows == n && nc > 0 && nc < n &&
                        (int64_t)Ph.rp.size() == (int64_t)n + 1 && Ph.rp[0] == 0 &&
                        (int64_t)Ph.ci.size() == Ph.rp[n] && Ph.v.size() == Ph.ci.size(),
                    CHRONOS_EINVAL,
                    "caller's prolongation of level " + std::to_string(level) +
                        " must be n x nc CSR with 0 < nc < n");
    for (int i = 0; i < n; ++i) {
      CHRONOS_REQUIRE(Ph.rp[i + 1] >= Ph.rp[i], CHRONOS_EINVAL,
                      "caller's prolongation: decreasing row pointers");
      for (int64_t k = Ph.rp[i]; k < Ph.rp[i + 1]; ++k)
        CHRONOS_REQUIRE(Ph.ci[k] >= 0 && Ph.ci[k] < nc && (k == Ph.rp[i] || Ph.ci[k] > Ph.ci[k - 1]) &&
                            std::isfinite(Ph.v[k]),
                        CHRONOS_EINVAL,
                        "caller's prolongation: columns must be ascending in [0, nc), values finite");
    }
    ph4.end();
  } else {
  // ---- test space, coarsening --------------------------------------------
  SetupPhase ph3("chronos setup: coarsening", &T[3]);
  qr_orthonormalize(n, ntv, TV.data());
  HostCSR S;
  std::vector<int> fcn;
  if (gpu_coarsening(prm.SoC_type)) {
    coarsen_device(n, L.A.rp, L.A.ci, L.A.v64, prm.SoC_type, prm.soc_tau, rng, S, fcn, &nc,
                   st);
  } else {
    S = soc_matrix(Al, prm.SoC_type, prm.soc_tau);
    fcn = pmis_split(Al, S, rng, &nc);
  }
  CHRONOS_REQUIRE(nc > 0 && nc < n, CHRONOS_EINVAL, "coarsening produced no usable coarse level");
  ph3.end();
  // ---- BAMG prolongation -----------------------------------------------------
  SetupPhase ph4("chronos setup: prolongation", &T[4]);
  std::vector<int> fc0(n);
  std::vector<int> clist;
  clist.reserve(nc);
  for (int i = 0; i < n; ++i) {
    fc0[i] = fcn[i] > 0 ? fcn[i] - 1 : -1;
    if (fcn[i] > 0) clist.push_back(i);
  }
  std::vector<double> TVr((size_t)n * ntv);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < ntv; ++j) TVr[(size_t)i * ntv + j] = TV[(size_t)j * n + i];
  BamgParams bp{prm.itmax_vol, prm.dist_min, prm.dist_max, ntv,
                prm.prol_np > 0 ? prm.prol_np : nth, prm.maxcond, prm.maxrownrm, prm.tol_vol,
                prm.eps_prol};
  std::vector<int> c_mark;
  Ph = gpu_bamg() && ntv <= 16
           ? bamg_prolongation_device(bp, S, fc0, nc, TVr.data(), ntv, c_mark, st)
                  : bamg_prolongation(bp, S, fc0, nc, TVr.data(), ntv, c_mark);
  if (pemin == "SMOOTH") Ph = smooth_prolongation(Al, L.A, Ph, st);
  if (pemin == "EMIN") {
    // prolong.m:207-235: S_emin is DOM strength of A with threshold patt_tau
    // either way (the coarsening's S when it is DOM with tau = patt_tau,
    // cpt_SoC_dom(patt_tau, A) otherwise), computed on the fly on the GPU
    EminStrength str;
    str.arp = L.A.rp.get();
    str.aci = L.A.ci.get();
    str.av = L.A.v64.get();
    str.n = n;
    str.nnz = L.A.nnz;
    str.tau = prm.patt_tau;
    for (int i = 0; i < n; ++i)
      str.max_row = std::max<int>(str.max_row, (int)(Al.rp[i + 1] - Al.rp[i]));
    const std::vector<int> prp = rp32(Ph);
    const CsrRef P0{n, nc, prp.data(), Ph.ci.data(), Ph.v.data()};
    DevPattern patt;
    emin_pattern_device(prm.patt_pow, n, nc, str, P0, fc0, prm.nnzr_max, ntv, false, patt, st);
    EminParams ep;
    ep.itmax = prm.itmax_emin;
    ep.energ_tol = prm.energ_tol;
    ep.condmax = prm.condmax_emin;
    ep.prec = prm.prec_emin;
    ep.solv = prm.solv_emin;
    ep.spd = true;
    double info[12];
    Ph = emin_device(ep, n, nc, L.A.rp.get(), L.A.ci.get(), L.A.v64.get(), P0, patt, fc0,
                     TVr.data(), ntv, st, info);
    if (std::getenv("CHRONOS_TUNE_VERBOSE"))
      std::fprintf(stderr, "chronos setup: level %d EMIN pattern %lld entries, %d CG steps, "
                   "%d SVD rows, %.3f s\n", level, (long long)patt.nnz, (int)info[7],
                   (int)info[6], info[5]);
  }
  std::vector<double> TVn((size_t)nc * ntv);
  for (int j = 0; j < ntv; ++j)
    for (int c = 0; c < nc; ++c) TVn[(size_t)j * nc + c] = TV[(size_t)j * n + clist[c]];
  TV.swap(TVn);
  ph4.end();
  }
  // ---- Galerkin on the GPU ---------------------------------------------------
  SetupPhase ph9("chronos setup: layouts", &T[9]);
  L.nc = nc;
  upload_csr(Ph, L.P, fp32, st);
  upload_transpose(L.P, L.Pt, fp32, st, &Ph);
  ph9.end();
  SetupPhase ph5("chronos setup: galerkin", &T[5]);
  DBuf<int> aprp, apci, acrp, acci;
  DBuf<double> apv, acv;
  int64_t nnz_ap = 0, nnz_ac = 0;
  spgemm_device(n, nc, L.A.rp, L.A.ci, L.A.v64, L.P.rp, L.P.ci, L.P.v64, aprp, apci, apv,
                &nnz_ap, st);
  spgemm_device(nc, nc, L.Pt.rp, L.Pt.ci, L.Pt.v64, aprp, apci, apv, acrp, acci, acv, &nnz_ac,
                st);
  HostCSR Ac = download_csr(nc, nc, acrp, acci, acv, nnz_ac, st);
  ph5.end();
  alloc_vectors(L, H.precision, st);
  Al = std::move(Ac);
}

std::unique_ptr<Hier> HierBuilder::finish(bool tune) {
  std::array<double, 12> &T = h_->times;
  {
    Active act(active_);
    if (tune) {
      SetupPhase ph10("chronos setup: autotune", &T[10]);
      tune_hierarchy(*h_);
    }
    CHRONOS_CUDA(cudaStreamSynchronize(h_->st));
  }
  T[7] = active_;
  double named = 0.0;
  for (int k : {0, 1, 2, 3, 4, 5, 6, 8, 9, 10}) named += T[k];
  T[11] = std::max(0.0, T[7] - named);
  return std::move(h_);
}

std::unique_ptr<Hier> build_hierarchy(const chronos_params &prm, HostCSR A0, int ntv0,
                                      const double *TV0, bool tune, const ProlongFn *prolong) {
  HierBuilder b(prm, std::move(A0), ntv0, TV0, prolong);
  while (b.begin_level()) b.end_level(b.fsai_numeric_single());
  return b.finish(tune);
}

void tune_hierarchy(Hier &h) {
  const bool fp32 = h.precision == CHRONOS_FP32;
  const int fmt = h.prm.spmv_format;
  // SpMV lane counts
  for (auto &L : h.levels) {
    autotune_lanes(L.A, fp32, h.st, fmt);
    if (!L.coarsest) {
      autotune_lanes(L.G, fp32, h.st, fmt);
      autotune_lanes(L.Gt, fp32, h.st, fmt);
      autotune_lanes(L.P, fp32, h.st, fmt);
      autotune_lanes(L.Pt, fp32, h.st, fmt);
    }
  }
  // the level-1 FP64 operator of the outer PCG
  if (fp32 && h.prm.exact_outer) autotune_lanes(h.levels[0].A, false, h.st);
  CHRONOS_CUDA(cudaStreamSynchronize(h.st));
}

// ---------------------------------------------------------------------------
// Hierarchy files: "CHRNHIER", format version, the parameter block, then per
// level n, nc, coarsest, omega, lambda and A, followed by G and P (smoothing
// levels) or the n x n inverse W (coarsest).  CSR as nrows, ncols, nnz, int64
// row pointers, int32 columns, FP64 values; all little-endian, as written.
// ---------------------------------------------------------------------------
namespace {

constexpr char kHierMagic[8] = {'C', 'H', 'R', 'N', 'H', 'I', 'E', 'R'};
constexpr uint32_t kHierVersion = 1;

struct FileW {
  FILE *f;
  explicit FileW(const char *path) : f(std::fopen(path, "wb")) {
    CHRONOS_REQUIRE(f, CHRONOS_EIO, std::string("cannot write ") + path);
  }
  ~FileW() { if (f) std::fclose(f); }
  void put(const void *p, size_t bytes) {
    CHRONOS_REQUIRE(bytes == 0 || std::fwrite(p, 1, bytes, f) == bytes, CHRONOS_EIO,
                    "short write of the hierarchy file");
  }
  template <typename T> void val(const T &v) { put(&v, sizeof(T)); }
  void close() {
    CHRONOS_REQUIRE(std::fclose(f) == 0, CHRONOS_EIO, "closing the hierarchy file failed");
    f = nullptr;
  }
};

struct FileR {
  FILE *f;
  explicit FileR(const char *path) : f(std::fopen(path, "rb")) {
    CHRONOS_REQUIRE(f, CHRONOS_EIO, std::string("cannot read ") + path);
  }
  ~FileR() { if (f) std::fclose(f); }
  void get(void *p, size_t bytes) {
    CHRONOS_REQUIRE(bytes == 0 || std::fread(p, 1, bytes, f) == bytes, CHRONOS_EIO,
                    "truncated hierarchy file");
  }
  template <typename T> T val() {
    T v;
    get(&v, sizeof(T));
    return v;
  }
  // bytes between the read position and the end of the file
  int64_t remaining() {
    const long pos = std::ftell(f);
    CHRONOS_REQUIRE(pos >= 0 && std::fseek(f, 0, SEEK_END) == 0, CHRONOS_EIO,
                    "cannot seek in the hierarchy file");
    const long end = std::ftell(f);
    CHRONOS_REQUIRE(end >= pos && std::fseek(f, pos, SEEK_SET) == 0, CHRONOS_EIO,
                    "cannot seek in the hierarchy file");
    return (int64_t)(end - pos);
  }
};

void write_csr(FileW &w, const HostCSR &m) {
  w.val<int32_t>(m.nrows);
  w.val<int32_t>(m.ncols);
  w.val<int64_t>(m.nnz());
  w.put(m.rp.data(), sizeof(int64_t) * m.rp.size());
  w.put(m.ci.data(), sizeof(int) * (size_t)m.nnz());
  w.put(m.v.data(), sizeof(double) * (size_t)m.nnz());
}

HostCSR read_csr(FileR &r) {
  HostCSR m;
  m.nrows = r.val<int32_t>();
  m.ncols = r.val<int32_t>();
  const int64_t nnz = r.val<int64_t>();
  CHRONOS_REQUIRE(m.nrows >= 0 && m.ncols >= 0 && nnz >= 0 && nnz < INT32_MAX, CHRONOS_EIO,
                  "bad matrix header in the hierarchy file");
  // a corrupt header must not size host buffers beyond what the file holds
  const int64_t need = 8 * ((int64_t)m.nrows + 1) + 12 * nnz;
  CHRONOS_REQUIRE(need <= r.remaining(), CHRONOS_EIO,
                  "truncated hierarchy file (matrix header larger than the file)");
  m.rp.resize((size_t)m.nrows + 1);
  m.ci.resize(nnz);
  m.v.resize(nnz);
  r.get(m.rp.data(), sizeof(int64_t) * m.rp.size());
  r.get(m.ci.data(), sizeof(int) * (size_t)nnz);
  r.get(m.v.data(), sizeof(double) * (size_t)nnz);
  CHRONOS_REQUIRE(m.rp[0] == 0 && m.rp[m.nrows] == nnz, CHRONOS_EIO,
                  "bad row pointers in the hierarchy file");
  for (int i = 0; i < m.nrows; ++i)
    CHRONOS_REQUIRE(m.rp[i + 1] >= m.rp[i], CHRONOS_EIO, "bad row pointers in the hierarchy file");
  for (int64_t k = 0; k < nnz; ++k)
    CHRONOS_REQUIRE(m.ci[k] >= 0 && m.ci[k] < m.ncols, CHRONOS_EIO,
                    "column out of range in the hierarchy file");
  return m;
}

HostCSR fetch_csr(const DMat &d, cudaStream_t st) {
  return download_csr(d.nrows, d.ncols, d.rp, d.ci, d.v64, d.nnz, st);
}

}  // namespace

void save_hierarchy(const Hier &h, const char *path) {
  CHRONOS_REQUIRE(path, CHRONOS_EINVAL, "null path");
  FileW w(path);
  w.put(kHierMagic, sizeof(kHierMagic));
  w.val<uint32_t>(kHierVersion);
  w.val<uint32_t>((uint32_t)sizeof(chronos_params));
  w.put(&h.prm, sizeof(chronos_params));
  w.val<int32_t>((int32_t)h.levels.size());
  for (const Level &L : h.levels) {
    w.val<int32_t>(L.n);
    w.val<int32_t>(L.nc);
    w.val<int32_t>(L.coarsest ? 1 : 0);
    w.val<double>(L.omega);
    w.val<double>(L.lambda);
    write_csr(w, fetch_csr(L.A, h.st));
    if (L.coarsest) {
      std::vector<double> W((size_t)L.n * L.n);
      L.W.download(W.data(), W.size(), h.st);
      CHRONOS_CUDA(cudaStreamSynchronize(h.st));
      w.put(W.data(), sizeof(double) * W.size());
    } else {
      write_csr(w, fetch_csr(L.G, h.st));
      write_csr(w, fetch_csr(L.P, h.st));
    }
  }
  w.close();
}

std::unique_ptr<Hier> load_hierarchy(const char *path) {
  CHRONOS_REQUIRE(path, CHRONOS_EINVAL, "null path");
  const double t_start = now_s();
  FileR r(path);
  char magic[8];
  r.get(magic, sizeof(magic));
  CHRONOS_REQUIRE(std::memcmp(magic, kHierMagic, sizeof(magic)) == 0, CHRONOS_EIO,
                  std::string(path) + " is not a hierarchy file");
  CHRONOS_REQUIRE(r.val<uint32_t>() == kHierVersion, CHRONOS_EIO,
                  "unsupported hierarchy file version");
  CHRONOS_REQUIRE(r.val<uint32_t>() == sizeof(chronos_params), CHRONOS_EIO,
                  "hierarchy file written with another parameter layout");
  chronos_params prm;
  r.get(&prm, sizeof(prm));
  CHRONOS_REQUIRE(prm.precision == CHRONOS_FP32 || prm.precision == CHRONOS_FP64, CHRONOS_EIO,
                  "bad precision in the hierarchy file");
  const int nlev = r.val<int32_t>();
  CHRONOS_REQUIRE(nlev >= 1 && nlev <= 64, CHRONOS_EIO, "bad level count in the hierarchy file");
  auto h = std::make_unique<Hier>();
  h->prm = prm;
  h->precision = prm.precision;
  const bool fp32 = prm.precision == CHRONOS_FP32;
  CHRONOS_CUDA(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
  cudaStream_t st = h->st;
  int nprev = -1;
  for (int l = 0; l < nlev; ++l) {
    h->levels.emplace_back();
    Level &L = h->levels.back();
    L.n = r.val<int32_t>();
    L.nc = r.val<int32_t>();
    L.coarsest = r.val<int32_t>() != 0;
    L.omega = r.val<double>();
    L.lambda = r.val<double>();
    CHRONOS_REQUIRE(L.n > 0 && (nprev < 0 || L.n == nprev) && L.coarsest == (l == nlev - 1),
                    CHRONOS_EIO, "inconsistent levels in the hierarchy file");
    const HostCSR A = read_csr(r);
    CHRONOS_REQUIRE(A.nrows == L.n && A.ncols == L.n, CHRONOS_EIO,
                    "operator size differs from its level in the hierarchy file");
    upload_csr(A, L.A, fp32, st);
    if (prm.use_bsr) attach_sell3(A, L.A, fp32, st);
    if (L.coarsest) {
      CHRONOS_REQUIRE(L.n <= 8192, CHRONOS_EIO, "coarsest level larger than 8192 rows");
      std::vector<double> W((size_t)L.n * L.n);
      r.get(W.data(), sizeof(double) * W.size());
      L.W.upload(W, st);
    } else {
      const HostCSR G = read_csr(r), P = read_csr(r);
      CHRONOS_REQUIRE(G.nrows == L.n && G.ncols == L.n && P.nrows == L.n && P.ncols == L.nc &&
                          L.nc > 0 && L.nc < L.n,
                      CHRONOS_EIO, "smoother or prolongation size differs in the hierarchy file");
      upload_csr(G, L.G, fp32, st);
      upload_transpose(L.G, L.Gt, fp32, st, &G);
      upload_csr(P, L.P, fp32, st);
      upload_transpose(L.P, L.Pt, fp32, st, &P);
    }
    alloc_vectors(L, h->precision, st);
    nprev = L.coarsest ? -1 : L.nc;
  }
  tune_hierarchy(*h);
  h->times[7] = now_s() - t_start;
  return h;
}

// ---------------------------------------------------------------------------
// V-cycle
// ---------------------------------------------------------------------------

// Deterministic dot of two device vectors into *out (used when the top level
// is also the coarsest).
__global__ void k_dot_store(int n, const double *a, const double *b, double *part,
                            unsigned *ticket, double *out) {
  pdl_begin();
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s += a[i] * b[i];
  double v[1] = {s};
  grid_reduce<1>(v, part, ticket, StoreScalar{out});
}

template <typename T, typename BT, typename OT, bool TOP>
static void vcycle_level(Hier &h, int l, const BT *b, OT *out, const double *dw, double *dot_out) {
  Level &L = h.levels[l];
  cudaStream_t st = h.st;
  const int n = L.n;
  double *part = h.pcg.part.get();
  unsigned *tick = h.pcg.tickets.get();
  if (L.coarsest) {
    dense_matvec<BT, OT>(n, L.W.get(), b, out, st);
    if (TOP && dw) {
      launch_pdl(k_dot_store, std::min(num_sms() * 4, (int)ceil_div(n, 256)), 256, st, n,
                 (const double *)out, dw, part, tick, dot_out);
      CHRONOS_CHECK_LAUNCH();
    }
    return;
  }
  T *x = L.x<T>(), *r = L.r<T>(), *t = L.t<T>();
  const T w = (T)L.omega;
  const DMat &A = L.A, &G = L.G, &Gt = L.Gt, &P = L.P, &Pt = L.Pt;
  // presmooth from x0 = 0: x = w G'(G b)
  mat_apply<T, BT, T, T, MODE_PLAIN, false>(st, G, vals<T>(G), b, nullptr, t, T(1));
  mat_apply<T, T, T, T, MODE_SCALE, false>(st, Gt, vals<T>(Gt), t, nullptr, x, w);
  for (int k = 1; k < h.prm.nupre; ++k) {
    op_apply<T, T, BT, T, MODE_RESID, false>(st, A, x, b, r, T(1));
    mat_apply<T, T, T, T, MODE_PLAIN, false>(st, G, vals<T>(G), r, nullptr, t, T(1));
    mat_apply<T, T, T, T, MODE_AXPY, false>(st, Gt, vals<T>(Gt), t, x, x, w);
  }
  // residual and restriction
  op_apply<T, T, BT, T, MODE_RESID, false>(st, A, x, b, r, T(1));
  Level &C = h.levels[l + 1];
  mat_apply<T, T, T, T, MODE_PLAIN, false>(st, Pt, vals<T>(Pt), r, nullptr,
                                           C.b<T>(), T(1));
  vcycle_level<T, T, T, false>(h, l + 1, C.b<T>(), C.x<T>(), nullptr, nullptr);
  // prolongation and correction
  mat_apply<T, T, T, T, MODE_AXPY, false>(st, P, vals<T>(P), C.x<T>(), x, x, T(1));
  // postsmooth
  const int npost = h.prm.nupost;
  for (int k = 0; k < npost; ++k) {
    op_apply<T, T, BT, T, MODE_RESID, false>(st, A, x, b, r, T(1));
    mat_apply<T, T, T, T, MODE_PLAIN, false>(st, G, vals<T>(G), r, nullptr, t, T(1));
    if (k + 1 < npost) {
      mat_apply<T, T, T, T, MODE_AXPY, false>(st, Gt, vals<T>(Gt), t, x, x, w);
    } else if (TOP && dw) {
      mat_apply<T, T, T, OT, MODE_AXPY, true>(st, Gt, vals<T>(Gt), t, x, out,
                                              w, dw, part, tick, dot_out);
    } else {
      mat_apply<T, T, T, OT, MODE_AXPY, false>(st, Gt, vals<T>(Gt), t, x, out, w);
    }
  }
  if (npost == 0) {
    // out = x + 0 * (G' t): copy / convert through the same epilogue
    if (TOP && dw)
      mat_apply<T, T, T, OT, MODE_AXPY, true>(st, Gt, vals<T>(Gt), t, x, out,
                                              T(0), dw, part, tick, dot_out);
    else
      mat_apply<T, T, T, OT, MODE_AXPY, false>(st, Gt, vals<T>(Gt), t, x, out,
                                               T(0));
  }
}

void Hier::vcycle(const double *b, double *out, const double *dw, double *dot_out) {
  if (precision == CHRONOS_FP32)
    vcycle_level<float, double, double, true>(*this, 0, b, out, dw, dot_out);
  else
    vcycle_level<double, double, double, true>(*this, 0, b, out, dw, dot_out);
}

__global__ void k_f32_to_f64(int64_t n, const float *__restrict__ a, double *__restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (double)a[i];
}

void Hier::vcycle_f32(const float *b, float *out) {
  if (precision == CHRONOS_FP32) {
    vcycle_level<float, float, float, true>(*this, 0, b, out, nullptr, nullptr);
    return;
  }
  // FP64 hierarchy: FP64 copies of the vectors around the cycle
  const int n = levels[0].n;
  if (stage_b.size() < (size_t)n) {
    stage_b.alloc(n);
    stage_x.alloc(n);
  }
  k_f32_to_f64<<<std::min<int64_t>(ceil_div(n, 256), (int64_t)num_sms() * 8), 256, 0, st>>>(
      n, b, stage_b.get());
  CHRONOS_CHECK_LAUNCH();
  vcycle(stage_b.get(), stage_x.get(), nullptr, nullptr);
  convert_f64_to_f32(n, stage_x.get(), out, st);
}

void Hier::apply_A(const double *x, double *y) {
  op_apply<double, double, double, double, MODE_PLAIN, false>(st, levels[0].A, x,
                                                              (const double *)nullptr, y, 1.0);
}

// ---------------------------------------------------------------------------
// PCG_CJ
// ---------------------------------------------------------------------------

// p = pres (first iteration) or p = pres + beta p, beta = -(pres'axp)/ptap.
__global__ void k_pcg_p_update(int n, const double *__restrict__ pres, double *__restrict__ p,
                               const double *__restrict__ sc) {
  pdl_begin();
  const bool first = sc[SC_ITER] < 0.5;
  const double beta = first ? 0.0 : -sc[SC_PRES_AXP] / sc[SC_PTAP];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = first ? pres[i] : pres[i] + beta * p[i];
}

struct FinAlpha {
  double *sc;
  __device__ void operator()(const double *t) const {
    const double ptap = t[0], pres = t[1];
    sc[SC_PTAP] = ptap;
    sc[SC_PRES] = pres;
    if (!(ptap > 0.0) || !isfinite(pres)) {     // breakdown: p'Ap <= 0 or NaN
      sc[SC_BREAKDOWN] = 1.0;
      sc[SC_ALPHA] = 0.0;
    } else {
      sc[SC_ALPHA] = pres / ptap;
    }
  }
};

// axp = A p with ptap = p'axp and p'res, accumulated in FP64; the stored
// values VT are the FP64 operator (exact PCG_CJ arithmetic) or the FP32 copy
// of the hierarchy (with true-residual replacement, see FinResidual).  Rows
// as in k_csrh_apply: L-lane groups, long rows on whole warps.
template <typename VT, int L, bool I16>
__global__ void __launch_bounds__(kApplyThreads)
k_pcg_spmv(int n, const int *__restrict__ rp, const int *__restrict__ ci,
           const int *__restrict__ cbase, const uint16_t *__restrict__ c16,
           const VT *__restrict__ v, const double *__restrict__ p,
           const double *__restrict__ res, double *__restrict__ axp, int short_blocks,
           int lthresh, const int *__restrict__ longrows, int nlong, double *part,
           unsigned *ticket, double *sc) {
  pdl_begin();
  const int lane = threadIdx.x & 31;
  double d0 = 0.0, d1 = 0.0;
  if ((int)blockIdx.x < short_blocks) {
    constexpr int R = 32 / L;
    const int g = lane / L, gl = lane & (L - 1);
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (short_blocks * blockDim.x) >> 5;
    for (int base = warp * R; base < n; base += nwarps * R) {
      const int row = base + g;
      double a = 0.0;
      bool live = false;
      if (row < n) {
        const int s = __ldg(rp + row), e = __ldg(rp + row + 1);
        if (e - s <= lthresh) {
          live = true;
          a = csr_row_dot<double, VT, double, L, I16>(s + gl, e, I16 ? __ldg(cbase + row) : 0,
                                                      ci, c16, v, p);
        }
      }
      a = group_sum<L>(a);
      if (live && gl == 0) {
        axp[row] = a;
        const double pi = p[row];
        d0 += pi * a;
        d1 += pi * res[row];
      }
    }
  } else {
    const int warp = ((blockIdx.x - short_blocks) * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = ((gridDim.x - short_blocks) * blockDim.x) >> 5;
    for (int i = warp; i < nlong; i += nwarps) {
      const int row = __ldg(longrows + i);
      const int s = __ldg(rp + row), e = __ldg(rp + row + 1);
      double a = csr_row_dot<double, VT, double, 32, I16>(
          s + lane, e, I16 ? __ldg(cbase + row) : 0, ci, c16, v, p);
      a = warp_sum(a);
      if (lane == 0) {
        axp[row] = a;
        const double pi = p[row];
        d0 += pi * a;
        d1 += pi * res[row];
      }
    }
  }
  double vals2[2] = {d0, d1};
  grid_reduce<2>(vals2, part, ticket, FinAlpha{sc});
}

// The three row sums of one block row of the sliced 3x3 block form (lane's
// slots; the T partial sums are combined by the caller), accumulated in AT.
template <typename AT, typename VT, typename XT>
__device__ __forceinline__ void sell3_rows(int off, int w, const int *__restrict__ sci,
                                           const VT *__restrict__ V, int64_t nslots,
                                           const XT *__restrict__ x, AT &s0, AT &s1, AT &s2) {
#pragma unroll 2
  for (int j = 0; j < w; ++j) {
    const int k = off + 32 * j;
    const int col = 3 * __ldg(sci + k);
    const AT xa = (AT)__ldg(x + col), xb = (AT)__ldg(x + col + 1), xc = (AT)__ldg(x + col + 2);
    s0 += (AT)__ldg(V + k) * xa + (AT)__ldg(V + nslots + k) * xb +
          (AT)__ldg(V + 2 * nslots + k) * xc;
    s1 += (AT)__ldg(V + 3 * nslots + k) * xa + (AT)__ldg(V + 4 * nslots + k) * xb +
          (AT)__ldg(V + 5 * nslots + k) * xc;
    s2 += (AT)__ldg(V + 6 * nslots + k) * xa + (AT)__ldg(V + 7 * nslots + k) * xb +
          (AT)__ldg(V + 8 * nslots + k) * xc;
  }
}

// The same on the sliced 3x3 block form (see k_sell3_apply).
template <typename VT, int T>
__global__ void __launch_bounds__(kApplyThreads)
k_pcg_spmv_sell3(int nb, int nchunk, const int *__restrict__ choff, const int *__restrict__ chw,
                 const int *__restrict__ sci, const VT *__restrict__ V, int64_t nslots,
                 const double *__restrict__ p, const double *__restrict__ res,
                 double *__restrict__ axp, double *part, unsigned *ticket, double *sc) {
  pdl_begin();
  constexpr int C = 32 / T;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double d0 = 0.0, d1 = 0.0;
  for (int c = warp; c < nchunk; c += nwarps) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    sell3_rows<double, VT, double>(__ldg(choff + c) + lane, __ldg(chw + c), sci, V, nslots, p,
                                   s0, s1, s2);
    if (T > 1) {
      s0 = slot_sum<T>(s0);
      s1 = slot_sum<T>(s1);
      s2 = slot_sum<T>(s2);
    }
    const int br = C * c + (lane & (C - 1));
    if (lane < C && br < nb) {
      const double s[3] = {s0, s1, s2};
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const int row = 3 * br + r;
        axp[row] = s[r];
        const double pi = p[row];
        d0 += pi * s[r];
        d1 += pi * res[row];
      }
    }
  }
  double vals2[2] = {d0, d1};
  grid_reduce<2>(vals2, part, ticket, FinAlpha{sc});
}

static int pcg_grid(const DMat &A, int *short_blocks) {
  const int cap = num_sms() * 8;
  if (A.nb > 0) {
    *short_blocks = 0;
    return std::min(cap, (int)ceil_div(A.nchunk, kApplyThreads / 32));
  }
  const int lb = long_blocks(A, cap);
  const int sb = std::min<int>(ceil_div(A.nrows, kApplyThreads / A.lanes), cap - lb);
  *short_blocks = sb;
  return sb + lb;
}

// axp = A p with ptap and p'res, through the block form when A has one; FP32
// stored values when fp32vals (the FP32 hierarchy's copy), FP64 otherwise.
static void launch_pcg_spmv(cudaStream_t st, const DMat &A, bool fp32vals, const double *p,
                            const double *res, double *axp, double *part, unsigned *tick,
                            double *sc) {
  int sb = 0;
  const int grid = pcg_grid(A, &sb);
  if (A.nb > 0) {
#define CHRONOS_PCGS_CASE(TT)                                                                  \
  case TT:                                                                                     \
    if (fp32vals)                                                                              \
      launch_pdl(k_pcg_spmv_sell3<float, TT>, grid, kApplyThreads, st, A.nb, A.nchunk,         \
                 A.choff.get(), A.chw.get(), A.sci.get(), A.bv32.get(), A.nslots, p, res, axp, \
                 part, tick, sc);                                                              \
    else                                                                                       \
      launch_pdl(k_pcg_spmv_sell3<double, TT>, grid, kApplyThreads, st, A.nb, A.nchunk,        \
                 A.choff.get(), A.chw.get(), A.sci.get(), A.bv64.get(), A.nslots, p, res, axp, \
                 part, tick, sc);                                                              \
    break;
    switch (A.sell_T) {
      CHRONOS_PCGS_CASE(1)
      CHRONOS_PCGS_CASE(2)
      CHRONOS_PCGS_CASE(4)
      default: throw Error(CHRONOS_EINVAL, "bad threads per block row");
    }
#undef CHRONOS_PCGS_CASE
  } else {
#define CHRONOS_PCG_LAUNCH(VT, VALS, LL, I16)                                                  \
  launch_pdl(k_pcg_spmv<VT, LL, I16>, grid, kApplyThreads, st, A.nrows, A.rp.get(), A.ci.get(),  \
             A.cbase.get(), A.c16.get(), VALS, p, res, axp, sb, A.lthresh, A.longrows.get(),    \
             A.nlong, part, tick, sc)
#define CHRONOS_PCG_CASE(LL)                                                                   \
  case LL:                                                                                     \
    if (fp32vals) {                                                                            \
      if (A.idx16) CHRONOS_PCG_LAUNCH(float, A.v32.get(), LL, true);                           \
      else CHRONOS_PCG_LAUNCH(float, A.v32.get(), LL, false);                                  \
    } else {                                                                                   \
      if (A.idx16) CHRONOS_PCG_LAUNCH(double, A.v64.get(), LL, true);                          \
      else CHRONOS_PCG_LAUNCH(double, A.v64.get(), LL, false);                                 \
    }                                                                                          \
    break;
    switch (A.lanes) {
      CHRONOS_PCG_CASE(1)
      CHRONOS_PCG_CASE(2)
      CHRONOS_PCG_CASE(4)
      CHRONOS_PCG_CASE(8)
      CHRONOS_PCG_CASE(16)
      CHRONOS_PCG_CASE(32)
      default: throw Error(CHRONOS_EINVAL, "bad lane count");
    }
#undef CHRONOS_PCG_CASE
#undef CHRONOS_PCG_LAUNCH
  }
  CHRONOS_CHECK_LAUNCH();
}

// End of an iteration's x/res update (PCG_CJ.m:58-64).  Exact mode: the
// recursive residual decides the stop.  Replacement mode (outer operator
// from stored FP32 values): the recursive residual is replaced by the FP64
// true residual (k_pcg_replace) when it has fallen below replace_ratio times
// its largest value since the last replacement, when it passes the
// tolerance, and at itmax; the stop is then decided on the true residual.
struct FinResidual {
  double *sc, *resvec;
  cudaGraphConditionalHandle handle;
  int use_cond, mixed;
  __device__ void operator()(const double *t) const {
    const double rn = sqrt(t[0]);
    const double resiter = rn / sc[SC_BNORM];
    const double it = sc[SC_ITER] + 1.0;
    sc[SC_ITER] = it;
    sc[SC_RR] = t[0];
    sc[SC_RESITER] = resiter;
    resvec[(int)it] = resiter;
    const bool bad = sc[SC_BREAKDOWN] != 0.0 || !isfinite(resiter);
    bool stop;
    if (mixed) {
      const double rmax = fmax(sc[SC_RMAX], rn);
      sc[SC_RMAX] = rmax;
      const bool rep = !bad && (rn < sc[SC_RATIO] * rmax || resiter < sc[SC_TOL] ||
                                it >= sc[SC_ITMAX]);
      sc[SC_REPLACE] = rep ? 1.0 : 0.0;
      stop = bad;                      // otherwise k_pcg_replace decides when it runs
    } else {
      stop = resiter < sc[SC_TOL] || it >= sc[SC_ITMAX] || bad;
    }
    if (use_cond) cudaGraphSetConditional(handle, stop ? 0u : 1u);
  }
};

// x += alpha p; res -= alpha axp; ||res||^2; stopping test of PCG_CJ.m:58-64.
__global__ void __launch_bounds__(256)
k_pcg_xr_update(int n, double *__restrict__ x, double *__restrict__ res,
                const double *__restrict__ p, const double *__restrict__ axp, double *part,
                unsigned *ticket, double *sc, double *resvec, cudaGraphConditionalHandle handle,
                int use_cond, int mixed) {
  pdl_begin();
  const double alpha = sc[SC_ALPHA];
  double rr = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    const double ri = res[i] - alpha * axp[i];
    res[i] = ri;
    rr += ri * ri;
  }
  double v[1] = {rr};
  grid_reduce<1>(v, part, ticket, FinResidual{sc, resvec, handle, use_cond, mixed});
}

// Stop decision on the true residual after a replacement.
struct FinReplace {
  double *sc, *resvec;
  cudaGraphConditionalHandle handle;
  int use_cond;
  __device__ void operator()(const double *t) const {
    const double rn = sqrt(t[0]);
    const double resiter = rn / sc[SC_BNORM];
    const double it = sc[SC_ITER];
    sc[SC_RR] = t[0];
    sc[SC_RESITER] = resiter;
    sc[SC_RMAX] = rn;
    resvec[(int)it] = resiter;
    const bool stop = resiter < sc[SC_TOL] || it >= sc[SC_ITMAX] || !isfinite(resiter);
    if (use_cond) cudaGraphSetConditional(handle, stop ? 0u : 1u);
  }
};

// res = b - A x with the FP64 operator and ||res||^2, only when the previous
// kernel flagged a replacement (every block reads the same flag, so the grid
// returns as a whole otherwise).
template <int L, bool I16>
__global__ void __launch_bounds__(kApplyThreads)
k_pcg_replace(int n, const int *__restrict__ rp, const int *__restrict__ ci,
              const int *__restrict__ cbase, const uint16_t *__restrict__ c16,
              const double *__restrict__ v, const double *__restrict__ x,
              const double *__restrict__ b, double *__restrict__ res, int short_blocks,
              int lthresh, const int *__restrict__ longrows, int nlong, double *part,
              unsigned *ticket, double *sc, double *resvec, cudaGraphConditionalHandle handle,
              int use_cond) {
  pdl_begin();
  if (sc[SC_REPLACE] == 0.0) return;
  const int lane = threadIdx.x & 31;
  double rr = 0.0;
  if ((int)blockIdx.x < short_blocks) {
    constexpr int R = 32 / L;
    const int g = lane / L, gl = lane & (L - 1);
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (short_blocks * blockDim.x) >> 5;
    for (int base = warp * R; base < n; base += nwarps * R) {
      const int row = base + g;
      double a = 0.0;
      bool live = false;
      if (row < n) {
        const int s = __ldg(rp + row), e = __ldg(rp + row + 1);
        if (e - s <= lthresh) {
          live = true;
          a = csr_row_dot<double, double, double, L, I16>(
              s + gl, e, I16 ? __ldg(cbase + row) : 0, ci, c16, v, x);
        }
      }
      a = group_sum<L>(a);
      if (live && gl == 0) {
        const double r = b[row] - a;
        res[row] = r;
        rr += r * r;
      }
    }
  } else {
    const int warp = ((blockIdx.x - short_blocks) * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = ((gridDim.x - short_blocks) * blockDim.x) >> 5;
    for (int i = warp; i < nlong; i += nwarps) {
      const int row = __ldg(longrows + i);
      const int s = __ldg(rp + row), e = __ldg(rp + row + 1);
      double a = csr_row_dot<double, double, double, 32, I16>(
          s + lane, e, I16 ? __ldg(cbase + row) : 0, ci, c16, v, x);
      a = warp_sum(a);
      if (lane == 0) {
        const double r = b[row] - a;
        res[row] = r;
        rr += r * r;
      }
    }
  }
  double vals[1] = {rr};
  grid_reduce<1>(vals, part, ticket, FinReplace{sc, resvec, handle, use_cond});
}

template <int T>
__global__ void __launch_bounds__(kApplyThreads)
k_pcg_replace_sell3(int nb, int nchunk, const int *__restrict__ choff,
                    const int *__restrict__ chw, const int *__restrict__ sci,
                    const double *__restrict__ V, int64_t nslots, const double *__restrict__ x,
                    const double *__restrict__ b, double *__restrict__ res, double *part,
                    unsigned *ticket, double *sc, double *resvec,
                    cudaGraphConditionalHandle handle, int use_cond) {
  pdl_begin();
  if (sc[SC_REPLACE] == 0.0) return;
  constexpr int C = 32 / T;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double rr = 0.0;
  for (int c = warp; c < nchunk; c += nwarps) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    sell3_rows<double, double, double>(__ldg(choff + c) + lane, __ldg(chw + c), sci, V, nslots,
                                       x, s0, s1, s2);
    if (T > 1) {
      s0 = slot_sum<T>(s0);
      s1 = slot_sum<T>(s1);
      s2 = slot_sum<T>(s2);
    }
    const int br = C * c + (lane & (C - 1));
    if (lane < C && br < nb) {
      const double s[3] = {s0, s1, s2};
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const int row = 3 * br + r;
        const double rv = b[row] - s[r];
        res[row] = rv;
        rr += rv * rv;
      }
    }
  }
  double vals[1] = {rr};
  grid_reduce<1>(vals, part, ticket, FinReplace{sc, resvec, handle, use_cond});
}

static void launch_pcg_replace(cudaStream_t st, const DMat &A, const double *x, const double *b,
                               double *res, double *part, unsigned *tick, double *sc,
                               double *resvec, cudaGraphConditionalHandle handle, int use_cond) {
  int sb = 0;
  const int grid = pcg_grid(A, &sb);
  if (A.nb > 0) {
#define CHRONOS_REP3_CASE(TT)                                                                  \
  case TT:                                                                                     \
    launch_pdl(k_pcg_replace_sell3<TT>, grid, kApplyThreads, st, A.nb, A.nchunk,               \
               A.choff.get(), A.chw.get(), A.sci.get(), A.bv64.get(), A.nslots, x, b, res, part, \
               tick, sc, resvec, handle, use_cond);                                            \
    break;
    switch (A.sell_T) {
      CHRONOS_REP3_CASE(1)
      CHRONOS_REP3_CASE(2)
      CHRONOS_REP3_CASE(4)
      default: throw Error(CHRONOS_EINVAL, "bad threads per block row");
    }
#undef CHRONOS_REP3_CASE
  } else {
#define CHRONOS_REP_CASE(LL)                                                                   \
  case LL:                                                                                     \
    if (A.idx16)                                                                               \
      launch_pdl(k_pcg_replace<LL, true>, grid, kApplyThreads, st, A.nrows, A.rp.get(),        \
                 A.ci.get(), A.cbase.get(), A.c16.get(), A.v64.get(), x, b, res, sb, A.lthresh,\
                 A.longrows.get(), A.nlong, part, tick, sc, resvec, handle, use_cond);         \
    else                                                                                       \
      launch_pdl(k_pcg_replace<LL, false>, grid, kApplyThreads, st, A.nrows, A.rp.get(),       \
                 A.ci.get(), A.cbase.get(), A.c16.get(), A.v64.get(), x, b, res, sb, A.lthresh,\
                 A.longrows.get(), A.nlong, part, tick, sc, resvec, handle, use_cond);         \
    break;
    switch (A.lanes) {
      CHRONOS_REP_CASE(1)
      CHRONOS_REP_CASE(2)
      CHRONOS_REP_CASE(4)
      CHRONOS_REP_CASE(8)
      CHRONOS_REP_CASE(16)
      CHRONOS_REP_CASE(32)
      default: throw Error(CHRONOS_EINVAL, "bad lane count");
    }
#undef CHRONOS_REP_CASE
  }
  CHRONOS_CHECK_LAUNCH();
}

static int reduce_blocks(int n) {
  return std::max(1, std::min(num_sms() * 8, (int)ceil_div(n, 256)));
}

// True when the outer PCG applies the stored FP32 values with true-residual
// replacement (FP32 hierarchy, exact_outer = 0).
static bool mixed_outer(const Hier &h) {
  return h.precision == CHRONOS_FP32 && !h.prm.exact_outer && !h.use_user_op;
}

static void drop_pcg_graph(PcgState &s) {
  if (s.exec) { cudaGraphExecDestroy(s.exec); s.exec = nullptr; }
  if (s.graph) { cudaGraphDestroy(s.graph); s.graph = nullptr; }
}

void Hier::set_outer_operator(const HostCSR *A) {
  if (A) {
    CHRONOS_REQUIRE(A->nrows == levels[0].n && A->ncols == levels[0].n, CHRONOS_EINVAL,
                    "the operator must have the hierarchy's level-1 size");
    CHRONOS_CUDA(cudaStreamSynchronize(st));   // the previous operator may still be in use
    user_op = DMat();
    upload_csr(*A, user_op, false, st);
    autotune_lanes(user_op, false, st);
    drop_pcg_graph(pcg);                       // the graph holds the operator's pointers
    use_user_op = true;
  } else if (use_user_op) {
    CHRONOS_CUDA(cudaStreamSynchronize(st));
    drop_pcg_graph(pcg);
    use_user_op = false;
    user_op = DMat();
  }
}

// Captures one PCG_CJ iteration (PCG_CJ.m:36-64) into the current stream capture.
static void capture_iteration(Hier &h, cudaGraphConditionalHandle handle, int use_cond) {
  PcgState &s = h.pcg;
  cudaStream_t st = h.st;
  const int n = s.n;
  const int nb = reduce_blocks(n);
  const bool mixed = mixed_outer(h);
  double *sc = s.sc.get();
  // pres = M^{-1} res  (with pres'axp for beta)
  h.vcycle(s.res.get(), s.pres.get(), s.axp.get(), sc + SC_PRES_AXP);
  launch_pdl(k_pcg_p_update, nb, 256, st, n, (const double *)s.pres.get(), s.p.get(),
             (const double *)sc);
  CHRONOS_CHECK_LAUNCH();
  unsigned *tk = s.tickets.get();
  launch_pcg_spmv(st, h.outer_A(), mixed, s.p.get(), s.res.get(), s.axp.get(),
                  s.part.get() + 4 * 3 * 2048, tk + 1, sc);
  launch_pdl(k_pcg_xr_update, nb, 256, st, n, s.x.get(), s.res.get(), (const double *)s.p.get(),
             (const double *)s.axp.get(), s.part.get() + 8 * 3 * 2048, tk + 2, sc,
             s.resvec.get(), handle, use_cond, mixed ? 1 : 0);
  CHRONOS_CHECK_LAUNCH();
  if (mixed)
    launch_pcg_replace(st, h.levels[0].A, s.x.get(), s.b.get(), s.res.get(),
                       s.part.get() + 10 * 3 * 2048, tk + 4, sc, s.resvec.get(), handle,
                       use_cond);
}

static void ensure_pcg_state(Hier &h, int itmax) {
  PcgState &s = h.pcg;
  const int n = h.levels[0].n;
  if (s.n != n) {
    s.n = n;
    s.x.alloc(n); s.res.alloc(n); s.p.alloc(n); s.axp.alloc(n); s.pres.alloc(n); s.b.alloc(n);
    s.sc.alloc(SC_COUNT);
    s.part.alloc((size_t)12 * 3 * 2048);
    s.tickets.alloc(8);
    s.tickets.zero(h.st);
    s.axp.zero(h.st);
    s.p.zero(h.st);
  }
  if (s.resvec_cap < itmax + 1) {
    // resvec is baked into the graph: rebuild it when the buffer moves
    s.resvec.alloc((size_t)itmax + 1);
    s.resvec_cap = itmax + 1;
    drop_pcg_graph(s);
  }
}

static void build_pcg_graph(Hier &h) {
  PcgState &s = h.pcg;
  cudaStream_t st = h.st;
  if (s.exec) return;
  if (h.prm.use_graph) {
    CHRONOS_CUDA(cudaGraphCreate(&s.graph, 0));
    cudaGraphConditionalHandle handle;
    CHRONOS_CUDA(cudaGraphConditionalHandleCreate(&handle, s.graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = handle;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    CHRONOS_CUDA(cudaGraphAddNode(&node, s.graph, nullptr, 0, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    CHRONOS_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal));
    try {
      capture_iteration(h, handle, 1);
    } catch (...) {
      cudaGraph_t dummy;
      cudaStreamEndCapture(st, &dummy);
      throw;
    }
    CHRONOS_CUDA(cudaStreamEndCapture(st, &body));
    CHRONOS_CUDA(cudaGraphInstantiate(&s.exec, s.graph, 0));
    s.conditional = true;
  } else {
    CHRONOS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
      capture_iteration(h, 0, 0);
    } catch (...) {
      cudaGraph_t dummy;
      cudaStreamEndCapture(st, &dummy);
      throw;
    }
    CHRONOS_CUDA(cudaStreamEndCapture(st, &s.graph));
    CHRONOS_CUDA(cudaGraphInstantiate(&s.exec, s.graph, 0));
    s.conditional = false;
  }
}

static double replace_ratio(const Hier &h) {
  const double r = h.prm.replace_ratio;
  return (r > 0.0 && r < 1.0) ? r : 0.01;
}

__global__ void k_pcg_init(double *sc, double *resvec, double tol, double itmax, double ratio) {
  // sc[SC_BNORM], sc[SC_RR] hold ||b||^2 and ||r0||^2 from the reductions
  const double bn = sqrt(sc[SC_BNORM]);
  sc[SC_BNORM] = bn;
  sc[SC_RESITER] = sqrt(sc[SC_RR]) / bn;
  sc[SC_RMAX] = sqrt(sc[SC_RR]);
  sc[SC_REPLACE] = 0.0;
  sc[SC_RATIO] = ratio;
  resvec[0] = sc[SC_RESITER];
  sc[SC_ITER] = 0.0;
  sc[SC_TOL] = tol;
  sc[SC_ITMAX] = itmax;
  sc[SC_BREAKDOWN] = 0.0;
}

void Hier::pcg_solve(const double *b, double *x, int itmax, double tol, int *iters, int *flag,
                     std::vector<double> *resvec_out, double *seconds) {
  ensure_pcg_state(*this, std::max(itmax, 1));
  PcgState &s = pcg;
  const int n = s.n;
  cudaEvent_t e0, e1;
  CHRONOS_CUDA(cudaEventCreate(&e0));
  CHRONOS_CUDA(cudaEventCreate(&e1));
  CHRONOS_CUDA(cudaEventRecord(e0, st));
  // res = b - A x0, ||b||, ||res|| (PCG_CJ.m:11-30)
  CHRONOS_CUDA(cudaMemcpyAsync(s.x.get(), x, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  if (mixed_outer(*this))
    CHRONOS_CUDA(cudaMemcpyAsync(s.b.get(), b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  op_apply<double, double, double, double, MODE_RESID, false>(st, outer_A(), s.x.get(), b,
                                                              s.res.get(), 1.0);
  const int nb = reduce_blocks(n);
  double *part = s.part.get();
  k_dot_store<<<nb, 256, 0, st>>>(n, b, b, part, s.tickets.get() + 3, s.sc.get() + SC_BNORM);
  CHRONOS_CHECK_LAUNCH();
  k_dot_store<<<nb, 256, 0, st>>>(n, s.res.get(), s.res.get(), part, s.tickets.get() + 3,
                                   s.sc.get() + SC_RR);
  CHRONOS_CHECK_LAUNCH();
  k_pcg_init<<<1, 1, 0, st>>>(s.sc.get(), s.resvec.get(), tol, (double)itmax,
                              replace_ratio(*this));
  CHRONOS_CHECK_LAUNCH();
  double sc_h[SC_COUNT];
  CHRONOS_CUDA(cudaMemcpyAsync(sc_h, s.sc.get(), sizeof(sc_h), cudaMemcpyDeviceToHost, st));
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  int it = 0;
  if (sc_h[SC_BNORM] == 0.0) {                 // PCG_CJ.m:12-16
    CHRONOS_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
    CHRONOS_CUDA(cudaStreamSynchronize(st));
    *iters = 0;
    *flag = 0;
    if (resvec_out) resvec_out->assign(1, 0.0);
    if (seconds) *seconds = 0.0;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return;
  }
  if (itmax > 0) {
    build_pcg_graph(*this);
    if (s.conditional) {
      CHRONOS_CUDA(cudaGraphLaunch(s.exec, st));
    } else {
      double *pinned = nullptr;
      CHRONOS_CUDA(cudaMallocHost(&pinned, sizeof(double) * SC_COUNT));
      for (int k = 0; k < itmax; ++k) {
        CHRONOS_CUDA(cudaGraphLaunch(s.exec, st));
        CHRONOS_CUDA(cudaMemcpyAsync(pinned, s.sc.get(), sizeof(double) * SC_COUNT,
                                     cudaMemcpyDeviceToHost, st));
        CHRONOS_CUDA(cudaStreamSynchronize(st));
        const double r = pinned[SC_RESITER];
        if (r < tol || pinned[SC_BREAKDOWN] != 0.0 || !std::isfinite(r)) break;
      }
      cudaFreeHost(pinned);
    }
  }
  CHRONOS_CUDA(cudaMemcpyAsync(x, s.x.get(), sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  CHRONOS_CUDA(cudaEventRecord(e1, st));
  CHRONOS_CUDA(cudaMemcpyAsync(sc_h, s.sc.get(), sizeof(sc_h), cudaMemcpyDeviceToHost, st));
  CHRONOS_CUDA(cudaEventSynchronize(e1));
  CHRONOS_CUDA(cudaStreamSynchronize(st));
  float ms = 0.f;
  CHRONOS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  it = (int)(sc_h[SC_ITER] + 0.5);
  *iters = it;
  const double resiter = sc_h[SC_RESITER];
  *flag = (resiter > tol || !std::isfinite(resiter)) ? 1 : 0;   // PCG_CJ.m:69-71
  if (sc_h[SC_BREAKDOWN] != 0.0) *flag = 1;
  if (resvec_out) {
    resvec_out->resize(it + 1);
    s.resvec.download(resvec_out->data(), it + 1, st);
    CHRONOS_CUDA(cudaStreamSynchronize(st));
  }
  if (seconds) *seconds = ms * 1e-3;
  if (sc_h[SC_BREAKDOWN] != 0.0)
    throw Error(CHRONOS_EBREAKDOWN, "PCG breakdown: p'Ap <= 0 or NaN at iteration " +
                                        std::to_string(it));
}

// The whole solve queued on st with no host synchronisation: initial
// residual, the conditional-graph loop, the copy of x and of the scalars to a
// pinned host buffer.  b must not be zero (the caller checks ||b||: PCG_CJ.m
// returns x = 0 without iterating then).  pcg_collect reads the outcome once
// st has drained.
void Hier::pcg_enqueue(const double *b, double *x, int itmax, double tol) {
  CHRONOS_REQUIRE(prm.use_graph, CHRONOS_EINVAL, "queued solves need use_graph = 1");
  ensure_pcg_state(*this, std::max(itmax, 1));
  build_pcg_graph(*this);
  PcgState &s = pcg;
  const int n = s.n;
  if (!s.sc_pinned) CHRONOS_CUDA(cudaMallocHost(&s.sc_pinned, sizeof(double) * SC_COUNT));
  CHRONOS_CUDA(cudaMemcpyAsync(s.x.get(), x, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  if (mixed_outer(*this))
    CHRONOS_CUDA(cudaMemcpyAsync(s.b.get(), b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  op_apply<double, double, double, double, MODE_RESID, false>(st, outer_A(), s.x.get(), b,
                                                              s.res.get(), 1.0);
  const int nb = reduce_blocks(n);
  k_dot_store<<<nb, 256, 0, st>>>(n, b, b, s.part.get(), s.tickets.get() + 3,
                                   s.sc.get() + SC_BNORM);
  CHRONOS_CHECK_LAUNCH();
  k_dot_store<<<nb, 256, 0, st>>>(n, s.res.get(), s.res.get(), s.part.get(), s.tickets.get() + 3,
                                   s.sc.get() + SC_RR);
  CHRONOS_CHECK_LAUNCH();
  k_pcg_init<<<1, 1, 0, st>>>(s.sc.get(), s.resvec.get(), tol, (double)itmax,
                              replace_ratio(*this));
  CHRONOS_CHECK_LAUNCH();
  if (itmax > 0) CHRONOS_CUDA(cudaGraphLaunch(s.exec, st));
  CHRONOS_CUDA(cudaMemcpyAsync(x, s.x.get(), sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  CHRONOS_CUDA(cudaMemcpyAsync(s.sc_pinned, s.sc.get(), sizeof(double) * SC_COUNT,
                               cudaMemcpyDeviceToHost, st));
}

void Hier::pcg_collect(double tol, int *iters, int *flag) const {
  const double *sc = pcg.sc_pinned;
  CHRONOS_REQUIRE(sc, CHRONOS_EINVAL, "no queued solve to collect");
  *iters = (int)(sc[SC_ITER] + 0.5);
  const double r = sc[SC_RESITER];
  *flag = (r > tol || !std::isfinite(r) || sc[SC_BREAKDOWN] != 0.0) ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Profiling: algorithmic bytes and CUDA-event timings of the hot kernels
// ---------------------------------------------------------------------------

// Compulsory traffic of one CSR apply of M (values s bytes, int32 indices):
// nnz*(s+4) + (rows+1)*4 + x (ncols*sx) + y (rows*sy) + extra row vectors.
static double apply_bytes(const DMat &M, double s, double sx, double sy, double extra_per_row) {
  // block form: 9 values + one block-column index per 3x3 block (true blocks:
  // the chunk padding is not algorithmic traffic)
  // CSR: 4-byte columns, or 2-byte offsets plus a 4-byte base per row
  const double mat = M.nb > 0    ? (double)M.nnzb * (9.0 * s + 4.0) + (M.nchunk + 1.0) * 8.0
                     : M.idx16 ? (double)M.nnz * (s + 2.0) + (M.nrows + 1.0) * 4.0 + M.nrows * 4.0
                               : (double)M.nnz * (s + 4.0) + (M.nrows + 1.0) * 4.0;
  return mat + M.ncols * sx + M.nrows * (sy + extra_per_row);
}

static double vcycle_bytes_level(const Hier &h, int l, double s, double sb, double sout, bool top) {
  const Level &L = h.levels[l];
  const int n = L.n;
  if (L.coarsest) return (double)n * n * 8.0 + n * (sb + sout);
  double b = 0.0;
  b += apply_bytes(L.G, s, sb, s, 0.0);                     // t = G b
  b += apply_bytes(L.Gt, s, s, s, 0.0);                     // x = w G' t
  for (int k = 1; k < h.prm.nupre; ++k)
    b += apply_bytes(L.A, s, s, s, sb) + apply_bytes(L.G, s, s, s, 0.0) +
         apply_bytes(L.Gt, s, s, s, s);
  b += apply_bytes(L.A, s, s, s, sb);                       // r = b - A x
  b += apply_bytes(L.Pt, s, s, s, 0.0);                     // b_c = P' r
  b += vcycle_bytes_level(h, l + 1, s, s, s, false);
  b += apply_bytes(L.P, s, s, s, s);                        // x = x + P x_c
  for (int k = 0; k < h.prm.nupost; ++k) {
    const bool last = k + 1 == h.prm.nupost;
    b += apply_bytes(L.A, s, s, s, sb);                     // r = b - A x
    b += apply_bytes(L.G, s, s, s, 0.0);                    // t = G r
    b += apply_bytes(L.Gt, s, s, last ? sout : s, s + (top && last ? 8.0 : 0.0));
  }
  return b;
}

static int vcycle_kernels(const Hier &h) {
  int k = 0;
  for (const auto &L : h.levels) {
    if (L.coarsest) { k += 1; break; }
    k += 2 + 3 * (h.prm.nupre - 1) + 2 + 1 + 3 * h.prm.nupost + (h.prm.nupost == 0 ? 1 : 0);
  }
  if (h.levels[0].coarsest) k += 1;                         // the separate dot
  return k;
}

void Hier::profile(int reps, chronos_profile *out) {
  reps = std::max(reps, 1);
  const int n = levels[0].n;
  const bool fp32 = precision == CHRONOS_FP32;
  const double s = fp32 ? 4.0 : 8.0;
  ensure_pcg_state(*this, 16);
  PcgState &ps = pcg;
  DBuf<double> b(n), x(n), w(n);
  std::vector<double> hb(n);
  for (int i = 0; i < n; ++i) hb[i] = std::sin(0.37 * i + 1.0);
  b.upload(hb, st);
  w.upload(hb, st);
  cudaEvent_t e0, e1;
  CHRONOS_CUDA(cudaEventCreate(&e0));
  CHRONOS_CUDA(cudaEventCreate(&e1));
  auto time_it = [&](const std::function<void()> &f) {
    f();
    CHRONOS_CUDA(cudaEventRecord(e0, st));
    for (int r = 0; r < reps; ++r) f();
    CHRONOS_CUDA(cudaEventRecord(e1, st));
    CHRONOS_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    CHRONOS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    return (double)ms / reps;
  };
  out->vcycle_ms = time_it([&] { vcycle(b.get(), x.get(), w.get(), ps.sc.get() + SC_PRES_AXP); });
  out->vcycle_bytes = vcycle_bytes_level(*this, 0, s, 8.0, 8.0, true);
  const Level &L0 = levels[0];
  const DMat &A = L0.A;
  if (!L0.coarsest) {
    out->top_apply_ms = time_it([&] {
      if (fp32)
        op_apply<float, float, double, float, MODE_RESID, false>(st, A, L0.x32.get(), b.get(),
                                                                L0.r32.get(), 1.0f);
      else
        op_apply<double, double, double, double, MODE_RESID, false>(st, A, L0.x64.get(), b.get(),
                                                                   L0.r64.get(), 1.0);
    });
    out->top_apply_bytes = apply_bytes(A, s, s, s, 8.0);
  } else {
    out->top_apply_ms = 0.0;
    out->top_apply_bytes = 0.0;
  }
  // outer SpMV with its two dots, as captured in the PCG iteration (stored
  // FP32 values with FP64 accumulation, or FP64 values)
  double *part = ps.part.get() + 4 * 3 * 2048;
  CHRONOS_CUDA(cudaMemcpyAsync(ps.p.get(), b.get(), sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  CHRONOS_CUDA(cudaMemcpyAsync(ps.res.get(), b.get(), sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  out->outer_spmv_ms = time_it([&] {
    launch_pcg_spmv(st, A, mixed_outer(*this), ps.p.get(), ps.res.get(), ps.axp.get(), part,
                    ps.tickets.get() + 1, ps.sc.get());
  });
  out->outer_spmv_bytes = apply_bytes(A, mixed_outer(*this) ? 4.0 : 8.0, 8.0, 8.0, 16.0);
  out->iteration_bytes = out->vcycle_bytes + out->outer_spmv_bytes + 3.0 * n * 8 + 6.0 * n * 8;
  out->kernels_per_iteration = vcycle_kernels(*this) + 3 + (mixed_outer(*this) ? 1 : 0);
  out->kernels_per_solve = 4;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CHRONOS_CUDA(cudaStreamSynchronize(st));
}

}  // namespace chronos
