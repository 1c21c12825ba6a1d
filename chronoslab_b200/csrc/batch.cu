// Batch of independent SPD problems of uneven sizes: one hierarchy per
// problem (each exactly what a single chronos_amg_setup builds).  The batch
// solve either runs the grouped path of group.cu (batch_grouped = 1, the
// default: one launch sequence for the whole batch) or queues every
// problem's whole PCG_CJ -- one conditional-graph launch each -- on its own
// stream with no host synchronisation in between, largest problems first.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <exception>
#include <memory>
#include <mutex>
#include <numeric>
#include <thread>
#include <vector>

#include <omp.h>

#include "group.h"

namespace chronos {

static double now_seconds() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Batch {
  std::vector<std::unique_ptr<Hier>> h;
  // setup wall clock (s): first levels begun, batched FSAI numeric phase of
  // the first levels, the rest of the hierarchies, tuning / grouping, total
  double wall[5] = {0, 0, 0, 0, 0};
  std::vector<int> order;           // largest level-1 operator first
  std::unique_ptr<GroupSolve> group;
};

}  // namespace chronos

using namespace chronos;

struct chronos_batch {
  Batch b;
};

template <typename F>
static int batch_guard(F &&f) {
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
  }
}

extern "C" {

int chronos_batch_setup(const chronos_params *prm, int nprob, const int *n,
                        const int *const *iat_h, const int *const *ja_h,
                        const double *const *val_h, chronos_batch **out) {
  return batch_guard([&] {
    CHRONOS_REQUIRE(prm && n && iat_h && ja_h && val_h && out && nprob > 0, CHRONOS_EINVAL,
                    "bad argument");
    CHRONOS_REQUIRE(prm->use_graph || prm->batch_grouped, CHRONOS_EINVAL,
                    "per-problem batched solves need use_graph = 1");
    auto bt = std::make_unique<chronos_batch>();
    for (int p = 0; p < nprob; ++p)
      CHRONOS_REQUIRE(n[p] > 0 && iat_h[p] && iat_h[p][0] == 0, CHRONOS_EINVAL,
                      "problem " + std::to_string(p) + ": 0-based CSR expected");
    // The problems' first levels are begun together (operator upload, FSAI
    // pattern on the host) on a few host threads at once, largest problems
    // first, each on its own stream with its share of the OpenMP threads;
    // the FSAI numeric phase of all first levels -- most of the batch's rows --
    // then runs as one batched launch per tile size (fsai_numeric_batched,
    // tile sizes tuned per batch shape); then every problem goes on alone on
    // the host threads, largest first: its first level ended (omega,
    // coarsening, prolongation, Galerkin) and its deeper levels built as a
    // single setup builds them.  Every hierarchy is what a single
    // chronos_amg_setup builds; lane counts are tuned afterwards on a quiet
    // GPU: the grouped solve's stacked operators, or each problem's own for
    // the per-problem path.
    DeferFrees defer_frees;          // no thread's free waits on the others' queued work
    bt->b.h.resize(nprob);
    const int hw = std::max(1, (int)std::thread::hardware_concurrency());
    const int nworkers = std::max(1, std::min({nprob, 8, std::max(1, hw / 2)}));
    int dev = 0;
    CHRONOS_CUDA(cudaGetDevice(&dev));
    // runs f(p) for every p of `items`, in that order, on the worker threads;
    // the first error is rethrown
    auto parallel = [&](const std::vector<int> &items, const auto &f) {
      std::atomic<size_t> next{0};
      std::mutex emu;
      std::exception_ptr err;
      auto worker = [&] {
        const int omp_saved = omp_get_max_threads();   // the calling thread gets it back
        try {
          CHRONOS_CUDA(cudaSetDevice(dev));
          omp_set_num_threads(std::max(1, hw / nworkers));
          for (size_t k = next++; k < items.size(); k = next++) {
            {
              std::lock_guard<std::mutex> lk(emu);
              if (err) break;
            }
            f(items[k]);
          }
        } catch (...) {
          std::lock_guard<std::mutex> lk(emu);
          if (!err) err = std::current_exception();
        }
        omp_set_num_threads(omp_saved);
      };
      std::vector<std::thread> pool;
      const int nw = std::min<int>(nworkers, (int)items.size());
      for (int w = 1; w < nw; ++w) pool.emplace_back(worker);
      worker();
      for (auto &t : pool) t.join();
      if (err) std::rethrow_exception(err);
    };
    std::vector<int> largest(nprob);
    std::iota(largest.begin(), largest.end(), 0);
    std::stable_sort(largest.begin(), largest.end(), [&](int a, int c) {
      return iat_h[a][n[a]] > iat_h[c][n[c]];
    });
    std::vector<std::unique_ptr<HierBuilder>> builders(nprob);
    std::vector<char> more(nprob, 0);
    double *wall = bt->b.wall;
    const double t0 = now_seconds();
    parallel(largest, [&](int p) {
      HostCSR A;
      A.nrows = A.ncols = n[p];
      A.rp.assign(iat_h[p], iat_h[p] + n[p] + 1);
      A.ci.assign(ja_h[p], ja_h[p] + A.rp[n[p]]);
      A.v.assign(val_h[p], val_h[p] + A.rp[n[p]]);
      // scalar problems: the constant vector as TV0 (as aspAMG_main.m:92-95
      // for a .mat without a test space), padded with random columns if ntv > 1
      std::vector<double> ones(n[p], 1.0);
      builders[p] = std::make_unique<HierBuilder>(*prm, A, 1, ones.data());
      more[p] = builders[p]->begin_level() ? 1 : 0;
    });
    const double t1 = now_seconds();
    std::vector<int> batched;
    std::vector<FsaiJob> jobs;
    for (int p : largest)
      if (more[p]) {
        batched.push_back(p);
        jobs.push_back(builders[p]->fsai_job());
      }
    std::vector<int> flag_of(nprob, 0);
    if (!jobs.empty()) {
      cudaStream_t bst;
      CHRONOS_CUDA(cudaStreamCreateWithFlags(&bst, cudaStreamNonBlocking));
      std::vector<int> fl;
      try {
        fl = fsai_numeric_batched(jobs, bst);
      } catch (...) {
        cudaStreamDestroy(bst);
        throw;
      }
      cudaStreamDestroy(bst);
      const double share = (now_seconds() - t1) / (double)jobs.size();
      for (size_t k = 0; k < batched.size(); ++k) {
        flag_of[batched[k]] = fl[k];
        builders[batched[k]]->add_numeric_time(share);
      }
    }
    const double t2 = now_seconds();
    parallel(largest, [&](int p) {
      HierBuilder &b = *builders[p];
      if (more[p]) {
        b.end_level(flag_of[p]);
        while (b.begin_level()) b.end_level(b.fsai_numeric_single());
      }
      bt->b.h[p] = b.finish(false);
      builders[p].reset();
    });
    const double t3 = now_seconds();
    wall[0] = t1 - t0;
    wall[1] = t2 - t1;
    wall[2] = t3 - t2;
    bt->b.order.resize(nprob);
    std::iota(bt->b.order.begin(), bt->b.order.end(), 0);
    std::stable_sort(bt->b.order.begin(), bt->b.order.end(), [&](int a, int c) {
      return bt->b.h[a]->levels[0].A.nnz > bt->b.h[c]->levels[0].A.nnz;
    });
    if (prm->batch_grouped && group_supported(bt->b.h)) bt->b.group = group_build(bt->b.h, *prm);
    CHRONOS_REQUIRE(bt->b.group || prm->use_graph, CHRONOS_EINVAL,
                    "these problems need the per-problem batch path, which needs use_graph = 1");
    // the grouped solve tunes its stacked operators itself; the per-problem
    // path runs each problem's own operators
    if (!bt->b.group)
      for (auto &h : bt->b.h) tune_hierarchy(*h);
    bt->b.wall[3] = now_seconds() - t3;
    bt->b.wall[4] = now_seconds() - t0;
    *out = bt.release();
  });
}

int chronos_batch_solve(chronos_batch *bt, const double *const *b_h, double *const *x_h,
                        int itmax, double tol, int *iters, int *flags, double *seconds) {
  return batch_guard([&] {
    CHRONOS_REQUIRE(bt && b_h && x_h && iters && flags, CHRONOS_EINVAL, "null argument");
    Batch &B = bt->b;
    const int np = (int)B.h.size();
    if (B.group) {
      std::vector<const double *> bb(b_h, b_h + np);
      std::vector<double *> xx(x_h, x_h + np);
      group_solve(*B.group, bb, xx, itmax, tol, iters, flags, seconds);
      return;
    }
    std::vector<DBuf<double>> bd(np), xd(np);
    std::vector<char> zero(np, 0);
    for (int p = 0; p < np; ++p) {
      Hier &h = *B.h[p];
      const int n = h.levels[0].n;
      double s = 0.0;
      for (int i = 0; i < n; ++i) s += b_h[p][i] * b_h[p][i];
      zero[p] = s == 0.0;
      bd[p].upload(b_h[p], n, h.st);
      xd[p].upload(x_h[p], n, h.st);
      CHRONOS_CUDA(cudaStreamSynchronize(h.st));
    }
    cudaStream_t fork;
    CHRONOS_CUDA(cudaStreamCreateWithFlags(&fork, cudaStreamNonBlocking));
    cudaEvent_t start;
    std::vector<cudaEvent_t> done(np);
    CHRONOS_CUDA(cudaEventCreate(&start));
    for (auto &e : done) CHRONOS_CUDA(cudaEventCreate(&e));
    CHRONOS_CUDA(cudaEventRecord(start, fork));
    for (int p : B.order) {
      Hier &h = *B.h[p];
      CHRONOS_CUDA(cudaStreamWaitEvent(h.st, start, 0));
      if (!zero[p]) h.pcg_enqueue(bd[p].get(), xd[p].get(), itmax, tol);
      CHRONOS_CUDA(cudaEventRecord(done[p], h.st));
    }
    float ms = 0.f;
    for (int p = 0; p < np; ++p) {
      CHRONOS_CUDA(cudaEventSynchronize(done[p]));
      float t = 0.f;
      CHRONOS_CUDA(cudaEventElapsedTime(&t, start, done[p]));
      ms = std::max(ms, t);
    }
    for (int p = 0; p < np; ++p) {
      Hier &h = *B.h[p];
      const int n = h.levels[0].n;
      if (zero[p]) {                       // PCG_CJ.m:12-16
        std::fill(x_h[p], x_h[p] + n, 0.0);
        iters[p] = 0;
        flags[p] = 0;
        continue;
      }
      xd[p].download(x_h[p], n, h.st);
      CHRONOS_CUDA(cudaStreamSynchronize(h.st));
      h.pcg_collect(tol, &iters[p], &flags[p]);
    }
    cudaEventDestroy(start);
    for (auto &e : done) cudaEventDestroy(e);
    cudaStreamDestroy(fork);
    if (seconds) *seconds = ms * 1e-3;
  });
}

int chronos_batch_setup_wall(const chronos_batch *bt, double *t5) {
  return batch_guard([&] {
    CHRONOS_REQUIRE(bt && t5, CHRONOS_EINVAL, "bad argument");
    for (int i = 0; i < 5; ++i) t5[i] = bt->b.wall[i];
  });
}

int chronos_batch_setup_phases(const chronos_batch *bt, double *t, int n) {
  return batch_guard([&] {
    CHRONOS_REQUIRE(bt && t && n >= 0, CHRONOS_EINVAL, "bad argument");
    for (int i = 0; i < n; ++i) t[i] = 0.0;
    for (const auto &h : bt->b.h)
      for (int i = 0; i < n && i < (int)h->times.size(); ++i) t[i] += h->times[i];
  });
}

int chronos_batch_info(const chronos_batch *bt, int p, int *nlev, int *n0) {
  return batch_guard([&] {
    CHRONOS_REQUIRE(bt && nlev && n0 && p >= 0 && p < (int)bt->b.h.size(), CHRONOS_EINVAL,
                    "bad argument");
    *nlev = (int)bt->b.h[p]->levels.size();
    *n0 = bt->b.h[p]->levels[0].n;
  });
}

int chronos_batch_free(chronos_batch *bt) {
  return batch_guard([&] { delete bt; });
}

}  // extern "C"
