// Shared helpers of the chronos_b200 library: status handling, device buffers,
// warp/block reductions.  sm_100a only.
#pragma once

#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "errors.h"

namespace chronos {

#define CHRONOS_CUDA(call)                                                        \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      throw ::chronos::Error(CHRONOS_ECUDA, std::string(#call) + ": " +             \
                                                cudaGetErrorString(e_) + " at " +   \
                                                __FILE__ + ":" + std::to_string(__LINE__)); \
    }                                                                               \
  } while (0)

#define CHRONOS_CHECK_LAUNCH() CHRONOS_CUDA(cudaGetLastError())

// Bytes held by live DBuf allocations of this process, and the cap that
// CHRONOS_DEVICE_ALLOC_CAP (bytes; unset or 0: none) puts on them.  The cap
// turns an allocation beyond it into CHRONOS_ENOMEM exactly as a failing
// cudaMalloc would, so out-of-memory handling is testable without filling a
// GPU.
inline std::atomic<int64_t> &device_bytes_live() {
  static std::atomic<int64_t> live{0};
  return live;
}
inline int64_t device_alloc_cap() {
  static const int64_t cap = [] {
    const char *e = std::getenv("CHRONOS_DEVICE_ALLOC_CAP");
    return e ? (int64_t)std::atoll(e) : (int64_t)0;
  }();
  return cap;
}

// Deferred frees.  cudaFree waits for all work queued on the device, so
// while a batch setup builds hierarchies on several host threads, one
// thread's free of a setup temporary would wait for every other thread's
// queued kernels.  Inside a DeferFrees scope (any thread) the buffers a DBuf
// lets go of are kept -- never reused -- and freed when the outermost scope
// ends, after one device synchronisation.  They stay counted in
// device_bytes_live() until then.
struct DeferredFrees {
  std::mutex mu;
  std::vector<std::pair<void *, int64_t>> list;
  std::atomic<int> depth{0};
};
inline DeferredFrees &deferred_frees() {
  static DeferredFrees d;
  return d;
}
inline void flush_deferred_frees() {
  DeferredFrees &d = deferred_frees();
  std::vector<std::pair<void *, int64_t>> list;
  {
    std::lock_guard<std::mutex> lk(d.mu);
    list.swap(d.list);
  }
  if (list.empty()) return;
  cudaDeviceSynchronize();
  for (auto &e : list) {
    cudaFree(e.first);
    device_bytes_live() -= e.second;
  }
}
class DeferFrees {
 public:
  DeferFrees() { deferred_frees().depth++; }
  ~DeferFrees() {
    if (--deferred_frees().depth == 0) flush_deferred_frees();
  }
  DeferFrees(const DeferFrees &) = delete;
  DeferFrees &operator=(const DeferFrees &) = delete;
};

// Owning device allocation (cudaMalloc / cudaFree), movable, typed.
template <typename T>
class DBuf {
 public:
  DBuf() = default;
  explicit DBuf(size_t n) { alloc(n); }
  ~DBuf() { release(); }
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  DBuf(DBuf &&o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
  DBuf &operator=(DBuf &&o) noexcept {
    if (this != &o) { release(); p_ = o.p_; n_ = o.n_; o.p_ = nullptr; o.n_ = 0; }
    return *this;
  }
  void alloc(size_t n) {
    release();
    if (n == 0) return;
    const int64_t bytes = (int64_t)(n * sizeof(T)), cap = device_alloc_cap();
    if (cap > 0 && device_bytes_live().load() + bytes > cap)
      throw Error(CHRONOS_ENOMEM, "allocation of " + std::to_string(bytes) +
                                      " bytes beyond CHRONOS_DEVICE_ALLOC_CAP");
    cudaError_t e = cudaMalloc(&p_, n * sizeof(T));
    if (e != cudaSuccess) {
      p_ = nullptr;
      cudaGetLastError();
      throw Error(CHRONOS_ENOMEM, "cudaMalloc of " + std::to_string(n * sizeof(T)) +
                                      " bytes failed: " + cudaGetErrorString(e));
    }
    n_ = n;
    device_bytes_live() += bytes;
  }
  void release() {
    if (p_) {
      DeferredFrees &d = deferred_frees();
      if (d.depth.load() > 0) {
        std::lock_guard<std::mutex> lk(d.mu);
        d.list.emplace_back(p_, (int64_t)(n_ * sizeof(T)));
      } else {
        cudaFree(p_);
        device_bytes_live() -= (int64_t)(n_ * sizeof(T));
      }
    }
    p_ = nullptr;
    n_ = 0;
  }
  void upload(const T *h, size_t n, cudaStream_t s = 0) {
    if (n_ < n) alloc(n);
    if (n) CHRONOS_CUDA(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void upload(const std::vector<T> &h, cudaStream_t s = 0) { upload(h.data(), h.size(), s); }
  void download(T *h, size_t n, cudaStream_t s = 0) const {
    if (n) CHRONOS_CUDA(cudaMemcpyAsync(h, p_, n * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
  std::vector<T> to_host(cudaStream_t s = 0) const {
    std::vector<T> h(n_);
    download(h.data(), n_, s);
    CHRONOS_CUDA(cudaStreamSynchronize(s));
    return h;
  }
  void zero(cudaStream_t s = 0) {
    if (n_) CHRONOS_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s));
  }
  T *get() const { return p_; }
  size_t size() const { return n_; }
  operator T *() const { return p_; }

 private:
  T *p_ = nullptr;
  size_t n_ = 0;
};

// ---- device helpers ------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over groups of L consecutive lanes (L a power of two <= 32); every lane
// of the group ends with the group sum.
template <int L, typename T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block reduction of one double per thread; result valid in
// thread 0.  blockDim.x must be a multiple of 32 and <= 1024.
__device__ __forceinline__ double block_sum(double v, double *smem32) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) smem32[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (wid == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    r = lane < nw ? smem32[lane] : 0.0;
    r = warp_sum(r);
  }
  __syncthreads();
  return r;
}

// ---- programmatic dependent launch ------------------------------------------
// Kernels of the solve loop begin with pdl_begin(): griddepcontrol.wait
// returns once the preceding kernel of the stream has completed and its
// writes are visible (a no-op for a kernel launched without the attribute),
// then griddepcontrol.launch_dependents lets the next kernel's blocks be
// scheduled while this one drains.  Nothing is read or written before the
// wait, so the order of memory effects is the plain stream order.
__device__ __forceinline__ void pdl_begin() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" :::);
}

// Programmatic dependent launch is on unless CHRONOS_PDL=0 in the environment.
inline bool pdl_enabled() {
  static const int on = [] {
    const char *e = std::getenv("CHRONOS_PDL");
    return (e && e[0] == '0') ? 0 : 1;
  }();
  return on != 0;
}

// Launch of a kernel that begins with pdl_begin(), with the programmatic
// stream serialization attribute when enabled.
template <typename... KArgs, typename... Args>
void launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  CHRONOS_CUDA(cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...));
}

inline int num_sms() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    CHRONOS_CUDA(cudaGetDevice(&dev));
    CHRONOS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  }
  return sms;
}

inline unsigned ceil_div(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

}  // namespace chronos
