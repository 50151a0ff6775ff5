// Device memory and common helpers of the engine: errors, the per-device
// cache of large arrays (DevicePool), typed device arrays (DevArray), the
// FFT tables of the generic kernels, set-up timing marks and NVTX ranges.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <memory>
#include <chrono>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>
#include "agdeblend_gpu.h"
#include "fast.cuh"
#include "kernels.cuh"
#include "plan.hpp"
#include "wavelet_fast.cuh"
#include "line_dft.cuh"
#include "nn_api.hpp"
#include "space_tc.cuh"

namespace agd {

// NVTX range over a scope (host phases of a call, visible in nsys / ncu
// timelines as "agd <phase>")
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

// Parts of the engine set-up on stderr when AGD_GPU_TIMING=1: host wall
// clock since the previous mark of this thread, after a device
// synchronisation (reset: start a new sequence without printing).
inline void setup_mark(const char *part, bool reset = false) {
  static const bool on = [] {
    const char *env = std::getenv("AGD_GPU_TIMING");
    return env != nullptr && env[0] == '1';
  }();
  if (!on) return;
  static thread_local std::chrono::steady_clock::time_point t;
  cudaDeviceSynchronize();
  const auto n = std::chrono::steady_clock::now();
  if (!reset)
    std::fprintf(stderr, "agd timing:   set-up/%-12s %8.2f ms\n", part,
                 std::chrono::duration<double, std::milli>(n - t).count());
  t = n;
}

struct DeviceError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

static void check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    char buf[512];
    std::snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    throw DeviceError(buf);
  }
}
#define CK(x) check((x), #x)

// Device blocks of finished problems kept for the next problem on the same
// device: a deblending call allocates its large arrays (model, intermediates,
// traces, records) once per call, and a fresh cudaMalloc of gigabytes costs
// page mapping that can exceed the solve itself.  Blocks enter the cache
// only from the destructor of an engine whose stream has been synchronised,
// so no kernel can still use them.  Best fit within a factor of two; at most
// half the device memory is held (AGD_GPU_CACHE=0 disables the cache;
// agd_gpu_release_cache frees it).
class DevicePool {
 public:
  static void *take(size_t bytes) {
    if (injected_alloc_failure()) throw DeviceError("injected device allocation failure");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (enabled()) {
      std::lock_guard<std::mutex> g(mu());
      auto &m = free_blocks()[dev];
      auto it = m.lower_bound(bytes);
      if (it != m.end() && it->first <= 2 * bytes + (size_t(1) << 20)) {
        void *p = it->second;
        held() -= it->first;
        m.erase(it);
        return p;
      }
    }
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaErrorMemoryAllocation) {
      cudaGetLastError();
      release_device(dev);
      e = cudaMalloc(&p, bytes);
    }
    CK(e);
    std::lock_guard<std::mutex> g(mu());
    sizes()[p] = bytes;
    return p;
  }

  static void put(void *p) {
    if (p == nullptr) return;
    int dev = 0;
    size_t total = 0;
    if (!enabled() || cudaGetDevice(&dev) != cudaSuccess || (total = device_total(dev)) == 0) {
      drop(p);
      return;
    }
    std::lock_guard<std::mutex> g(mu());
    const size_t bytes = sizes()[p];
    if (held() + bytes > total / 2) {
      sizes().erase(p);
      cudaFree(p);
      return;
    }
    free_blocks()[dev].emplace(bytes, p);
    held() += bytes;
  }

  static void release_device(int dev) {
    std::lock_guard<std::mutex> g(mu());
    auto &m = free_blocks()[dev];
    for (auto &kv : m) {
      held() -= kv.first;
      sizes().erase(kv.second);
      cudaFree(kv.second);
    }
    m.clear();
  }

  static void release_all() {
    std::vector<int> devs;
    {
      std::lock_guard<std::mutex> g(mu());
      for (auto &kv : free_blocks()) devs.push_back(kv.first);
    }
    int cur = 0;
    cudaGetDevice(&cur);
    for (int d : devs) {
      cudaSetDevice(d);
      release_device(d);
    }
    cudaSetDevice(cur);
  }

 private:
  // the device's memory size, queried once (a memory-information query on
  // every return would cost a driver call each)
  static size_t device_total(int dev) {
    {
      std::lock_guard<std::mutex> g(mu());
      auto it = totals().find(dev);
      if (it != totals().end()) return it->second;
    }
    size_t freeb = 0, total = 0;
    if (cudaMemGetInfo(&freeb, &total) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    std::lock_guard<std::mutex> g(mu());
    totals()[dev] = total;
    return total;
  }
  static std::map<int, size_t> &totals() {
    static std::map<int, size_t> m;
    return m;
  }
  static bool enabled() {
    static const bool on = [] {
      const char *env = std::getenv("AGD_GPU_CACHE");
      return !(env != nullptr && env[0] == '0');
    }();
    return on;
  }
  static void drop(void *p) {
    {
      std::lock_guard<std::mutex> g(mu());
      sizes().erase(p);
    }
    cudaFree(p);
  }
  static std::mutex &mu() {
    static std::mutex m;
    return m;
  }
  static std::map<int, std::multimap<size_t, void *>> &free_blocks() {
    static std::map<int, std::multimap<size_t, void *>> m;
    return m;
  }
  static std::map<void *, size_t> &sizes() {
    static std::map<void *, size_t> m;
    return m;
  }
  static size_t &held() {
    static size_t h = 0;
    return h;
  }
};

template <typename T>
class DevArray {
 public:
  DevArray() = default;
  DevArray(const DevArray &) = delete;
  DevArray &operator=(const DevArray &) = delete;
  DevArray(DevArray &&o) noexcept : p_(o.p_), n_(o.n_), pooled_(o.pooled_) {
    o.p_ = nullptr;
    o.n_ = 0;
    o.pooled_ = false;
  }
  DevArray &operator=(DevArray &&o) noexcept {
    if (this != &o) {
      release();
      p_ = o.p_;
      n_ = o.n_;
      pooled_ = o.pooled_;
      o.p_ = nullptr;
      o.n_ = 0;
      o.pooled_ = false;
    }
    return *this;
  }
  ~DevArray() { release(); }
  void alloc(size_t n) {
    release();
    if (n && injected_alloc_failure())
      throw DeviceError("injected device allocation failure");
    if (n) CK(cudaMalloc(reinterpret_cast<void **>(&p_), n * sizeof(T)));
    n_ = n;
  }
  // From the device cache; the array must live until its engine's stream
  // is idle (engine members: the engine synchronises before destruction).
  void alloc_pooled(size_t n) {
    release();
    if (n) {
      p_ = static_cast<T *>(DevicePool::take(n * sizeof(T)));
      pooled_ = true;
    }
    n_ = n;
  }
  void upload(const std::vector<T> &v, cudaStream_t s) {
    alloc(v.size());
    if (n_) CK(cudaMemcpyAsync(p_, v.data(), n_ * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  T *get() const { return p_; }
  size_t size() const { return n_; }
  size_t bytes() const { return n_ * sizeof(T); }
  void release() {
    if (p_) {
      if (pooled_)
        DevicePool::put(p_);
      else
        cudaFree(p_);
    }
    p_ = nullptr;
    n_ = 0;
    pooled_ = false;
  }

 private:
  T *p_ = nullptr;
  size_t n_ = 0;
  bool pooled_ = false;
};

// Distinct FFT lengths with their radix lists and twiddle tables.
template <typename R>
struct FftTable {
  std::vector<FftDesc> descs;
  std::vector<Cx<R>> tw;
  std::map<int, int> index;

  int get(int n) {
    auto it = index.find(n);
    if (it != index.end()) return it->second;
    FftDesc d{};
    d.n = n;
    d.nf = 0;
    int m = n;
    for (int r : {4, 2, 3, 5}) {
      while (m % r == 0) {
        d.radix[d.nf++] = r;
        m /= r;
      }
    }
    for (int p = 7; m > 1; p += 2) {
      while (m % p == 0) {
        if (d.nf >= kMaxFactors) throw DeviceError("FFT length has too many factors");
        d.radix[d.nf++] = p;
        m /= p;
      }
    }
    d.tw_off = (long)tw.size();
    for (int k = 0; k < n; ++k) {
      const double a = -2.0 * 3.14159265358979323846 * (double)k / (double)n;
      Cx<R> w;
      w.x = (R)std::cos(a);
      w.y = (R)std::sin(a);
      tw.push_back(w);
    }
    const int id = (int)descs.size();
    descs.push_back(d);
    index[n] = id;
    return id;
  }
};

static int optin_smem() {
  int dev = 0;
  int v = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  return v;
}

}  // namespace agd
