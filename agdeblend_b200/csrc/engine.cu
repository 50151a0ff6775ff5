// Device engine of the deblending path: turns a Plan into device tables and
// launch lists, runs the operator, the ISTA solver and blending, and exports
// the C API (include/agdeblend.h) and the extension API
// (include/agdeblend_gpu.h).  Built twice: float (libagdeblend.so) and, with
// -DAGD_DOUBLE, double (libagdeblend_double.so).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "agdeblend_gpu.h"
#include "fast.cuh"
#include "kernels.cuh"
#include "plan.hpp"
#include "wavelet_fast.cuh"

namespace agd {

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

template <typename T>
class DevArray {
 public:
  DevArray() = default;
  DevArray(const DevArray &) = delete;
  DevArray &operator=(const DevArray &) = delete;
  DevArray(DevArray &&o) noexcept : p_(o.p_), n_(o.n_) {
    o.p_ = nullptr;
    o.n_ = 0;
  }
  DevArray &operator=(DevArray &&o) noexcept {
    if (this != &o) {
      release();
      p_ = o.p_;
      n_ = o.n_;
      o.p_ = nullptr;
      o.n_ = 0;
    }
    return *this;
  }
  ~DevArray() { release(); }
  void alloc(size_t n) {
    release();
    if (n) CK(cudaMalloc(reinterpret_cast<void **>(&p_), n * sizeof(T)));
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
    if (p_) cudaFree(p_);
    p_ = nullptr;
    n_ = 0;
  }

 private:
  T *p_ = nullptr;
  size_t n_ = 0;
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

template <typename R>
class Engine {
 public:
  using C = Cx<R>;

  struct AxisLaunch {
    DevArray<AxisJob<R>> jobs;
    DevArray<int> cta_job;
    DevArray<long> cta_line0;
    int n_cta = 0;
    int lpc = 0;
    size_t smem = 0;
  };
  struct TimeLaunch {
    DevArray<int> cta_job;
    DevArray<int> cta_trace0;
    int n_cta = 0;
    int nb = 0;
    size_t smem = 0;
  };
  struct GatherLaunch {
    DevArray<Contrib> contrib;
    DevArray<long> chunk_ptr;
    int n_chunk = 0;
    int chunk = 512;
    long n_contrib = 0;
  };

  Plan plan;
  cudaStream_t stream = nullptr;
  int smem_max = 0;
  FftTable<R> fft;
  DevArray<FftDesc> d_descs;
  DevArray<C> d_tw;

  DevArray<C> X, S0, S1, G;
  DevArray<R> Y, rec_d, rec_r, data_dev;
  DevArray<uint8_t> mute;
  DevArray<R> space_scale, space_fold, time_taper;
  DevArray<long> blend_rec;
  DevArray<int> blend_ts, blend_n;
  DevArray<int> wsrc;
  DevArray<C> spectra;
  DevArray<long> spec_off;
  DevArray<long> wt_dst;  // trace buffer offset of each window trace
  DevArray<int> wt_C;
  DevArray<TimeJob<R>> time_jobs;
  DevArray<WaveletJob<R>> wav_jobs;
  DevArray<long> out_ptr, out_src, out_dst;
  DevArray<int> out_nt;
  DevArray<R> scalar;
  DevArray<double> dscalar;

  std::vector<AxisLaunch> fwd, adj_update, adj_plain;
  TimeLaunch time_fwd, time_adj, wav;

  // shape-specialised path (fast.cuh), used when every window has the same
  // space and time FFT lengths and an instantiation exists
  using SpaceFwdFn = void (*)(PlaneBatches<R>);
  using SpaceAdjFn = void (*)(PlaneBatches<R>, int, R, R, const R *, R *);
  using TimeFwdFn = void (*)(const TimeJob<R> *, const int *, const int *);
  using TimeAdjFn = void (*)(const TimeJob<R> *, const int *, const int *, const R *, int);
  static constexpr int kTimeNB = 32;  // traces per block of the fast time kernels
  struct PlaneLaunch {
    DevArray<PlaneBatch<R>> batch;
    int n_batch = 0;
    int grid = 0;
    int nt = 0;
    size_t smem = 0;
    PlaneBatches<R> batches() const { return PlaneBatches<R>{batch.get(), n_batch}; }
  };
  bool fast = false;
  SpaceFwdFn sp_fwd = nullptr;
  SpaceAdjFn sp_adj = nullptr;
  TimeFwdFn tm_fwd = nullptr;
  TimeAdjFn tm_adj = nullptr;
  int nt_fwd = 0, np_fwd = 0, nt_adj = 0, np_adj = 0;  // threads, planes per batch
  size_t smem_fwd = 0, smem_adj = 0;
  int n_sm = 148;
  PlaneLaunch pl_fwd, pl_adj, pl_adj_plain;
  TimeLaunch tf_fast, ta_fast;
  DevArray<TimeJob<R>> time_jobs_fast;
  GatherLaunch g_fwd, g_input;
  std::vector<long> trace_off;   // per window, in reals
  std::vector<long> patch_off;   // per patch, in reals
  long n_wtraces = 0;
  long data_size = 0;
  long out_traces = 0;
  bool wavelets = false;
  // prime-factor wavelet kernel (wavelet_fast.cuh), used when every window's
  // trace length factors into supported coprime prime powers
  bool wav_fast = false;
  DevArray<WaveletFastJob<R>> wavf_jobs;
  DevArray<int> kperm;
  TimeLaunch wavf;
  R stepsize = 0;

  explicit Engine(Plan &&p) : plan(std::move(p)) {
    CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    smem_max = optin_smem();
    {
      int dev = 0;
      CK(cudaGetDevice(&dev));
      CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
    }
    set_smem_limits();
    build();
  }

  ~Engine() {
    if (stream) {
      cudaStreamSynchronize(stream);
      release_graph();
      cudaStreamDestroy(stream);
    }
  }

  size_t device_bytes() const {
    return X.bytes() + S0.bytes() + S1.bytes() + G.bytes() + Y.bytes() + rec_d.bytes() +
           rec_r.bytes() + data_dev.bytes() + mute.bytes() + g_fwd.contrib.bytes() +
           g_input.contrib.bytes();
  }

  // Opt every dynamic-shared-memory kernel in to the device limit minus its
  // own static shared memory; smem_max becomes the smallest such limit.
  template <typename K>
  int opt_in(K kernel, int limit) {
    cudaFuncAttributes fa;
    CK(cudaFuncGetAttributes(&fa, kernel));
    const int dyn = limit - (int)fa.sharedSizeBytes;
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
    return dyn;
  }

  void set_smem_limits() {
    const int limit = smem_max;
    smem_max = std::min({opt_in(axis_pass<R>, limit), opt_in(time_c2r_ola<R>, limit),
                         opt_in(time_r2c<R>, limit), opt_in(wavelet_apply<R>, limit),
                         opt_in(wavelet_fast<R>, limit)});
  }

  // twiddle tables of the register DFTs in constant memory of the current
  // device (fast.cuh), shared by the fast space, time and wavelet kernels
  void upload_twiddles() {
    std::vector<C> tw(kTwTotal);
    for (int i = 0, off = 0; i < kNumTw; off += kTwSizes[i], ++i)
      for (int k = 0; k < kTwSizes[i]; ++k) {
        const double a = -2.0 * 3.14159265358979323846 * (double)k / (double)kTwSizes[i];
        tw[off + k].x = (R)std::cos(a);
        tw[off + k].y = (R)std::sin(a);
      }
    if (sizeof(R) == sizeof(float))
      CK(cudaMemcpyToSymbol(c_tw_f, tw.data(), tw.size() * sizeof(C)));
    else
      CK(cudaMemcpyToSymbol(c_tw_d, tw.data(), tw.size() * sizeof(C)));
  }

  // C = product of pairwise coprime prime powers with a register DFT
  static bool pfa_shape(int N, PfaShape &sh) {
    static const int kOk[] = {2, 3, 4, 5, 7, 8, 9, 11, 13, 16, 17, 19, 23, 25, 27, 32};
    sh = PfaShape{};
    sh.N = N;
    int n = N;
    for (int p = 2; n > 1; ++p) {
      if (n % p) continue;
      int q = 1;
      while (n % p == 0) {
        n /= p;
        q *= p;
      }
      if (std::find(std::begin(kOk), std::end(kOk), q) == std::end(kOk) ||
          sh.nf == kPfaMaxFactors)
        return false;
      sh.f[sh.nf++] = q;
    }
    for (int i = 0; i < sh.nf; ++i) {
      sh.s[i] = N / sh.f[i];
      sh.inv[i] = 1;
      while ((long)sh.s[i] * sh.inv[i] % sh.f[i] != 1 % sh.f[i]) ++sh.inv[i];
    }
    return true;
  }

  // position -> frequency after the forward passes (Chinese remainder map)
  static void pfa_kperm(const PfaShape &sh, std::vector<int> &out) {
    const long N = sh.N;
    for (long p = 0; p < N; ++p) {
      long k = 0;
      for (int i = 0; i < sh.nf; ++i) {
        const long ki = p * sh.inv[i] % sh.f[i];
        const long ei = (long)sh.s[i] * sh.inv[i] % N;
        k = (k + ki * ei) % N;
      }
      out.push_back((int)k);
    }
  }

  void build_wavelet_fast(const std::vector<WaveletJob<R>> &wj,
                          const std::vector<long> &wt_base) {
    const char *env = std::getenv("AGD_GPU_GENERIC");
    if (env != nullptr && env[0] == '1') return;
    const int nw = (int)plan.windows.size();
    std::vector<WaveletFastJob<R>> jobs(nw);
    std::vector<int> perm;
    std::map<int, long> perm_off;
    int n_max = 1;
    for (int w = 0; w < nw; ++w) {
      WaveletFastJob<R> &j = jobs[w];
      const int N = plan.windows[w].C;
      if (!pfa_shape(N, j.sh)) return;
      if (!perm_off.count(N)) {
        perm_off[N] = (long)perm.size();
        pfa_kperm(j.sh, perm);
      }
      n_max = std::max(n_max, N);
    }
    const size_t per_pair = (size_t)n_max * sizeof(C);
    const int np = (int)std::max<size_t>(1, std::min<size_t>(4, 60000 / per_pair));
    if (per_pair * np > (size_t)smem_max) return;
    kperm.upload(perm, stream);
    std::vector<int> cj, cp;
    for (int w = 0; w < nw; ++w) {
      const WindowPlan &W = plan.windows[w];
      WaveletFastJob<R> &j = jobs[w];
      j.y = wj[w].y;
      j.src = wj[w].src;
      j.kperm = kperm.get() + perm_off[W.C];
      j.blend_rec = blend_rec.get() + wt_base[w];
      j.blend_ts = blend_ts.get() + wt_base[w];
      j.blend_n = blend_n.get() + wt_base[w];
      j.n_traces = W.n_traces;
      for (int p = 0; p < (W.n_traces + 1) / 2; p += np) {
        cj.push_back(w);
        cp.push_back(p);
      }
    }
    wavf_jobs.upload(jobs, stream);
    wavf.cta_job.upload(cj, stream);
    wavf.cta_trace0.upload(cp, stream);
    wavf.n_cta = (int)cj.size();
    wavf.nb = np;
    wavf.smem = per_pair * np;
    upload_twiddles();
    wav_fast = true;
  }

  // ---------------------------------------------------------------- set-up

  void make_axis_launch(AxisLaunch &L, const std::vector<AxisJob<R>> &jobs) {
    if (jobs.empty()) return;
    int n_max = 1;
    for (const auto &j : jobs) n_max = std::max(n_max, fft.descs[j.fft].n);
    const size_t per_line = 2 * (size_t)n_max * sizeof(C);
    const size_t budget = 64 * 1024;
    int lpc = (int)std::max<size_t>(1, budget / per_line);
    lpc = std::min(lpc, 256);
    if (per_line * lpc > (size_t)smem_max) throw DeviceError("space axis too long");
    std::vector<int> cj;
    std::vector<long> cl;
    for (size_t i = 0; i < jobs.size(); ++i) {
      const long lines = jobs[i].outer * jobs[i].inner;
      for (long q = 0; q < lines; q += lpc) {
        cj.push_back((int)i);
        cl.push_back(q);
      }
    }
    L.jobs.upload(jobs, stream);
    L.cta_job.upload(cj, stream);
    L.cta_line0.upload(cl, stream);
    L.n_cta = (int)cj.size();
    L.lpc = lpc;
    L.smem = per_line * lpc;
  }

  void make_time_launch(TimeLaunch &L, size_t per_trace, int nb_cap) {
    int nb = nb_cap;
    while (nb > 1 && per_trace * nb > (size_t)std::min(smem_max, 160 * 1024)) nb /= 2;
    if (per_trace * nb > (size_t)smem_max)
      throw DeviceError("time window or trace too long for shared memory");
    std::vector<int> cj, ct;
    for (size_t w = 0; w < plan.windows.size(); ++w) {
      for (int t = 0; t < plan.windows[w].n_traces; t += nb) {
        cj.push_back((int)w);
        ct.push_back(t);
      }
    }
    L.cta_job.upload(cj, stream);
    L.cta_trace0.upload(ct, stream);
    L.n_cta = (int)cj.size();
    L.nb = nb;
    L.smem = per_trace * nb;
  }

  // Candidate instantiations of the fast space kernels for one padded shape
  // P0..P2 (window lengths 4P/5): threads, planes per batch, stages and
  // blocks per SM.  The two-stage kernels fill most of the shared memory with
  // one block per SM; the one-stage kernels run two or three blocks per SM
  // (two for 40-point lines, whose registers do not fit three).  The
  // fastest of each list is picked by timing on the problem (autotune_space).
  struct FwdVariant {
    SpaceFwdFn fn;
    int nt, np, stages;
    size_t smem;
  };
  struct AdjVariant {
    SpaceAdjFn fn;
    int nt, np, stages;
    size_t smem;
  };
  std::vector<FwdVariant> fwd_vars;
  std::vector<AdjVariant> adj_vars;
  int fwd_pick = 0, adj_pick = 0;

  template <int D, int P0, int P1, int P2, int NT, int NP, int ST, int MB>
  void add_fwd() {
    using Sh = PlaneShape<D, P0, P1, P2>;
    fwd_vars.push_back(FwdVariant{space_fwd_fast<R, D, P0, P1, P2, NT, NP, ST, MB>, NT, NP, ST,
                                  (size_t)ST * NP * Sh::size * sizeof(C)});
  }

  template <int D, int P0, int P1, int P2, int NT, int NP, int ST, int MB>
  void add_adj() {
    using Sh = PlaneShape<D, P0, P1, P2>;
    const size_t x = ST == 2 ? (size_t)NP * Sh::dense_P : 0;
    adj_vars.push_back(AdjVariant{space_adj_fast<R, D, P0, P1, P2, NT, NP, ST, MB>, NT, NP, ST,
                                  ((size_t)ST * NP * Sh::size + x) * sizeof(C)});
  }

  template <int D, int P0, int P1, int P2>
  static bool shape_is(const WindowPlan &W) {
    const int P[3] = {P0, P1, P2};
    if (W.D != D) return false;
    for (int d = 0; d < D; ++d)
      if (W.P[d] != P[d]) return false;
    return true;
  }

  bool space_cases(const WindowPlan &W) {
    fwd_vars.clear();
    adj_vars.clear();
    if constexpr (sizeof(R) == sizeof(float)) {
      if (shape_is<1, 40, 1, 1>(W)) {
        add_fwd<1, 40, 1, 1, 256, 256, 2, 1>();
        add_fwd<1, 40, 1, 1, 256, 96, 1, 2>();
        add_adj<1, 40, 1, 1, 192, 192, 2, 1>();
        add_adj<1, 40, 1, 1, 256, 96, 1, 2>();
      } else if (shape_is<1, 20, 1, 1>(W)) {
        add_fwd<1, 20, 1, 1, 256, 256, 2, 1>();
        add_fwd<1, 20, 1, 1, 256, 128, 1, 3>();
        add_adj<1, 20, 1, 1, 256, 256, 2, 1>();
        add_adj<1, 20, 1, 1, 256, 128, 1, 3>();
      } else if (shape_is<2, 20, 40, 1>(W)) {
        add_fwd<2, 20, 40, 1, 384, 16, 2, 1>();
        add_fwd<2, 20, 40, 1, 256, 12, 1, 2>();
        add_adj<2, 20, 40, 1, 384, 11, 2, 1>();
        add_adj<2, 20, 40, 1, 256, 12, 1, 2>();
      } else if (shape_is<2, 20, 20, 1>(W)) {
        add_fwd<2, 20, 20, 1, 384, 24, 2, 1>();
        add_fwd<2, 20, 20, 1, 256, 12, 1, 3>();
        add_adj<2, 20, 20, 1, 384, 20, 2, 1>();
        add_adj<2, 20, 20, 1, 256, 12, 1, 3>();
      } else if (shape_is<2, 40, 40, 1>(W)) {
        add_fwd<2, 40, 40, 1, 320, 8, 2, 1>();
        add_fwd<2, 40, 40, 1, 256, 6, 1, 2>();
        add_adj<2, 40, 40, 1, 256, 5, 2, 1>();
        add_adj<2, 40, 40, 1, 256, 6, 1, 2>();
      } else if (shape_is<3, 20, 20, 20>(W)) {
        add_fwd<3, 20, 20, 20, 512, 1, 2, 1>();
        add_fwd<3, 20, 20, 20, 256, 1, 1, 3>();
        add_adj<3, 20, 20, 20, 512, 1, 2, 1>();
        add_adj<3, 20, 20, 20, 256, 1, 1, 3>();
      }
    } else {
      // double: the two-stage kernels only (one-stage kernels with several
      // blocks per SM would spill), and one stage for the 20x20x20 planes
      if (shape_is<1, 40, 1, 1>(W)) {
        add_fwd<1, 40, 1, 1, 256, 128, 2, 1>();
        add_adj<1, 40, 1, 1, 192, 96, 2, 1>();
      } else if (shape_is<1, 20, 1, 1>(W)) {
        add_fwd<1, 20, 1, 1, 256, 256, 2, 1>();
        add_adj<1, 20, 1, 1, 256, 160, 2, 1>();
      } else if (shape_is<2, 20, 40, 1>(W)) {
        add_fwd<2, 20, 40, 1, 384, 8, 2, 1>();
        add_adj<2, 20, 40, 1, 384, 5, 2, 1>();
      } else if (shape_is<2, 20, 20, 1>(W)) {
        add_fwd<2, 20, 20, 1, 384, 12, 2, 1>();
        add_adj<2, 20, 20, 1, 384, 10, 2, 1>();
      } else if (shape_is<2, 40, 40, 1>(W)) {
        add_fwd<2, 40, 40, 1, 320, 4, 2, 1>();
        add_adj<2, 40, 40, 1, 256, 2, 2, 1>();
      } else if (shape_is<3, 20, 20, 20>(W)) {
        add_fwd<3, 20, 20, 20, 256, 1, 1, 1>();
        add_adj<3, 20, 20, 20, 256, 1, 1, 1>();
      }
    }
    return !fwd_vars.empty() && !adj_vars.empty();
  }

  // Times every candidate (one warm-up launch, then two timed ones with CUDA
  // events on the engine's stream, forward X -> S0 and adjoint S0 -> X with
  // the update epilogue) and keeps the fastest.  Choices are remembered per
  // shape, precision, problem size class and device, so later problems of
  // the same kind skip the timing.  AGD_GPU_SPACE_VARIANT="f,a" forces the
  // candidates (tests).
  void autotune_space(const std::vector<PlaneJob<R>> &jf, const std::vector<PlaneJob<R>> &ja,
                      const std::vector<long> &planes) {
    fwd_pick = adj_pick = 0;
    const char *env = std::getenv("AGD_GPU_SPACE_VARIANT");
    if (env != nullptr && env[0] != '\0') {
      int f = 0, a = 0;
      if (std::sscanf(env, "%d,%d", &f, &a) == 2) {
        fwd_pick = std::max(0, std::min(f, (int)fwd_vars.size() - 1));
        adj_pick = std::max(0, std::min(a, (int)adj_vars.size() - 1));
        return;
      }
    }
    if (fwd_vars.size() == 1 && adj_vars.size() == 1) return;
    long total = 0;
    for (long v : planes) total += v;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    const WindowPlan &W = plan.windows[0];
    char key[128];
    std::snprintf(key, sizeof key, "%d:%d:%d:%d:%d:%d:%d", dev, (int)sizeof(R), W.D, W.P[0],
                  W.D > 1 ? W.P[1] : 1, W.D > 2 ? W.P[2] : 1,
                  (int)std::log2((double)std::max(1L, total)));
    static std::mutex mu;
    static std::map<std::string, std::pair<int, int>> cache;
    {
      std::lock_guard<std::mutex> g(mu);
      auto it = cache.find(key);
      if (it != cache.end()) {
        fwd_pick = it->second.first;
        adj_pick = it->second.second;
        return;
      }
    }
    CK(cudaMemsetAsync(X.get(), 0, X.bytes(), stream));
    CK(cudaMemsetAsync(S0.get(), 0, S0.bytes(), stream));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    auto timed = [&](auto launch) {
      launch();
      CK(cudaEventRecord(e0, stream));
      launch();
      launch();
      CK(cudaEventRecord(e1, stream));
      CK(cudaEventSynchronize(e1));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      return ms;
    };
    float best = 1e30f;
    for (size_t v = 0; v < fwd_vars.size(); ++v) {
      const FwdVariant &fv = fwd_vars[v];
      if (fv.smem > (size_t)smem_max) continue;
      PlaneLaunch L;
      make_plane_launch(L, jf, planes, fv.nt, fv.np, fv.smem, fv.fn);
      const float ms = timed([&] {
        fv.fn<<<L.grid, L.nt, L.smem, stream>>>(L.batches());
        CK(cudaGetLastError());
      });
      if (ms < best) {
        best = ms;
        fwd_pick = (int)v;
      }
    }
    best = 1e30f;
    for (size_t v = 0; v < adj_vars.size(); ++v) {
      const AdjVariant &av = adj_vars[v];
      if (av.smem > (size_t)smem_max) continue;
      PlaneLaunch L;
      make_plane_launch(L, ja, planes, av.nt, av.np, av.smem, av.fn);
      const float ms = timed([&] {
        av.fn<<<L.grid, L.nt, L.smem, stream>>>(L.batches(), kUpdateThreshold, (R)0, (R)0,
                                                 nullptr, scalar.get());
        CK(cudaGetLastError());
      });
      if (ms < best) {
        best = ms;
        adj_pick = (int)v;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::lock_guard<std::mutex> g(mu);
    cache[key] = {fwd_pick, adj_pick};
  }

  bool pick_fast() {
    if (plan.windows.empty()) return false;
    const char *env = std::getenv("AGD_GPU_GENERIC");
    if (env != nullptr && env[0] == '1') return false;
    const WindowPlan &W0 = plan.windows[0];
    for (const WindowPlan &W : plan.windows) {
      if (W.D != W0.D || W.Pt != W0.Pt || W.Lt != W0.Lt || W.Lt % 2 != 0) return false;
      // the kernels assume L = 4P/5 in space and Lt = 2h = 4Pt/5 in time
      if (W.Lt * 5 != W.Pt * 4) return false;
      for (int d = 0; d < W.D; ++d)
        if (W.P[d] != W0.P[d] || W.L[d] * 5 != W.P[d] * 4) return false;
    }
    if (!space_cases(W0)) return false;
    if (W0.Pt == 320) {
      tm_fwd = time_fwd_fast<R, 16, 10, kTimeNB>;
      tm_adj = time_adj_fast<R, 16, 10, kTimeNB>;
    } else if (W0.Pt == 160) {
      tm_fwd = time_fwd_fast<R, 8, 10, kTimeNB>;
      tm_adj = time_adj_fast<R, 8, 10, kTimeNB>;
    } else {
      return false;
    }
    return true;
  }

  // Persistent, double-buffered batches of np planes; grid = resident blocks.
  template <typename K>
  void make_plane_launch(PlaneLaunch &L, const std::vector<PlaneJob<R>> &jobs,
                         const std::vector<long> &planes, int nt, int np, size_t smem,
                         K kernel) {
    if (smem > (size_t)smem_max) throw DeviceError("space planes too large");
    std::vector<PlaneBatch<R>> bt;
    for (size_t i = 0; i < jobs.size(); ++i)
      for (long q = 0; q < planes[i]; q += np) {
        PlaneBatch<R> x{};
        x.src = jobs[i].src + q * jobs[i].src_plane;
        x.dst = jobs[i].dst + q * jobs[i].dst_plane;
        x.count = (int)std::min<long>(np, planes[i] - q);
        bt.push_back(x);
      }
    L.batch.upload(bt, stream);
    L.n_batch = (int)bt.size();
    L.nt = nt;
    L.smem = smem;
    int per_sm = 1;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, nt, L.smem));
    L.grid = std::max(1, std::min(L.n_batch, std::max(per_sm, 1) * n_sm));
  }

  void build_fast(const std::vector<TimeJob<R>> &tj_generic) {
    const int limit = optin_smem();
    int dyn = std::min(opt_in(tm_fwd, limit), opt_in(tm_adj, limit));
    for (const FwdVariant &v : fwd_vars) dyn = std::min(dyn, opt_in(v.fn, limit));
    for (const AdjVariant &v : adj_vars) dyn = std::min(dyn, opt_in(v.fn, limit));
    smem_max = std::min(smem_max, dyn);
    upload_twiddles();
    const int nw = (int)plan.windows.size();
    std::vector<PlaneJob<R>> jf(nw), ja(nw);
    const WindowPlan &W0 = plan.windows[0];
    long dense_P = 1, dense_L = 1;
    for (int d = 0; d < W0.D; ++d) {
      dense_P *= W0.P[d];
      dense_L *= W0.L[d];
    }
    std::vector<long> planes(nw);
    std::vector<TimeJob<R>> tj = tj_generic;
    for (int w = 0; w < nw; ++w) {
      const WindowPlan &W = plan.windows[w];
      planes[w] = (long)W.T * W.F;
      PlaneJob<R> j{};
      j.src = X.get() + W.model_off;
      j.dst = S0.get() + W.model_off;
      j.src_plane = dense_P;
      j.dst_plane = dense_L;
      jf[w] = j;
      j.src = S0.get() + W.model_off;
      j.dst = X.get() + W.model_off;
      j.src_plane = dense_L;
      j.dst_plane = dense_P;
      ja[w] = j;
      tj[w].z = S0.get() + W.model_off;
    }
    autotune_space(jf, ja, planes);
    const FwdVariant &fv = fwd_vars[fwd_pick];
    const AdjVariant &av = adj_vars[adj_pick];
    sp_fwd = fv.fn;
    sp_adj = av.fn;
    nt_fwd = fv.nt;
    np_fwd = fv.np;
    smem_fwd = fv.smem;
    nt_adj = av.nt;
    np_adj = av.np;
    smem_adj = av.smem;
    make_plane_launch(pl_fwd, jf, planes, nt_fwd, np_fwd, smem_fwd, sp_fwd);
    make_plane_launch(pl_adj, ja, planes, nt_adj, np_adj, smem_adj, sp_adj);
    pending_plane_plain = ja;
    pending_planes = planes;
    time_jobs_fast.upload(tj, stream);
    const int h = plan.windows[0].h;
    const int LS = plan.windows[0].Pt / 2 + 1;
    const size_t per_fwd = 2 * (size_t)LS * sizeof(C) + (size_t)h * sizeof(R);
    const size_t per_adj = (size_t)LS * sizeof(C) + 2 * (size_t)(2 * h) * sizeof(R);
    make_fixed_time_launch(tf_fast, per_fwd * kTimeNB);
    make_fixed_time_launch(ta_fast, per_adj * kTimeNB);
  }

  std::vector<PlaneJob<R>> pending_plane_plain;
  std::vector<long> pending_planes;

  void make_fixed_time_launch(TimeLaunch &L, size_t smem) {
    if (smem > (size_t)smem_max) throw DeviceError("time window too long for shared memory");
    std::vector<int> cj, ct;
    for (size_t w = 0; w < plan.windows.size(); ++w)
      for (int t = 0; t < plan.windows[w].n_traces; t += kTimeNB) {
        cj.push_back((int)w);
        ct.push_back(t);
      }
    L.cta_job.upload(cj, stream);
    L.cta_trace0.upload(ct, stream);
    L.n_cta = (int)cj.size();
    L.nb = kTimeNB;
    L.smem = smem;
  }

  void make_gather(GatherLaunch &G, const std::vector<Contrib> &list, long record_size) {
    G.n_chunk = (int)((record_size + G.chunk - 1) / G.chunk);
    std::vector<long> count(G.n_chunk + 1, 0);
    for (const Contrib &c : list) {
      if (c.n <= 0) continue;
      const long a = c.rec / G.chunk;
      const long b = (c.rec + c.n - 1) / G.chunk;
      for (long k = a; k <= b; ++k) count[k + 1]++;
    }
    for (int k = 0; k < G.n_chunk; ++k) count[k + 1] += count[k];
    std::vector<Contrib> flat(count[G.n_chunk]);
    std::vector<long> fill(count.begin(), count.end() - 1);
    for (const Contrib &c : list) {
      if (c.n <= 0) continue;
      const long a = c.rec / G.chunk;
      const long b = (c.rec + c.n - 1) / G.chunk;
      for (long k = a; k <= b; ++k) flat[fill[k]++] = c;
    }
    G.contrib.upload(flat, stream);
    G.chunk_ptr.upload(count, stream);
    G.n_contrib = (long)list.size();
  }

  void build() {
    const long M = plan.model_size;
    const int nw = (int)plan.windows.size();
    // ---- FFT tables and per-window trace tables
    int Pt_max = 1, C_max = 1, maxD = 0;
    trace_off.assign(nw, 0);
    long toff = 0;
    std::vector<R> sscale, sfold, ttaper;
    std::vector<long> brec, wdst;
    std::vector<int> bts, bn, ws, wC;
    std::vector<long> ttaper_off(nw);
    std::vector<TimeJob<R>> tj(nw);
    std::vector<WaveletJob<R>> wj(nw);
    std::vector<long> wt_base(nw);
    for (int w = 0; w < nw; ++w) {
      const WindowPlan &W = plan.windows[w];
      trace_off[w] = toff;
      wt_base[w] = (long)sscale.size();
      for (int t = 0; t < W.n_traces; ++t) {
        // scaler then space tapers from the last dim to the first, the
        // multiplication order of src/fk.c:343-347
        R s = W.scaler;
        R fold = (R)1;
        int r = t;
        int coord[kMaxSpaceDims];
        for (int d = W.D - 1; d >= 0; --d) {
          coord[d] = r % W.L[d];
          r /= W.L[d];
        }
        for (int d = W.D - 1; d >= 0; --d) {
          s *= W.taper[d][coord[d]];
          fold *= W.taper[d][coord[d]];
        }
        sscale.push_back(s);
        sfold.push_back(fold);
        brec.push_back(W.blend[t].rec);
        bts.push_back(W.blend[t].trace_start);
        bn.push_back(W.blend[t].n);
        ws.push_back(W.wavelet_src.empty() ? -1 : W.wavelet_src[t]);
        wdst.push_back(toff + (long)t * W.C);
        wC.push_back(W.C);
      }
      ttaper_off[w] = (long)ttaper.size();
      ttaper.insert(ttaper.end(), W.taper[W.D].begin(), W.taper[W.D].end());
      toff += (long)W.n_traces * W.C;
      Pt_max = std::max(Pt_max, W.Pt);
      C_max = std::max(C_max, W.C);
      maxD = std::max(maxD, W.D);
      if (!W.wavelet_src.empty()) wavelets = true;
    }
    n_wtraces = (long)sscale.size();
    space_scale.upload(sscale, stream);
    space_fold.upload(sfold, stream);
    time_taper.upload(ttaper, stream);
    blend_rec.upload(brec, stream);
    blend_ts.upload(bts, stream);
    blend_n.upload(bn, stream);
    wsrc.upload(ws, stream);
    wt_dst.upload(wdst, stream);
    wt_C.upload(wC, stream);

    fast = pick_fast();
    X.alloc(M);
    S0.alloc(M);
    if (!fast) S1.alloc(M);
    Y.alloc(toff);
    rec_d.alloc(plan.record_size);
    rec_r.alloc(plan.record_size);
    scalar.alloc(1);
    dscalar.alloc(1);
    {
      std::vector<uint8_t> m(plan.record_size, 0);
      for (const auto &mu : plan.mute)
        for (int k = 0; k < mu.second; ++k) m[mu.first + k] = 1;
      mute.upload(m, stream);
    }
    C *Sb[2] = {S0.get(), S1.get()};

    // ---- time-axis jobs
    for (int w = 0; w < nw; ++w) {
      const WindowPlan &W = plan.windows[w];
      TimeJob<R> &j = tj[w];
      j.z = Sb[(W.D - 1) & 1] + W.model_off;
      j.y = Y.get() + trace_off[w];
      j.space_scale = space_scale.get() + wt_base[w];
      j.time_taper = time_taper.get() + ttaper_off[w];
      j.blend_rec = blend_rec.get() + wt_base[w];
      j.blend_ts = blend_ts.get() + wt_base[w];
      j.blend_n = blend_n.get() + wt_base[w];
      j.n_traces = W.n_traces;
      j.T = W.T;
      j.F = W.F;
      j.Lt = W.Lt;
      j.Pt = W.Pt;
      j.h = W.h;
      j.n_fk = W.n_fk;
      j.C = W.C;
      j.fft = fft.get(W.Pt);
      WaveletJob<R> &v = wj[w];
      v.y = Y.get() + trace_off[w];
      v.src = wsrc.get() + wt_base[w];
      v.n_traces = W.n_traces;
      v.C = W.C;
      v.fft = wavelets ? fft.get(W.C) : 0;
    }
    time_jobs.upload(tj, stream);
    if (fast) build_fast(tj);
    const size_t per_trace_time = 2 * (size_t)Pt_max * sizeof(C) + (size_t)C_max * sizeof(R);
    make_time_launch(time_fwd, per_trace_time, 16);
    make_time_launch(time_adj, per_trace_time, 16);
    if (wavelets) {
      wav_jobs.upload(wj, stream);
      make_time_launch(wav, 2 * (size_t)C_max * sizeof(C), 8);
      // spectra table
      std::vector<C> sp;
      std::vector<long> so;
      for (const auto &s : plan.spectra) {
        so.push_back((long)sp.size());
        for (const auto &v : s) {
          C c;
          c.x = (R)v.real();
          c.y = (R)v.imag();
          sp.push_back(c);
        }
      }
      spectra.upload(sp, stream);
      spec_off.upload(so, stream);
      build_wavelet_fast(wj, wt_base);
    }

    // ---- space-axis passes (generic path)
    if (fast) maxD = 0;
    fwd.resize(maxD);
    adj_update.resize(maxD);
    adj_plain.resize(maxD);
    for (int k = 0; k < maxD; ++k) {
      std::vector<AxisJob<R>> jf, ju, jp;
      for (int w = 0; w < nw; ++w) {
        const WindowPlan &W = plan.windows[w];
        if (W.D <= k) continue;
        const long TF = (long)W.T * W.F;
        {  // forward: axis D-1-k, inverse FFT, crop P -> L
          const int a = W.D - 1 - k;
          AxisJob<R> j{};
          long outer = TF;
          for (int d = 0; d < a; ++d) outer *= W.P[d];
          int inner = 1;
          for (int d = a + 1; d < W.D; ++d) inner *= W.L[d];
          j.src = (k == 0 ? X.get() : Sb[(k - 1) & 1]) + W.model_off;
          j.dst = Sb[k & 1] + W.model_off;
          j.outer = outer;
          j.inner = inner;
          j.n_in = W.P[a];
          j.n_out = W.L[a];
          j.fft = fft.get(W.P[a]);
          jf.push_back(j);
        }
        {  // adjoint: axis k, zero-pad L -> P, forward FFT
          const int a = k;
          AxisJob<R> j{};
          long outer = TF;
          for (int d = 0; d < a; ++d) outer *= W.P[d];
          int inner = 1;
          for (int d = a + 1; d < W.D; ++d) inner *= W.L[d];
          j.src = Sb[(W.D - 1 + k) & 1] + W.model_off;
          j.outer = outer;
          j.inner = inner;
          j.n_in = W.L[a];
          j.n_out = W.P[a];
          j.fft = fft.get(W.P[a]);
          const bool last = (k == W.D - 1);
          j.last = last ? 1 : 0;
          j.dst = last ? X.get() + W.model_off : Sb[(W.D + k) & 1] + W.model_off;
          ju.push_back(j);
          j.dst = last ? nullptr : Sb[(W.D + k) & 1] + W.model_off;  // G set lazily
          jp.push_back(j);
        }
      }
      make_axis_launch(fwd[k], jf);
      make_axis_launch(adj_update[k], ju);
      pending_plain.push_back(jp);
    }

    // ---- forward blend: window traces into the record, window then trace
    {
      std::vector<Contrib> list;
      for (int w = 0; w < nw; ++w) {
        const WindowPlan &W = plan.windows[w];
        for (int t = 0; t < W.n_traces; ++t) {
          const BlendCoord &b = W.blend[t];
          if (b.rec < 0) continue;
          Contrib c{b.rec, trace_off[w] + (long)t * W.C + b.trace_start, b.n, 0};
          list.push_back(c);
        }
      }
      make_gather(g_fwd, list, plan.record_size);
    }

    // ---- input blend and output gather tables (patch traces)
    patch_off.assign(plan.n_patches, 0);
    long poff = 0;
    for (int p = 0; p < plan.n_patches; ++p) {
      patch_off[p] = poff;
      poff += (long)plan.n_traces[p] * plan.n_times[p];
    }
    data_size = poff;
    data_dev.alloc(data_size);
    {
      std::vector<std::vector<long>> cover;  // per global patch trace
      std::vector<long> tr_base(plan.n_patches);
      long ntr = 0;
      for (int p = 0; p < plan.n_patches; ++p) {
        tr_base[p] = ntr;
        ntr += plan.n_traces[p];
      }
      cover.resize(ntr);
      for (int w = 0; w < nw; ++w) {
        const WindowPlan &W = plan.windows[w];
        for (int t = 0; t < W.n_traces; ++t)
          cover[tr_base[W.patch] + W.trace_index[t]].push_back(trace_off[w] + (long)t * W.C +
                                                              W.h);
      }
      std::vector<long> ptr(ntr + 1, 0), src, dst(ntr);
      std::vector<int> nt(ntr);
      for (int p = 0; p < plan.n_patches; ++p) {
        for (int t = 0; t < plan.n_traces[p]; ++t) {
          const long g = tr_base[p] + t;
          dst[g] = patch_off[p] + (long)t * plan.n_times[p];
          nt[g] = plan.n_times[p];
        }
      }
      for (long g = 0; g < ntr; ++g) {
        ptr[g + 1] = ptr[g] + (long)cover[g].size();
        src.insert(src.end(), cover[g].begin(), cover[g].end());
      }
      out_ptr.upload(ptr, stream);
      out_src.upload(src, stream);
      out_dst.upload(dst, stream);
      out_nt.upload(nt, stream);
      out_traces = ntr;
    }
    d_descs.upload(fft.descs, stream);
    d_tw.upload(fft.tw, stream);
    CK(cudaStreamSynchronize(stream));
  }

  std::vector<std::vector<AxisJob<R>>> pending_plain;

  void ensure_plain_adjoint() {
    if (G.get() != nullptr || plan.model_size == 0) return;
    G.alloc(plan.model_size);
    if (fast) {
      std::vector<PlaneJob<R>> jobs = pending_plane_plain;
      for (size_t w = 0; w < jobs.size(); ++w) jobs[w].dst = G.get() + plan.windows[w].model_off;
      make_plane_launch(pl_adj_plain, jobs, pending_planes, nt_adj, np_adj, smem_adj, sp_adj);
      CK(cudaStreamSynchronize(stream));
      return;
    }
    for (size_t k = 0; k < pending_plain.size(); ++k) {
      auto jobs = pending_plain[k];
      size_t i = 0;
      for (int w = 0; w < (int)plan.windows.size(); ++w) {
        const WindowPlan &W = plan.windows[w];
        if (W.D <= (int)k) continue;
        if ((int)k == W.D - 1) jobs[i].dst = G.get() + W.model_off;
        ++i;
      }
      make_axis_launch(adj_plain[k], jobs);
    }
    CK(cudaStreamSynchronize(stream));
  }

  void set_input_gather(const std::vector<Contrib> &list) {
    make_gather(g_input, list, plan.record_size);
  }

  // ---------------------------------------------------------------- launches

  void launch_axis(const AxisLaunch &L, int inverse, int epilogue, R step, R lamb,
                   const R *lamb_dev = nullptr) {
    if (L.n_cta == 0) return;
    axis_pass<R><<<L.n_cta, kThreads, L.smem, stream>>>(
        L.jobs.get(), L.cta_job.get(), L.cta_line0.get(), L.lpc, d_descs.get(), d_tw.get(),
        inverse, epilogue, step, lamb, lamb_dev, scalar.get());
    CK(cudaGetLastError());
  }

  void launch_gather(const GatherLaunch &Gl, const R *src, R *out, int mode, bool use_mute,
                     const R *d, const R *taper, int taper_len, double *sumsq) {
    if (Gl.n_chunk == 0) return;
    blend_gather<R><<<Gl.n_chunk, kThreads, 0, stream>>>(
        Gl.contrib.get(), Gl.chunk_ptr.get(), Gl.chunk, plan.record_size, src, out, mode,
        use_mute ? mute.get() : nullptr, d, taper, taper_len, sumsq);
    CK(cudaGetLastError());
  }

  void launch_space_fwd() {
    if (pl_fwd.n_batch == 0) return;
    sp_fwd<<<pl_fwd.grid, pl_fwd.nt, pl_fwd.smem, stream>>>(pl_fwd.batches());
    CK(cudaGetLastError());
  }

  void launch_space_adj(const PlaneLaunch &L, int epilogue, R step, R lamb,
                        const R *lamb_dev = nullptr) {
    if (L.n_batch == 0) return;
    sp_adj<<<L.grid, L.nt, L.smem, stream>>>(L.batches(), epilogue, step, lamb, lamb_dev,
                                             scalar.get());
    CK(cudaGetLastError());
  }

  void launch_time_fwd() {
    if (fast) {
      if (tf_fast.n_cta)
        tm_fwd<<<tf_fast.n_cta, kThreads, tf_fast.smem, stream>>>(
            time_jobs_fast.get(), tf_fast.cta_job.get(), tf_fast.cta_trace0.get());
    } else if (time_fwd.n_cta) {
      time_c2r_ola<R><<<time_fwd.n_cta, kThreads, time_fwd.smem, stream>>>(
          time_jobs.get(), time_fwd.cta_job.get(), time_fwd.cta_trace0.get(), time_fwd.nb,
          d_descs.get(), d_tw.get());
    }
    CK(cudaGetLastError());
  }

  // Y = W F X  (window traces of the current model)
  void forward_traces() {
    if (fast) {
      launch_space_fwd();
      launch_time_fwd();
      if (wavelets) launch_wavelet(+1);
      return;
    }
    for (size_t k = 0; k < fwd.size(); ++k) launch_axis(fwd[k], 1, kStore, 0, 0);
    if (time_fwd.n_cta) {
      time_c2r_ola<R><<<time_fwd.n_cta, kThreads, time_fwd.smem, stream>>>(
          time_jobs.get(), time_fwd.cta_job.get(), time_fwd.cta_trace0.get(), time_fwd.nb,
          d_descs.get(), d_tw.get());
      CK(cudaGetLastError());
    }
    if (wavelets) launch_wavelet(+1);
  }

  // in place on the window traces (direction +1), or from the record into
  // the window traces (direction -1, prime-factor kernel only)
  void launch_wavelet_fast(int direction, const R *record) {
    if (!wavf.n_cta) return;
    wavelet_fast<R><<<wavf.n_cta, kWavThreads, wavf.smem, stream>>>(
        wavf_jobs.get(), wavf.cta_job.get(), wavf.cta_trace0.get(), wavf.nb, spectra.get(),
        spec_off.get(), direction, record);
    CK(cudaGetLastError());
  }

  void launch_wavelet(int direction) {
    if (wav_fast) {
      launch_wavelet_fast(direction, nullptr);
      return;
    }
    if (!wav.n_cta) return;
    wavelet_apply<R><<<wav.n_cta, kThreads, wav.smem, stream>>>(
        wav_jobs.get(), wav.cta_job.get(), wav.cta_trace0.get(), wav.nb, d_descs.get(),
        d_tw.get(), spectra.get(), spec_off.get(), direction);
    CK(cudaGetLastError());
  }

  // Z = F_t^H B^H W^H record, per window (before the space passes)
  void adjoint_time(const R *record) {
    if (wavelets && wav_fast) {
      launch_wavelet_fast(-1, record);
    } else if (wavelets) {
      if (n_wtraces)
        extract_traces<R><<<(unsigned)n_wtraces, kThreads, 0, stream>>>(
            blend_rec.get(), blend_ts.get(), blend_n.get(), wt_dst.get(), wt_C.get(), record,
            Y.get());
      CK(cudaGetLastError());
      launch_wavelet(-1);
    }
    if (fast) {
      if (ta_fast.n_cta)
        tm_adj<<<ta_fast.n_cta, kThreads, ta_fast.smem, stream>>>(
            time_jobs_fast.get(), ta_fast.cta_job.get(), ta_fast.cta_trace0.get(), record,
            wavelets ? 0 : 1);
      CK(cudaGetLastError());
    } else if (time_adj.n_cta) {
      time_r2c<R><<<time_adj.n_cta, kThreads, time_adj.smem, stream>>>(
          time_jobs.get(), time_adj.cta_job.get(), time_adj.cta_trace0.get(), time_adj.nb,
          d_descs.get(), d_tw.get(), record, wavelets ? 0 : 1);
      CK(cudaGetLastError());
    }
  }

  // X <- threshold(X - step * A^H record, lamb); lambda is read from
  // lamb_dev instead when given (graph replays)
  void adjoint_update(const R *record, R step, R lamb, bool track_max,
                      const R *lamb_dev = nullptr) {
    adjoint_time(record);
    if (fast) {
      launch_space_adj(pl_adj, track_max ? kUpdateMax : kUpdateThreshold, step, lamb, lamb_dev);
      return;
    }
    for (size_t k = 0; k < adj_update.size(); ++k)
      launch_axis(adj_update[k], 0, track_max ? kUpdateMax : kUpdateThreshold, step, lamb,
                  lamb_dev);
  }

  // ---------------------------------------------------------------- graphs

  // One ISTA iteration (forward, residual, next lambda, adjoint update)
  // captured once and replayed; lambda comes from a device table indexed by
  // a device counter the graph advances.
  DevArray<R> lamb_table, lamb_cur;
  DevArray<int> lamb_counter;
  cudaGraphExec_t iter_graph = nullptr;

  void release_graph() {
    if (iter_graph != nullptr) {
      cudaGraphExecDestroy(iter_graph);
      iter_graph = nullptr;
    }
  }

  // table[k] = lambda used after iteration k + 1.  The captured graph holds
  // the table's address, so the table keeps its allocation while it is
  // large enough; growing it drops the graph (re-captured on next use).
  void load_schedule(const std::vector<R> &table) {
    if (table.size() > lamb_table.size()) {
      release_graph();
      CK(cudaStreamSynchronize(stream));
      lamb_table.alloc(table.size());
    }
    CK(cudaMemcpyAsync(lamb_table.get(), table.data(), table.size() * sizeof(R),
                       cudaMemcpyHostToDevice, stream));
    if (lamb_cur.get() == nullptr) lamb_cur.alloc(1);
    if (lamb_counter.get() == nullptr) lamb_counter.alloc(1);
    CK(cudaMemsetAsync(lamb_counter.get(), 0, sizeof(int), stream));
  }

  void iteration_body(bool want_norm) {
    forward_traces();
    residual(want_norm);
    next_lambda<R><<<1, 32, 0, stream>>>(lamb_table.get(), lamb_counter.get(), lamb_cur.get());
    CK(cudaGetLastError());
    adjoint_update(rec_r.get(), stepsize, (R)0, false, lamb_cur.get());
  }

  void capture_iteration() {
    if (iter_graph != nullptr) return;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    try {
      iteration_body(false);
    } catch (...) {
      cudaStreamEndCapture(stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    CK(cudaStreamEndCapture(stream, &g));
    const cudaError_t e = cudaGraphInstantiate(&iter_graph, g, 0);
    cudaGraphDestroy(g);
    CK(e);
  }

  void replay_iteration() { CK(cudaGraphLaunch(iter_graph, stream)); }

  void residual(bool want_norm) {
    double *ss = nullptr;
    if (want_norm) {
      CK(cudaMemsetAsync(dscalar.get(), 0, sizeof(double), stream));
      ss = dscalar.get();
    }
    launch_gather(g_fwd, Y.get(), rec_r.get(), kGatherResidual, true, rec_d.get(), nullptr, 0,
                  ss);
  }

  double read_dscalar() {
    double v = 0;
    CK(cudaMemcpyAsync(&v, dscalar.get(), sizeof(double), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    return v;
  }

  R read_scalar() {
    R v = 0;
    CK(cudaMemcpyAsync(&v, scalar.get(), sizeof(R), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    return v;
  }

  double record_norm(const R *rec) {
    CK(cudaMemsetAsync(dscalar.get(), 0, sizeof(double), stream));
    if (plan.record_size)
      record_sumsq<R><<<grid_for(plan.record_size), kThreads, 0, stream>>>(
          rec, plan.record_size, dscalar.get());
    CK(cudaGetLastError());
    return std::sqrt(read_dscalar());
  }

  static unsigned grid_for(long n) {
    long g = (n + kThreads - 1) / kThreads;
    return (unsigned)std::max<long>(1, std::min<long>(g, 148L * 16));
  }

  // 0.5 / max(1, max blended sum of the space tapers)   (src/model.c:1230-1312)
  R compute_stepsize() {
    if (n_wtraces) {
      fill_traces<R><<<(unsigned)std::min<long>(n_wtraces, 148L * 64), kThreads, 0, stream>>>(
          Y.get(), space_fold.get(), wt_dst.get(), wt_C.get(), n_wtraces);
      CK(cudaGetLastError());
    }
    launch_gather(g_fwd, Y.get(), rec_r.get(), kGatherSum, false, nullptr, nullptr, 0, nullptr);
    R one = (R)1;
    CK(cudaMemcpyAsync(scalar.get(), &one, sizeof(R), cudaMemcpyHostToDevice, stream));
    if (plan.record_size)
      record_max<R><<<grid_for(plan.record_size), kThreads, 0, stream>>>(
          rec_r.get(), plan.record_size, scalar.get());
    CK(cudaGetLastError());
    const R factor = read_scalar();
    stepsize = (R)0.5 / factor;
    return stepsize;
  }

  void upload_data(R const *const *data) {
    for (int p = 0; p < plan.n_patches; ++p) {
      const long n = (long)plan.n_traces[p] * plan.n_times[p];
      if (n)
        CK(cudaMemcpyAsync(data_dev.get() + patch_off[p], data[p], n * sizeof(R),
                           cudaMemcpyHostToDevice, stream));
    }
  }

  void download_data(R *const *data) {
    for (int p = 0; p < plan.n_patches; ++p) {
      const long n = (long)plan.n_traces[p] * plan.n_times[p];
      if (n)
        CK(cudaMemcpyAsync(data[p], data_dev.get() + patch_off[p], n * sizeof(R),
                           cudaMemcpyDeviceToHost, stream));
    }
    CK(cudaStreamSynchronize(stream));
  }

  // d = mute(mean blend of the patch data at the raw shot times)
  void blend_input(const long *const *shottimes, const int *const *channels,
                   const enum AGDTraceType *const *trace_types) {
    if (g_input.n_chunk == 0 && plan.record_size) {
      std::vector<Contrib> list;
      for (int p = 0; p < plan.n_patches; ++p) {
        const int nt = plan.n_times[p];
        for (int t = 0; t < plan.n_traces[p]; ++t) {
          const BlendCoord b = plan.coord_of(shottimes[p][t], nt, channels[p][t],
                                             (int)trace_types[p][t]);
          if (b.rec < 0) continue;
          list.push_back(Contrib{b.rec, patch_off[p] + (long)t * nt + b.trace_start, b.n, 0});
        }
      }
      set_input_gather(list);
    }
    launch_gather(g_input, data_dev.get(), rec_d.get(), kGatherMean, true, nullptr, nullptr, 0,
                  nullptr);
  }

  void output() {
    forward_traces();
    if (out_traces)
      output_gather<R><<<(unsigned)out_traces, kThreads, 0, stream>>>(
          out_ptr.get(), out_src.get(), out_dst.get(), out_nt.get(), Y.get(), data_dev.get());
    CK(cudaGetLastError());
  }

  // Initial step: x = -step * A^H d, lambda_0 = sqrt(max |x|^2)
  R initial_step() {
    if (plan.model_size) CK(cudaMemsetAsync(X.get(), 0, X.bytes(), stream));
    CK(cudaMemsetAsync(scalar.get(), 0, sizeof(R), stream));
    adjoint_update(rec_d.get(), stepsize, (R)0, true);
    const R m = read_scalar();
    return (R)std::sqrt(m);
  }

  void threshold_model(R lamb) {
    if (plan.model_size)
      model_threshold<R><<<grid_for(plan.model_size), kThreads, 0, stream>>>(
          X.get(), plan.model_size, lamb);
    CK(cudaGetLastError());
  }

  // Thresholds after the initial step: the schedule of src/agdeblend.c:
  // 526-533,588-589,623-627 evaluated in AGD_TYPE on the host.
  static std::vector<R> schedule_table(R lamb0, R initial_factor, int n_its, R *first) {
    const Schedule sc = lambda_schedule(initial_factor, n_its);
    const R linear_slope = sc.linear_slope * lamb0;
    R lamb = lamb0 * initial_factor;
    *first = lamb;
    std::vector<R> t(n_its > 1 ? n_its - 1 : 1, (R)0);
    for (int it = 1; it < n_its; ++it) {
      if (it < sc.first_linear_it)
        lamb *= sc.decay;
      else
        lamb = (R)(n_its - 1 - it) * linear_slope;
      t[it - 1] = lamb;
    }
    return t;
  }

  // the solver of agd_deblend (src/agdeblend.c:584-633); iterations replay a
  // captured CUDA graph unless residuals are printed
  void solve(R initial_factor, int n_its, int print_freq) {
    R lamb0 = initial_step();
    R first = 0;
    const std::vector<R> table = schedule_table(lamb0, initial_factor, n_its, &first);
    threshold_model(first);
    load_schedule(table);
    if (print_freq > 0) {
      const double r = record_norm(rec_d.get());
      std::printf("Iteration 0 Residual %f\n", r);
      for (int it = 1; it < n_its; ++it) {
        const bool print_residual = it % print_freq == 0;
        iteration_body(print_residual);
        if (print_residual)
          std::printf("Iteration %d Residual %f\n", it, std::sqrt(read_dscalar()));
      }
    } else if (n_its > 1) {
      capture_iteration();
      for (int it = 1; it < n_its; ++it) replay_iteration();
    }
    output();
  }

  // host <-> device model in the reference layout
  void model_from_ref(const R *host) {
    DevArray<C> tmp;
    tmp.alloc(plan.model_size);
    if (!plan.model_size) return;
    CK(cudaMemcpyAsync(tmp.get(), host, tmp.bytes(), cudaMemcpyHostToDevice, stream));
    for (const WindowPlan &W : plan.windows)
      model_layout<R><<<grid_for(W.model_size), kThreads, 0, stream>>>(
          tmp.get() + W.model_off, X.get() + W.model_off, W.T, W.F, W.plane(), 1);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream));
  }

  void model_to_ref(const C *dev, R *host) {
    DevArray<C> tmp;
    tmp.alloc(plan.model_size);
    if (!plan.model_size) return;
    for (const WindowPlan &W : plan.windows)
      model_layout<R><<<grid_for(W.model_size), kThreads, 0, stream>>>(
          dev + W.model_off, tmp.get() + W.model_off, W.T, W.F, W.plane(), 0);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(host, tmp.get(), tmp.bytes(), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
  }
};

using EngineR = Engine<real>;

}  // namespace agd

// ==================================================================== C API

struct agd_gpu_problem {
  std::unique_ptr<agd::EngineR> eng;
  // kept for blend_input (raw shot times, channels, trace types)
  std::vector<std::vector<long>> shottimes;
  std::vector<std::vector<int>> channels;
  std::vector<std::vector<AGDTraceType>> trace_types;
  std::vector<const long *> st_p;
  std::vector<const int *> ch_p;
  std::vector<const AGDTraceType *> tt_p;

  void input_blend() {
    eng->blend_input(st_p.data(), ch_p.data(), tt_p.data());
  }
};

namespace {

agd::ProblemArgs make_args(int n_patches, int const *volumes, int const *n_dims,
                           int const *const *window_shapes, int const *const *coords,
                           int const *const *shapes, long int const *const *shottimes,
                           int const *const *channels,
                           enum AGDTraceType const *const *trace_types,
                           int const *wavelet_lengths, int const *const *wavelet_idxs,
                           AGD_TYPE const *const *wavelets) {
  return agd::ProblemArgs{n_patches,  volumes,     n_dims,   window_shapes,
                          coords,     shapes,      shottimes, channels,
                          trace_types, wavelet_lengths, wavelet_idxs, wavelets};
}

int create_problem(const agd::ProblemArgs &a, agd_gpu_problem **out) {
  *out = nullptr;
  agd::Plan plan;
  if (agd::build_plan(a, plan)) return 1;
  auto *pb = new agd_gpu_problem();
  try {
    pb->shottimes.resize(a.n_patches);
    pb->channels.resize(a.n_patches);
    pb->trace_types.resize(a.n_patches);
    for (int p = 0; p < a.n_patches; ++p) {
      const int n = plan.n_traces[p];
      pb->shottimes[p].assign(a.shottimes[p], a.shottimes[p] + n);
      pb->channels[p].assign(a.channels[p], a.channels[p] + n);
      pb->trace_types[p].assign(a.trace_types[p], a.trace_types[p] + n);
      pb->st_p.push_back(pb->shottimes[p].data());
      pb->ch_p.push_back(pb->channels[p].data());
      pb->tt_p.push_back(pb->trace_types[p].data());
    }
    pb->eng.reset(new agd::EngineR(std::move(plan)));
    pb->eng->compute_stepsize();
  } catch (const std::exception &e) {
    std::fprintf(stderr, "ERROR: %s\n", e.what());
    delete pb;
    return 1;
  }
  *out = pb;
  return 0;
}

template <typename F>
int guarded(const char *name, F &&f) {
  try {
    return f();
  } catch (const std::exception &e) {
    std::fprintf(stderr, "ERROR: %s\nERROR in %s\n", e.what(), name);
    return 1;
  }
}

}  // namespace

extern "C" {

int agd_gpu_problem_create(int n_patches, int const *volumes, int const *n_dims,
                           int const *const *window_shapes, int const *const *coords,
                           int const *const *shapes, long int const *const *shottimes,
                           int const *const *channels,
                           enum AGDTraceType const *const *trace_types,
                           int const *wavelet_lengths, int const *const *wavelet_idxs,
                           AGD_TYPE const *const *wavelets, agd_gpu_problem **problem) {
  if (problem == nullptr) return 1;
  const agd::ProblemArgs a =
      make_args(n_patches, volumes, n_dims, window_shapes, coords, shapes, shottimes,
                channels, trace_types, wavelet_lengths, wavelet_idxs, wavelets);
  // Validation with a dummy non-null data array (data is checked per call).
  std::vector<AGD_TYPE *> dummy(n_patches > 0 ? n_patches : 1, (AGD_TYPE *)1);
  if (agd::check_deblend_inputs(a, (AGD_TYPE)1, 1, dummy.data())) return 1;
  return create_problem(a, problem);
}

void agd_gpu_problem_destroy(agd_gpu_problem *problem) { delete problem; }

int agd_gpu_problem_info(agd_gpu_problem const *pb, long int *info) {
  if (pb == nullptr || info == nullptr) return 1;
  const agd::EngineR &e = *pb->eng;
  info[0] = (long)e.plan.windows.size();
  info[1] = e.plan.model_size;
  info[2] = e.plan.record_size;
  info[3] = e.n_wtraces;
  long segs = 0;
  for (const auto &c : e.plan.intervals) segs += (long)c.size();
  info[4] = segs;
  info[5] = (long)e.plan.mute.size();
  info[6] = (long)e.device_bytes();
  info[7] = e.g_fwd.n_contrib;
  info[8] = e.fast ? 1 : 0;
  info[9] = e.wav_fast ? 1 : 0;
  info[10] = e.fast ? e.fwd_pick : -1;
  info[11] = e.fast ? e.adj_pick : -1;
  info[12] = (long)e.fwd_vars.size();
  info[13] = (long)e.adj_vars.size();
  return 0;
}

int agd_gpu_stepsize(agd_gpu_problem *pb, AGD_TYPE *stepsize) {
  if (pb == nullptr || stepsize == nullptr) return 1;
  *stepsize = pb->eng->stepsize;
  return 0;
}

int agd_gpu_forward(agd_gpu_problem *pb, AGD_TYPE const *model, AGD_TYPE *record) {
  if (pb == nullptr || model == nullptr || record == nullptr) return 1;
  return guarded("agd_gpu_forward", [&] {
    agd::EngineR &e = *pb->eng;
    e.model_from_ref(model);
    e.forward_traces();
    e.launch_gather(e.g_fwd, e.Y.get(), e.rec_r.get(), agd::kGatherSum, true, nullptr, nullptr,
                    0, nullptr);
    if (e.plan.record_size)
      agd::CK(cudaMemcpyAsync(record, e.rec_r.get(), e.rec_r.bytes(), cudaMemcpyDeviceToHost,
                              e.stream));
    agd::CK(cudaStreamSynchronize(e.stream));
    return 0;
  });
}

int agd_gpu_adjoint(agd_gpu_problem *pb, AGD_TYPE const *record, AGD_TYPE *model) {
  if (pb == nullptr || model == nullptr || record == nullptr) return 1;
  return guarded("agd_gpu_adjoint", [&] {
    agd::EngineR &e = *pb->eng;
    e.ensure_plain_adjoint();
    if (e.plan.record_size)
      agd::CK(cudaMemcpyAsync(e.rec_r.get(), record, e.rec_r.bytes(), cudaMemcpyHostToDevice,
                              e.stream));
    e.adjoint_time(e.rec_r.get());
    if (e.fast) e.launch_space_adj(e.pl_adj_plain, agd::kStore, 0, 0);
    for (size_t k = 0; k < e.adj_plain.size(); ++k)
      e.launch_axis(e.adj_plain[k], 0, agd::kStore, 0, 0);
    e.model_to_ref(e.G.get(), model);
    return 0;
  });
}

int agd_gpu_blend_input(agd_gpu_problem *pb, AGD_TYPE const *const *data, AGD_TYPE *record) {
  if (pb == nullptr || data == nullptr || record == nullptr) return 1;
  return guarded("agd_gpu_blend_input", [&] {
    agd::EngineR &e = *pb->eng;
    e.upload_data(data);
    pb->input_blend();
    if (e.plan.record_size)
      agd::CK(cudaMemcpyAsync(record, e.rec_d.get(), e.rec_d.bytes(), cudaMemcpyDeviceToHost,
                              e.stream));
    agd::CK(cudaStreamSynchronize(e.stream));
    return 0;
  });
}

int agd_gpu_set_output(agd_gpu_problem *pb, AGD_TYPE const *model, AGD_TYPE *const *data) {
  if (pb == nullptr || model == nullptr || data == nullptr) return 1;
  return guarded("agd_gpu_set_output", [&] {
    agd::EngineR &e = *pb->eng;
    e.model_from_ref(model);
    e.output();
    e.download_data(data);
    return 0;
  });
}

int agd_gpu_solve(agd_gpu_problem *pb, AGD_TYPE initial_factor, int n_its, int print_freq,
                  AGD_TYPE *const *data) {
  if (pb == nullptr || data == nullptr) return 1;
  if (n_its <= 0) {
    std::fprintf(stderr, "ERROR: n_its must be > 0\n");
    return 1;
  }
  return guarded("agd_deblend", [&] {
    agd::EngineR &e = *pb->eng;
    e.upload_data(data);
    pb->input_blend();
    e.solve(initial_factor, n_its, print_freq);
    e.download_data(data);
    return 0;
  });
}

int agd_gpu_time_iterations(agd_gpu_problem *pb, AGD_TYPE const *const *data,
                            AGD_TYPE initial_factor, int n_its, int warmup, int steps,
                            double *timing) {
  if (pb == nullptr || data == nullptr || timing == nullptr || steps <= 0 || n_its < 2 ||
      warmup < 0)
    return 1;
  return guarded("agd_gpu_time_iterations", [&] {
    agd::EngineR &e = *pb->eng;
    e.upload_data(data);
    pb->input_blend();
    const AGD_TYPE lamb0 = e.initial_step();
    AGD_TYPE first = 0;
    const std::vector<AGD_TYPE> sched =
        agd::EngineR::schedule_table(lamb0, initial_factor, n_its, &first);
    e.threshold_model(first);
    // thresholds for every replay: the schedule, repeated if the run is
    // longer than n_its - 1 iterations
    const int total = warmup + steps + 2;
    std::vector<AGD_TYPE> table(total);
    for (int k = 0; k < total; ++k) table[k] = sched[k % sched.size()];
    e.load_schedule(table);
    e.capture_iteration();
    for (int i = 0; i < warmup; ++i) e.replay_iteration();
    cudaEvent_t ev[4];
    for (auto &v : ev) agd::CK(cudaEventCreate(&v));
    agd::CK(cudaEventRecord(ev[0], e.stream));
    for (int i = 0; i < steps; ++i) e.replay_iteration();
    agd::CK(cudaEventRecord(ev[1], e.stream));
    // one more iteration split into its forward and adjoint halves
    agd::CK(cudaEventRecord(ev[2], e.stream));
    e.forward_traces();
    e.residual(false);
    agd::CK(cudaEventRecord(ev[3], e.stream));
    agd::CK(cudaEventSynchronize(ev[3]));
    float ms_total = 0, ms_fwd = 0;
    agd::CK(cudaEventElapsedTime(&ms_total, ev[0], ev[1]));
    agd::CK(cudaEventElapsedTime(&ms_fwd, ev[2], ev[3]));
    agd::CK(cudaEventRecord(ev[2], e.stream));
    e.adjoint_update(e.rec_r.get(), e.stepsize, table[warmup + steps], false);
    agd::CK(cudaEventRecord(ev[3], e.stream));
    agd::CK(cudaEventSynchronize(ev[3]));
    float ms_adj = 0;
    agd::CK(cudaEventElapsedTime(&ms_adj, ev[2], ev[3]));
    for (auto &v : ev) cudaEventDestroy(v);
    timing[0] = ms_total;
    timing[1] = ms_fwd;
    timing[2] = ms_adj;
    timing[3] = steps;
    return 0;
  });
}

int agd_gpu_profile_iteration(agd_gpu_problem *pb, AGD_TYPE lamb, double *ms) {
  if (pb == nullptr || ms == nullptr) return 1;
  return guarded("agd_gpu_profile_iteration", [&] {
    agd::EngineR &e = *pb->eng;
    for (int i = 0; i < 16; ++i) ms[i] = 0.0;
    std::vector<cudaEvent_t> ev;
    auto mark = [&] {
      cudaEvent_t v;
      agd::CK(cudaEventCreate(&v));
      agd::CK(cudaEventRecord(v, e.stream));
      ev.push_back(v);
    };
    const int nf = e.fast ? 1 : (int)e.fwd.size();
    mark();
    for (int k = 0; k < nf; ++k) {
      if (e.fast)
        e.launch_space_fwd();
      else
        e.launch_axis(e.fwd[k], 1, agd::kStore, 0, 0);
      mark();
    }
    e.launch_time_fwd();
    mark();
    if (e.wavelets) e.launch_wavelet(+1);
    mark();
    e.residual(false);
    mark();
    e.adjoint_time(e.rec_r.get());
    mark();
    for (int k = 0; k < nf; ++k) {
      if (e.fast)
        e.launch_space_adj(e.pl_adj, agd::kUpdateThreshold, e.stepsize, lamb);
      else
        e.launch_axis(e.adj_update[k], 0, agd::kUpdateThreshold, e.stepsize, lamb);
      mark();
    }
    agd::CK(cudaEventSynchronize(ev.back()));
    auto dt = [&](int a, int b) {
      float v = 0;
      agd::CK(cudaEventElapsedTime(&v, ev[a], ev[b]));
      return (double)v;
    };
    // [0] forward space passes, [1] time c2r + overlap-add, [2] wavelet
    // forward, [3] blend gather + residual, [4] adjoint time (incl. gather
    // and wavelet), [5] adjoint space passes incl. update, [6..9] forward
    // passes by index, [10..13] adjoint passes by index, [14] passes count
    for (int k = 0; k < nf && k < 4; ++k) ms[6 + k] = dt(k, k + 1);
    ms[0] = dt(0, nf);
    ms[1] = dt(nf, nf + 1);
    ms[2] = dt(nf + 1, nf + 2);
    ms[3] = dt(nf + 2, nf + 3);
    ms[4] = dt(nf + 3, nf + 4);
    for (int k = 0; k < nf && k < 4; ++k) ms[10 + k] = dt(nf + 4 + k, nf + 5 + k);
    ms[5] = dt(nf + 4, nf + 4 + nf);
    ms[14] = nf;
    for (auto v : ev) cudaEventDestroy(v);
    return 0;
  });
}

int agd_plan_export(int n_patches, int const *volumes, int const *n_dims,
                    int const *const *window_shapes, int const *const *coords,
                    int const *const *shapes, long int const *const *shottimes,
                    int const *const *channels, enum AGDTraceType const *const *trace_types,
                    int const *wavelet_lengths, int const *const *wavelet_idxs,
                    AGD_TYPE const *const *wavelets, long int *info, int *win,
                    long int *blend) {
  if (info == nullptr) return 1;
  const agd::ProblemArgs a =
      make_args(n_patches, volumes, n_dims, window_shapes, coords, shapes, shottimes,
                channels, trace_types, wavelet_lengths, wavelet_idxs, wavelets);
  std::vector<AGD_TYPE *> dummy(n_patches > 0 ? n_patches : 1, (AGD_TYPE *)1);
  if (agd::check_deblend_inputs(a, (AGD_TYPE)1, 1, dummy.data())) return 1;
  agd::Plan plan;
  if (agd::build_plan(a, plan)) return 1;
  long ntr = 0;
  for (const auto &w : plan.windows) ntr += w.n_traces;
  long segs = 0;
  for (const auto &c : plan.intervals) segs += (long)c.size();
  info[0] = (long)plan.windows.size();
  info[1] = plan.model_size;
  info[2] = plan.record_size;
  info[3] = ntr;
  info[4] = segs;
  info[5] = (long)plan.mute.size();
  info[6] = 0;
  info[7] = 0;
  if (win != nullptr) {
    for (size_t i = 0; i < plan.windows.size(); ++i) {
      const agd::WindowPlan &w = plan.windows[i];
      int *o = win + 32 * i;
      std::memset(o, 0, 32 * sizeof(int));
      o[0] = w.patch;
      o[1] = w.D;
      o[2] = w.T;
      o[3] = w.F;
      o[4] = w.Lt;
      o[5] = w.Pt;
      o[6] = w.h;
      o[7] = w.n_fk;
      o[8] = w.C;
      o[9] = w.n_traces;
      for (int d = 0; d < w.D; ++d) {
        o[10 + d] = w.L[d];
        o[14 + d] = w.P[d];
      }
      for (int k = 0; k < 2 * w.D + 2; ++k) o[18 + k] = w.use_taper[k];
    }
  }
  if (blend != nullptr) {
    long k = 0;
    for (const auto &w : plan.windows)
      for (const auto &b : w.blend) {
        blend[3 * k] = b.rec;
        blend[3 * k + 1] = b.trace_start;
        blend[3 * k + 2] = b.n;
        ++k;
      }
  }
  return 0;
}

int agd_deblend(int n_patches, int const *volumes, int const *n_dims,
                int const *const *window_shapes, int const *const *coords,
                int const *const *shapes, long int const *const *shottimes,
                int const *const *channels, enum AGDTraceType const *const *trace_types,
                int const *wavelet_lengths, int const *const *wavelet_idxs,
                AGD_TYPE const *const *wavelets, AGD_TYPE const initial_factor, int n_its,
                int print_freq, AGD_TYPE *const *data) {
  const agd::ProblemArgs a =
      make_args(n_patches, volumes, n_dims, window_shapes, coords, shapes, shottimes,
                channels, trace_types, wavelet_lengths, wavelet_idxs, wavelets);
  if (agd::check_deblend_inputs(a, initial_factor, n_its, data)) {
    std::fprintf(stderr, "ERROR in agd_deblend\n");
    return 1;
  }
  agd_gpu_problem *pb = nullptr;
  if (create_problem(a, &pb)) {
    std::fprintf(stderr, "ERROR in agd_deblend\n");
    return 1;
  }
  if (pb->eng->stepsize > (AGD_TYPE)0.3)
    std::printf("WARNING: There does not appear to be any overlap between shots\n");
  const int rc = agd_gpu_solve(pb, initial_factor, n_its, print_freq, data);
  delete pb;
  return rc;
}

}  // extern "C"
