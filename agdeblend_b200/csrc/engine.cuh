// The device engine of the deblending path: turns a Plan into device tables
// and launch lists (window classes, autotuned kernel candidates), runs the
// operator, the ISTA solver as a captured CUDA graph, the precision modes and
// the warm start.  Templated on the real type (float / double).
#pragma once

#include "engine_memory.cuh"

namespace agd {

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
  // windows with one space axis of a length without a shape-specialised
  // kernel, on the line kernels (line_dft.cuh)
  struct LineLaunch {
    DevArray<LineJob<R>> jobs;
    DevArray<int> cta_job;
    DevArray<long> cta_line0;
    int n_cta = 0;
    size_t smem = 0;
  };
  LineLaunch line_fwd, line_adj, line_adj_plain;
  DevArray<R> line_tab;        // per (P, L): forward and adjoint cos / sin tables
  std::vector<char> win_line;  // 1: window on the line kernels
  std::vector<LineJob<R>> line_adj_host;  // adjoint jobs (the plain adjoint's, re-aimed)
  TimeLaunch time_fwd, time_adj, wav;

  // Shape-specialised kernels (fast.cuh).  Windows are grouped into classes
  // of equal padded space and time lengths; every class with an
  // instantiation runs the fast kernels, the remaining windows run the
  // generic ones (kernels.cuh).
  using SpaceFwdFn = void (*)(PlaneBatches<R>);
  using SpaceAdjFn = void (*)(PlaneBatches<R>, int, R, R, const R *, const R *, R *);
  using TimeFwdFn = void (*)(const TimeJob<R> *, const int *, const int *);
  using TimeAdjFn = void (*)(const TimeJob<R> *, const int *, const int *, const R *, int);
  struct PlaneLaunch {
    DevArray<PlaneBatch<R>> batch;
    int n_batch = 0;
    int grid = 0;
    int nt = 0;
    size_t smem = 0;
    PlaneBatches<R> batches() const { return PlaneBatches<R>{batch.get(), n_batch}; }
  };
  struct FwdVariant {
    SpaceFwdFn fn;
    int nt, np, stages;
    size_t smem;
    const char *name;  // kernel family (as profilers list it)
  };
  struct AdjVariant {
    SpaceAdjFn fn;
    int nt, np, stages;
    size_t smem;
    const char *name;  // kernel family (as profilers list it)
  };
  // windows of one padded space shape on the fast space kernels
  struct FastClass {
    std::vector<int> win;  // windows of the class
    std::vector<FwdVariant> fwd_vars;
    std::vector<AdjVariant> adj_vars;
    int fwd_pick = 0, adj_pick = 0;
    PlaneLaunch pl_fwd, pl_adj, pl_adj_plain;
    std::vector<PlaneJob<R>> fwd_jobs;    // forward jobs
    std::vector<PlaneJob<R>> plain_jobs;  // adjoint jobs without the update
    // split-BF16 tensor-core kernels (precision mode 1, space_tc.cuh)
    bool tc = false;
    PlaneLaunch tc_fwd, tc_adj, tc_adj_plain;
    std::vector<long> planes;             // (t, f) planes per window
    const FwdVariant &fv() const { return fwd_vars[fwd_pick]; }
    const AdjVariant &av() const { return adj_vars[adj_pick]; }
  };
  // windows of one padded time length on the fast time kernels (whatever
  // kernels serve their space axes), with candidate instantiations (traces
  // per block, padded line stride, blocks per SM) picked by timing
  struct TimeFwdVariant {
    TimeFwdFn fn;
    int nb;
    size_t smem;
    const char *name;  // kernel family (as profilers list it)
  };
  struct TimeAdjVariant {
    TimeAdjFn fn;
    int nb;
    size_t smem;
    const char *name;  // kernel family (as profilers list it)
  };
  struct TimeGroup {
    std::vector<int> win;
    std::vector<TimeFwdVariant> fwd_vars;
    std::vector<TimeAdjVariant> adj_vars;
    int fwd_pick = 0, adj_pick = 0;
    TimeLaunch tf, ta;
    const TimeFwdVariant &fv() const { return fwd_vars[fwd_pick]; }
    const TimeAdjVariant &av() const { return adj_vars[adj_pick]; }
  };
  std::vector<std::unique_ptr<FastClass>> classes;
  std::vector<std::unique_ptr<TimeGroup>> tgroups;
  std::vector<int> win_class;   // per window: its space class, or -1 (generic)
  std::vector<int> win_tgroup;  // per window: its time group, or -1 (generic)
  int n_generic = 0;            // windows on the generic space kernels
  int max_d_generic = 0;        // space dimensions of those windows
  int n_sm = 148;
  int sm_smem = 233472;      // shared memory per SM (bytes)
  int block_reserved = 1024;  // shared memory the system reserves per block
  GatherLaunch g_fwd, g_input;
  std::vector<long> trace_off;   // per window, in reals
  std::vector<long> patch_off;   // per patch, in reals
  long n_wtraces = 0;
  long data_size = 0;
  long out_traces = 0;
  bool wavelets = false;
  // independent problems solved together (plan.n_problems > 1): step sizes,
  // thresholds and maxima are per problem, read by the adjoint kernels
  bool multi = false;
  std::vector<R> steps;        // per problem
  DevArray<R> step_dev, pmax;  // per problem
  // prime-factor wavelet kernel (wavelet_fast.cuh), used when every window's
  // trace length factors into supported coprime prime powers
  bool wav_fast = false;
  DevArray<WaveletFastJob<R>> wavf_jobs;
  DevArray<unsigned short> pfa_map;  // per trace length: qmap [C], kpos [C]
  TimeLaunch wavf;
  using WaveletFn = void (*)(const WaveletFastJob<R> *, const int *, const int *, int,
                             const C *, const long *, int, const R *);
  WaveletFn wav_fn = nullptr;
  R stepsize = 0;

  explicit Engine(Plan &&p) : plan(std::move(p)) {
    CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    smem_max = optin_smem();
    {
      int dev = 0;
      CK(cudaGetDevice(&dev));
      CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
      CK(cudaDeviceGetAttribute(&sm_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
      CK(cudaDeviceGetAttribute(&block_reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev));
    }
    set_smem_limits();
    try {
      build();
    } catch (...) {
      // nothing of this engine may still run when its arrays are released
      cudaStreamSynchronize(stream);
      release_graph();
      cudaStreamDestroy(stream);
      stream = nullptr;
      throw;
    }
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
                         opt_in(line_dft_fwd<R>, limit), opt_in(line_dft_adj<R>, limit)});
    if constexpr (sizeof(R) == sizeof(float))
      smem_max = std::min({smem_max, opt_in(wavelet_fast<R, 2, 17>, limit),
                           opt_in(wavelet_fast<R, 3, 17>, limit),
                           opt_in(wavelet_fast<R, 4, 17>, limit),
                           opt_in(wavelet_fast<R, 2, 32>, limit),
                           opt_in(wavelet_fast<R, 3, 32>, limit)});
    else
      smem_max = std::min({smem_max, opt_in(wavelet_fast<R, 1, 17>, limit),
                           opt_in(wavelet_fast<R, 2, 17>, limit),
                           opt_in(wavelet_fast<R, 1, 32>, limit)});
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

  // C = product of pairwise coprime prime powers with a register DFT; the
  // even factor (if any) is the outermost axis, so the innermost axis, whose
  // lines start f apart, has an odd extent (no shared-memory bank conflicts)
  static bool pfa_shape(int N, PfaShape &sh) {
    static const int kOk[] = {2, 3, 4, 5, 7, 8, 9, 11, 13, 16, 17, 19, 23, 25, 27, 32};
    if (N < 2 || N > 65535) return false;
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
    int g = 1;
    for (int i = sh.nf - 1; i >= 0; --i) {
      sh.g[i] = g;
      sh.inv_g[i] = 1.0f / (float)g;
      sh.inv_lines[i] = (float)sh.f[i] / (float)N;
      g *= sh.f[i];
    }
    return true;
  }

  // qmap[t]: dense position of sample t (coordinates t mod f_i);
  // kpos[k]: dense position of frequency k after the forward passes
  // (coordinates k s_i^-1 mod f_i, s_i = C / f_i)
  static void pfa_tables(const PfaShape &sh, std::vector<unsigned short> &out) {
    const long N = sh.N;
    long inv[kPfaMaxFactors];
    for (int i = 0; i < sh.nf; ++i) {
      const long s = N / sh.f[i];
      inv[i] = 1;
      while (s * inv[i] % sh.f[i] != 1 % sh.f[i]) ++inv[i];
    }
    for (long t = 0; t < N; ++t) {
      long q = 0;
      for (int i = 0; i < sh.nf; ++i) q += t % sh.f[i] * sh.g[i];
      out.push_back((unsigned short)q);
    }
    for (long k = 0; k < N; ++k) {
      long q = 0;
      for (int i = 0; i < sh.nf; ++i) q += k * inv[i] % sh.f[i] * sh.g[i];
      out.push_back((unsigned short)q);
    }
  }

  void build_wavelet_fast(const std::vector<WaveletJob<R>> &wj,
                          const std::vector<long> &wt_base) {
    const char *env = std::getenv("AGD_GPU_GENERIC");
    if (env != nullptr && env[0] == '1') return;
    const int nw = (int)plan.windows.size();
    std::vector<WaveletFastJob<R>> jobs(nw);
    std::vector<unsigned short> perm;
    std::map<int, long> perm_off;
    int fmax = 1;  // largest factor of any trace length
    int n_max = 1;
    for (int w = 0; w < nw; ++w) {
      WaveletFastJob<R> &j = jobs[w];
      const int N = plan.windows[w].C;
      if (!pfa_shape(N, j.sh)) return;
      for (int i = 0; i < j.sh.nf; ++i) fmax = std::max(fmax, j.sh.f[i]);
      if (!perm_off.count(N)) {
        perm_off[N] = (long)perm.size();
        pfa_tables(j.sh, perm);
      }
      n_max = std::max(n_max, N);
    }
    const size_t per_pair = (size_t)n_max * sizeof(C);
    if (per_pair > (size_t)smem_max) return;
    pfa_map.upload(perm, stream);
    for (int w = 0; w < nw; ++w) {
      const WindowPlan &W = plan.windows[w];
      WaveletFastJob<R> &j = jobs[w];
      j.y = wj[w].y;
      j.src = wj[w].src;
      j.qmap = pfa_map.get() + perm_off[W.C];
      j.kpos = j.qmap + W.C;
      j.blend_rec = blend_rec.get() + wt_base[w];
      j.blend_ts = blend_ts.get() + wt_base[w];
      j.blend_n = blend_n.get() + wt_base[w];
      j.n_traces = W.n_traces;
    }
    wavf_jobs.upload(jobs, stream);
    upload_twiddles();
    // candidates: blocks per SM and pairs per block (about a third of the
    // SM's shared memory per block at three blocks)
    struct Cand {
      WaveletFn fn;
      int np;
    };
    std::vector<Cand> cands;
    auto pairs = [&](size_t budget) {
      return (int)std::max<size_t>(1, std::min<size_t>(4, budget / per_pair));
    };
    if (fmax <= 17) {
      if constexpr (sizeof(R) == sizeof(float)) {
        cands.push_back(Cand{wavelet_fast<R, 2, 17>, pairs(80000)});
        cands.push_back(Cand{wavelet_fast<R, 3, 17>, pairs(60000)});
        cands.push_back(Cand{wavelet_fast<R, 3, 17>, pairs(40000)});
        cands.push_back(Cand{wavelet_fast<R, 4, 17>, pairs(40000)});
      } else {
        cands.push_back(Cand{wavelet_fast<R, 1, 17>, pairs(80000)});
        cands.push_back(Cand{wavelet_fast<R, 2, 17>, pairs(80000)});
      }
    } else {
      if constexpr (sizeof(R) == sizeof(float)) {
        cands.push_back(Cand{wavelet_fast<R, 2, 32>, pairs(60000)});
        cands.push_back(Cand{wavelet_fast<R, 3, 32>, pairs(60000)});
        cands.push_back(Cand{wavelet_fast<R, 3, 32>, pairs(40000)});
      } else {
        cands.push_back(Cand{wavelet_fast<R, 1, 32>, pairs(60000)});
      }
    }
    auto launch_for = [&](TimeLaunch &L, int np) {
      std::vector<int> cj, cp;
      for (int w = 0; w < nw; ++w)
        for (int p = 0; p < (plan.windows[w].n_traces + 1) / 2; p += np) {
          cj.push_back(w);
          cp.push_back(p);
        }
      L.cta_job.upload(cj, stream);
      L.cta_trace0.upload(cp, stream);
      L.n_cta = (int)cj.size();
      L.nb = np;
      L.smem = per_pair * np;
    };
    int pick = 0;
    const char *force = std::getenv("AGD_GPU_WAVELET_VARIANT");
    if (force != nullptr && force[0] != '\0') {
      pick = std::max(0, std::min(std::atoi(force), (int)cands.size() - 1));
    } else if (cands.size() > 1) {
      pick = autotune_wavelet(cands.size(), [&](size_t v, TimeLaunch &L) {
        launch_for(L, cands[v].np);
        return cands[v].fn;
      });
    }
    wav_candidates = (int)cands.size();
    wav_pick = pick;
    wav_fn = cands[pick].fn;
    launch_for(wavf, cands[pick].np);
    wav_fast = true;
  }

  int wav_candidates = 0, wav_pick = -1;

  // Times the wavelet candidates (both directions, three rounds, CUDA
  // events), cached per device, precision, trace length and size class.
  template <typename Make>
  int autotune_wavelet(size_t n, Make make) {
    long traces = 0;
    int c_max = 0;
    for (const WindowPlan &W : plan.windows) {
      traces += W.n_traces;
      c_max = std::max(c_max, W.C);
    }
    int dev = 0;
    CK(cudaGetDevice(&dev));
    char key[96];
    std::snprintf(key, sizeof key, "wav:%d:%d:%d:%d", dev, (int)sizeof(R), c_max,
                  (int)std::log2((double)std::max(1L, traces)));
    static std::mutex mu;
    static std::map<std::string, int> cache;
    {
      std::lock_guard<std::mutex> lk(mu);
      auto it = cache.find(key);
      if (it != cache.end()) return it->second;
    }
    CK(cudaMemsetAsync(Y.get(), 0, Y.bytes(), stream));
    CK(cudaMemsetAsync(rec_d.get(), 0, rec_d.bytes(), stream));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    std::vector<TimeLaunch> ls(n);
    std::vector<WaveletFn> fns(n);
    std::vector<float> best(n, 1e30f);
    for (size_t v = 0; v < n; ++v) fns[v] = make(v, ls[v]);
    for (int round = 0; round < 3; ++round)
      for (size_t v = 0; v < n; ++v) {
        const TimeLaunch &L = ls[v];
        if (L.smem > (size_t)smem_max || L.n_cta == 0) continue;
        auto run = [&] {
          fns[v]<<<L.n_cta, kWavThreads, L.smem, stream>>>(
              wavf_jobs.get(), L.cta_job.get(), L.cta_trace0.get(), L.nb, spectra.get(),
              spec_off.get(), +1, nullptr);
          fns[v]<<<L.n_cta, kWavThreads, L.smem, stream>>>(
              wavf_jobs.get(), L.cta_job.get(), L.cta_trace0.get(), L.nb, spectra.get(),
              spec_off.get(), -1, rec_d.get());
          CK(cudaGetLastError());
        };
        run();
        CK(cudaEventRecord(e0, stream));
        run();
        CK(cudaEventRecord(e1, stream));
        CK(cudaEventSynchronize(e1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        best[v] = std::min(best[v], ms);
      }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const int pick = (int)(std::min_element(best.begin(), best.end()) - best.begin());
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = pick;
    return pick;
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

  // CTAs of nb traces over every window, or (generic_only) over the windows
  // of the generic kernels
  void make_time_launch(TimeLaunch &L, size_t per_trace, int nb_cap, bool generic_only) {
    int nb = nb_cap;
    while (nb > 1 && per_trace * nb > (size_t)std::min(smem_max, 160 * 1024)) nb /= 2;
    if (per_trace * nb > (size_t)smem_max)
      throw DeviceError("time window or trace too long for shared memory");
    std::vector<int> cj, ct;
    for (size_t w = 0; w < plan.windows.size(); ++w) {
      if (generic_only && win_tgroup[w] >= 0) continue;
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
  // blocks per SM.  Two-stage kernels either fill most of the shared memory
  // with one block per SM or take a third of it per block with two blocks
  // per SM; the one-stage kernels run two or three blocks per SM (two for
  // 40-point lines, whose registers do not fit three).  The
  // fastest of each list is picked by timing on the problem (autotune_space).
  template <int D, int P0, int P1, int P2, int NT, int NP, int ST, int MB>
  static void add_fwd(FastClass &c) {
    using Sh = PlaneShape<D, P0, P1, P2>;
    c.fwd_vars.push_back(FwdVariant{space_fwd_fast<R, D, P0, P1, P2, NT, NP, ST, MB>, NT, NP,
                                    ST, (size_t)ST * NP * Sh::size * sizeof(C), "space_fwd_fast"});
  }

  template <int D, int P0, int P1, int P2, int NT, int NP, int ST, int MB>
  static void add_adj(FastClass &c) {
    using Sh = PlaneShape<D, P0, P1, P2>;
    const size_t x = ST == 2 ? (size_t)NP * Sh::dense_P : 0;
    c.adj_vars.push_back(AdjVariant{space_adj_fast<R, D, P0, P1, P2, NT, NP, ST, MB>, NT, NP,
                                    ST, ((size_t)ST * NP * Sh::size + x) * sizeof(C), "space_adj_fast"});
  }

  // row-fused candidates (fast.cuh space_fwd_rows / space_adj_rows)
  template <int D, int P0, int P1, int P2, int NT, int NP, int MB>
  static void add_fwd_rows(FastClass &c) {
    using Sh = PlaneShape<D, P0, P1, P2>;
    c.fwd_vars.push_back(FwdVariant{space_fwd_rows<R, D, P0, P1, P2, NT, NP, MB>, NT, NP, 1,
                                    (size_t)NP * Sh::size * sizeof(C), "space_fwd_rows"});
  }

  template <int D, int P0, int P1, int P2, int NT, int NP, int ST, int MB>
  static void add_adj_rows(FastClass &c) {
    using Sh = PlaneShape<D, P0, P1, P2>;
    c.adj_vars.push_back(AdjVariant{space_adj_rows<R, D, P0, P1, P2, NT, NP, ST, MB>, NT, NP,
                                    ST, (size_t)ST * NP * Sh::size * sizeof(C), "space_adj_rows"});
  }

  // pipelined adjoint candidates (fast.cuh space_adj_pipe): NP dense
  // cropped staging planes and NP padded work planes
  template <int D, int P0, int P1, int P2, int NT, int NP, int MB, bool XS = false>
  static void add_adj_pipe(FastClass &c) {
    using Sh = PlaneShape<D, P0, P1, P2>;
    const size_t stg = (size_t)NP * Sh::dense_L;
    const size_t work = (size_t)NP * Sh::size;
    const size_t x = XS ? (size_t)NP * Sh::dense_P : 0;
    c.adj_vars.push_back(AdjVariant{space_adj_pipe<R, D, P0, P1, P2, NT, NP, MB, XS>, NT, NP,
                                    XS ? 4 : 3,
                                    (stg + stg % 2 + work + work % 2 + x) * sizeof(C), "space_adj_pipe"});
  }

  template <int D, int P0, int P1, int P2>
  static bool shape_is(const WindowPlan &W) {
    const int P[3] = {P0, P1, P2};
    if (W.D != D) return false;
    for (int d = 0; d < D; ++d)
      if (W.P[d] != P[d]) return false;
    return true;
  }

  static bool space_cases(const WindowPlan &W, FastClass &c) {
    c.fwd_vars.clear();
    c.adj_vars.clear();
    if constexpr (sizeof(R) == sizeof(float)) {
      if (shape_is<1, 40, 1, 1>(W)) {
        add_fwd<1, 40, 1, 1, 256, 256, 2, 1>(c);
        add_fwd<1, 40, 1, 1, 256, 96, 1, 2>(c);
        add_fwd<1, 40, 1, 1, 256, 96, 2, 2>(c);
        add_adj<1, 40, 1, 1, 192, 192, 2, 1>(c);
        add_adj<1, 40, 1, 1, 256, 96, 1, 2>(c);
        add_adj<1, 40, 1, 1, 256, 96, 2, 2>(c);
        add_fwd_rows<1, 40, 1, 1, 256, 64, 2>(c);
        add_adj_rows<1, 40, 1, 1, 256, 64, 2, 2>(c);
        add_adj_pipe<1, 40, 1, 1, 256, 128, 2>(c);
      } else if (shape_is<1, 20, 1, 1>(W)) {
        add_fwd<1, 20, 1, 1, 256, 256, 2, 1>(c);
        add_fwd<1, 20, 1, 1, 256, 128, 1, 3>(c);
        add_fwd<1, 20, 1, 1, 256, 128, 2, 2>(c);
        add_adj<1, 20, 1, 1, 256, 256, 2, 1>(c);
        add_adj<1, 20, 1, 1, 256, 128, 1, 3>(c);
        add_adj<1, 20, 1, 1, 256, 128, 2, 2>(c);
        add_fwd_rows<1, 20, 1, 1, 256, 128, 3>(c);
        add_adj_rows<1, 20, 1, 1, 256, 128, 2, 2>(c);
        add_adj_pipe<1, 20, 1, 1, 256, 160, 3>(c);
        add_adj_pipe<1, 20, 1, 1, 256, 256, 2>(c);
      } else if (shape_is<2, 20, 40, 1>(W)) {
        add_fwd<2, 20, 40, 1, 384, 16, 2, 1>(c);
        add_fwd<2, 20, 40, 1, 256, 12, 1, 2>(c);
        add_fwd<2, 20, 40, 1, 256, 6, 2, 2>(c);
        add_fwd<2, 20, 40, 1, 192, 6, 1, 3>(c);
        add_adj<2, 20, 40, 1, 384, 11, 2, 1>(c);
        add_adj<2, 20, 40, 1, 256, 12, 1, 2>(c);
        add_adj<2, 20, 40, 1, 256, 5, 2, 2>(c);
        add_fwd_rows<2, 20, 40, 1, 256, 8, 2>(c);
        add_adj_rows<2, 20, 40, 1, 256, 6, 2, 2>(c);
        add_adj_pipe<2, 20, 40, 1, 256, 6, 2>(c);
        add_adj_pipe<2, 20, 40, 1, 256, 5, 2, true>(c);
        add_adj_pipe<2, 20, 40, 1, 256, 8, 2>(c);
      } else if (shape_is<2, 20, 20, 1>(W)) {
        add_fwd<2, 20, 20, 1, 384, 24, 2, 1>(c);
        add_fwd<2, 20, 20, 1, 256, 12, 1, 3>(c);
        add_fwd<2, 20, 20, 1, 256, 12, 2, 2>(c);
        add_adj<2, 20, 20, 1, 384, 20, 2, 1>(c);
        add_adj<2, 20, 20, 1, 256, 12, 1, 3>(c);
        add_adj<2, 20, 20, 1, 256, 10, 2, 2>(c);
        add_fwd_rows<2, 20, 20, 1, 256, 12, 3>(c);
        add_adj_rows<2, 20, 20, 1, 256, 10, 2, 2>(c);
        add_adj_pipe<2, 20, 20, 1, 256, 12, 3>(c);
        add_adj_pipe<2, 20, 20, 1, 256, 16, 2>(c);
        add_adj_pipe<2, 20, 20, 1, 256, 8, 2, true>(c);
      } else if (shape_is<2, 40, 40, 1>(W)) {
        add_fwd<2, 40, 40, 1, 320, 8, 2, 1>(c);
        add_fwd<2, 40, 40, 1, 256, 6, 1, 2>(c);
        add_fwd<2, 40, 40, 1, 256, 3, 2, 2>(c);
        add_adj<2, 40, 40, 1, 256, 5, 2, 1>(c);
        add_adj<2, 40, 40, 1, 256, 6, 1, 2>(c);
        add_adj<2, 40, 40, 1, 256, 2, 2, 2>(c);
        add_fwd_rows<2, 40, 40, 1, 256, 4, 2>(c);
        add_adj_rows<2, 40, 40, 1, 256, 3, 2, 2>(c);
        add_adj_pipe<2, 40, 40, 1, 256, 4, 2>(c);
      } else if (shape_is<3, 20, 20, 20>(W)) {
        add_fwd<3, 20, 20, 20, 512, 1, 2, 1>(c);
        add_fwd<3, 20, 20, 20, 256, 1, 1, 3>(c);
        add_fwd<3, 20, 20, 20, 416, 1, 1, 2>(c);
        add_fwd_rows<3, 20, 20, 20, 256, 1, 3>(c);
        add_adj<3, 20, 20, 20, 512, 1, 2, 1>(c);
        add_adj<3, 20, 20, 20, 256, 1, 1, 3>(c);
        add_adj_rows<3, 20, 20, 20, 512, 1, 2, 1>(c);
        add_adj_rows<3, 20, 20, 20, 256, 1, 1, 3>(c);
        add_adj_pipe<3, 20, 20, 20, 256, 1, 2>(c);
        add_adj_pipe<3, 20, 20, 20, 384, 1, 2>(c);
        add_adj_pipe<3, 20, 20, 20, 448, 1, 1, true>(c);
        add_adj_pipe<3, 20, 20, 20, 416, 1, 2>(c);
      }
    } else {
      // double: the two-stage kernels only (one-stage kernels with several
      // blocks per SM would spill), and one stage for the 20x20x20 planes
      if (shape_is<1, 40, 1, 1>(W)) {
        add_fwd<1, 40, 1, 1, 256, 128, 2, 1>(c);
        add_adj<1, 40, 1, 1, 192, 96, 2, 1>(c);
      } else if (shape_is<1, 20, 1, 1>(W)) {
        add_fwd<1, 20, 1, 1, 256, 256, 2, 1>(c);
        add_adj<1, 20, 1, 1, 256, 160, 2, 1>(c);
      } else if (shape_is<2, 20, 40, 1>(W)) {
        add_fwd<2, 20, 40, 1, 384, 8, 2, 1>(c);
        add_adj<2, 20, 40, 1, 384, 5, 2, 1>(c);
      } else if (shape_is<2, 20, 20, 1>(W)) {
        add_fwd<2, 20, 20, 1, 384, 12, 2, 1>(c);
        add_adj<2, 20, 20, 1, 384, 10, 2, 1>(c);
      } else if (shape_is<2, 40, 40, 1>(W)) {
        add_fwd<2, 40, 40, 1, 320, 4, 2, 1>(c);
        add_adj<2, 40, 40, 1, 256, 2, 2, 1>(c);
      } else if (shape_is<3, 20, 20, 20>(W)) {
        add_fwd<3, 20, 20, 20, 256, 1, 1, 1>(c);
        add_adj<3, 20, 20, 20, 256, 1, 1, 1>(c);
      }
    }
    return !c.fwd_vars.empty() && !c.adj_vars.empty();
  }

  // time-axis kernel candidates for Pt = 2 M1 M2: NB traces per block, line
  // stride LS (M + 1, or padded to 10 mod 16 complex so that the four-step
  // passes hit distinct banks), MB blocks per SM
  template <int M1, int M2, int NB, int LS, int MB>
  static void add_time(TimeGroup &g) {
    constexpr int M = M1 * M2;
    constexpr int H = 4 * M / 5;
    g.fwd_vars.push_back(TimeFwdVariant{time_fwd_fast<R, M1, M2, NB, LS, MB>, NB,
                                        2 * (size_t)NB * LS * sizeof(C) +
                                            (size_t)NB * H * sizeof(R), "time_fwd_fast"});
    g.adj_vars.push_back(TimeAdjVariant{time_adj_fast<R, M1, M2, NB, LS, MB>, NB,
                                        (size_t)NB * LS * sizeof(C) +
                                            2 * (size_t)NB * 2 * H * sizeof(R), "time_adj_fast"});
  }

  // fused candidates (fast.cuh time_fwd_fused / time_adj_fused), 256 / M1
  // traces per block
  template <int M1, int M2, int LSB, int LSW, int MB>
  static void add_time_fused(TimeGroup &g) {
    constexpr int M = M1 * M2;
    constexpr int H = 4 * M / 5;
    constexpr int NB = kThreads / M1;
    g.fwd_vars.push_back(TimeFwdVariant{time_fwd_fused<R, M1, M2, LSB, LSW, MB>, NB,
                                        ((size_t)2 * NB * LSB + (size_t)NB * LSW) * sizeof(C), "time_fwd_fused"});
    constexpr int LT = 2 * H;
    constexpr int LTP = LT + ((20 - LT % 32) + 32) % 32;  // as time_adj_fused
    g.adj_vars.push_back(TimeAdjVariant{time_adj_fused<R, M1, M2, LSW, MB>, NB,
                                        (size_t)NB * LSW * sizeof(C) +
                                            2 * (size_t)NB * LTP * sizeof(R), "time_adj_fused"});
  }

  static bool time_case(const WindowPlan &W, TimeGroup &g) {
    g.fwd_vars.clear();
    g.adj_vars.clear();
    if (W.Pt == 320) {
      add_time<16, 10, 32, 161, 1>(g);
      if constexpr (sizeof(R) == sizeof(float)) {
        add_time<16, 10, 32, 170, 2>(g);
        add_time<16, 10, 16, 170, 4>(g);
        add_time_fused<16, 10, 170, 186, 3>(g);
        add_time_fused<16, 10, 170, 186, 2>(g);
      }
    } else if (W.Pt == 160) {
      add_time<8, 10, 32, 81, 1>(g);
      if constexpr (sizeof(R) == sizeof(float)) {
        add_time<8, 10, 32, 90, 2>(g);
        add_time<8, 10, 16, 90, 4>(g);
        add_time_fused<8, 10, 90, 90, 3>(g);
        add_time_fused<8, 10, 90, 90, 2>(g);
      }
    } else {
      return false;
    }
    return true;
  }

  // the fast space kernels assume L = 4P/5 on every space axis, the fast
  // time kernels Lt = 2h = 4Pt/5
  static bool space_eligible(const WindowPlan &W) {
    for (int d = 0; d < W.D; ++d)
      if (W.L[d] * 5 != W.P[d] * 4) return false;
    return true;
  }
  static bool time_eligible(const WindowPlan &W) {
    return W.Lt % 2 == 0 && W.Lt * 5 == W.Pt * 4;
  }

  // Groups the windows into fast space classes and fast time groups
  // (AGD_GPU_GENERIC=1: none).
  void pick_classes() {
    const int nw = (int)plan.windows.size();
    win_class.assign(nw, -1);
    win_tgroup.assign(nw, -1);
    classes.clear();
    tgroups.clear();
    const char *env = std::getenv("AGD_GPU_GENERIC");
    const bool generic_only = env != nullptr && env[0] == '1';
    std::map<std::vector<int>, int> by_key;  // -1: no instantiation
    std::map<int, int> by_pt;
    for (int w = 0; w < nw && !generic_only; ++w) {
      const WindowPlan &W = plan.windows[w];
      if (time_eligible(W)) {
        auto it = by_pt.find(W.Pt);
        int k;
        if (it == by_pt.end()) {
          std::unique_ptr<TimeGroup> g(new TimeGroup());
          k = time_case(W, *g) ? (int)tgroups.size() : -1;
          if (k >= 0) tgroups.push_back(std::move(g));
          by_pt[W.Pt] = k;
        } else {
          k = it->second;
        }
        if (k >= 0) {
          win_tgroup[w] = k;
          tgroups[k]->win.push_back(w);
        }
      }
      if (!space_eligible(W)) continue;
      std::vector<int> key{W.D};
      for (int d = 0; d < W.D; ++d) key.push_back(W.P[d]);
      auto it = by_key.find(key);
      int k;
      if (it == by_key.end()) {
        std::unique_ptr<FastClass> c(new FastClass());
        if (space_cases(W, *c)) {
          k = (int)classes.size();
          classes.push_back(std::move(c));
        } else {
          k = -1;
        }
        by_key[key] = k;
      } else {
        k = it->second;
      }
      if (k < 0) continue;
      win_class[w] = k;
      classes[k]->win.push_back(w);
    }
    // one space axis of any other length up to kLineMaxP: line kernels,
    // when their blocks fit in shared memory
    win_line.assign(nw, 0);
    for (int w = 0; w < nw && !generic_only; ++w) {
      const WindowPlan &W = plan.windows[w];
      if (win_class[w] >= 0 || W.D != 1 || W.P[0] > kLineMaxP || W.P[0] < 3) continue;
      const int P = W.P[0], L = W.L[0];
      const int H = (P - 1) / 2;
      const size_t sf = line_fwd_smem<R>(P, H, (L + 3) / 4 * 4, 4);
      const size_t sa = line_adj_smem<R>(P, L, (P / 2 + 1 + 3) / 4 * 4, 4);
      if (std::max(sf, sa) <= (size_t)smem_max) win_line[w] = 1;
    }
    n_generic = 0;
    max_d_generic = 0;
    for (int w = 0; w < nw; ++w)
      if (win_class[w] < 0 && !win_line[w]) {
        ++n_generic;
        max_d_generic = std::max(max_d_generic, plan.windows[w].D);
      }
  }

  // Line-kernel jobs, tables and block lists (windows marked in win_line).
  // Tables per (P, L) in double precision, rounded once: forward rows
  // j = 1 .. (P-1)/2 over outputs k < L, adjoint rows j < L over k <= P/2,
  // cos / sin of 2 pi (j k mod P) / P, rows padded to a multiple of 4.
  void build_line_kernels() {
    const int nw = (int)plan.windows.size();
    std::vector<R> tab;
    std::map<std::pair<int, int>, std::pair<long, long>> off;  // (P, L) -> fwd, adj
    auto add_table = [&](int P, int rows, int j0, int kout, int kpad) {
      const long o = (long)tab.size();
      tab.resize(tab.size() + 2 * (size_t)rows * kpad, (R)0);
      for (int r = 0; r < rows; ++r)
        for (int k = 0; k < kout; ++k) {
          const long m = (long)(r + j0) * k % P;
          const double a = 2.0 * 3.14159265358979323846 * (double)m / (double)P;
          tab[o + (long)r * kpad + k] = (R)std::cos(a);
          tab[o + (long)rows * kpad + (long)r * kpad + k] = (R)std::sin(a);
        }
      return o;
    };
    std::vector<LineJob<R>> jf, ja;
    std::vector<long> tf, ta;  // table offsets of each job
    for (int w = 0; w < nw; ++w) {
      if (!win_line[w]) continue;
      const WindowPlan &W = plan.windows[w];
      const int P = W.P[0], L = W.L[0];
      const int H = (P - 1) / 2;
      const int kpf = (L + 3) / 4 * 4, kpa = (P / 2 + 1 + 3) / 4 * 4;
      auto it = off.find({P, L});
      if (it == off.end())
        it = off.emplace(std::make_pair(P, L),
                         std::make_pair(add_table(P, H, 1, L, kpf),
                                        add_table(P, L, 0, P / 2 + 1, kpa)))
                 .first;
      const long lines = (long)W.T * W.F;
      LineJob<R> f{};
      f.src = X.get() + W.model_off;
      f.dst = S0.get() + W.model_off;
      f.lines = lines;
      f.P = P;
      f.L = L;
      f.rows = H;
      f.kout = L;
      f.kpad = kpf;
      f.pid = W.problem;
      LineJob<R> a = f;
      a.src = S0.get() + W.model_off;
      a.dst = X.get() + W.model_off;
      a.rows = L;
      a.kout = P / 2 + 1;
      a.kpad = kpa;
      f.nl = line_pick_nl(P, L, true);
      a.nl = line_pick_nl(P, L, false);
      jf.push_back(f);
      ja.push_back(a);
      tf.push_back(it->second.first);
      ta.push_back(it->second.second);
    }
    if (jf.empty()) return;
    line_tab.upload(tab, stream);
    for (size_t i = 0; i < jf.size(); ++i) {
      jf[i].tab_c = line_tab.get() + tf[i];
      jf[i].tab_s = jf[i].tab_c + (long)jf[i].rows * jf[i].kpad;
      ja[i].tab_c = line_tab.get() + ta[i];
      ja[i].tab_s = ja[i].tab_c + (long)ja[i].rows * ja[i].kpad;
    }
    make_line_launch(line_fwd, jf, true);
    make_line_launch(line_adj, ja, false);
    line_adj_host = ja;
  }

  // Lines per block of a window: a multiple of 4 whose 4-line x 4-output
  // tiles best fill the block's threads, within a shared-memory budget of
  // three blocks per SM (two in double; more when even 4 lines need it),
  // counting the memory the system reserves per block and the kernels'
  // static arrays (at most 256 bytes).
  int line_pick_nl(int P, int L, bool fwd) const {
    const int H = (P - 1) / 2;
    const int kpad = fwd ? (L + 3) / 4 * 4 : (P / 2 + 1 + 3) / 4 * 4;
    auto smem = [&](int nl) {
      return fwd ? line_fwd_smem<R>(P, H, kpad, nl) : line_adj_smem<R>(P, L, kpad, nl);
    };
    const int blocks = sizeof(R) == sizeof(float) ? 3 : 2;
    const size_t budget =
        std::max<size_t>((size_t)(sm_smem / blocks - block_reserved - 256), smem(4));
    int best = 4;
    double best_eff = -1.0;
    for (int nl = 4; nl <= 64 && smem(nl) <= budget; nl += 4) {
      const int tiles = nl / 4 * (kpad / 4);
      const int rounds = (tiles + kLineThreads - 1) / kLineThreads;
      const double eff = (double)tiles / (rounds * kLineThreads);
      if (eff >= best_eff - 1e-9) {
        best_eff = eff;
        best = nl;
      }
    }
    return best;
  }

  void make_line_launch(LineLaunch &Lc, const std::vector<LineJob<R>> &jobs, bool fwd) {
    std::vector<int> cj;
    std::vector<long> cl;
    size_t smem = 0;
    for (size_t i = 0; i < jobs.size(); ++i) {
      const LineJob<R> &j = jobs[i];
      for (long l = 0; l < j.lines; l += j.nl) {
        cj.push_back((int)i);
        cl.push_back(l);
      }
      smem = std::max(smem, fwd ? line_fwd_smem<R>(j.P, j.rows, j.kpad, j.nl)
                                : line_adj_smem<R>(j.P, j.L, j.kpad, j.nl));
    }
    Lc.jobs.upload(jobs, stream);
    Lc.cta_job.upload(cj, stream);
    Lc.cta_line0.upload(cl, stream);
    Lc.n_cta = (int)cj.size();
    Lc.smem = smem;
  }

  // Times every candidate of a class (three rounds over the candidates, each
  // one warm-up launch and two timed ones with CUDA events on the engine's
  // stream; forward X -> S0, adjoint S0 -> X with the update epilogue) and
  // keeps the fastest.  Choices are
  // remembered per shape, precision, problem size class and device, so later
  // problems of the same kind skip the timing.  AGD_GPU_SPACE_VARIANT="f,a"
  // forces the candidates (tests).
  void autotune_space(FastClass &c, const std::vector<PlaneJob<R>> &jf,
                      const std::vector<PlaneJob<R>> &ja) {
    c.fwd_pick = c.adj_pick = 0;
    const char *env = std::getenv("AGD_GPU_SPACE_VARIANT");
    if (env != nullptr && env[0] != '\0') {
      int f = 0, a = 0;
      if (std::sscanf(env, "%d,%d", &f, &a) == 2) {
        c.fwd_pick = std::max(0, std::min(f, (int)c.fwd_vars.size() - 1));
        c.adj_pick = std::max(0, std::min(a, (int)c.adj_vars.size() - 1));
        return;
      }
    }
    if (c.fwd_vars.size() == 1 && c.adj_vars.size() == 1) return;
    long total = 0;
    for (long v : c.planes) total += v;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    const WindowPlan &W = plan.windows[c.win[0]];
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
        c.fwd_pick = it->second.first;
        c.adj_pick = it->second.second;
        return;
      }
    }
    // a non-zero model and a small threshold, so that the adjoint's update
    // takes the arithmetic path of real iterations (every byte 0x3f: about
    // 0.75 in float, 1.6e-4 in double)
    CK(cudaMemsetAsync(X.get(), 0x3f, X.bytes(), stream));
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
    // three rounds over all candidates, the best time of each counts
    const size_t nf = c.fwd_vars.size(), na = c.adj_vars.size();
    std::vector<PlaneLaunch> lf(nf), la(na);
    std::vector<float> tf(nf, 1e30f), ta(na, 1e30f);
    for (size_t v = 0; v < nf; ++v)
      if (c.fwd_vars[v].smem <= (size_t)smem_max)
        make_plane_launch(lf[v], jf, c.planes, c.fwd_vars[v].nt, c.fwd_vars[v].np,
                          c.fwd_vars[v].smem, c.fwd_vars[v].fn);
    for (size_t v = 0; v < na; ++v)
      if (c.adj_vars[v].smem <= (size_t)smem_max)
        make_plane_launch(la[v], ja, c.planes, c.adj_vars[v].nt, c.adj_vars[v].np,
                          c.adj_vars[v].smem, c.adj_vars[v].fn);
    for (int round = 0; round < 3; ++round) {
      for (size_t v = 0; v < nf; ++v) {
        const PlaneLaunch &L = lf[v];
        if (L.n_batch == 0) continue;
        const SpaceFwdFn fn = c.fwd_vars[v].fn;
        tf[v] = std::min(tf[v], timed([&] {
          fn<<<L.grid, L.nt, L.smem, stream>>>(L.batches());
          CK(cudaGetLastError());
        }));
      }
      for (size_t v = 0; v < na; ++v) {
        const PlaneLaunch &L = la[v];
        if (L.n_batch == 0) continue;
        const SpaceAdjFn fn = c.adj_vars[v].fn;
        ta[v] = std::min(ta[v], timed([&] {
          fn<<<L.grid, L.nt, L.smem, stream>>>(L.batches(), kUpdateThreshold, (R)0.5,
                                               (R)1e-6, nullptr, nullptr, scalar.get());
          CK(cudaGetLastError());
        }));
      }
    }
    c.fwd_pick = (int)(std::min_element(tf.begin(), tf.end()) - tf.begin());
    c.adj_pick = (int)(std::min_element(ta.begin(), ta.end()) - ta.begin());
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::lock_guard<std::mutex> g(mu);
    cache[key] = {c.fwd_pick, c.adj_pick};
  }

  // Persistent batches of np planes; grid = resident blocks.
  template <typename K>
  void make_plane_launch(PlaneLaunch &L, const std::vector<PlaneJob<R>> &jobs,
                         const std::vector<long> &planes, int nt, int np, size_t smem,
                         K kernel, size_t smem_limit = 0) {
    if (smem > (smem_limit ? smem_limit : (size_t)smem_max))
      throw DeviceError("space planes too large");
    std::vector<PlaneBatch<R>> bt;
    for (size_t i = 0; i < jobs.size(); ++i)
      for (long q = 0; q < planes[i]; q += np) {
        PlaneBatch<R> x{};
        x.src = jobs[i].src + q * jobs[i].src_plane;
        x.dst = jobs[i].dst + q * jobs[i].dst_plane;
        x.count = (int)std::min<long>(np, planes[i] - q);
        x.pid = jobs[i].pid;
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

  // shared-memory opt-in of every fast kernel of every class
  void opt_in_classes() {
    const int limit = optin_smem();
    int dyn = smem_max;
    for (const auto &gp : tgroups) {
      for (const TimeFwdVariant &v : gp->fwd_vars) dyn = std::min(dyn, opt_in(v.fn, limit));
      for (const TimeAdjVariant &v : gp->adj_vars) dyn = std::min(dyn, opt_in(v.fn, limit));
    }
    for (const auto &cp : classes) {
      for (const FwdVariant &v : cp->fwd_vars) dyn = std::min(dyn, opt_in(v.fn, limit));
      for (const AdjVariant &v : cp->adj_vars) dyn = std::min(dyn, opt_in(v.fn, limit));
    }
    smem_max = std::min(smem_max, dyn);
  }

  void build_class(FastClass &c) {
    const WindowPlan &W0 = plan.windows[c.win[0]];
    long dense_P = 1, dense_L = 1;
    for (int d = 0; d < W0.D; ++d) {
      dense_P *= W0.P[d];
      dense_L *= W0.L[d];
    }
    std::vector<PlaneJob<R>> jf, ja;
    c.planes.clear();
    for (int w : c.win) {
      const WindowPlan &W = plan.windows[w];
      c.planes.push_back((long)W.T * W.F);
      PlaneJob<R> j{};
      j.pid = W.problem;
      j.src = X.get() + W.model_off;
      j.dst = S0.get() + W.model_off;
      j.src_plane = dense_P;
      j.dst_plane = dense_L;
      jf.push_back(j);
      j.src = S0.get() + W.model_off;
      j.dst = X.get() + W.model_off;
      j.src_plane = dense_L;
      j.dst_plane = dense_P;
      ja.push_back(j);
    }
    autotune_space(c, jf, ja);
    make_plane_launch(c.pl_fwd, jf, c.planes, c.fv().nt, c.fv().np, c.fv().smem, c.fv().fn);
    make_plane_launch(c.pl_adj, ja, c.planes, c.av().nt, c.av().np, c.av().smem, c.av().fn);
    c.fwd_jobs = jf;
    c.plain_jobs = ja;
  }

  // ------------------------------------------------------------ precision modes
  //
  // Mode 0 (default): FP32 space kernels.  Mode 1: the space axes of every
  // window class of padded shape kTcP^3 and window kTcL^3 run as split-BF16
  // tensor-core contractions (space_tc.cuh); the time axis, the wavelet, the
  // blend and the update arithmetic stay FP32.  Float library only.
  static constexpr int kTcP = 20, kTcL = 16;
  using TcS = TcDft3<kTcP, kTcL>;
  int precision = 0;
  DevArray<uint16_t> tc_mat;  // forward hi | forward lo | adjoint hi | adjoint lo
  DevArray<int> tc_err;       // 1 when a tensor-core wait gave up
  long tc_windows = 0;

  static bool tc_shape(const WindowPlan &W) {
    return W.D == 3 && W.P[0] == kTcP && W.P[1] == kTcP && W.P[2] == kTcP && W.L[0] == kTcL &&
           W.L[1] == kTcL && W.L[2] == kTcL;
  }

  // BF16 bits of a float, rounded to nearest even (finite values)
  static uint16_t bf16_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
  }
  static double bf16_value(uint16_t h) {
    const uint32_t u = (uint32_t)h << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
  }
  // hi, lo BF16 parts of v (v ~ hi + lo to about 16 significant bits)
  static void split_host(double v, uint16_t &hi, uint16_t &lo) {
    hi = bf16_bits((float)v);
    lo = bf16_bits((float)(v - bf16_value(hi)));
  }

  // B[n][k] of the forward (n = 2 i + (re, im) for output i < L, k = 2 j +
  // (re, im) for input j < P; exp(+2 pi i i j / P)) and of the adjoint (n = 2 k
  // + .. for output k < P, k = 2 j + .. for input j < L; exp(-2 pi i j k / P)),
  // as real matrices acting on interleaved (re, im) values, zero-padded to
  // the kernels' N x K; computed in double precision, then split.
  void upload_tc_matrices() {
    const int nf = TcS::kFwdN * TcS::kFwdK, na = TcS::kAdjN * TcS::kAdjK;
    std::vector<uint16_t> h(2 * nf + 2 * na, 0);
    const double two_pi = 6.283185307179586476925286766559;
    auto put = [&](int base, int n_off, int K, int row_i, int col_j, double c, double sgn_s) {
      // complex entry w = c + i s at (output row_i, input col_j), s = sgn_s
      const double vals[2][2] = {{c, -sgn_s}, {sgn_s, c}};
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
          uint16_t hi, lo;
          split_host(vals[a][b], hi, lo);
          const int idx = (2 * row_i + a) * K + 2 * col_j + b;
          h[base + idx] = hi;
          h[base + n_off + idx] = lo;
        }
    };
    for (int i = 0; i < kTcL; ++i)
      for (int j = 0; j < kTcP; ++j) {
        const double th = two_pi * (double)((i * j) % kTcP) / kTcP;
        put(0, nf, TcS::kFwdK, i, j, std::cos(th), std::sin(th));
      }
    for (int k = 0; k < kTcP; ++k)
      for (int j = 0; j < kTcL; ++j) {
        const double th = two_pi * (double)((j * k) % kTcP) / kTcP;
        put(2 * nf, na, TcS::kAdjK, k, j, std::cos(th), -std::sin(th));
      }
    tc_mat.alloc(h.size());
    CK(cudaMemcpyAsync(tc_mat.get(), h.data(), h.size() * sizeof(uint16_t),
                       cudaMemcpyHostToDevice, stream));
    tc_err.alloc(1);
    CK(cudaMemsetAsync(tc_err.get(), 0, sizeof(int), stream));
  }

  TcMatrices tc_fwd_mats() const {
    const int nf = TcS::kFwdN * TcS::kFwdK;
    return TcMatrices{tc_mat.get(), tc_mat.get() + nf};
  }
  TcMatrices tc_adj_mats() const {
    const int nf = TcS::kFwdN * TcS::kFwdK, na = TcS::kAdjN * TcS::kAdjK;
    return TcMatrices{tc_mat.get() + 2 * nf, tc_mat.get() + 2 * nf + na};
  }

  void build_tc_plain(FastClass &c) {
    if constexpr (std::is_same<R, float>::value) {
      std::vector<PlaneJob<R>> jobs = c.plain_jobs;
      for (size_t i = 0; i < jobs.size(); ++i)
        jobs[i].dst = G.get() + plan.windows[c.win[i]].model_off;
      make_plane_launch(c.tc_adj_plain, jobs, c.planes, kTcThreads, kTcBatch,
                        TcS::kAdjSmem, space_adj_tc<kTcP, kTcL>, (size_t)optin_smem());
      tc_grid(c.tc_adj_plain);
    }
  }

  static constexpr int kTcBatch = 4;  // planes per batch record of the tensor-core kernels
  // the tensor-core kernels are sized for two CTAs per SM (shared memory,
  // registers and TMEM columns), whatever the occupancy query answers
  void tc_grid(PlaneLaunch &L) const { L.grid = std::max(1, std::min(L.n_batch, 2 * n_sm)); }

  void set_precision(int mode) {
    if (mode != 0 && mode != 1) throw DeviceError("unknown precision mode");
    if (mode == precision) return;
    release_graph();
    CK(cudaStreamSynchronize(stream));
    for (auto &cp : classes) cp->tc = false;
    tc_windows = 0;
    if (mode == 1) {
      if constexpr (!std::is_same<R, float>::value) {
        throw DeviceError("the split-BF16 tensor-core kernels serve the float library only");
      } else {
        if (tc_mat.get() == nullptr) upload_tc_matrices();
        const int limit = optin_smem();
        if ((int)TcS::kFwdSmem > limit || (int)TcS::kAdjSmem > limit)
          throw DeviceError("not enough shared memory for the tensor-core kernels");
        CK(cudaFuncSetAttribute(space_fwd_tc<kTcP, kTcL>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, TcS::kFwdSmem));
        CK(cudaFuncSetAttribute(space_adj_tc<kTcP, kTcL>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, TcS::kAdjSmem));
        // all of the unified L1 / shared memory as shared memory: two CTAs per SM
        CK(cudaFuncSetAttribute(space_fwd_tc<kTcP, kTcL>,
                                cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        CK(cudaFuncSetAttribute(space_adj_tc<kTcP, kTcL>,
                                cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        for (auto &cp : classes) {
          FastClass &c = *cp;
          if (!tc_shape(plan.windows[c.win[0]])) continue;
          make_plane_launch(c.tc_fwd, c.fwd_jobs, c.planes, kTcThreads, kTcBatch,
                            TcS::kFwdSmem, space_fwd_tc<kTcP, kTcL>, (size_t)limit);
          make_plane_launch(c.tc_adj, c.plain_jobs, c.planes, kTcThreads, kTcBatch,
                            TcS::kAdjSmem, space_adj_tc<kTcP, kTcL>, (size_t)limit);
          tc_grid(c.tc_fwd);
          tc_grid(c.tc_adj);
          if (G.get() != nullptr) build_tc_plain(c);
          c.tc = true;
          tc_windows += (long)c.win.size();
        }
        CK(cudaStreamSynchronize(stream));
      }
    }
    precision = mode;
  }

  // error word of the tensor-core kernels (read after the stream's work)
  void check_tc_error() {
    if (precision != 1 || tc_err.get() == nullptr) return;
    int h = 0;
    CK(cudaMemcpyAsync(&h, tc_err.get(), sizeof(int), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    if (h) throw DeviceError("a tensor-core kernel gave up waiting for its MMAs");
  }

  void build_time_group(TimeGroup &g) {
    autotune_time(g);
    make_fixed_time_launch(g.tf, g.fv().smem, g.win, g.fv().nb);
    make_fixed_time_launch(g.ta, g.av().smem, g.win, g.av().nb);
  }

  // As autotune_space, for the candidates of a time group: forward
  // S0/S1 -> Y, adjoint record (or Y after the wavelet stage) -> S0/S1.
  // AGD_GPU_TIME_VARIANT="f,a" forces the candidates (tests).
  void autotune_time(TimeGroup &g) {
    g.fwd_pick = g.adj_pick = 0;
    const char *env = std::getenv("AGD_GPU_TIME_VARIANT");
    if (env != nullptr && env[0] != '\0') {
      int f = 0, a = 0;
      if (std::sscanf(env, "%d,%d", &f, &a) == 2) {
        g.fwd_pick = std::max(0, std::min(f, (int)g.fwd_vars.size() - 1));
        g.adj_pick = std::max(0, std::min(a, (int)g.adj_vars.size() - 1));
        return;
      }
    }
    if (g.fwd_vars.size() == 1 && g.adj_vars.size() == 1) return;
    long traces = 0;
    for (int w : g.win) traces += plan.windows[w].n_traces;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    char key[96];
    std::snprintf(key, sizeof key, "time:%d:%d:%d:%d:%d", dev, (int)sizeof(R),
                  plan.windows[g.win[0]].Pt, wavelets ? 1 : 0,
                  (int)std::log2((double)std::max(1L, traces)));
    static std::mutex mu;
    static std::map<std::string, std::pair<int, int>> cache;
    {
      std::lock_guard<std::mutex> lk(mu);
      auto it = cache.find(key);
      if (it != cache.end()) {
        g.fwd_pick = it->second.first;
        g.adj_pick = it->second.second;
        return;
      }
    }
    if (Y.get() != nullptr) CK(cudaMemsetAsync(Y.get(), 0, Y.bytes(), stream));
    if (rec_d.get() != nullptr) CK(cudaMemsetAsync(rec_d.get(), 0, rec_d.bytes(), stream));
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
    const size_t nf = g.fwd_vars.size(), na = g.adj_vars.size();
    std::vector<TimeLaunch> lf(nf), la(na);
    std::vector<float> tf(nf, 1e30f), ta(na, 1e30f);
    for (size_t v = 0; v < nf; ++v)
      if (g.fwd_vars[v].smem <= (size_t)smem_max)
        make_fixed_time_launch(lf[v], g.fwd_vars[v].smem, g.win, g.fwd_vars[v].nb);
    for (size_t v = 0; v < na; ++v)
      if (g.adj_vars[v].smem <= (size_t)smem_max)
        make_fixed_time_launch(la[v], g.adj_vars[v].smem, g.win, g.adj_vars[v].nb);
    const int from_record = wavelets ? 0 : 1;
    for (int round = 0; round < 3; ++round) {
      for (size_t v = 0; v < nf; ++v) {
        const TimeLaunch &L = lf[v];
        if (L.n_cta == 0) continue;
        const TimeFwdFn fn = g.fwd_vars[v].fn;
        tf[v] = std::min(tf[v], timed([&] {
          fn<<<L.n_cta, kThreads, L.smem, stream>>>(time_jobs.get(), L.cta_job.get(),
                                                    L.cta_trace0.get());
          CK(cudaGetLastError());
        }));
      }
      for (size_t v = 0; v < na; ++v) {
        const TimeLaunch &L = la[v];
        if (L.n_cta == 0) continue;
        const TimeAdjFn fn = g.adj_vars[v].fn;
        ta[v] = std::min(ta[v], timed([&] {
          fn<<<L.n_cta, kThreads, L.smem, stream>>>(time_jobs.get(), L.cta_job.get(),
                                                    L.cta_trace0.get(), rec_d.get(),
                                                    from_record);
          CK(cudaGetLastError());
        }));
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    g.fwd_pick = (int)(std::min_element(tf.begin(), tf.end()) - tf.begin());
    g.adj_pick = (int)(std::min_element(ta.begin(), ta.end()) - ta.begin());
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = {g.fwd_pick, g.adj_pick};
  }

  void make_fixed_time_launch(TimeLaunch &L, size_t smem, const std::vector<int> &wins,
                              int nb) {
    if (smem > (size_t)smem_max) throw DeviceError("time window too long for shared memory");
    std::vector<int> cj, ct;
    for (int w : wins)
      for (int t = 0; t < plan.windows[w].n_traces; t += nb) {
        cj.push_back(w);
        ct.push_back(t);
      }
    L.cta_job.upload(cj, stream);
    L.cta_trace0.upload(ct, stream);
    L.n_cta = (int)cj.size();
    L.nb = nb;
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
    setup_mark("", true);
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

    setup_mark("tables");
    pick_classes();
    X.alloc_pooled(M);
    S0.alloc_pooled(M);
    if (n_generic) S1.alloc_pooled(M);
    Y.alloc_pooled(toff);
    rec_d.alloc_pooled(plan.record_size);
    rec_r.alloc_pooled(plan.record_size);
    scalar.alloc(1);
    dscalar.alloc(1);
    multi = plan.n_problems > 1;
    if (multi) {
      step_dev.alloc(plan.n_problems);
      pmax.alloc(plan.n_problems);
    }
    {
      std::vector<uint8_t> m(plan.record_size, 0);
      for (const auto &mu : plan.mute)
        for (int k = 0; k < mu.second; ++k) m[mu.first + k] = 1;
      mute.upload(m, stream);
    }
    C *Sb[2] = {S0.get(), S1.get()};

    // ---- time-axis jobs (the space-axis intermediate: S0 for the fast
    // space kernels, the generic passes' last buffer otherwise)
    for (int w = 0; w < nw; ++w) {
      const WindowPlan &W = plan.windows[w];
      TimeJob<R> &j = tj[w];
      j.z = (win_class[w] >= 0 ? S0.get() : Sb[(W.D - 1) & 1]) + W.model_off;
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
    setup_mark("buffers");
    if (!classes.empty() || !tgroups.empty()) {
      opt_in_classes();
      upload_twiddles();
      for (auto &c : classes) build_class(*c);
      for (auto &g : tgroups) build_time_group(*g);
    }
    const size_t per_trace_time = 2 * (size_t)Pt_max * sizeof(C) + (size_t)C_max * sizeof(R);
    make_time_launch(time_fwd, per_trace_time, 16, true);
    make_time_launch(time_adj, per_trace_time, 16, true);
    if (wavelets) {
      wav_jobs.upload(wj, stream);
      make_time_launch(wav, 2 * (size_t)C_max * sizeof(C), 8, false);
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

    setup_mark("classes");
    // ---- one-axis windows of other lengths (line kernels)
    build_line_kernels();

    // ---- space-axis passes (generic path)
    maxD = max_d_generic;
    fwd.resize(maxD);
    adj_update.resize(maxD);
    adj_plain.resize(maxD);
    for (int k = 0; k < maxD; ++k) {
      std::vector<AxisJob<R>> jf, ju, jp;
      for (int w = 0; w < nw; ++w) {
        const WindowPlan &W = plan.windows[w];
        if (W.D <= k || win_class[w] >= 0 || win_line[w]) continue;
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
          j.pid = W.problem;
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
          j.pid = W.problem;
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

    setup_mark("line, generic");
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
    data_dev.alloc_pooled(data_size);
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
    G.alloc_pooled(plan.model_size);
    for (auto &cp : classes) {
      FastClass &c = *cp;
      std::vector<PlaneJob<R>> jobs = c.plain_jobs;
      for (size_t i = 0; i < jobs.size(); ++i)
        jobs[i].dst = G.get() + plan.windows[c.win[i]].model_off;
      make_plane_launch(c.pl_adj_plain, jobs, c.planes, c.av().nt, c.av().np, c.av().smem,
                        c.av().fn);
      if (c.tc) build_tc_plain(c);
    }
    for (size_t k = 0; k < pending_plain.size(); ++k) {
      auto jobs = pending_plain[k];
      size_t i = 0;
      for (int w = 0; w < (int)plan.windows.size(); ++w) {
        const WindowPlan &W = plan.windows[w];
        if (W.D <= (int)k || win_class[w] >= 0 || win_line[w]) continue;
        if ((int)k == W.D - 1) jobs[i].dst = G.get() + W.model_off;
        ++i;
      }
      make_axis_launch(adj_plain[k], jobs);
    }
    if (!line_adj_host.empty()) {
      std::vector<LineJob<R>> jobs = line_adj_host;
      size_t i = 0;
      for (int w = 0; w < (int)plan.windows.size(); ++w)
        if (win_line[w]) jobs[i++].dst = G.get() + plan.windows[w].model_off;
      make_line_launch(line_adj_plain, jobs, false);
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
        inverse, epilogue, step, lamb, multi ? step_dev.get() : nullptr, lamb_dev,
        multi ? pmax.get() : scalar.get());
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

  void launch_space_fwd(const FastClass &c) {
    if constexpr (std::is_same<R, float>::value) {
      if (c.tc) {
        if (c.tc_fwd.n_batch == 0) return;
        space_fwd_tc<kTcP, kTcL><<<c.tc_fwd.grid, kTcThreads, TcS::kFwdSmem, stream>>>(
            c.tc_fwd.batches(), tc_fwd_mats(), tc_err.get());
        CK(cudaGetLastError());
        return;
      }
    }
    if (c.pl_fwd.n_batch == 0) return;
    c.fv().fn<<<c.pl_fwd.grid, c.pl_fwd.nt, c.pl_fwd.smem, stream>>>(c.pl_fwd.batches());
    CK(cudaGetLastError());
  }

  void launch_space_adj(const FastClass &c, const PlaneLaunch &L, int epilogue, R step, R lamb,
                        const R *lamb_dev = nullptr) {
    if constexpr (std::is_same<R, float>::value) {
      if (c.tc) {
        const PlaneLaunch &T = &L == &c.pl_adj_plain ? c.tc_adj_plain : c.tc_adj;
        if (T.n_batch == 0) return;
        space_adj_tc<kTcP, kTcL><<<T.grid, kTcThreads, TcS::kAdjSmem, stream>>>(
            T.batches(), tc_adj_mats(), epilogue, step, lamb, multi ? step_dev.get() : nullptr,
            lamb_dev, multi ? pmax.get() : scalar.get(), tc_err.get());
        CK(cudaGetLastError());
        return;
      }
    }
    if (L.n_batch == 0) return;
    c.av().fn<<<L.grid, L.nt, L.smem, stream>>>(L.batches(), epilogue, step, lamb,
                                                 multi ? step_dev.get() : nullptr, lamb_dev,
                                                 multi ? pmax.get() : scalar.get());
    CK(cudaGetLastError());
  }

  // time c2r + taper + overlap-add of every window (fast time groups, then
  // the generic windows)
  void launch_time_fwd() {
    for (const auto &gp : tgroups) {
      const TimeGroup &g = *gp;
      if (!g.tf.n_cta) continue;
      g.fv().fn<<<g.tf.n_cta, kThreads, g.tf.smem, stream>>>(time_jobs.get(), g.tf.cta_job.get(),
                                                             g.tf.cta_trace0.get());
      CK(cudaGetLastError());
    }
    if (time_fwd.n_cta) {
      time_c2r_ola<R><<<time_fwd.n_cta, kThreads, time_fwd.smem, stream>>>(
          time_jobs.get(), time_fwd.cta_job.get(), time_fwd.cta_trace0.get(), time_fwd.nb,
          d_descs.get(), d_tw.get());
      CK(cudaGetLastError());
    }
  }

  // blend adjoint gather + taper + time r2c of every window, from the record
  // (from_record) or from the window traces (after the wavelet correlation)
  void launch_time_adj(const R *record, int from_record) {
    for (const auto &gp : tgroups) {
      const TimeGroup &g = *gp;
      if (!g.ta.n_cta) continue;
      g.av().fn<<<g.ta.n_cta, kThreads, g.ta.smem, stream>>>(
          time_jobs.get(), g.ta.cta_job.get(), g.ta.cta_trace0.get(), record, from_record);
      CK(cudaGetLastError());
    }
    if (time_adj.n_cta) {
      time_r2c<R><<<time_adj.n_cta, kThreads, time_adj.smem, stream>>>(
          time_jobs.get(), time_adj.cta_job.get(), time_adj.cta_trace0.get(), time_adj.nb,
          d_descs.get(), d_tw.get(), record, from_record);
      CK(cudaGetLastError());
    }
  }

  void launch_line_fwd() {
    if (line_fwd.n_cta == 0) return;
    line_dft_fwd<R><<<line_fwd.n_cta, kLineThreads, line_fwd.smem, stream>>>(
        line_fwd.jobs.get(), line_fwd.cta_job.get(), line_fwd.cta_line0.get());
    CK(cudaGetLastError());
  }

  void launch_line_adj(const LineLaunch &Lc, int epilogue, R step, R lamb,
                       const R *lamb_dev = nullptr) {
    if (Lc.n_cta == 0) return;
    line_dft_adj<R><<<Lc.n_cta, kLineThreads, Lc.smem, stream>>>(
        Lc.jobs.get(), Lc.cta_job.get(), Lc.cta_line0.get(), epilogue, step, lamb,
        multi ? step_dev.get() : nullptr, lamb_dev, multi ? pmax.get() : scalar.get());
    CK(cudaGetLastError());
  }

  void launch_space_fwd_all() {
    for (const auto &cp : classes) launch_space_fwd(*cp);
    launch_line_fwd();
    for (size_t k = 0; k < fwd.size(); ++k) launch_axis(fwd[k], 1, kStore, 0, 0);
  }

  void launch_space_adj_all(int epilogue, R step, R lamb, const R *lamb_dev) {
    for (const auto &cp : classes) launch_space_adj(*cp, cp->pl_adj, epilogue, step, lamb, lamb_dev);
    launch_line_adj(line_adj, epilogue, step, lamb, lamb_dev);
    for (size_t k = 0; k < adj_update.size(); ++k)
      launch_axis(adj_update[k], 0, epilogue, step, lamb, lamb_dev);
  }

  // Y = W F X  (window traces of the current model)
  void forward_traces() {
    launch_space_fwd_all();
    launch_time_fwd();
    if (wavelets) launch_wavelet(+1);
  }

  // in place on the window traces (direction +1), or from the record into
  // the window traces (direction -1, prime-factor kernel only)
  void launch_wavelet_fast(int direction, const R *record) {
    if (!wavf.n_cta) return;
    wav_fn<<<wavf.n_cta, kWavThreads, wavf.smem, stream>>>(
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
    launch_time_adj(record, wavelets ? 0 : 1);
  }

  // X <- threshold(X - step * A^H record, lamb); lambda is read from
  // lamb_dev instead when given (graph replays)
  void adjoint_update(const R *record, R step, R lamb, bool track_max,
                      const R *lamb_dev = nullptr) {
    adjoint_time(record);
    launch_space_adj_all(track_max ? kUpdateMax : kUpdateThreshold, step, lamb, lamb_dev);
  }

  // kernels launched by one ISTA iteration (iteration_body)
  int kernels_per_iteration() const {
    int n = 2 * (int)classes.size();  // space passes, forward and adjoint
    for (const auto &gp : tgroups) n += (gp->tf.n_cta ? 1 : 0) + (gp->ta.n_cta ? 1 : 0);
    for (const auto *v : {&fwd, &adj_update})
      for (const AxisLaunch &L : *v) n += L.n_cta ? 1 : 0;
    n += (line_fwd.n_cta ? 1 : 0) + (line_adj.n_cta ? 1 : 0);
    n += (time_fwd.n_cta ? 1 : 0) + (time_adj.n_cta ? 1 : 0);
    n += (g_fwd.n_chunk ? 1 : 0) + 1;  // residual gather, threshold schedule
    if (wavelets) n += wav_fast ? 2 : 3;
    return n;
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

  // table[k * n_problems + p] = lambda of problem p used after iteration
  // k + 1.  The captured graph holds
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
    if (lamb_cur.get() == nullptr) lamb_cur.alloc(plan.n_problems);
    if (lamb_counter.get() == nullptr) lamb_counter.alloc(1);
    CK(cudaMemsetAsync(lamb_counter.get(), 0, sizeof(int), stream));
  }

  void iteration_body(bool want_norm) {
    forward_traces();
    residual(want_norm);
    next_lambda<R><<<1, 256, 0, stream>>>(lamb_table.get(), lamb_counter.get(), lamb_cur.get(),
                                          plan.n_problems);
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

  // FP64 L2 norm of n values on the device
  double device_norm(const R *x, long n) {
    CK(cudaMemsetAsync(dscalar.get(), 0, sizeof(double), stream));
    if (n) record_sumsq<R><<<grid_for(n), kThreads, 0, stream>>>(x, n, dscalar.get());
    CK(cudaGetLastError());
    return std::sqrt(read_dscalar());
  }

  double record_norm(const R *rec) { return device_norm(rec, plan.record_size); }

  // Guard on the FP64 residual norm (no counterpart in the reference, whose
  // get_residual_norm, src/model.c:1343-1384, returns whatever it sums): a
  // NaN or Inf norm ends the call with an error instead of a NaN output.
  static void require_finite(double norm, const char *what) {
    if (!std::isfinite(norm))
      throw std::runtime_error(std::string(what) +
                               " is not finite (NaN or Inf values in the data)");
  }

  static unsigned grid_for(long n) {
    long g = (n + kThreads - 1) / kThreads;
    return (unsigned)std::max<long>(1, std::min<long>(g, 148L * 16));
  }

  // 0.5 / max(1, max blended sum of the space tapers)   (src/model.c:1230-1312)
  R compute_stepsize() {
    NvtxRange nv("agd step size");
    if (n_wtraces) {
      fill_traces<R><<<(unsigned)std::min<long>(n_wtraces, 148L * 64), kThreads, 0, stream>>>(
          Y.get(), space_fold.get(), wt_dst.get(), wt_C.get(), n_wtraces);
      CK(cudaGetLastError());
    }
    launch_gather(g_fwd, Y.get(), rec_r.get(), kGatherSum, false, nullptr, nullptr, 0, nullptr);
    if (multi) {  // one maximum per problem, over its record range
      const int np = plan.n_problems;
      std::vector<R> fac(np, (R)1);
      CK(cudaMemcpyAsync(pmax.get(), fac.data(), np * sizeof(R), cudaMemcpyHostToDevice,
                         stream));
      for (int p = 0; p < np; ++p)
        if (plan.problem_rec_size[p])
          record_max<R><<<grid_for(plan.problem_rec_size[p]), kThreads, 0, stream>>>(
              rec_r.get() + plan.problem_rec_off[p], plan.problem_rec_size[p], pmax.get() + p);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(fac.data(), pmax.get(), np * sizeof(R), cudaMemcpyDeviceToHost,
                         stream));
      CK(cudaStreamSynchronize(stream));
      steps.resize(np);
      for (int p = 0; p < np; ++p) steps[p] = (R)0.5 / fac[p];
      step_dev.upload(steps, stream);
      stepsize = steps[0];
      return stepsize;
    }
    R one = (R)1;
    CK(cudaMemcpyAsync(scalar.get(), &one, sizeof(R), cudaMemcpyHostToDevice, stream));
    if (plan.record_size)
      record_max<R><<<grid_for(plan.record_size), kThreads, 0, stream>>>(
          rec_r.get(), plan.record_size, scalar.get());
    CK(cudaGetLastError());
    const R factor = read_scalar();
    stepsize = (R)0.5 / factor;
    steps.assign(1, stepsize);
    return stepsize;
  }

  void upload_data(R const *const *data) {
    NvtxRange nv("agd upload");
    for (int p = 0; p < plan.n_patches; ++p) {
      const long n = (long)plan.n_traces[p] * plan.n_times[p];
      if (n)
        CK(cudaMemcpyAsync(data_dev.get() + patch_off[p], data[p], n * sizeof(R),
                           cudaMemcpyHostToDevice, stream));
    }
  }

  void download_data(R *const *data) {
    NvtxRange nv("agd download");
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
    NvtxRange nv("agd input blend");
    if (g_input.n_chunk == 0 && plan.record_size) {
      std::vector<Contrib> list;
      for (int p = 0; p < plan.n_patches; ++p) {
        const int nt = plan.n_times[p];
        for (int t = 0; t < plan.n_traces[p]; ++t) {
          const BlendCoord b = !plan.input_coord.empty()
                                   ? plan.input_coord[p][t]
                                   : plan.coord_of(shottimes[p][t], nt, channels[p][t],
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
    NvtxRange nv("agd output");
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

  // Initial step of problems solved together: x = -step_p A^H d per problem,
  // lambda_0 of each problem from its own model range
  std::vector<R> initial_steps() {
    const int np = plan.n_problems;
    if (plan.model_size) CK(cudaMemsetAsync(X.get(), 0, X.bytes(), stream));
    CK(cudaMemsetAsync(pmax.get(), 0, np * sizeof(R), stream));
    adjoint_update(rec_d.get(), stepsize, (R)0, true);
    std::vector<R> m(np);
    CK(cudaMemcpyAsync(m.data(), pmax.get(), np * sizeof(R), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    for (R &v : m) v = (R)std::sqrt(v);
    return m;
  }

  // Initial step, first threshold and the device schedule of every problem:
  // returns the table loaded on the device, rows x n_problems (the schedule
  // repeated when rows exceeds n_its - 1).
  std::vector<R> start_schedule(R initial_factor, int n_its, int rows) {
    NvtxRange nv("agd initial step");
    const int np = plan.n_problems;
    const std::vector<R> lamb0 = multi ? initial_steps() : std::vector<R>{initial_step()};
    std::vector<R> table((size_t)rows * np);
    for (int p = 0; p < np; ++p) {
      R first = 0;
      const std::vector<R> t = schedule_table(lamb0[p], initial_factor, n_its, &first);
      if (!multi) {
        threshold_model(first);
      } else if (plan.problem_model_size[p]) {
        model_threshold<R><<<grid_for(plan.problem_model_size[p]), kThreads, 0, stream>>>(
            X.get() + plan.problem_model_off[p], plan.problem_model_size[p], first);
        CK(cudaGetLastError());
      }
      for (int r = 0; r < rows; ++r) table[(size_t)r * np + p] = t[r % t.size()];
    }
    load_schedule(table);
    return table;
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
    solve_range(initial_factor, n_its, 0, n_its, print_freq, nullptr, nullptr);
  }

  // Iterations [begin, end) of the n_its schedule, for checkpoint / resume
  // and warm starts.  The whole solver state is the model and the iteration
  // number: the thresholds follow from lambda_0 of the initial step, which
  // is recomputed (it depends on the data only).  begin = 0 starts from the
  // initial step like solve(); begin > 0 starts from model_in, the model
  // after iteration begin - 1 (reference layout).  model_out, if given,
  // receives the model after iteration end - 1, and the patch data receive
  // that model's output.
  void solve_range(R initial_factor, int n_its, int begin, int end, int print_freq,
                   const R *model_in, R *model_out) {
    NvtxRange nv("agd solve");
    // the blended input's norm is the residual of the zero model
    const double r0 = record_norm(rec_d.get());
    require_finite(r0, "the norm of the blended input data");
    start_schedule(initial_factor, n_its, std::max(1, n_its - 1));
    int first = 1;
    if (begin > 0) {
      model_from_ref(model_in);
      const int counter = begin - 1;  // iteration `begin` uses table row begin - 1
      CK(cudaMemcpyAsync(lamb_counter.get(), &counter, sizeof(int), cudaMemcpyHostToDevice,
                         stream));
      CK(cudaStreamSynchronize(stream));
      first = begin;
    }
    if (print_freq > 0) {
      if (begin == 0) std::printf("Iteration 0 Residual %f\n", r0);
      for (int it = first; it < end; ++it) {
        const bool print_residual = it % print_freq == 0;
        iteration_body(print_residual);
        if (print_residual) {
          const double r = std::sqrt(read_dscalar());
          require_finite(r, "the residual norm");
          std::printf("Iteration %d Residual %f\n", it, r);
        }
      }
    } else if (end > first) {
      capture_iteration();
      for (int it = first; it < end; ++it) replay_iteration();
    }
    if (model_out != nullptr) model_to_ref(X.get(), model_out);
    output();
    check_tc_error();
    require_finite(device_norm(data_dev.get(), data_size), "the norm of the deblended output");
  }

  // ------------------------------------------------------------ warm start
  //
  // A model x0 whose FK operator reproduces an estimate v of the deblended
  // data: per window, x0_w = r2c(taper_w * v / fold2) / (N scaler) with
  // fold2 = sum over windows of taper_w^2 (space and time tapers at each
  // data sample).  Then F x0 = sum_w taper_w^2 v / fold2 = v exactly, since
  // within a zero-padded window c2r(r2c(u)) = N u.  The adjoint kernels
  // compute r2c(taper * .) * scaler with bins 1..(Pt-1)/2 doubled
  // (src/fk.c:375-452); with N scaler^2 = 1, x0 is the adjoint of v / fold2
  // with those bins halved.  With a source wavelet, v is first correlated
  // with it (the wavelet operator is all-pass: its adjoint inverts it on
  // live traces).  No counterpart in the reference, which starts from zero.
  DevArray<R> inv_fold2;  // 1 / fold2 per patch data sample
  DevArray<R> est_aux, est_tmp;  // the input and an estimate along another source axis
  // fold2 is at least 0.5^(D+1) (D space axes) on the samples the model
  // represents; with a source wavelet the last samples of a trace lie in the
  // tapered tail of the last time window, where fold2 falls towards 0: the
  // floor keeps 1 / fold2 bounded there (such samples are only approached).
  static constexpr R kFoldFloor = (R)0.05;

  void halve_model_interior() {
    for (const WindowPlan &W : plan.windows)
      if (W.model_size)
        halve_interior_bins<R><<<grid_for(W.model_size), kThreads, 0, stream>>>(
            X.get() + W.model_off, W.T, W.F, W.plane(), (W.Pt - 1) / 2);
    CK(cudaGetLastError());
  }

  // X <- adjoint of the window traces Y (no wavelet), bins halved
  void model_from_traces() {
    launch_time_adj(nullptr, 0);
    launch_space_adj_all(kStore, (R)0, (R)0, nullptr);
    halve_model_interior();
  }

  void scatter_to_traces(const R *data, const R *scale) {
    if (Y.get() != nullptr) CK(cudaMemsetAsync(Y.get(), 0, Y.bytes(), stream));
    if (out_traces)
      traces_from_data<R><<<(unsigned)out_traces, kThreads, 0, stream>>>(
          out_ptr.get(), out_src.get(), out_dst.get(), out_nt.get(), data, scale, Y.get());
    CK(cudaGetLastError());
  }

  void ensure_fold2() {
    if (inv_fold2.get() != nullptr || data_size == 0) return;
    inv_fold2.alloc(data_size);
    scatter_to_traces(nullptr, nullptr);  // ones on every data sample
    model_from_traces();
    launch_space_fwd_all();
    launch_time_fwd();
    if (out_traces)
      output_gather<R><<<(unsigned)out_traces, kThreads, 0, stream>>>(
          out_ptr.get(), out_src.get(), out_dst.get(), out_nt.get(), Y.get(), inv_fold2.get());
    reciprocal_floor<R><<<grid_for(data_size), kThreads, 0, stream>>>(inv_fold2.get(),
                                                                      data_size, kFoldFloor);
    CK(cudaGetLastError());
  }

  // X <- the warm model of the estimate held in data_dev
  void warm_model() {
    ensure_fold2();
    scatter_to_traces(data_dev.get(), inv_fold2.get());
    if (wavelets) launch_wavelet(-1);
    model_from_traces();
  }

  // The solver from a warm model: the initial step and the thresholds of
  // the n_its schedule as agd_gpu_solve computes them from the blended
  // input in rec_d, then X <- warm_model(estimate) and iterations [begin,
  // n_its) (begin >= 1: the schedule continues from iteration begin).
  void solve_warm(R initial_factor, int n_its, int begin, R const *const *estimate,
                  int print_freq) {
    const double r0 = record_norm(rec_d.get());
    require_finite(r0, "the norm of the blended input data");
    start_schedule(initial_factor, n_its, std::max(1, n_its - 1));
    upload_data(estimate);
    warm_iterations(n_its, begin, print_freq);
  }

  // data_dev holds the estimate; the schedule is loaded: X <- warm model,
  // then iterations [begin, n_its) and the output
  void warm_iterations(int n_its, int begin, int print_freq) {
    NvtxRange nv("agd warm iterations");
    require_finite(device_norm(data_dev.get(), data_size), "the norm of the estimate");
    warm_model();
    const int counter = begin - 1;  // iteration `begin` uses table row begin - 1
    CK(cudaMemcpyAsync(lamb_counter.get(), &counter, sizeof(int), cudaMemcpyHostToDevice,
                       stream));
    if (print_freq > 0) {
      for (int it = begin; it < n_its; ++it) {
        const bool print_residual = it % print_freq == 0;
        iteration_body(print_residual);
        if (print_residual) {
          const double r = std::sqrt(read_dscalar());
          require_finite(r, "the residual norm");
          std::printf("Iteration %d Residual %f\n", it, r);
        }
      }
    } else if (n_its > begin) {
      capture_iteration();
      for (int it = begin; it < n_its; ++it) replay_iteration();
    }
    output();
    check_tc_error();
    require_finite(device_norm(data_dev.get(), data_size), "the norm of the deblended output");
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
