// The C API of the library (include/agdeblend.h, include/agdeblend_gpu.h)
// over the device engine (engine.cuh).  Built twice: float (libagdeblend.so)
// and, with -DAGD_DOUBLE, double (libagdeblend_double.so).
#include "engine.cuh"

// ==================================================================== C API

struct agd_gpu_problem {
  std::unique_ptr<agd::EngineR> eng;
  std::vector<std::vector<int>> shapes;  // per patch: space sizes..., time samples
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

// A problem handle over a plan of one or more problems (args in problem
// order; their patches follow one another in the plan).
int create_from_plan(const std::vector<agd::ProblemArgs> &args, agd::Plan &&plan,
                     agd_gpu_problem **out) {
  *out = nullptr;
  auto *pb = new agd_gpu_problem();
  try {
    int gp = 0;
    for (const agd::ProblemArgs &a : args)
      for (int p = 0; p < a.n_patches; ++p, ++gp) {
        const int n = plan.n_traces[gp];
        pb->shottimes.emplace_back(a.shottimes[p], a.shottimes[p] + n);
        pb->shapes.emplace_back(a.shapes[p], a.shapes[p] + a.n_dims[a.volumes[p]]);
        pb->channels.emplace_back(a.channels[p], a.channels[p] + n);
        pb->trace_types.emplace_back(a.trace_types[p], a.trace_types[p] + n);
      }
    for (int p = 0; p < gp; ++p) {
      pb->st_p.push_back(pb->shottimes[p].data());
      pb->ch_p.push_back(pb->channels[p].data());
      pb->tt_p.push_back(pb->trace_types[p].data());
    }
    pb->eng.reset(new agd::EngineR(std::move(plan)));
    agd::setup_mark("blend, rest");
    pb->eng->compute_stepsize();
    agd::setup_mark("step size");
  } catch (const std::exception &e) {
    std::fprintf(stderr, "ERROR: %s\n", e.what());
    delete pb;
    return 1;
  }
  *out = pb;
  return 0;
}

// Phase times of an agd_deblend call on stderr when AGD_GPU_TIMING=1: host
// wall clock between marks, each mark after a device synchronisation.
struct PhaseTimer {
  bool on = false;
  std::chrono::steady_clock::time_point t;
  PhaseTimer() {
    const char *env = std::getenv("AGD_GPU_TIMING");
    on = env != nullptr && env[0] == '1';
    if (on) t = std::chrono::steady_clock::now();
  }
  void mark(const char *phase) {
    if (!on) return;
    cudaDeviceSynchronize();
    const auto n = std::chrono::steady_clock::now();
    std::fprintf(stderr, "agd timing: %-12s %8.2f ms\n", phase,
                 std::chrono::duration<double, std::milli>(n - t).count());
    t = n;
  }
};

int create_problem(const agd::ProblemArgs &a, agd_gpu_problem **out) {
  *out = nullptr;
  agd::Plan plan;
  if (agd::build_plan(a, plan)) return 1;
  return create_from_plan({a}, std::move(plan), out);
}

// Arguments of problem q of a batch call (each argument is an array over
// the problems of agd_deblend's argument).
agd::ProblemArgs batch_args(int q, int const *n_patches, int const *const *volumes,
                            int const *const *n_dims, int const *const *const *window_shapes,
                            int const *const *const *coords, int const *const *const *shapes,
                            long int const *const *const *shottimes,
                            int const *const *const *channels,
                            enum AGDTraceType const *const *const *trace_types,
                            int const *const *wavelet_lengths,
                            int const *const *const *wavelet_idxs,
                            AGD_TYPE const *const *const *wavelets) {
  return make_args(n_patches[q], volumes[q], n_dims[q], window_shapes[q], coords[q], shapes[q],
                   shottimes[q], channels[q], trace_types[q],
                   wavelet_lengths ? wavelet_lengths[q] : nullptr,
                   wavelet_idxs ? wavelet_idxs[q] : nullptr, wavelets ? wavelets[q] : nullptr);
}

int create_batch(const std::vector<agd::ProblemArgs> &args, agd_gpu_problem **out) {
  *out = nullptr;
  agd::Plan plan;
  if (agd::build_batch_plan(args, plan)) return 1;
  return create_from_plan(args, std::move(plan), out);
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
  long n_fast = 0;
  for (int c : e.win_class) n_fast += c >= 0 ? 1 : 0;
  const long nw = (long)e.plan.windows.size();
  info[8] = (nw > 0 && n_fast == nw) ? 1 : (n_fast > 0 ? 2 : 0);
  info[9] = e.wav_fast ? 1 : 0;
  info[10] = e.classes.empty() ? -1 : e.classes[0]->fwd_pick;
  info[11] = e.classes.empty() ? -1 : e.classes[0]->adj_pick;
  info[12] = e.classes.empty() ? 0 : (long)e.classes[0]->fwd_vars.size();
  info[13] = e.classes.empty() ? 0 : (long)e.classes[0]->adj_vars.size();
  info[14] = e.kernels_per_iteration();
  info[15] = (long)e.classes.size();
  info[16] = n_fast;
  info[17] = e.tgroups.empty() ? -1 : e.tgroups[0]->fwd_pick;
  info[18] = e.tgroups.empty() ? -1 : e.tgroups[0]->adj_pick;
  info[19] = e.tgroups.empty() ? 0 : (long)e.tgroups[0]->fwd_vars.size();
  info[20] = e.wav_fast ? e.wav_pick : -1;
  info[21] = e.wav_candidates;
  long n_line = 0;
  for (char c : e.win_line) n_line += c ? 1 : 0;
  info[22] = n_line;
  return 0;
}

int agd_gpu_problem_kernels(agd_gpu_problem const *pb, char *buf, int len) {
  if (pb == nullptr || buf == nullptr || len <= 0) return 1;
  const agd::EngineR &e = *pb->eng;
  const bool sc = !e.classes.empty(), tg = !e.tgroups.empty();
  const int n = std::snprintf(
      buf, (size_t)len, "space_fwd=%s space_adj=%s time_fwd=%s time_adj=%s wavelet=%s",
      !sc ? "axis_pass" : (e.classes[0]->tc ? "space_fwd_tc" : e.classes[0]->fv().name),
      !sc ? "axis_pass" : (e.classes[0]->tc ? "space_adj_tc" : e.classes[0]->av().name),
      tg ? e.tgroups[0]->fv().name : "time_c2r_ola", tg ? e.tgroups[0]->av().name : "time_r2c",
      !e.wavelets ? "none" : (e.wav_fast ? "wavelet_fast" : "wavelet_apply"));
  return n < 0 || n >= len ? 1 : 0;
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
    e.check_tc_error();
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
    for (const auto &cp : e.classes) e.launch_space_adj(*cp, cp->pl_adj_plain, agd::kStore, 0, 0);
    for (size_t k = 0; k < e.adj_plain.size(); ++k)
      e.launch_axis(e.adj_plain[k], 0, agd::kStore, 0, 0);
    e.launch_line_adj(e.line_adj_plain, agd::kStore, 0, 0);
    e.model_to_ref(e.G.get(), model);
    e.check_tc_error();
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

int agd_gpu_solve_range(agd_gpu_problem *pb, AGD_TYPE initial_factor, int n_its, int it_begin,
                        int it_end, int print_freq, AGD_TYPE const *model_in,
                        AGD_TYPE *model_out, AGD_TYPE *const *data) {
  if (pb == nullptr || data == nullptr) return 1;
  if (n_its <= 0 || it_begin < 0 || it_end < it_begin || it_end > n_its ||
      (it_begin > 0 && model_in == nullptr)) {
    std::fprintf(stderr,
                 "ERROR: need 0 <= it_begin <= it_end <= n_its, n_its > 0, and a model to "
                 "resume from when it_begin > 0\nERROR in agd_gpu_solve_range\n");
    return 1;
  }
  return guarded("agd_gpu_solve_range", [&] {
    agd::EngineR &e = *pb->eng;
    e.upload_data(data);
    pb->input_blend();
    e.solve_range(initial_factor, n_its, it_begin, it_end, print_freq, model_in, model_out);
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
    // thresholds for every replay: the schedule, repeated if the run is
    // longer than n_its - 1 iterations
    const std::vector<AGD_TYPE> table =
        e.start_schedule(initial_factor, n_its, warmup + steps + 2);
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
    e.adjoint_update(e.rec_r.get(), e.stepsize,
                     table[(size_t)(warmup + steps) * e.plan.n_problems], false);
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
    mark();
    e.launch_space_fwd_all();
    mark();
    e.launch_time_fwd();
    mark();
    if (e.wavelets) e.launch_wavelet(+1);
    mark();
    e.residual(false);
    mark();
    e.adjoint_time(e.rec_r.get());
    mark();
    e.launch_space_adj_all(agd::kUpdateThreshold, e.stepsize, lamb, nullptr);
    mark();
    agd::CK(cudaEventSynchronize(ev.back()));
    auto dt = [&](int a, int b) {
      float v = 0;
      agd::CK(cudaEventElapsedTime(&v, ev[a], ev[b]));
      return (double)v;
    };
    // [0] space passes of the forward operator (all windows), [1] time c2r +
    // overlap-add, [2] wavelet convolution, [3] blend gather + residual,
    // [4] adjoint time (incl. blend gather and wavelet correlation),
    // [5] adjoint space passes incl. the update; [6] = [0], [10] = [5] and
    // [14] = 1 (the space phases counted as one pass)
    for (int k = 0; k < 6; ++k) ms[k] = dt(k, k + 1);
    ms[6] = ms[0];
    ms[10] = ms[5];
    ms[14] = 1;
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
  PhaseTimer timer;
  timer.mark("validate");
  agd_gpu_problem *pb = nullptr;
  agd::Plan plan;
  if (agd::build_plan(a, plan)) {
    std::fprintf(stderr, "ERROR in agd_deblend\n");
    return 1;
  }
  timer.mark("plan");
  if (create_from_plan({a}, std::move(plan), &pb)) {
    std::fprintf(stderr, "ERROR in agd_deblend\n");
    return 1;
  }
  timer.mark("set-up");
  if (pb->eng->stepsize > (AGD_TYPE)0.3)
    std::printf("WARNING: There does not appear to be any overlap between shots\n");
  const int rc = guarded("agd_deblend", [&] {
    agd::EngineR &e = *pb->eng;
    e.upload_data(data);
    timer.mark("upload");
    pb->input_blend();
    timer.mark("input blend");
    e.solve(initial_factor, n_its, print_freq);
    timer.mark("solve");
    e.download_data(data);
    timer.mark("download");
    return 0;
  });
  delete pb;
  timer.mark("teardown");
  return rc;
}

int agd_gpu_batch_create(int n_problems, int const *n_patches, int const *const *volumes,
                         int const *const *n_dims, int const *const *const *window_shapes,
                         int const *const *const *coords, int const *const *const *shapes,
                         long int const *const *const *shottimes,
                         int const *const *const *channels,
                         enum AGDTraceType const *const *const *trace_types,
                         int const *const *wavelet_lengths, int const *const *const *wavelet_idxs,
                         AGD_TYPE const *const *const *wavelets, agd_gpu_problem **problem) {
  if (problem == nullptr || n_problems <= 0 || n_patches == nullptr || volumes == nullptr ||
      n_dims == nullptr || window_shapes == nullptr || coords == nullptr || shapes == nullptr ||
      shottimes == nullptr || channels == nullptr || trace_types == nullptr) {
    std::fprintf(stderr, "ERROR: invalid batch arguments\nERROR in agd_gpu_batch_create\n");
    return 1;
  }
  std::vector<agd::ProblemArgs> args;
  for (int q = 0; q < n_problems; ++q) {
    args.push_back(batch_args(q, n_patches, volumes, n_dims, window_shapes, coords, shapes,
                              shottimes, channels, trace_types, wavelet_lengths, wavelet_idxs,
                              wavelets));
    std::vector<AGD_TYPE *> dummy(n_patches[q] > 0 ? n_patches[q] : 1, (AGD_TYPE *)1);
    if (agd::check_deblend_inputs(args.back(), (AGD_TYPE)1, 1, dummy.data())) {
      std::fprintf(stderr, "ERROR in problem %d of agd_gpu_batch_create\n", q);
      return 1;
    }
  }
  return create_batch(args, problem);
}

void agd_gpu_release_cache(void) { agd::DevicePool::release_all(); }

int agd_gpu_solve_warm(agd_gpu_problem *pb, AGD_TYPE initial_factor, int n_its, int it_begin,
                       int print_freq, AGD_TYPE const *const *estimate, AGD_TYPE *const *data) {
  if (pb == nullptr || data == nullptr || estimate == nullptr) return 1;
  if (n_its <= 0 || it_begin < 1 || it_begin > n_its) {
    std::fprintf(stderr,
                 "ERROR: need n_its > 0 and 1 <= it_begin <= n_its\nERROR in agd_gpu_solve_warm\n");
    return 1;
  }
  return guarded("agd_gpu_solve_warm", [&] {
    agd::EngineR &e = *pb->eng;
    e.upload_data(data);
    pb->input_blend();
    e.solve_warm(initial_factor, n_its, it_begin, estimate, print_freq);
    e.download_data(data);
    return 0;
  });
}

namespace {

// Images for the network: every line of a patch along its trace axis (the
// space axis along which the shot times change least, but change: receiver
// gathers of consecutive shots) is one image of (traces x time samples).
// Source axes of a patch: the space axes along which the shot times change,
// by increasing mean |shot-time step| (the first: receiver gathers of
// consecutive shots).  Lines along any of them see the blending noise of
// other shots as incoherent.
std::vector<int> source_axes(const agd_gpu_problem &pb, size_t p) {
  const std::vector<int> &sh = pb.shapes[p];
  const int D = (int)sh.size() - 1;
  std::vector<long> stride(sh.size(), 1);
  for (int d = (int)sh.size() - 2; d >= 0; --d) stride[d] = stride[d + 1] * sh[d + 1];
  std::vector<std::pair<double, int>> found;
  for (int d = 0; d < D; ++d) {
    if (sh[d] < 2) continue;
    const long st = stride[d] / sh[D];  // trace stride of axis d
    double sum = 0;
    long cnt = 0;
    const long n_tr = (long)pb.shottimes[p].size();
    for (long t = 0; t < n_tr; ++t)
      if ((t / st) % sh[d] + 1 < sh[d]) {
        sum += std::fabs((double)(pb.shottimes[p][t + st] - pb.shottimes[p][t]));
        ++cnt;
      }
    const double m = cnt ? sum / cnt : 0;
    if (m > 0) found.emplace_back(m, d);
  }
  std::sort(found.begin(), found.end());
  std::vector<int> axes;
  for (const auto &f : found) axes.push_back(f.second);
  if (axes.empty()) axes.push_back(D - 1);
  return axes;
}

// Lines along source axis `which` of every patch (source axes in order of
// their shot-time step, smallest first; the first one where a patch has
// fewer), grouped by shape.  A network with in_ch = 2 k + 1 > 1 input
// channels gets the lines along each patch's slowest source axis instead
// (`which` ignored), each with the lines at offsets -1, +1, ..., -k, +k
// (clamped at the patch edge) along the next faster source axis - the shots
// fired just before and after - or itself where the patch has one source
// axis.
std::vector<agd::nn::ImageGroup> image_groups(const agd_gpu_problem &pb, size_t which,
                                              int in_ch) {
  std::vector<agd::nn::ImageGroup> groups;
  const agd::EngineR &e = *pb.eng;
  for (size_t p = 0; p < pb.shapes.size(); ++p) {
    const std::vector<int> &sh = pb.shapes[p];
    const int D = (int)sh.size() - 1;
    std::vector<long> stride(sh.size(), 1);
    for (int d = (int)sh.size() - 2; d >= 0; --d) stride[d] = stride[d + 1] * sh[d + 1];
    const std::vector<int> axes = source_axes(pb, p);
    const size_t ai = in_ch > 1 ? axes.size() - 1 : (which < axes.size() ? which : 0);
    const int axis = axes[ai];
    const int nbr_axis = in_ch > 1 && ai > 0 ? axes[ai - 1] : -1;
    agd::nn::ImageGroup *g = nullptr;
    for (auto &x : groups)
      if (x.rows == sh[axis] && x.cols == sh[D] && x.row_stride == stride[axis]) g = &x;
    if (g == nullptr) {
      groups.push_back(agd::nn::ImageGroup{});
      g = &groups.back();
      g->rows = sh[axis];
      g->cols = sh[D];
      g->row_stride = stride[axis];
    }
    // every combination of the other space indices
    const long n_img = stride[0] * sh[0] / ((long)sh[axis] * sh[D]);
    for (long i = 0; i < n_img; ++i) {
      long rem = i, off = 0;
      int j = 0;  // index along the neighbour axis
      for (int d = D - 1; d >= 0; --d) {
        if (d == axis) continue;
        const int idx = (int)(rem % sh[d]);
        if (d == nbr_axis) j = idx;
        off += idx * stride[d];
        rem /= sh[d];
      }
      const long b = e.patch_off[p] + off;
      g->base.push_back(b);
      for (int c = 1; c < in_ch; ++c) {
        if (nbr_axis < 0) {
          g->nbr.push_back(b);
          continue;
        }
        const int o = (c + 1) / 2 * (c % 2 ? -1 : 1);  // -1, +1, -2, +2, ...
        const int jn = std::min(std::max(j + o, 0), sh[nbr_axis] - 1);
        g->nbr.push_back(b + (long)(jn - j) * stride[nbr_axis]);
      }
    }
  }
  return groups;
}

size_t max_source_axes(const agd_gpu_problem &pb) {
  size_t n = 1;
  for (size_t p = 0; p < pb.shapes.size(); ++p) n = std::max(n, source_axes(pb, p).size());
  return n;
}

}  // namespace

int agd_gpu_solve_learned(agd_gpu_problem *pb, agd_nn *net, AGD_TYPE initial_factor, int n_its,
                          int it_begin, int print_freq, AGD_TYPE *const *data) {
  if (pb == nullptr || net == nullptr || data == nullptr) return 1;
  if (n_its <= 0 || it_begin < 1 || it_begin > n_its) {
    std::fprintf(stderr,
                 "ERROR: need n_its > 0 and 1 <= it_begin <= n_its\nERROR in agd_gpu_solve_learned\n");
    return 1;
  }
  return guarded("agd_gpu_solve_learned", [&] {
#ifdef AGD_DOUBLE
    throw std::runtime_error("the warm-start network serves the float library only");
#else
    agd::EngineR &e = *pb->eng;
    PhaseTimer timer;
    e.upload_data(data);
    pb->input_blend();
    timer.mark("upload+blend");
    const double r0 = e.record_norm(e.rec_d.get());
    agd::EngineR::require_finite(r0, "the norm of the blended input data");
    e.start_schedule(initial_factor, n_its, std::max(1, n_its - 1));
    timer.mark("initial step");
    // the pseudo-deblended input in data_dev becomes the network's estimate:
    // the mean of its estimates from the lines along every source axis, or
    // for a multi-channel network its estimate from the lines along the
    // slowest source axis with their neighbours
    const int in_ch = agd::nn::input_channels(net);
    const size_t n_axes = in_ch > 1 ? 1 : max_source_axes(*pb);
    // the input is read from an untouched copy when the estimate is written
    // over it while other images still read it (neighbour channels, more
    // axes); kept between calls: allocating half a gigabyte per call costs
    // more than the estimate
    const bool copy = n_axes > 1 || in_ch > 1;
    if (copy && e.est_aux.bytes() != (size_t)e.data_size * sizeof(float))
      e.est_aux.alloc(e.data_size);
    if (n_axes > 1 && e.est_tmp.bytes() != (size_t)e.data_size * sizeof(float))
      e.est_tmp.alloc(e.data_size);
    if (copy)
      agd::CK(cudaMemcpyAsync(e.est_aux.get(), e.data_dev.get(), e.data_size * sizeof(float),
                              cudaMemcpyDeviceToDevice, e.stream));
    const float *src = copy ? e.est_aux.get() : e.data_dev.get();
    agd::nn::estimate_images(net, src, e.data_dev.get(), image_groups(*pb, 0, in_ch), e.stream);
    for (size_t a = 1; a < n_axes; ++a) {
      // every sample of est_tmp is written (each trace lies on one line)
      agd::nn::estimate_images(net, src, e.est_tmp.get(), image_groups(*pb, a, in_ch),
                               e.stream);
      agd::mean_into<float><<<agd::EngineR::grid_for(e.data_size), agd::kThreads, 0,
                              e.stream>>>(e.data_dev.get(), e.est_tmp.get(), e.data_size,
                                          (float)a / (float)(a + 1));
      agd::CK(cudaGetLastError());
      agd::CK(cudaStreamSynchronize(e.stream));
    }
    timer.mark("estimate");
    e.warm_iterations(n_its, it_begin, print_freq);
    timer.mark("warm model+its");
    e.download_data(data);
    timer.mark("download");
#endif
    return 0;
  });
}

int agd_gpu_warm_model(agd_gpu_problem *pb, AGD_TYPE const *const *estimate, AGD_TYPE *model) {
  if (pb == nullptr || estimate == nullptr || model == nullptr) return 1;
  return guarded("agd_gpu_warm_model", [&] {
    agd::EngineR &e = *pb->eng;
    e.upload_data(estimate);
    e.warm_model();
    e.model_to_ref(e.X.get(), model);
    e.check_tc_error();
    return 0;
  });
}

int agd_gpu_problem_set_precision(agd_gpu_problem *pb, int precision, long int *tc_windows) {
  if (pb == nullptr) return 1;
  return guarded("agd_gpu_problem_set_precision", [&] {
    pb->eng->set_precision(precision);
    if (tc_windows != nullptr) *tc_windows = pb->eng->tc_windows;
    return 0;
  });
}

int agd_gpu_problem_steps(agd_gpu_problem const *pb, AGD_TYPE *steps) {
  if (pb == nullptr || steps == nullptr) return 1;
  const agd::EngineR &e = *pb->eng;
  for (size_t q = 0; q < e.steps.size(); ++q) steps[q] = e.steps[q];
  return 0;
}

int agd_deblend_batch(int n_problems, int const *n_patches, int const *const *volumes,
                      int const *const *n_dims, int const *const *const *window_shapes,
                      int const *const *const *coords, int const *const *const *shapes,
                      long int const *const *const *shottimes, int const *const *const *channels,
                      enum AGDTraceType const *const *const *trace_types,
                      int const *const *wavelet_lengths, int const *const *const *wavelet_idxs,
                      AGD_TYPE const *const *const *wavelets, AGD_TYPE initial_factor,
                      int n_its, AGD_TYPE *const *const *data) {
  if (n_problems <= 0 || n_patches == nullptr || data == nullptr) {
    std::fprintf(stderr, "ERROR: invalid batch arguments\nERROR in agd_deblend_batch\n");
    return 1;
  }
  PhaseTimer timer;
  std::vector<AGD_TYPE *> all_data;
  std::vector<agd::ProblemArgs> args;
  for (int q = 0; q < n_problems; ++q) {
    if (volumes == nullptr || n_dims == nullptr || window_shapes == nullptr ||
        coords == nullptr || shapes == nullptr || shottimes == nullptr || channels == nullptr ||
        trace_types == nullptr) {
      std::fprintf(stderr, "ERROR: invalid batch arguments\nERROR in agd_deblend_batch\n");
      return 1;
    }
    args.push_back(batch_args(q, n_patches, volumes, n_dims, window_shapes, coords, shapes,
                              shottimes, channels, trace_types, wavelet_lengths, wavelet_idxs,
                              wavelets));
    if (data[q] == nullptr ||
        agd::check_deblend_inputs(args.back(), initial_factor, n_its, data[q])) {
      std::fprintf(stderr, "ERROR in problem %d of agd_deblend_batch\n", q);
      return 1;
    }
    for (int p = 0; p < n_patches[q]; ++p) all_data.push_back(data[q][p]);
  }
  timer.mark("validate");
  agd_gpu_problem *pb = nullptr;
  agd::Plan plan;
  if (agd::build_batch_plan(args, plan)) {
    std::fprintf(stderr, "ERROR in agd_deblend_batch\n");
    return 1;
  }
  timer.mark("plan");
  if (create_from_plan(args, std::move(plan), &pb)) {
    std::fprintf(stderr, "ERROR in agd_deblend_batch\n");
    return 1;
  }
  timer.mark("set-up");
  const int rc = guarded("agd_deblend_batch", [&] {
    agd::EngineR &e = *pb->eng;
    e.upload_data(all_data.data());
    timer.mark("upload");
    pb->input_blend();
    timer.mark("input blend");
    e.solve(initial_factor, n_its, 0);
    timer.mark("solve");
    e.download_data(all_data.data());
    timer.mark("download");
    return 0;
  });
  delete pb;
  timer.mark("teardown");
  return rc;
}

}  // extern "C"
