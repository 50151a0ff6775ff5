// Host-side planning for the deblending path: input validation, windows,
// blend geometry and operator constants, computed once per agd_deblend /
// agd_blend call and flattened into device tables by engine.cu.
//
// The planning reproduces the reference's set_model (src/model.c:932-1065),
// set_blend_config (src/blend.c:629-691) and check_deblend_inputs
// (src/agdeblend.c:263-509) result for result; each function cites the part
// it mirrors.
#pragma once

#include <complex>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "agdeblend.h"

namespace agd {

using real = AGD_TYPE;

constexpr int kMaxSpaceDims = AGD_MAX_N_COORDS;

struct Interval {
  long start;
  long stop;
};

// Where one trace lands in the flat blended record (all (channel, interval)
// segments concatenated channel-major).  rec < 0: the trace is not blended.
struct BlendCoord {
  long rec;
  int trace_start;
  int n;
};

// One space window with its FK operator constants (src/fk.c:75-169).
struct WindowPlan {
  int patch = 0;
  int problem = 0;             // independent problem (batches of problems)
  int D = 0;                   // number of space dimensions
  int coords[kMaxSpaceDims] = {0};
  int L[kMaxSpaceDims] = {0};  // window length per space dim
  int P[kMaxSpaceDims] = {0};  // padded length per space dim
  int use_taper[2 * kMaxSpaceDims + 2] = {0};
  int Lt = 0, Pt = 0, F = 0, h = 0, T = 0;
  int n_fk = 0;  // time samples produced by the FK operator
  int C = 0;     // trace capacity (n_times_conv)
  int n_traces = 0;
  real scaler = 0;
  std::vector<real> taper[kMaxSpaceDims + 1];  // [D] is the time taper
  std::vector<int> trace_index;                // patch trace of each window trace
  std::vector<BlendCoord> blend;
  std::vector<int> wavelet_src;                // per trace, -1 = not convolved
  bool has_wavelet_traces = false;
  long model_off = 0;   // complex offset of the window's model
  long model_size = 0;  // T * F * prod(P)

  long plane() const {
    long n = 1;
    for (int d = 0; d < D; ++d) n *= P[d];
    return n;
  }
};

struct Plan {
  int n_patches = 0;
  std::vector<int> volume;     // per patch
  std::vector<int> n_space;    // per patch: space dims
  std::vector<std::vector<int>> shape;  // per patch, space..., time
  std::vector<int> n_traces;   // per patch
  std::vector<int> n_times;    // per patch (data)
  std::vector<int> n_fk, conv; // per patch
  std::vector<int> lt;         // per patch: time window length

  // blend configuration
  std::vector<int> channel_values;
  std::vector<std::vector<Interval>> intervals;  // per channel
  std::vector<std::vector<long>> seg_off;        // per channel, per interval
  long record_size = 0;
  // lookups built with the configuration: channel value -> index; per
  // channel the intervals sorted by start (start, position in `intervals`)
  // and the longest interval, which bounds how far back a search by start
  // must look
  std::unordered_map<int, int> channel_lookup;
  std::vector<std::vector<std::pair<long, int>>> by_start;
  std::vector<long> max_len;
  std::vector<std::pair<long, int>> mute;        // (flat start, n)

  std::vector<WindowPlan> windows;
  long model_size = 0;  // complex elements over all windows

  // wavelet source configurations (src/wavelet.c:19-70): phase-only spectra
  std::vector<int> wavelet_n;                      // transform length
  std::vector<std::vector<std::complex<double>>> spectra;

  // Independent problems planned together (build_batch_plan): each keeps
  // its record range, model range, step size and threshold schedule.  A
  // single agd_deblend problem has n_problems = 1 and empty tables.
  int n_problems = 1;
  std::vector<long> problem_rec_off, problem_rec_size;
  std::vector<long> problem_model_off, problem_model_size;
  // blend coordinates of every patch trace at its raw shot time (the
  // pseudo-deblending input), when the channel tables above do not hold
  // every problem
  std::vector<std::vector<BlendCoord>> input_coord;

  int channel_index(int value, int trace_type) const;
  BlendCoord coord_of(long shottime, int n_times, int channel, int trace_type) const;
};

struct ProblemArgs {
  int n_patches;
  const int *volumes;
  const int *n_dims;
  const int *const *window_shapes;
  const int *const *coords;
  const int *const *shapes;
  const long *const *shottimes;
  const int *const *channels;
  const enum AGDTraceType *const *trace_types;
  const int *wavelet_lengths;
  const int *const *wavelet_idxs;
  const real *const *wavelets;
};

// check_deblend_inputs (src/agdeblend.c:263-431): prints the reference's
// messages on failure and returns 1.
int check_deblend_inputs(const ProblemArgs &a, real initial_factor, int n_its,
                         real *const *data);

// set_model + the wavelet spectra; returns 1 (after printing) on failure.
int build_plan(const ProblemArgs &a, Plan &plan);

// Plans independent problems one by one and concatenates them: patches,
// windows, records and models follow one another in problem order, each
// window tagged with its problem.  Returns 1 (after printing) on failure.
int build_batch_plan(const std::vector<ProblemArgs> &args, Plan &plan);

// Blend configuration of arbitrary trace sets (used by agd_blend and by
// build_plan): set_blend_config, src/blend.c:629-691.
void build_blend_config(int n_patches, const int *n_traces, const int *n_times,
                        const long *const *shottimes, const int *const *channels,
                        const enum AGDTraceType *const *trace_types, Plan &plan);

// Phase-only, 1/n scaled spectrum of a zero-padded wavelet
// (transform_wavelets, src/wavelet.c:188-237).
std::vector<std::complex<double>> wavelet_spectrum(const real *w, int len, int n);

// Hann taper (set_taper_window, src/fk.c:28-73).
std::vector<real> taper_window(int length, int left, int right);

// Test hook for the error paths: with AGD_GPU_FAIL_ALLOC=n in the
// environment, the n-th device allocation counted from when the variable was
// set (or last changed) reports failure, so tests can walk every allocation
// of a call and check that the call returns 1 and releases what it held,
// without any fault on the GPU.
bool injected_alloc_failure();

// lambda schedule constants (src/agdeblend.c:526-533) in AGD_TYPE.
struct Schedule {
  real decay;
  int first_linear_it;
  real linear_slope;  // before multiplication by lambda_0
};
Schedule lambda_schedule(real initial_factor, int n_its);

}  // namespace agd
