// Host planning for the deblending path.  See plan.hpp.
#include "plan.hpp"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <mutex>
#include <set>
#include <string>

namespace agd {

namespace {

constexpr double kPi = 3.14159265358979323846;

int fail(const char *msg) {
  std::fprintf(stderr, "%s", msg);
  return 1;
}

int check_positive(int v, const char *name) {
  if (v <= 0) {
    std::fprintf(stderr, "ERROR: %s must be > 0\n", name);
    return 1;
  }
  return 0;
}

int check_non_null(const void *p, const char *name) {
  if (p == nullptr) {
    std::fprintf(stderr, "ERROR: %s must not be NULL\n", name);
    return 1;
  }
  return 0;
}

int space_traces(int n_space, const int *shape) {
  int n = 1;
  for (int d = 0; d < n_space; ++d) n *= shape[d];
  return n;
}

// Number of volumes: largest volume index + 1 (src/utils.c:59-67).
int count_volumes(int n_patches, const int *volumes) {
  int m = 0;
  for (int p = 0; p < n_patches; ++p) m = volumes[p] > m ? volumes[p] : m;
  return m + 1;
}

// Wavelet length per volume from its first live trace, 1 if none or no
// wavelets (set_volume_wavelet_lengths, src/utils.c:72-123).
int volume_wavelet_lengths(const ProblemArgs &a, const std::vector<int> &n_traces,
                           std::vector<int> &out) {
  int const nv = count_volumes(a.n_patches, a.volumes);
  out.assign(nv, 0);
  if (a.wavelet_idxs == nullptr) {
    out.assign(nv, 1);
    return 0;
  }
  for (int p = 0; p < a.n_patches; ++p) {
    int const v = a.volumes[p];
    if (out[v] != 0) continue;
    for (int t = 0; t < n_traces[p]; ++t) {
      if (a.trace_types[p][t] == AGDLive) {
        out[v] = a.wavelet_lengths[a.wavelet_idxs[p][t]];
        if (out[v] <= 0) return fail("ERROR: Wavelet lengths must be positive\n");
        break;
      }
    }
  }
  for (int &v : out)
    if (v == 0) v = 1;
  return 0;
}

bool overlaps(const Interval &a, const Interval &b) {
  return a.start < b.stop && a.stop > b.start;
}

bool adjacent(const Interval &a, const Interval &b) {
  return a.start == b.stop || a.stop == b.start;
}

// A channel's interval list under the reference's merge rule
// (src/blend.c:113-151): the first entry, in list order, that overlaps or
// touches the new span absorbs it; then, scanning on in list order, entries
// that touch the *new* span (not the grown entry) are absorbed and removed,
// and the scan resumes one position past the removed entry - so the entry
// that moves into the freed position is skipped.
//
// Entries are numbered in creation order; as new entries are appended and
// removals keep the order of the others, list order is number order.  A
// start-sorted index finds the entries touching a span (starts up to the
// span's end, back to the longest entry's length before its start), and the
// set of live numbers gives each removed entry's successor, so one merge
// costs O(k log n) for k candidates instead of a scan of the whole list.
class IntervalList {
 public:
  void add(const Interval &nw) {
    std::vector<int> touch;
    auto it = by_start_.upper_bound(std::make_pair(nw.stop, INT_MAX));
    while (it != by_start_.begin()) {
      --it;
      if (it->first + max_len_ < nw.start) break;
      if (iv_[it->second].stop >= nw.start) touch.push_back(it->second);
    }
    if (touch.empty()) {
      insert(nw);
      return;
    }
    std::sort(touch.begin(), touch.end());
    const int first = touch[0];
    Interval g = iv_[first];
    if (nw.start < g.start) g.start = nw.start;
    if (nw.stop > g.stop) g.stop = nw.stop;
    int cursor = first;
    size_t k = 1;
    for (;;) {
      while (k < touch.size() && touch[k] <= cursor) ++k;
      if (k == touch.size()) break;
      const int e = touch[k++];
      if (iv_[e].start < g.start) g.start = iv_[e].start;
      if (iv_[e].stop > g.stop) g.stop = iv_[e].stop;
      erase(e);
      auto s = live_.upper_bound(e);
      if (s == live_.end()) break;
      cursor = *s;  // moved into the freed position: not examined
    }
    replace(first, g);
  }

  std::vector<Interval> list() const {
    std::vector<Interval> out;
    out.reserve(live_.size());
    for (int id : live_) out.push_back(iv_[id]);
    return out;
  }

 private:
  void insert(const Interval &v) {
    const int id = (int)iv_.size();
    iv_.push_back(v);
    live_.insert(id);
    by_start_.insert(std::make_pair(v.start, id));
    max_len_ = std::max(max_len_, v.stop - v.start);
  }
  void erase(int id) {
    live_.erase(id);
    by_start_.erase(std::make_pair(iv_[id].start, id));
  }
  void replace(int id, const Interval &v) {
    by_start_.erase(std::make_pair(iv_[id].start, id));
    iv_[id] = v;
    by_start_.insert(std::make_pair(v.start, id));
    max_len_ = std::max(max_len_, v.stop - v.start);
  }

  std::vector<Interval> iv_;                 // by number
  std::set<int> live_;                       // numbers in the list
  std::set<std::pair<long, int>> by_start_;  // (start, number) of live entries
  long max_len_ = 0;
};

// Patch neighbour tapers (src/model.c:20-50,149-188).
std::vector<std::vector<int>> patch_use_taper(const ProblemArgs &a) {
  std::vector<std::vector<int>> ut(a.n_patches);
  for (int p = 0; p < a.n_patches; ++p) {
    int const v = a.volumes[p];
    int const nd = a.n_dims[v] - 1;
    ut[p].assign(2 * nd, 0);
    for (int q = 0; q < a.n_patches; ++q) {
      if (q == p || a.volumes[q] != v) continue;
      bool neighbour = true;
      for (int d = 0; d < nd; ++d) {
        int const c = a.coords[p][d];
        int const o = a.coords[q][d];
        if (o != c - 1 && o != c && o != c + 1) neighbour = false;
      }
      if (!neighbour) continue;
      for (int d = 0; d < nd; ++d) {
        int const c = a.coords[p][d];
        int const o = a.coords[q][d];
        if (o == c - 1)
          ut[p][2 * d] = 1;
        else if (o == c + 1)
          ut[p][2 * d + 1] = 1;
      }
    }
  }
  return ut;
}

}  // namespace

std::vector<real> taper_window(int length, int left, int right) {
  int const tl = length / 2;
  std::vector<real> w(length, (real)1);
  // The expression order and AGD_TYPE arithmetic follow src/fk.c:39-61 so the
  // table is bit-identical to the reference's.
  if (left) {
    for (int i = 0; i < tl; ++i) {
      w[i] = (real)0.5 * ((real)1 - (real)std::cos((real)2 * (real)kPi * (real)i /
                                                   (real)(2 * tl)));
    }
  }
  if (right) {
    for (int i = 0; i < tl; ++i) {
      w[length - tl + i] =
          (real)0.5 * ((real)1 - (real)std::cos((real)2 * (real)kPi * (real)(tl + i) /
                                                (real)(2 * tl)));
    }
  }
  return w;
}

std::vector<std::complex<double>> wavelet_spectrum(const real *w, int len, int n) {
  std::vector<std::complex<double>> out(n / 2 + 1);
  for (int k = 0; k <= n / 2; ++k) {
    double re = 0.0;
    double im = 0.0;
    for (int t = 0; t < len && t < n; ++t) {
      double const ang = -2.0 * kPi * (double)((long)k * t % n) / (double)n;
      re += (double)w[t] * std::cos(ang);
      im += (double)w[t] * std::sin(ang);
    }
    double const phase = std::atan2(im, re);
    out[k] = std::complex<double>(std::cos(phase) / n, std::sin(phase) / n);
  }
  return out;
}

Schedule lambda_schedule(real initial_factor, int n_its) {
  // Evaluated in AGD_TYPE with the C library's functions, as
  // src/agdeblend.c:526-533 does.
  Schedule s;
#ifdef AGD_DOUBLE
  s.decay = std::exp(std::log(AGD_TARGET_LAMB / initial_factor) / (real)n_its);
  s.first_linear_it = (int)((std::log(s.decay) * ((real)n_its - (real)1) + (real)1) /
                            std::log(s.decay));
  s.linear_slope = initial_factor * std::pow(s.decay, (real)s.first_linear_it) /
                   (real)(n_its - 1 - s.first_linear_it);
#else
  s.decay = expf(logf(AGD_TARGET_LAMB / initial_factor) / (real)n_its);
  s.first_linear_it = (int)((logf(s.decay) * ((real)n_its - 1.0f) + 1.0f) / logf(s.decay));
  s.linear_slope = initial_factor * powf(s.decay, (real)s.first_linear_it) /
                   (real)(n_its - 1 - s.first_linear_it);
#endif
  return s;
}

int Plan::channel_index(int value, int trace_type) const {
  if (trace_type == AGDMissing) return -1;
  if (!channel_lookup.empty() || channel_values.empty()) {
    auto it = channel_lookup.find(value);
    return it == channel_lookup.end() ? -1 : it->second;
  }
  for (size_t i = 0; i < channel_values.size(); ++i)
    if (channel_values[i] == value) return (int)i;
  return -1;
}

BlendCoord Plan::coord_of(long shottime, int n_times, int channel, int trace_type) const {
  // set_blend_coords (src/blend.c:693-726): first interval of the channel
  // (in list order) that strictly overlaps the trace span, clipped to it.
  // The candidates come from the start-sorted index: intervals starting
  // before the span ends, back to max_len before the span starts.
  BlendCoord c{-1, 0, 0};
  int const ci = channel_index(channel, trace_type);
  if (trace_type == AGDMissing || ci < 0) return c;
  Interval const span{shottime, shottime + n_times};
  const std::vector<Interval> &ivs = intervals[ci];
  int best = -1;
  if (ci < (int)by_start.size()) {
    const auto &idx = by_start[ci];
    auto it = std::lower_bound(idx.begin(), idx.end(), std::make_pair(span.stop, -1));
    while (it != idx.begin()) {
      --it;
      if (it->first + max_len[ci] <= span.start) break;
      if (overlaps(span, ivs[it->second]) && (best < 0 || it->second < best)) best = it->second;
    }
  } else {
    for (size_t i = 0; i < ivs.size() && best < 0; ++i)
      if (overlaps(span, ivs[i])) best = (int)i;
  }
  if (best >= 0) {
    const Interval &iv = ivs[best];
    long const s = span.start > iv.start ? span.start : iv.start;
    long const e = span.stop < iv.stop ? span.stop : iv.stop;
    c.rec = seg_off[ci][best] + (s - iv.start);
    c.trace_start = (int)(s - span.start);
    c.n = (int)(e - s);
  }
  return c;
}

void build_blend_config(int n_patches, const int *n_traces, const int *n_times,
                        const long *const *shottimes, const int *const *channels,
                        const enum AGDTraceType *const *trace_types, Plan &plan) {
  // Unique channels in first-appearance order, missing traces ignored
  // (src/blend.c:176-223); a hash map gives each trace its channel index.
  plan.channel_values.clear();
  plan.channel_lookup.clear();
  for (int p = 0; p < n_patches; ++p) {
    for (int t = 0; t < n_traces[p]; ++t) {
      if (trace_types[p][t] == AGDMissing) continue;
      int const c = channels[p][t];
      if (plan.channel_lookup.emplace(c, (int)plan.channel_values.size()).second)
        plan.channel_values.push_back(c);
    }
  }
  size_t const nch = plan.channel_values.size();
  std::vector<IntervalList> record_lists(nch), mute_lists(nch);
  // Per-channel record intervals and bad-trace mute intervals
  // (src/blend.c:305-342).
  for (int p = 0; p < n_patches; ++p) {
    for (int t = 0; t < n_traces[p]; ++t) {
      int const ci = plan.channel_index(channels[p][t], trace_types[p][t]);
      if (ci < 0) continue;
      Interval const iv{shottimes[p][t], shottimes[p][t] + n_times[p]};
      record_lists[ci].add(iv);
      if (trace_types[p][t] == AGDBad) mute_lists[ci].add(iv);
    }
  }
  plan.intervals.assign(nch, {});
  std::vector<std::vector<Interval>> mutes(nch);
  plan.by_start.assign(nch, {});
  plan.max_len.assign(nch, 0);
  for (size_t c = 0; c < nch; ++c) {
    plan.intervals[c] = record_lists[c].list();
    mutes[c] = mute_lists[c].list();
    for (size_t i = 0; i < plan.intervals[c].size(); ++i) {
      const Interval &iv = plan.intervals[c][i];
      plan.by_start[c].emplace_back(iv.start, (int)i);
      plan.max_len[c] = std::max(plan.max_len[c], iv.stop - iv.start);
    }
    std::sort(plan.by_start[c].begin(), plan.by_start[c].end());
  }
  plan.seg_off.assign(nch, {});
  long off = 0;
  for (size_t c = 0; c < nch; ++c) {
    for (const Interval &iv : plan.intervals[c]) {
      plan.seg_off[c].push_back(off);
      off += iv.stop - iv.start;
    }
  }
  plan.record_size = off;
  // Mute spans clipped to each overlapping record interval, intervals in
  // list order (src/blend.c:585-627)
  plan.mute.clear();
  for (size_t c = 0; c < nch; ++c) {
    const auto &idx = plan.by_start[c];
    for (const Interval &m : mutes[c]) {
      std::vector<int> hit;
      auto it = std::lower_bound(idx.begin(), idx.end(), std::make_pair(m.stop, -1));
      while (it != idx.begin()) {
        --it;
        if (it->first + plan.max_len[c] <= m.start) break;
        if (overlaps(m, plan.intervals[c][it->second])) hit.push_back(it->second);
      }
      std::sort(hit.begin(), hit.end());
      for (int i : hit) {
        const Interval &iv = plan.intervals[c][i];
        long const s = m.start < iv.start ? iv.start : m.start;
        long const e = m.stop > iv.stop ? iv.stop : m.stop;
        plan.mute.emplace_back(plan.seg_off[c][i] + (s - iv.start), (int)(e - s));
      }
    }
  }
}

int check_deblend_inputs(const ProblemArgs &a, real initial_factor, int n_its,
                         real *const *data) {
  auto err = [] { return fail("ERROR in agd_deblend inputs\n"); };
  if (check_positive(a.n_patches, "n_patches")) return err();
  if (check_positive(n_its, "n_its")) return err();
  if (initial_factor <= (real)0 || initial_factor > (real)1) {
    std::fprintf(stderr, "ERROR: initial_factor must be in (0, 1]\n");
    return err();
  }
  if (check_non_null(a.volumes, "volumes")) return err();
  if (check_non_null(a.n_dims, "n_dims")) return err();
  if (check_non_null(a.window_shapes, "window_shapes")) return err();
  if (check_non_null(a.coords, "coords")) return err();
  if (check_non_null(a.shapes, "shapes")) return err();
  if (check_non_null(a.shottimes, "shottimes")) return err();
  if (check_non_null(a.channels, "channels")) return err();
  if (check_non_null(a.trace_types, "trace_types")) return err();
  if (check_non_null(data, "data")) return err();

  for (int p = 0; p < a.n_patches; ++p) {
    int const v = a.volumes[p];
    if (v < 0) {
      std::fprintf(stderr, "ERROR: volumes must not be negative\n");
      return err();
    }
    if (check_non_null(a.coords[p], "coords")) return err();
    if (check_non_null(a.shottimes[p], "shottimes")) return err();
    if (check_non_null(a.channels[p], "channels")) return err();
    if (check_non_null(a.trace_types[p], "trace_types")) return err();
    if (check_non_null(data[p], "data")) return err();
    int const nd = a.n_dims[v];
    if (nd <= 1) {
      std::fprintf(stderr, "ERROR: n_dims must be > 1\n");
      return err();
    }
    if (nd - 1 > AGD_MAX_N_COORDS) {
      std::fprintf(stderr,
                   "ERROR: AGD_MAX_N_COORDS is currently set to %d, "
                   "but %d space dimensions have been requested. "
                   "Please increase AGD_MAX_N_COORDS in the source code and recompile\n",
                   AGD_MAX_N_COORDS, nd - 1);
      return err();
    }
    if (check_non_null(a.window_shapes[v], "window_shapes")) return err();
    if (check_non_null(a.shapes[p], "shapes")) return err();
    int const max_n_times = a.shapes[p][nd - 1] + a.window_shapes[v][nd - 1];
    size_t window_size = 1;
    size_t n_tr = 1;
    for (int d = 0; d < nd; ++d) {
      int const w = a.window_shapes[v][d];
      int const s = a.shapes[p][d];
      if (w < 2) {
        std::fprintf(stderr, "ERROR: window_shapes must be at least 2\n");
        return err();
      }
      if (w != s && w % 2 != 0) {
        std::fprintf(stderr,
                     "ERROR: window_shapes must be even if it doesn't cover the whole "
                     "dimension\n");
        return err();
      }
      if (w > s) {
        std::fprintf(stderr, "ERROR: window_shape must not be bigger than patch shape\n");
        return err();
      }
    }
    for (int d = 0; d < nd - 1; ++d) {
      window_size *= (size_t)a.window_shapes[v][d];
      n_tr *= (size_t)a.shapes[p][d];
    }
    if (2 * window_size * (size_t)max_n_times >= (size_t)INT_MAX) {
      std::fprintf(stderr, "ERROR: The window for volume %d is too big\n", v);
      return err();
    }
    if (n_tr >= (size_t)INT_MAX) {
      std::fprintf(stderr, "ERROR: Patches must have fewer than %d traces\n", INT_MAX);
      return err();
    }
  }

  if (a.wavelet_lengths != nullptr || a.wavelet_idxs != nullptr || a.wavelets != nullptr) {
    if (check_non_null(a.wavelet_lengths, "wavelet_lengths")) return err();
    if (check_non_null(a.wavelet_idxs, "wavelet_idxs")) return err();
    if (check_non_null(a.wavelets, "wavelets")) return err();
    std::vector<int> n_traces(a.n_patches);
    for (int p = 0; p < a.n_patches; ++p)
      n_traces[p] = space_traces(a.n_dims[a.volumes[p]] - 1, a.shapes[p]);
    for (int p = 0; p < a.n_patches; ++p)
      if (check_non_null(a.wavelet_idxs[p], "wavelet_idxs")) return err();
    for (int p = 0; p < a.n_patches; ++p)
      for (int t = 0; t < n_traces[p]; ++t)
        if (a.trace_types[p][t] == AGDLive && a.wavelet_idxs[p][t] < 0) {
          std::fprintf(stderr, "ERROR: wavelet_idx must not be negative\n");
          return err();
        }
    std::vector<int> vwl;
    if (volume_wavelet_lengths(a, n_traces, vwl)) return err();
    int n_wavelets = 0;
    for (int p = 0; p < a.n_patches; ++p) {
      int const v = a.volumes[p];
      for (int t = 0; t < n_traces[p]; ++t) {
        if (a.trace_types[p][t] != AGDLive) continue;
        int const wi = a.wavelet_idxs[p][t];
        if (wi + 1 > n_wavelets) n_wavelets = wi + 1;
        if (a.wavelet_lengths[wi] != vwl[v]) {
          std::fprintf(stderr,
                       "ERROR: wavelets in the same volume must have the same length\n");
          return err();
        }
      }
    }
    for (int i = 0; i < n_wavelets; ++i)
      if (check_non_null(a.wavelets[i], "wavelets")) return err();
  }
  return 0;
}

int build_plan(const ProblemArgs &a, Plan &plan) {
  auto err = [] { return fail("ERROR in set_model\n"); };
  int const np = a.n_patches;
  plan.n_patches = np;
  plan.volume.assign(a.volumes, a.volumes + np);
  plan.n_space.resize(np);
  plan.shape.resize(np);
  plan.n_traces.resize(np);
  plan.n_times.resize(np);
  plan.lt.resize(np);
  for (int p = 0; p < np; ++p) {
    int const nd = a.n_dims[a.volumes[p]];
    plan.n_space[p] = nd - 1;
    plan.shape[p].assign(a.shapes[p], a.shapes[p] + nd);
    plan.n_traces[p] = space_traces(nd - 1, a.shapes[p]);
    plan.n_times[p] = a.shapes[p][nd - 1];
    plan.lt[p] = a.window_shapes[a.volumes[p]][nd - 1];
  }
  std::vector<int> vwl;
  if (volume_wavelet_lengths(a, plan.n_traces, vwl)) return err();

  // Model time lengths (src/model.c:326-357).
  plan.n_fk.resize(np);
  plan.conv.resize(np);
  for (int p = 0; p < np; ++p) {
    int const h = plan.lt[p] / 2;
    int const wl = vwl[a.volumes[p]];
    int const n_before = plan.n_times[p] - wl + 1;
    int const n_tw = (n_before + h - 1) / h + 1;
    plan.n_fk[p] = (n_tw + 1) * h;
    plan.conv[p] = plan.n_fk[p] + wl - 1;
  }

  // Shot times moved earlier by the time taper (src/model.c:424-446).
  std::vector<std::vector<long>> shifted(np);
  std::vector<const long *> shifted_p(np);
  for (int p = 0; p < np; ++p) {
    shifted[p].resize(plan.n_traces[p]);
    for (int t = 0; t < plan.n_traces[p]; ++t)
      shifted[p][t] = a.shottimes[p][t] - plan.lt[p] / 2;
    shifted_p[p] = shifted[p].data();
  }
  build_blend_config(np, plan.n_traces.data(), plan.conv.data(), shifted_p.data(),
                     a.channels, a.trace_types, plan);

  // Space windows (src/model.c:456-745).
  std::vector<std::vector<int>> put = patch_use_taper(a);
  for (int p = 0; p < np; ++p) {
    int const v = a.volumes[p];
    for (int d = 0; d < plan.n_space[p]; ++d) {
      if ((put[p][2 * d] || put[p][2 * d + 1]) && a.window_shapes[v][d] % 2 == 1) {
        std::fprintf(stderr,
                     "ERROR: window shapes may only be odd if there is no tapering. "
                     "Patch %d touches another patch in dimension %d and so will be "
                     "tapered, but has window shape %d.\n",
                     p, d, a.window_shapes[v][d]);
        fail("ERROR in set_space_window\n");
        return err();
      }
    }
  }

  plan.windows.clear();
  std::vector<std::pair<long, int>> src_keys;  // (wavelet index, length)
  long model_off = 0;
  for (int p = 0; p < np; ++p) {
    int const v = a.volumes[p];
    int const D = plan.n_space[p];
    int n_win[kMaxSpaceDims];
    std::vector<int> starts[kMaxSpaceDims], lens[kMaxSpaceDims];
    int total = 1;
    for (int d = 0; d < D; ++d) {
      int const n = a.shapes[p][d];
      int const L = a.window_shapes[v][d];
      int const tl = L / 2;
      n_win[d] = (L == n) ? 1 : n / tl - 1;
      int const base = (n - tl) / n_win[d] + tl;
      int const n_larger = n - tl - (base - tl) * n_win[d];
      int start = 0;
      for (int i = 0; i < n_win[d]; ++i) {
        int const len = base + (i < n_larger ? 1 : 0);
        starts[d].push_back(start);
        lens[d].push_back(len);
        start += len - tl;
      }
      total *= n_win[d];
    }
    for (int wi = 0; wi < total; ++wi) {
      // window grid index, last space dim fastest
      int idx[kMaxSpaceDims];
      int rem = wi;
      for (int d = D - 1; d >= 0; --d) {
        idx[d] = rem % n_win[d];
        rem /= n_win[d];
      }
      WindowPlan w;
      w.patch = p;
      w.D = D;
      w.n_traces = 1;
      for (int d = 0; d < D; ++d) {
        w.coords[d] = starts[d][idx[d]];
        w.L[d] = lens[d][idx[d]];
        w.use_taper[2 * d] = idx[d] == 0 ? put[p][2 * d] : 1;
        w.use_taper[2 * d + 1] = idx[d] == n_win[d] - 1 ? put[p][2 * d + 1] : 1;
        w.n_traces *= w.L[d];
      }
      // Window traces in C order over the window's space dims
      // (set_window_arrays, src/model.c:748-805).
      w.trace_index.resize(w.n_traces);
      bool any_live = false;
      for (int t = 0; t < w.n_traces; ++t) {
        int r = t;
        long pt = 0;
        long stride = 1;
        for (int d = D - 1; d >= 0; --d) {
          int const k = r % w.L[d];
          r /= w.L[d];
          pt += (long)(w.coords[d] + k) * stride;
          stride *= a.shapes[p][d];
        }
        w.trace_index[t] = (int)pt;
        if (a.trace_types[p][pt] == AGDLive) any_live = true;
      }
      if (!any_live) continue;  // src/model.c:999-1006

      // FK operator constants (src/fk.c:75-169).
      w.Lt = plan.lt[p];
      w.h = w.Lt / 2;
      w.n_fk = plan.n_fk[p];
      w.C = plan.conv[p];
      w.T = w.n_fk / w.h - 1;
      long n_padded = 1;
      for (int d = 0; d < D; ++d) {
        w.P[d] = (int)std::ceil((real)w.L[d] * ((real)1 + AGD_PAD_FRACTION));
        n_padded *= w.P[d];
      }
      w.Pt = (int)std::ceil((real)w.Lt * ((real)1 + AGD_PAD_FRACTION));
      n_padded *= w.Pt;
      w.F = w.Pt / 2 + 1;
      w.scaler = (real)1 / (real)std::sqrt((real)n_padded);
      w.use_taper[2 * D] = 1;
      w.use_taper[2 * D + 1] = 1;
      for (int d = 0; d < D; ++d)
        w.taper[d] = taper_window(w.L[d], w.use_taper[2 * d], w.use_taper[2 * d + 1]);
      w.taper[D] = taper_window(w.Lt, 1, 1);

      // Wavelet source configurations (src/wavelet.c:19-70).
      if (a.wavelet_idxs != nullptr) {
        w.wavelet_src.assign(w.n_traces, -1);
        for (int t = 0; t < w.n_traces; ++t) {
          int const pt = w.trace_index[t];
          if (a.trace_types[p][pt] != AGDLive) continue;
          std::pair<long, int> key{a.wavelet_idxs[p][pt], w.C};
          int s = -1;
          for (size_t k = 0; k < src_keys.size(); ++k)
            if (src_keys[k] == key) s = (int)k;
          if (s < 0) {
            s = (int)src_keys.size();
            src_keys.push_back(key);
            plan.wavelet_n.push_back(w.C);
            plan.spectra.push_back(wavelet_spectrum(a.wavelets[key.first],
                                                    a.wavelet_lengths[key.first], w.C));
          }
          w.wavelet_src[t] = s;
          w.has_wavelet_traces = true;
        }
      }

      // Blend coordinates of each window trace on the shifted shot times
      // (set_blend_params, src/blend.c:728-760).
      w.blend.resize(w.n_traces);
      for (int t = 0; t < w.n_traces; ++t) {
        int const pt = w.trace_index[t];
        w.blend[t] = plan.coord_of(shifted[p][pt], w.C, a.channels[p][pt],
                                   a.trace_types[p][pt]);
      }
      w.model_size = (long)w.T * w.F * w.plane();
      w.model_off = model_off;
      model_off += w.model_size;
      plan.windows.push_back(std::move(w));
    }
  }
  plan.model_size = model_off;
  return 0;
}

}  // namespace agd

namespace agd {

int build_batch_plan(const std::vector<ProblemArgs> &args, Plan &out) {
  out = Plan{};
  out.n_problems = (int)args.size();
  // the wavelet stage runs on every window of a plan or on none
  for (const ProblemArgs &a : args)
    if ((a.wavelet_idxs != nullptr) != (args[0].wavelet_idxs != nullptr))
      return fail("ERROR: the problems of a batch must all have wavelets or all have none\n");
  for (size_t q = 0; q < args.size(); ++q) {
    const ProblemArgs &a = args[q];
    Plan sub;
    if (build_plan(a, sub)) return 1;
    const int patch_base = out.n_patches;
    const long rec_base = out.record_size;
    const long model_base = out.model_size;
    const int spec_base = (int)out.spectra.size();
    out.problem_rec_off.push_back(rec_base);
    out.problem_rec_size.push_back(sub.record_size);
    out.problem_model_off.push_back(model_base);
    out.problem_model_size.push_back(sub.model_size);
    out.n_patches += sub.n_patches;
    auto append = [](auto &dst, const auto &src) { dst.insert(dst.end(), src.begin(), src.end()); };
    append(out.volume, sub.volume);
    append(out.n_space, sub.n_space);
    append(out.shape, sub.shape);
    append(out.n_traces, sub.n_traces);
    append(out.n_times, sub.n_times);
    append(out.n_fk, sub.n_fk);
    append(out.conv, sub.conv);
    append(out.lt, sub.lt);
    append(out.intervals, sub.intervals);
    append(out.wavelet_n, sub.wavelet_n);
    append(out.spectra, sub.spectra);
    for (const auto &m : sub.mute) out.mute.emplace_back(m.first + rec_base, m.second);
    // blend coordinates of the patch traces at their raw shot times
    for (int p = 0; p < sub.n_patches; ++p) {
      std::vector<BlendCoord> c(sub.n_traces[p]);
      for (int t = 0; t < sub.n_traces[p]; ++t) {
        c[t] = sub.coord_of(a.shottimes[p][t], sub.n_times[p], a.channels[p][t],
                            (int)a.trace_types[p][t]);
        if (c[t].rec >= 0) c[t].rec += rec_base;
      }
      out.input_coord.push_back(std::move(c));
    }
    for (WindowPlan &W : sub.windows) {
      W.patch += patch_base;
      W.problem = (int)q;
      W.model_off += model_base;
      for (BlendCoord &b : W.blend)
        if (b.rec >= 0) b.rec += rec_base;
      for (int &s : W.wavelet_src)
        if (s >= 0) s += spec_base;
      out.windows.push_back(std::move(W));
    }
    out.record_size += sub.record_size;
    out.model_size += sub.model_size;
  }
  return 0;
}

}  // namespace agd

namespace agd {

bool injected_alloc_failure() {
  const char *env = std::getenv("AGD_GPU_FAIL_ALLOC");
  if (env == nullptr || env[0] == '\0') return false;
  static std::mutex mu;
  static std::string last;
  static long count = 0;
  std::lock_guard<std::mutex> g(mu);
  if (last != env) {
    last = env;
    count = 0;
  }
  return ++count == std::atol(env);
}

}  // namespace agd
