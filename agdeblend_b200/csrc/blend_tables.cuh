// Host tables of one agd_blend call, shared by agd_blend (blend.cu) and
// agd_blend_device_noalloc (blend_noalloc.cu) so that both entry points read
// the same contribution lists, mute mask, mean-mode weights and output trace
// coordinates (reference src/agdeblend.c:800-938, src/blend.c:936-1292).
#pragma once

#include <cmath>
#include <cstdint>
#include <vector>

#include "agdeblend.h"
#include "kernels.cuh"
#include "plan.hpp"

namespace agd {

struct BlendTables {
  static constexpr int kChunk = 512;  // record samples per blend_gather block
  long record_size = 0;
  int mode = kGatherSum;
  // input traces: patch offsets in the concatenated input, total samples
  std::vector<long> in_off;
  long in_size = 0;
  // per record chunk, the runs of input samples overlapping it (CSR), in
  // patch-then-trace order so that sums follow the serial reference's order
  std::vector<long> ptr;
  std::vector<Contrib> flat;
  std::vector<uint8_t> mute;  // one byte per record sample, 1 = bad-trace span
  std::vector<real> taper;    // mean-mode edge weights (src/blend.c:1174-1178)
  // output traces: where each reads the record and writes the output
  std::vector<long> out_off;
  long out_size = 0;
  std::vector<long> o_rec, o_dst;
  std::vector<int> o_ts, o_n, o_nt;

  long n_chunk() const { return (long)ptr.size() - 1; }
  long n_out() const { return (long)o_rec.size(); }
};

// Blend configuration of the input traces (set_blend_config,
// src/blend.c:629-691) flattened into BlendTables.  Any mode other than sum
// and overwrite takes the mean, as the reference's else branch does.
inline void build_blend_tables(int n_patches, const int *n_traces, const int *n_times,
                               const long *const *shottimes, const int *const *channels,
                               const enum AGDTraceType *const *trace_types,
                               enum AGDBlendMode blend_mode, int taper_length,
                               int n_patches_out, const int *n_traces_out,
                               const int *n_times_out, const long *const *shottimes_out,
                               const int *const *channels_out,
                               const enum AGDTraceType *const *trace_types_out,
                               BlendTables &bt) {
  Plan plan;
  build_blend_config(n_patches, n_traces, n_times, shottimes, channels, trace_types, plan);
  const long R = plan.record_size;
  bt.record_size = R;
  bt.mode = blend_mode == AGDBlendSum         ? kGatherSum
            : blend_mode == AGDBlendOverwrite ? kGatherOverwrite
                                              : kGatherMean;
  // contributions of the input traces, patch then trace order
  std::vector<Contrib> list;
  bt.in_off.assign(n_patches, 0);
  bt.in_size = 0;
  for (int p = 0; p < n_patches; ++p) {
    bt.in_off[p] = bt.in_size;
    for (int t = 0; t < n_traces[p]; ++t) {
      const BlendCoord b =
          plan.coord_of(shottimes[p][t], n_times[p], channels[p][t], (int)trace_types[p][t]);
      if (b.rec >= 0 && b.n > 0)
        list.push_back(Contrib{b.rec, bt.in_size + (long)t * n_times[p] + b.trace_start, b.n, 0});
    }
    bt.in_size += (long)n_traces[p] * n_times[p];
  }
  const int chunk = BlendTables::kChunk;
  const long n_chunk = (R + chunk - 1) / chunk;
  bt.ptr.assign(n_chunk + 1, 0);
  for (const auto &c : list)
    for (long k = c.rec / chunk; k <= (c.rec + c.n - 1) / chunk; ++k) bt.ptr[k + 1]++;
  for (long k = 0; k < n_chunk; ++k) bt.ptr[k + 1] += bt.ptr[k];
  bt.flat.assign(bt.ptr[n_chunk], Contrib{});
  {
    std::vector<long> fill(bt.ptr.begin(), bt.ptr.end() - 1);
    for (const auto &c : list)
      for (long k = c.rec / chunk; k <= (c.rec + c.n - 1) / chunk; ++k) bt.flat[fill[k]++] = c;
  }
  bt.mute.assign(R, 0);
  for (const auto &m : plan.mute)
    for (int k = 0; k < m.second; ++k) bt.mute[m.first + k] = 1;
  // mean-mode edge weights, expression as src/blend.c:1174-1178
  bt.taper.clear();
  if (bt.mode == kGatherMean && taper_length > 1) {
    bt.taper.resize(taper_length);
    for (int i = 0; i < taper_length; ++i)
      bt.taper[i] = (real)std::cos((real)0.5 * (real)3.14159265358979323846 *
                                   (real)(taper_length - i) / (real)(taper_length + 1));
  }
  // output traces
  bt.out_off.assign(n_patches_out, 0);
  bt.out_size = 0;
  bt.o_rec.clear();
  bt.o_dst.clear();
  bt.o_ts.clear();
  bt.o_n.clear();
  bt.o_nt.clear();
  for (int p = 0; p < n_patches_out; ++p) {
    bt.out_off[p] = bt.out_size;
    for (int t = 0; t < n_traces_out[p]; ++t) {
      const BlendCoord b = plan.coord_of(shottimes_out[p][t], n_times_out[p], channels_out[p][t],
                                         (int)trace_types_out[p][t]);
      bt.o_rec.push_back(b.rec);
      bt.o_ts.push_back(b.trace_start);
      bt.o_n.push_back(b.n);
      bt.o_dst.push_back(bt.out_size + (long)t * n_times_out[p]);
      bt.o_nt.push_back(n_times_out[p]);
    }
    bt.out_size += (long)n_traces_out[p] * n_times_out[p];
  }
}

}  // namespace agd
