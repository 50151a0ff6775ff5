// agd_blend on the GPU: blend traces into continuous records (sum, mean with
// cosine edge weights, or overwrite), mute bad traces, and read output traces
// back (reference src/agdeblend.c:651-938, src/blend.c:936-1292).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <vector>

#include "agdeblend.h"
#include "blend_tables.cuh"
#include "kernels.cuh"
#include "plan.hpp"

namespace {

using agd::real;

int fail_blend(const char *msg) {
  std::fprintf(stderr, "%s", msg);
  std::fprintf(stderr, "ERROR in agd_blend inputs\n");
  return 1;
}

// check_blend_inputs (src/agdeblend.c:651-732)
int check_blend_inputs(int n_patches, const int *n_traces, const int *n_times,
                       const long *const *shottimes, const int *const *channels,
                       const enum AGDTraceType *const *trace_types, real *const *data,
                       enum AGDBlendMode blend_mode, int taper_length, int n_patches_out,
                       const int *n_traces_out, const int *n_times_out,
                       const long *const *shottimes_out, const int *const *channels_out,
                       const enum AGDTraceType *const *trace_types_out,
                       real *const *data_out) {
  char buf[256];
  auto pos = [&](int v, const char *name) {
    if (v > 0) return 0;
    std::snprintf(buf, sizeof(buf), "ERROR: %s must be > 0\n", name);
    return fail_blend(buf);
  };
  auto nn = [&](const void *p, const char *name) {
    if (p != nullptr) return 0;
    std::snprintf(buf, sizeof(buf), "ERROR: %s must not be NULL\n", name);
    return fail_blend(buf);
  };
  if (pos(n_patches, "n_patches")) return 1;
  // the reference checks n_patches again under this name (src/agdeblend.c:667)
  if (pos(n_patches, "n_patches_out")) return 1;
  if (nn(n_traces, "n_traces_per_volume") || nn(n_traces_out, "n_traces_per_volume_out") ||
      nn(n_times, "n_times_per_volume") || nn(n_times_out, "n_times_per_volume_out") ||
      nn(shottimes, "shottimes") || nn(shottimes_out, "shottimes_out") ||
      nn(channels, "channels") || nn(channels_out, "channels_out") ||
      nn(trace_types, "trace_types") || nn(trace_types_out, "trace_types_out") ||
      nn(data, "data") || nn(data_out, "data_out"))
    return 1;
  for (int p = 0; p < n_patches; ++p) {
    if (pos(n_traces[p], "n_traces_per_volume") || pos(n_times[p], "n_times_per_volume") ||
        nn(shottimes[p], "shottimes") || nn(channels[p], "channels") ||
        nn(trace_types[p], "trace_types") || nn(data[p], "data"))
      return 1;
  }
  for (int p = 0; p < n_patches_out; ++p) {
    if (pos(n_traces_out[p], "n_traces_per_volume_out") ||
        pos(n_times_out[p], "n_times_per_volume_out") || nn(shottimes_out[p], "shottimes_out") ||
        nn(channels_out[p], "channels_out") || nn(trace_types_out[p], "trace_types_out") ||
        nn(data_out[p], "data_out"))
      return 1;
    for (int t = 0; t < n_traces_out[p]; ++t)
      if (trace_types_out[p][t] == AGDBad)
        return fail_blend("ERROR: Output trace types may not be AGDBad\n");
  }
  if (blend_mode == AGDBlendMean && taper_length < 0)
    return fail_blend("ERROR: taper_length must be >= 0 when blend_mode is AGDBlendMean\n");
  return 0;
}

struct Dev {
  void *p = nullptr;
  ~Dev() {
    if (p) cudaFree(p);
  }
};

// cudaMalloc, or a reported failure under the test hook AGD_GPU_FAIL_ALLOC
cudaError_t dev_alloc(void **p, size_t bytes) {
  if (agd::injected_alloc_failure()) return cudaErrorMemoryAllocation;
  return cudaMalloc(p, bytes);
}

#define BCK(x)                                                                \
  do {                                                                        \
    cudaError_t e_ = (x);                                                     \
    if (e_ != cudaSuccess) {                                                  \
      std::fprintf(stderr, "ERROR: %s: %s\n", #x, cudaGetErrorString(e_));    \
      goto err;                                                               \
    }                                                                         \
  } while (0)

}  // namespace

extern "C" int agd_blend(int n_patches, int const *n_traces, int const *n_times,
                         long int const *const *shottimes, int const *const *channels,
                         enum AGDTraceType const *const *trace_types, AGD_TYPE *const *data,
                         enum AGDBlendMode blend_mode, int taper_length, int n_patches_out,
                         int const *n_traces_out, int const *n_times_out,
                         long int const *const *shottimes_out,
                         int const *const *channels_out,
                         enum AGDTraceType const *const *trace_types_out,
                         AGD_TYPE *const *data_out) {
  if (check_blend_inputs(n_patches, n_traces, n_times, shottimes, channels, trace_types, data,
                         blend_mode, taper_length, n_patches_out, n_traces_out, n_times_out,
                         shottimes_out, channels_out, trace_types_out, data_out)) {
    std::fprintf(stderr, "ERROR in agd_blend\n");
    return 1;
  }
  agd::BlendTables bt;
  agd::build_blend_tables(n_patches, n_traces, n_times, shottimes, channels, trace_types,
                          blend_mode, taper_length, n_patches_out, n_traces_out, n_times_out,
                          shottimes_out, channels_out, trace_types_out, bt);
  const long R = bt.record_size;
  const long n_chunk = bt.n_chunk();
  const long n_out_tr = bt.n_out();
  const long in_size = bt.in_size, out_size = bt.out_size;
  const std::vector<long> &in_off = bt.in_off, &out_off = bt.out_off;
  const std::vector<long> &ptr = bt.ptr;
  const std::vector<agd::Contrib> &flat = bt.flat;
  const std::vector<uint8_t> &mute = bt.mute;
  const std::vector<real> &taper = bt.taper;
  const std::vector<long> &o_rec = bt.o_rec, &o_dst = bt.o_dst;
  const std::vector<int> &o_ts = bt.o_ts, &o_n = bt.o_n, &o_nt = bt.o_nt;

  cudaStream_t s = nullptr;
  Dev d_in, d_rec, d_flat, d_ptr, d_mute, d_taper, d_out, d_orec, d_ots, d_on, d_odst, d_ont;
  BCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  BCK(dev_alloc(&d_in.p, std::max<long>(in_size, 1) * sizeof(real)));
  BCK(dev_alloc(&d_rec.p, std::max<long>(R, 1) * sizeof(real)));
  BCK(dev_alloc(&d_flat.p, std::max<size_t>(flat.size(), 1) * sizeof(agd::Contrib)));
  BCK(dev_alloc(&d_ptr.p, ptr.size() * sizeof(long)));
  BCK(dev_alloc(&d_mute.p, std::max<long>(R, 1)));
  BCK(dev_alloc(&d_taper.p, std::max<size_t>(taper.size(), 1) * sizeof(real)));
  BCK(dev_alloc(&d_out.p, std::max<long>(out_size, 1) * sizeof(real)));
  BCK(dev_alloc(&d_orec.p, std::max<long>(n_out_tr, 1) * sizeof(long)));
  BCK(dev_alloc(&d_ots.p, std::max<long>(n_out_tr, 1) * sizeof(int)));
  BCK(dev_alloc(&d_on.p, std::max<long>(n_out_tr, 1) * sizeof(int)));
  BCK(dev_alloc(&d_odst.p, std::max<long>(n_out_tr, 1) * sizeof(long)));
  BCK(dev_alloc(&d_ont.p, std::max<long>(n_out_tr, 1) * sizeof(int)));
  for (int p = 0; p < n_patches; ++p)
    BCK(cudaMemcpyAsync((real *)d_in.p + in_off[p], data[p],
                        (size_t)n_traces[p] * n_times[p] * sizeof(real), cudaMemcpyHostToDevice,
                        s));
  if (!flat.empty())
    BCK(cudaMemcpyAsync(d_flat.p, flat.data(), flat.size() * sizeof(agd::Contrib),
                        cudaMemcpyHostToDevice, s));
  BCK(cudaMemcpyAsync(d_ptr.p, ptr.data(), ptr.size() * sizeof(long), cudaMemcpyHostToDevice, s));
  if (R) BCK(cudaMemcpyAsync(d_mute.p, mute.data(), R, cudaMemcpyHostToDevice, s));
  if (!taper.empty())
    BCK(cudaMemcpyAsync(d_taper.p, taper.data(), taper.size() * sizeof(real),
                        cudaMemcpyHostToDevice, s));
  if (n_out_tr) {
    BCK(cudaMemcpyAsync(d_orec.p, o_rec.data(), n_out_tr * sizeof(long), cudaMemcpyHostToDevice, s));
    BCK(cudaMemcpyAsync(d_ots.p, o_ts.data(), n_out_tr * sizeof(int), cudaMemcpyHostToDevice, s));
    BCK(cudaMemcpyAsync(d_on.p, o_n.data(), n_out_tr * sizeof(int), cudaMemcpyHostToDevice, s));
    BCK(cudaMemcpyAsync(d_odst.p, o_dst.data(), n_out_tr * sizeof(long), cudaMemcpyHostToDevice, s));
    BCK(cudaMemcpyAsync(d_ont.p, o_nt.data(), n_out_tr * sizeof(int), cudaMemcpyHostToDevice, s));
  }
  if (n_chunk > 0) {
    agd::blend_gather<real><<<(unsigned)n_chunk, agd::kThreads, 0, s>>>(
        (const agd::Contrib *)d_flat.p, (const long *)d_ptr.p, agd::BlendTables::kChunk, R,
        (const real *)d_in.p, (real *)d_rec.p, bt.mode, (const uint8_t *)d_mute.p, nullptr,
        (const real *)d_taper.p,
        (int)taper.size(), nullptr);
    BCK(cudaGetLastError());
  }
  if (n_out_tr) {
    agd::extract_traces<real><<<(unsigned)n_out_tr, agd::kThreads, 0, s>>>(
        (const long *)d_orec.p, (const int *)d_ots.p, (const int *)d_on.p,
        (const long *)d_odst.p, (const int *)d_ont.p, (const real *)d_rec.p, (real *)d_out.p);
    BCK(cudaGetLastError());
  }
  for (int p = 0; p < n_patches_out; ++p)
    BCK(cudaMemcpyAsync(data_out[p], (real *)d_out.p + out_off[p],
                        (size_t)n_traces_out[p] * n_times_out[p] * sizeof(real),
                        cudaMemcpyDeviceToHost, s));
  BCK(cudaStreamSynchronize(s));
  cudaStreamDestroy(s);
  return 0;
err:
  if (s) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  std::fprintf(stderr, "ERROR in agd_blend\n");
  return 1;
}
