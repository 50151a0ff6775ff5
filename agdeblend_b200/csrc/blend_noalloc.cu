// agd_blend_device_noalloc: blending for callers that cannot allocate device
// memory.
//
// Some callers may not call cudaMalloc at all: plugin hosts and frameworks
// that own every byte of device memory through their own pool (an
// allocation behind their back can fail or break their accounting), or
// real-time code that has to avoid the allocator's latency and possible
// failure.  This entry point does the work of agd_blend
// on data that is already on the device, and keeps every intermediate (the
// blended record and the lookup tables the kernels read) in one fixed array
// that is part of the library image: kScratchBytes of device memory that
// every GPU which loads the library holds until the process exits.
//
// The array's name in host code is only a host-side handle, not a device
// address, so the device address is looked up with cudaGetSymbolAddress the
// first time the entry point runs on a device (with that device current) and
// cached per device for the life of the process.  That first call therefore
// does set-up work and should happen before any stream capture begins.  The
// cached address belongs to the device's context at that time: resetting the
// device (cudaDeviceReset, or destroying and re-creating its primary context)
// between calls is not supported.
//
// All calls on one device share that device's array, and the array keeps
// whatever the previous call left in it.  Nothing here relies on it starting
// at zero: every record sample is written by the blend kernel before it is
// read, and every table is copied in before the kernels run.  Calls whose GPU
// work overlaps on the same device - two host threads calling at once, say -
// race on the array and corrupt each other's results.  Every call copies its
// tables from temporary host memory and then waits on `stream` until its own
// work has finished (the calling thread blocks), so consecutive calls from
// one host thread never overlap.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>
#include <vector>

#include "agdeblend_gpu.h"
#include "blend_tables.cuh"
#include "kernels.cuh"
#include "plan.hpp"

namespace {

using agd::real;

// Fixed scratch: 16 MiB per device.
constexpr size_t kScratchBytes = size_t(16) << 20;
static __device__ __align__(256) unsigned char g_blend_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void *g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device (looked up once
// per device).
int scratch_address(void **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    std::fprintf(stderr, "ERROR: agd_blend_device_noalloc: no usable current device\n");
    return 1;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (g_scratch_ptr[dev] == nullptr) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_blend_scratch);
    if (e != cudaSuccess || p == nullptr) {
      std::fprintf(stderr, "ERROR: agd_blend_device_noalloc: cudaGetSymbolAddress: %s\n",
                   cudaGetErrorString(e));
      return 1;
    }
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return 0;
}

size_t align_up(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace

extern "C" int agd_blend_device_noalloc(
    int n_patches, int const *n_traces, int const *n_times, long int const *const *shottimes,
    int const *const *channels, enum AGDTraceType const *const *trace_types,
    AGD_TYPE const *data_dev, enum AGDBlendMode blend_mode, int taper_length,
    int n_patches_out, int const *n_traces_out, int const *n_times_out,
    long int const *const *shottimes_out, int const *const *channels_out,
    enum AGDTraceType const *const *trace_types_out, AGD_TYPE *data_out_dev, void *stream_ptr) {
  const char *name = "agd_blend_device_noalloc";
  if (n_patches <= 0 || n_patches_out <= 0 || n_traces == nullptr || n_times == nullptr ||
      shottimes == nullptr || channels == nullptr || trace_types == nullptr ||
      data_dev == nullptr || n_traces_out == nullptr || n_times_out == nullptr ||
      shottimes_out == nullptr || channels_out == nullptr || trace_types_out == nullptr ||
      data_out_dev == nullptr) {
    std::fprintf(stderr, "ERROR: %s: invalid arguments\n", name);
    return 1;
  }
  for (int p = 0; p < n_patches; ++p)
    if (n_traces[p] <= 0 || n_times[p] <= 0 || shottimes[p] == nullptr ||
        channels[p] == nullptr || trace_types[p] == nullptr) {
      std::fprintf(stderr, "ERROR: %s: invalid input patch %d\n", name, p);
      return 1;
    }
  for (int p = 0; p < n_patches_out; ++p) {
    if (n_traces_out[p] <= 0 || n_times_out[p] <= 0 || shottimes_out[p] == nullptr ||
        channels_out[p] == nullptr || trace_types_out[p] == nullptr) {
      std::fprintf(stderr, "ERROR: %s: invalid output patch %d\n", name, p);
      return 1;
    }
    for (int t = 0; t < n_traces_out[p]; ++t)
      if (trace_types_out[p][t] == AGDBad) {
        std::fprintf(stderr, "ERROR: Output trace types may not be AGDBad\n");
        return 1;
      }
  }
  if (blend_mode == AGDBlendMean && taper_length < 0) {
    std::fprintf(stderr, "ERROR: taper_length must be >= 0 when blend_mode is AGDBlendMean\n");
    return 1;
  }
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);

  // host tables: the same ones agd_blend builds
  agd::BlendTables bt;
  agd::build_blend_tables(n_patches, n_traces, n_times, shottimes, channels, trace_types,
                          blend_mode, taper_length, n_patches_out, n_traces_out, n_times_out,
                          shottimes_out, channels_out, trace_types_out, bt);
  const long R = bt.record_size;
  const long n_chunk = bt.n_chunk();
  const long n_out = bt.n_out();
  const std::vector<long> &ptr = bt.ptr;
  const std::vector<agd::Contrib> &flat = bt.flat;
  const std::vector<real> &taper = bt.taper;

  // carve the fixed scratch array
  size_t off = 0;
  const size_t at_record = off;
  off = align_up(off + (size_t)R * sizeof(real));
  const size_t at_ptr = off;
  off = align_up(off + ptr.size() * sizeof(long));
  const size_t at_flat = off;
  off = align_up(off + flat.size() * sizeof(agd::Contrib));
  const size_t at_mute = off;
  off = align_up(off + (size_t)R);
  const size_t at_taper = off;
  off = align_up(off + taper.size() * sizeof(real));
  const size_t at_orec = off;
  off = align_up(off + (size_t)n_out * sizeof(long));
  const size_t at_odst = off;
  off = align_up(off + (size_t)n_out * sizeof(long));
  const size_t at_ots = off;
  off = align_up(off + (size_t)n_out * sizeof(int));
  const size_t at_on = off;
  off = align_up(off + (size_t)n_out * sizeof(int));
  const size_t at_ont = off;
  off = align_up(off + (size_t)n_out * sizeof(int));
  if (off > kScratchBytes) {
    std::fprintf(stderr,
                 "ERROR: %s: this blend needs %zu bytes of device scratch; the fixed limit is "
                 "%zu bytes (16 MiB). Use agd_blend for larger problems.\n",
                 name, off, kScratchBytes);
    return 1;
  }
  void *base_v = nullptr;
  if (scratch_address(&base_v)) return 1;
  unsigned char *base = static_cast<unsigned char *>(base_v);
  auto put = [&](size_t at, const void *src, size_t bytes) {
    return bytes == 0 ? cudaSuccess
                      : cudaMemcpyAsync(base + at, src, bytes, cudaMemcpyHostToDevice, stream);
  };
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = put(at_ptr, ptr.data(), ptr.size() * sizeof(long));
  if (e == cudaSuccess) e = put(at_flat, flat.data(), flat.size() * sizeof(agd::Contrib));
  if (e == cudaSuccess) e = put(at_mute, bt.mute.data(), (size_t)R);
  if (e == cudaSuccess) e = put(at_taper, taper.data(), taper.size() * sizeof(real));
  if (e == cudaSuccess) e = put(at_orec, bt.o_rec.data(), (size_t)n_out * sizeof(long));
  if (e == cudaSuccess) e = put(at_odst, bt.o_dst.data(), (size_t)n_out * sizeof(long));
  if (e == cudaSuccess) e = put(at_ots, bt.o_ts.data(), (size_t)n_out * sizeof(int));
  if (e == cudaSuccess) e = put(at_on, bt.o_n.data(), (size_t)n_out * sizeof(int));
  if (e == cudaSuccess) e = put(at_ont, bt.o_nt.data(), (size_t)n_out * sizeof(int));
  real *record = reinterpret_cast<real *>(base + at_record);
  if (e == cudaSuccess && n_chunk > 0) {
    agd::blend_gather<real><<<(unsigned)n_chunk, agd::kThreads, 0, stream>>>(
        reinterpret_cast<const agd::Contrib *>(base + at_flat),
        reinterpret_cast<const long *>(base + at_ptr), agd::BlendTables::kChunk, R, data_dev,
        record, bt.mode,
        reinterpret_cast<const uint8_t *>(base + at_mute), nullptr,
        reinterpret_cast<const real *>(base + at_taper), (int)taper.size(), nullptr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && n_out > 0) {
    agd::extract_traces<real><<<(unsigned)n_out, agd::kThreads, 0, stream>>>(
        reinterpret_cast<const long *>(base + at_orec), reinterpret_cast<const int *>(base + at_ots),
        reinterpret_cast<const int *>(base + at_on), reinterpret_cast<const long *>(base + at_odst),
        reinterpret_cast<const int *>(base + at_ont), record, data_out_dev);
    e = cudaGetLastError();
  }
  const cudaError_t es = cudaStreamSynchronize(stream);
  if (e == cudaSuccess) e = es;
  if (e != cudaSuccess) {
    std::fprintf(stderr, "ERROR: %s: %s\n", name, cudaGetErrorString(e));
    return 1;
  }
  return 0;
}
