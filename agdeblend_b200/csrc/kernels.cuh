// CUDA kernels of the deblending operator A = M B W F and its adjoint.
//
// Device layouts (per window w, offsets from the window tables):
//   model X      [T][F][P_0..P_{D-1}] complex, F = Pt/2 + 1   (f-major planes)
//   spatial Z    [T][F][L_0..L_{D-1}] complex  (model after the space IFFTs)
//   traces Y     [n_traces][C] real            (window traces, C = n_times_conv)
//   record       flat real array of every (channel, interval) segment
//
// Forward  A x : axis_pass (space IFFT per axis, crop P->L) -> time_c2r_ola
//                (time c2r, taper, overlap-add) -> [wavelet_apply] ->
//                blend_gather (ordered sum into the record, mute, residual)
// Adjoint A^H r: time_r2c (blend adjoint gather, taper, time r2c, x2 bins)
//                -> axis_pass (zero-pad L->P, space FFT per axis) with the
//                ISTA update and soft threshold fused into the last pass.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fft.cuh"

namespace agd {

constexpr int kThreads = 256;

// ------------------------------------------------------------ job records

// One window's pass along one space axis.  Lines are indexed q = o*inner + i
// over a [outer][n][inner] tensor.
template <typename R>
struct AxisJob {
  const Cx<R> *src;
  Cx<R> *dst;
  long outer;
  int inner;
  int n_in;   // elements per line read (zero-padded up to the FFT length)
  int n_out;  // elements per line written (first n_out of the FFT output)
  int fft;    // FftDesc index
  int last;   // 1: the window's final pass, which takes the launch's epilogue
  int pid;    // problem of the window (per-problem step, threshold, maximum)
};

enum AxisEpilogue : int {
  kStore = 0,          // dst = result
  kUpdateThreshold = 1,  // dst = soft_threshold(dst - step * result, lamb)
  kUpdateMax = 2,      // dst = dst - step * result; track max |dst|^2
};

// Per-window constants of the time-axis kernels.
template <typename R>
struct TimeJob {
  Cx<R> *z;              // window's [T][F][n_traces] block
  R *y;                  // window's [n_traces][C] trace block
  const R *space_scale;  // per trace: scaler * product of space tapers
  const R *time_taper;   // [Lt]
  const long *blend_rec; // per trace: flat record start, or -1
  const int *blend_ts;   // per trace: first blended sample of the trace
  const int *blend_n;    // per trace: number of blended samples
  int n_traces, T, F, Lt, Pt, h, n_fk, C;
  int fft;               // FftDesc index of length Pt
};

template <typename R>
struct WaveletJob {
  R *y;                 // [n_traces][C]
  const int *src;       // per trace spectrum index or -1
  int n_traces, C;
  int fft;              // FftDesc index of length C
};

// A contiguous run of one source trace added into the record.
struct Contrib {
  long rec;  // flat record index of the first sample
  long src;  // index of the first sample in the source array
  int n;     // samples
  int pad;
};

enum GatherMode : int {
  kGatherSum = 0,
  kGatherMean = 1,
  kGatherOverwrite = 2,
  kGatherResidual = 3,  // out = mask ? 0 : sum - d
};

// ------------------------------------------------------------ helpers

template <typename R>
__device__ __forceinline__ R mul_rn(R a, R b);
template <>
__device__ __forceinline__ float mul_rn<float>(float a, float b) {
  return __fmul_rn(a, b);
}
template <>
__device__ __forceinline__ double mul_rn<double>(double a, double b) {
  return __dmul_rn(a, b);
}
template <typename R>
__device__ __forceinline__ R add_rn(R a, R b);
template <>
__device__ __forceinline__ float add_rn<float>(float a, float b) {
  return __fadd_rn(a, b);
}
template <>
__device__ __forceinline__ double add_rn<double>(double a, double b) {
  return __dadd_rn(a, b);
}
template <typename R>
__device__ __forceinline__ R sub_rn(R a, R b);
template <>
__device__ __forceinline__ float sub_rn<float>(float a, float b) {
  return __fsub_rn(a, b);
}
template <>
__device__ __forceinline__ double sub_rn<double>(double a, double b) {
  return __dsub_rn(a, b);
}

// |x|^2 rounded per operation, as the reference's abs_sq (src/model.c:1409)
template <typename R>
__device__ __forceinline__ R abs_sq(Cx<R> x) {
  return add_rn<R>(mul_rn<R>(x.x, x.x), mul_rn<R>(x.y, x.y));
}

// Soft threshold: |x|^2 <= lamb^2 -> 0, else x * (|x| - lamb) / |x|
// (src/model.c:1392-1423).
template <typename R>
__device__ __forceinline__ Cx<R> soft_threshold(Cx<R> x, R lamb, R lamb_sq) {
  const R a2 = abs_sq<R>(x);
  if (a2 <= lamb_sq) return cmake<Cx<R>>((R)0, (R)0);
  const R a = sqrt(a2);
  const R s = (a - lamb) / a;
  return cmake<Cx<R>>(x.x * s, x.y * s);
}

// Atomic max for non-negative floating values through their bit patterns.
__device__ __forceinline__ void atomic_max_nonneg(float *addr, float v) {
  atomicMax(reinterpret_cast<unsigned int *>(addr), __float_as_uint(v));
}
__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long *>(addr),
            (unsigned long long)__double_as_longlong(v));
}

template <typename R>
__device__ R block_max(R v, R *red) {
  for (int o = 16; o > 0; o >>= 1) {
    R w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < (int)(blockDim.x >> 5) ? red[lane] : (R)0;
    for (int o = 16; o > 0; o >>= 1) {
      R w = __shfl_xor_sync(0xffffffffu, v, o);
      v = w > v ? w : v;
    }
  }
  return v;
}

__device__ inline double block_sum(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  return v;
}

// ------------------------------------------------------------ space axes

// One FFT pass along one space axis for a list of windows.  Block b handles
// lines [cta_line0[b], +lines_per_cta) of job cta_job[b].
template <typename R>
__global__ void __launch_bounds__(kThreads)
    axis_pass(const AxisJob<R> *__restrict__ jobs, const int *__restrict__ cta_job,
              const long *__restrict__ cta_line0, int lines_per_cta,
              const FftDesc *__restrict__ descs, const Cx<R> *__restrict__ tw,
              int inverse, int epilogue, R step_arg, R lamb_arg, const R *step_dev,
              const R *lamb_dev, R *max_out) {
  using C = Cx<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const AxisJob<R> job = jobs[cta_job[blockIdx.x]];
  const FftDesc &d = descs[job.fft];
  const int n = d.n;
  const long lines = job.outer * job.inner;
  const int epi = job.last ? epilogue : (int)kStore;  // block-uniform
  const long q0 = cta_line0[blockIdx.x];
  const int nl = (int)((lines - q0) < lines_per_cta ? (lines - q0) : lines_per_cta);
  C *a = reinterpret_cast<C *>(smem_raw);
  C *b = a + (long)lines_per_cta * n;
  const int inner = job.inner;
  const int total = nl * n;

  // load (zero-pad elements n_in..n-1)
  if (inner == 1) {
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
      const int i = idx / n;
      const int e = idx - i * n;
      const long q = q0 + i;
      a[idx] = e < job.n_in ? job.src[q * job.n_in + e] : cmake<C>((R)0, (R)0);
    }
  } else {
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
      const int e = idx / nl;
      const int i = idx - e * nl;
      const long q = q0 + i;
      const long o = q / inner;
      const long r = q - o * inner;
      a[(long)i * n + e] = e < job.n_in ? job.src[(o * job.n_in + e) * inner + r]
                                        : cmake<C>((R)0, (R)0);
    }
  }
  __syncthreads();
  C *res = block_fft<R>(a, b, nl, d, tw, inverse);

  R local_max = (R)0;
  const int total_out = nl * job.n_out;
  // the threshold comes from device memory when the launch is replayed from
  // a CUDA graph (one captured iteration, a different lambda each replay);
  // step_dev: independent problems solved together, per-problem scalars
  const bool multi = step_dev != nullptr;
  const R step = multi ? step_dev[job.pid] : step_arg;
  const R lamb = lamb_dev != nullptr ? lamb_dev[multi ? job.pid : 0] : lamb_arg;
  const R lamb_sq = lamb * lamb;
  for (int idx = threadIdx.x; idx < total_out; idx += blockDim.x) {
    int i, e;
    if (inner == 1) {
      i = idx / job.n_out;
      e = idx - i * job.n_out;
    } else {
      e = idx / nl;
      i = idx - e * nl;
    }
    const long q = q0 + i;
    const long o = q / inner;
    const long r = q - o * inner;
    const long di = (o * job.n_out + e) * inner + r;
    const C g = res[(long)i * n + e];
    if (epi == kStore) {
      job.dst[di] = g;
    } else {
      // x <- x - step * g   (src/model.c:1149-1154), then threshold
      const C x = job.dst[di];
      C xn = cmake<C>(sub_rn<R>(x.x, mul_rn<R>(step, g.x)),
                      sub_rn<R>(x.y, mul_rn<R>(step, g.y)));
      if (epi == kUpdateThreshold) {
        xn = soft_threshold<R>(xn, lamb, lamb_sq);
      } else {
        const R a2 = abs_sq<R>(xn);
        local_max = a2 > local_max ? a2 : local_max;
      }
      job.dst[di] = xn;
    }
  }
  if (epi == kUpdateMax) {
    __shared__ R red[32];
    const R m = block_max<R>(local_max, red);
    if (threadIdx.x == 0) atomic_max_nonneg(max_out + (multi ? job.pid : 0), m);
  }
}

// ------------------------------------------------------------ time axis

// Forward time axis: for every time window t, c2r of the F bins of each
// trace (Hermitian extension to Pt points, inverse FFT, real part), crop to
// Lt, scale by the space and time tapers and overlap-add at hop h into the
// trace; writes [n_traces][C] with zeros after n_fk (src/fk.c:307-373).
template <typename R>
__global__ void __launch_bounds__(kThreads)
    time_c2r_ola(const TimeJob<R> *__restrict__ jobs, const int *__restrict__ cta_job,
                 const int *__restrict__ cta_trace0, int nb_max,
                 const FftDesc *__restrict__ descs, const Cx<R> *__restrict__ tw) {
  using C = Cx<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const TimeJob<R> job = jobs[cta_job[blockIdx.x]];
  const FftDesc &d = descs[job.fft];
  const int t0 = cta_trace0[blockIdx.x];
  const int nb = min(nb_max, job.n_traces - t0);
  const int Pt = job.Pt;
  C *a = reinterpret_cast<C *>(smem_raw);
  C *b = a + (long)nb_max * Pt;
  R *y = reinterpret_cast<R *>(b + (long)nb_max * Pt);
  const int Cn = job.C;  // row pitch of the trace buffer
  for (int idx = threadIdx.x; idx < nb * Cn; idx += blockDim.x) y[idx] = (R)0;
  const int half = (Pt - 1) / 2;  // bins mirrored by the Hermitian extension
  for (int t = 0; t < job.T; ++t) {
    const C *zt = job.z + (long)t * job.F * job.n_traces + t0;
    for (int idx = threadIdx.x; idx < nb * job.F; idx += blockDim.x) {
      const int f = idx / nb;
      const int i = idx - f * nb;
      const C v = zt[(long)f * job.n_traces + i];
      a[i * Pt + f] = v;
      if (f >= 1 && f <= half) a[i * Pt + Pt - f] = cmake<C>(v.x, -v.y);
    }
    __syncthreads();
    C *res = block_fft<R>(a, b, nb, d, tw, 1);
    for (int idx = threadIdx.x; idx < nb * job.Lt; idx += blockDim.x) {
      const int i = idx / job.Lt;
      const int j = idx - i * job.Lt;
      const R u = res[i * Pt + j].x;
      // Samples past the trace capacity (only possible for an odd time
      // window spanning the whole trace) are dropped.
      const int s = t * job.h + j;
      if (s < Cn) y[i * Cn + s] += (u * job.space_scale[t0 + i]) * job.time_taper[j];
    }
    __syncthreads();
    if (res != a) {  // keep `a` as the load buffer
      C *tmp = a;
      a = b;
      b = tmp;
    }
  }
  for (int idx = threadIdx.x; idx < nb * Cn; idx += blockDim.x)
    job.y[(long)t0 * Cn + idx] = y[idx];
}

// Adjoint time axis: gather each trace (from the record through its blend
// coordinates, or from the trace buffer), then for every time window t take
// the Lt samples from t*h scaled by the tapers, zero-pad to Pt, forward FFT,
// keep F bins and double bins 1..(Pt-1)/2 (src/fk.c:375-452,
// src/blend.c:1262-1292).
template <typename R>
__global__ void __launch_bounds__(kThreads)
    time_r2c(const TimeJob<R> *__restrict__ jobs, const int *__restrict__ cta_job,
             const int *__restrict__ cta_trace0, int nb_max,
             const FftDesc *__restrict__ descs, const Cx<R> *__restrict__ tw,
             const R *__restrict__ record, int from_record) {
  using C = Cx<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const TimeJob<R> job = jobs[cta_job[blockIdx.x]];
  const FftDesc &d = descs[job.fft];
  const int t0 = cta_trace0[blockIdx.x];
  const int nb = min(nb_max, job.n_traces - t0);
  const int Pt = job.Pt;
  const int Cn = job.C;
  C *a = reinterpret_cast<C *>(smem_raw);
  C *b = a + (long)nb_max * Pt;
  R *y = reinterpret_cast<R *>(b + (long)nb_max * Pt);
  for (int idx = threadIdx.x; idx < nb * Cn; idx += blockDim.x) {
    const int i = idx / Cn;
    const int j = idx - i * Cn;
    const int tr = t0 + i;
    R v = (R)0;
    if (from_record) {
      const long rec = job.blend_rec[tr];
      const int ts = job.blend_ts[tr];
      if (rec >= 0 && j >= ts && j < ts + job.blend_n[tr]) v = record[rec + (j - ts)];
    } else {
      v = job.y[(long)tr * job.C + j];
    }
    y[idx] = v;
  }
  __syncthreads();
  const int half = (Pt - 1) / 2;
  for (int t = 0; t < job.T; ++t) {
    for (int idx = threadIdx.x; idx < nb * Pt; idx += blockDim.x) {
      const int i = idx / Pt;
      const int j = idx - i * Pt;
      R v = (R)0;
      const int s = t * job.h + j;
      if (j < job.Lt && s < Cn)
        v = (y[i * Cn + s] * job.space_scale[t0 + i]) * job.time_taper[j];
      a[idx] = cmake<C>(v, (R)0);
    }
    __syncthreads();
    C *res = block_fft<R>(a, b, nb, d, tw, 0);
    C *zt = job.z + (long)t * job.F * job.n_traces + t0;
    for (int idx = threadIdx.x; idx < nb * job.F; idx += blockDim.x) {
      const int f = idx / nb;
      const int i = idx - f * nb;
      C v = res[i * Pt + f];
      if (f >= 1 && f <= half) v = cmake<C>(v.x * (R)2, v.y * (R)2);
      zt[(long)f * job.n_traces + i] = v;
    }
    __syncthreads();
    if (res != a) {
      C *tmp = a;
      a = b;
      b = tmp;
    }
  }
}

// ------------------------------------------------------------ wavelets

// Phase-only wavelet convolution (direction +1) or correlation (-1) of each
// trace, as an unnormalised length-C transform pair with the 1/C-scaled
// spectrum; traces without a spectrum only go through the transform pair
// (src/wavelet.c:239-301).
template <typename R>
__global__ void __launch_bounds__(kThreads)
    wavelet_apply(const WaveletJob<R> *__restrict__ jobs, const int *__restrict__ cta_job,
                  const int *__restrict__ cta_trace0, int nb_max,
                  const FftDesc *__restrict__ descs, const Cx<R> *__restrict__ tw,
                  const Cx<R> *__restrict__ spectra, const long *__restrict__ spec_off,
                  int direction) {
  using C = Cx<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const WaveletJob<R> job = jobs[cta_job[blockIdx.x]];
  const FftDesc &d = descs[job.fft];
  const int t0 = cta_trace0[blockIdx.x];
  const int nb = min(nb_max, job.n_traces - t0);
  const int n = job.C;
  C *a = reinterpret_cast<C *>(smem_raw);
  C *b = a + (long)nb_max * n;
  for (int idx = threadIdx.x; idx < nb * n; idx += blockDim.x)
    a[idx] = cmake<C>(job.y[(long)t0 * n + idx], (R)0);
  __syncthreads();
  C *res = block_fft<R>(a, b, nb, d, tw, 0);
  C *other = res == a ? b : a;
  for (int idx = threadIdx.x; idx < nb * n; idx += blockDim.x) {
    const int i = idx / n;
    const int k = idx - i * n;
    const int s = job.src[t0 + i];
    C v = res[idx];
    if (s >= 0) {
      const C *sp = spectra + spec_off[s];
      C w = k <= n / 2 ? sp[k] : cmake<C>(sp[n - k].x, -sp[n - k].y);
      if (direction < 0) w.y = -w.y;
      v = cmul(v, w);
    }
    res[idx] = v;
  }
  __syncthreads();
  C *out = block_fft<R>(res, other, nb, d, tw, 1);
  for (int idx = threadIdx.x; idx < nb * n; idx += blockDim.x)
    job.y[(long)t0 * n + idx] = out[idx].x;
}

// ------------------------------------------------------------ blending

// Ordered gather into the blended record.  Block b owns record samples
// [b*chunk, (b+1)*chunk) (chunk <= 4 * blockDim) and visits the
// contributions overlapping its chunk in the reference's order (window, then
// trace), so sums are formed in the same order as its serial blend loops
// (src/blend.c:936-1027,1155-1260).  The contribution list is staged in
// shared memory in tiles of kGatherTile; each thread keeps the sums of its
// samples in registers across the tiles.
constexpr int kGatherTile = 256;
constexpr int kGatherSpt = 4;  // samples per thread at most

template <typename R>
__global__ void __launch_bounds__(kThreads)
    blend_gather(const Contrib *__restrict__ contrib, const long *__restrict__ chunk_ptr,
                 int chunk, long record_size, const R *__restrict__ src, R *out,
                 int mode, const uint8_t *__restrict__ mute, const R *__restrict__ d,
                 const R *__restrict__ taper, int taper_len, double *sumsq) {
  __shared__ Contrib tile[kGatherTile];
  const long c0 = (long)blockIdx.x * chunk;
  const long b0 = chunk_ptr[blockIdx.x];
  const long b1 = chunk_ptr[blockIdx.x + 1];
  R acc[kGatherSpt], cnt[kGatherSpt];
#pragma unroll
  for (int q = 0; q < kGatherSpt; ++q) acc[q] = cnt[q] = (R)0;
  for (long base = b0; base < b1; base += kGatherTile) {
    const int nt = (int)min((long)kGatherTile, b1 - base);
    __syncthreads();
    for (int i = threadIdx.x; i < nt; i += blockDim.x) tile[i] = contrib[base + i];
    __syncthreads();
    if (mode != kGatherMean && chunk == 2 * (int)blockDim.x) {
      // two samples per thread, four contributions per step: eight loads in
      // flight, added in list order (the order of the serial sum).  A run
      // lies inside the record, so samples past its end are never covered.
      const long s0 = c0 + threadIdx.x;
      const bool ovw = mode == kGatherOverwrite;
      R a0 = acc[0], a1 = acc[1];
      int c = 0;
      for (; c + 4 <= nt; c += 4) {
        R v[4][2];
        bool k[4][2];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const Contrib cu = tile[c + u];
          const long o = s0 - cu.rec;
          k[u][0] = (unsigned long)o < (unsigned long)cu.n;
          k[u][1] = (unsigned long)(o + blockDim.x) < (unsigned long)cu.n;
          v[u][0] = k[u][0] ? src[cu.src + o] : (R)0;
          v[u][1] = k[u][1] ? src[cu.src + o + blockDim.x] : (R)0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (k[u][0]) a0 = ovw ? v[u][0] : a0 + v[u][0];
          if (k[u][1]) a1 = ovw ? v[u][1] : a1 + v[u][1];
        }
      }
      for (; c < nt; ++c) {
        const Contrib ca = tile[c];
        const long oa = s0 - ca.rec;
        if ((unsigned long)oa < (unsigned long)ca.n) {
          const R v = src[ca.src + oa];
          a0 = ovw ? v : a0 + v;
        }
        if ((unsigned long)(oa + blockDim.x) < (unsigned long)ca.n) {
          const R v = src[ca.src + oa + blockDim.x];
          a1 = ovw ? v : a1 + v;
        }
      }
      acc[0] = a0;
      acc[1] = a1;
      continue;
    }
#pragma unroll
    for (int q = 0; q < kGatherSpt; ++q) {
      const int k = threadIdx.x + q * blockDim.x;
      const long s = c0 + k;
      if (k >= chunk || s >= record_size) continue;
      R a = acc[q], w_sum = cnt[q];
      for (int c = 0; c < nt; ++c) {
        const Contrib cb = tile[c];
        const long off = s - cb.rec;
        if (off < 0 || off >= cb.n) continue;
        const R v = src[cb.src + off];
        if (mode == kGatherOverwrite) {
          a = v;
        } else if (mode == kGatherMean) {
          R w = (R)1;
          if (taper_len > 1) {
            const int t = (int)off;
            const int to_end = cb.n - 1 - t;
            const int edge = t < to_end ? t : to_end;
            if (edge < taper_len) w = taper[edge];
          }
          a += v * w;
          w_sum += w;
        } else {
          a += v;
        }
      }
      acc[q] = a;
      cnt[q] = w_sum;
    }
  }
  double local = 0.0;
#pragma unroll
  for (int q = 0; q < kGatherSpt; ++q) {
    const int k = threadIdx.x + q * blockDim.x;
    const long s = c0 + k;
    if (k >= chunk || s >= record_size) continue;
    R a = acc[q];
    if (mode == kGatherMean && cnt[q] > (R)0) a /= cnt[q];
    if (mode == kGatherResidual) a = a - d[s];
    if (mute != nullptr && mute[s]) a = (R)0;
    out[s] = a;
    local += (double)a * (double)a;
  }
  if (sumsq != nullptr) {
    __shared__ double red[32];
    const double t = block_sum(local, red);
    if (threadIdx.x == 0) atomicAdd(sumsq, t);
  }
}

// Sum of window traces into the patch data: data[trace][t] = sum over the
// windows covering the trace (window order) of Y[w][wt][h + t]
// (set_output, src/model.c:1425-1515).  One block per patch trace.
template <typename R>
__global__ void __launch_bounds__(kThreads)
    output_gather(const long *__restrict__ out_ptr, const long *__restrict__ out_src,
                  const long *__restrict__ out_dst, const int *__restrict__ out_nt,
                  const R *__restrict__ y, R *data) {
  const long tr = blockIdx.x;
  const long b0 = out_ptr[tr];
  const long b1 = out_ptr[tr + 1];
  const int nt = out_nt[tr];
  R *dst = data + out_dst[tr];
  for (int t = threadIdx.x; t < nt; t += blockDim.x) {
    R acc = (R)0;
    for (long c = b0; c < b1; ++c) acc += y[out_src[c] + t];
    dst[t] = acc;
  }
}

// Output traces read back from the record: zeros outside the blended span,
// all zeros for traces without one (blend_adjoint, src/blend.c:1262-1292).
// One block per output trace.
template <typename R>
__global__ void __launch_bounds__(kThreads)
    extract_traces(const long *__restrict__ rec, const int *__restrict__ ts,
                   const int *__restrict__ n, const long *__restrict__ dst_off,
                   const int *__restrict__ nt, const R *__restrict__ record, R *out) {
  const long tr = blockIdx.x;
  const long r = rec[tr];
  const int s = ts[tr];
  const int m = n[tr];
  R *dst = out + dst_off[tr];
  for (int t = threadIdx.x; t < nt[tr]; t += blockDim.x)
    dst[t] = (r >= 0 && t >= s && t < s + m) ? record[r + (t - s)] : (R)0;
}

// Traces of per-trace constants (the stepsize probe, src/model.c:1239-1276):
// trace k (of every window) gets value[k] at y[dst[k] .. dst[k] + len[k]).
template <typename R>
__global__ void fill_traces(R *y, const R *__restrict__ value, const long *__restrict__ dst,
                            const int *__restrict__ len, long n_traces) {
  for (long k = blockIdx.x; k < n_traces; k += gridDim.x) {
    const R v = value[k];
    R *row = y + dst[k];
    for (int t = threadIdx.x; t < len[k]; t += blockDim.x) row[t] = v;
  }
}

template <typename R>
__global__ void record_max(const R *__restrict__ x, long n, R *out) {
  __shared__ R red[32];
  R m = (R)0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    m = x[i] > m ? x[i] : m;
  m = block_max<R>(m, red);
  if (threadIdx.x == 0) atomic_max_nonneg(out, m);
}

template <typename R>
__global__ void record_sumsq(const R *__restrict__ x, long n, double *out) {
  __shared__ double red[32];
  double s = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    s += (double)x[i] * (double)x[i];
  s = block_sum(s, red);
  if (threadIdx.x == 0) atomicAdd(out, s);
}

// Advances the threshold schedule on the device: out[0..n) = row *counter
// of table (n thresholds per iteration, one per problem solved together),
// then ++*counter.  One block; captured in the per-iteration CUDA graph.
template <typename R>
__global__ void next_lambda(const R *__restrict__ table, int *counter, R *out, int n) {
  const int k = *counter;
  for (int i = threadIdx.x; i < n; i += blockDim.x) out[i] = table[(long)k * n + i];
  __syncthreads();
  if (threadIdx.x == 0) *counter = k + 1;
}

// Window traces from patch data (the transpose of output_gather): for every
// patch trace and every window trace covering it, y[src + t] = data[dst + t]
// * scale[dst + t] (scale NULL: 1; data NULL: 1) for t < nt.  One block per
// patch trace; y is zeroed beforehand.
template <typename R>
__global__ void __launch_bounds__(kThreads)
    traces_from_data(const long *__restrict__ out_ptr, const long *__restrict__ out_src,
                     const long *__restrict__ out_dst, const int *__restrict__ out_nt,
                     const R *__restrict__ data, const R *__restrict__ scale, R *y) {
  const long tr = blockIdx.x;
  const long b0 = out_ptr[tr];
  const long b1 = out_ptr[tr + 1];
  const int nt = out_nt[tr];
  const long d0 = out_dst[tr];
  for (int t = threadIdx.x; t < nt; t += blockDim.x) {
    R v = data != nullptr ? data[d0 + t] : (R)1;
    if (scale != nullptr) v *= scale[d0 + t];
    for (long c = b0; c < b1; ++c) y[out_src[c] + t] = v;
  }
}

// running mean: acc = w acc + (1 - w) x
template <typename R>
__global__ void mean_into(R *acc, const R *x, long n, R w) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    acc[i] = w * acc[i] + ((R)1 - w) * x[i];
}

// x = 1 / max(x, floor) where x > 0 (else 0)
template <typename R>
__global__ void reciprocal_floor(R *x, long n, R floor) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    x[i] = x[i] > (R)0 ? (R)1 / (x[i] > floor ? x[i] : floor) : (R)0;
}

// Halves the time-frequency planes f = 1 .. (Pt - 1) / 2 of one window's
// model ([T][F][plane] complex): undoes the factor 2 that the adjoint
// applies to those bins (src/fk.c:446), leaving the plain r2c.
template <typename R>
__global__ void halve_interior_bins(Cx<R> *x, int T, int F, long plane, int f_last) {
  const long n = (long)T * F * plane;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    const int f = (int)((i / plane) % F);
    if (f >= 1 && f <= f_last) {
      x[i].x *= (R)0.5;
      x[i].y *= (R)0.5;
    }
  }
}

template <typename R>
__global__ void model_threshold(Cx<R> *x, long n, R lamb) {
  const R lamb_sq = lamb * lamb;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    x[i] = soft_threshold<R>(x[i], lamb, lamb_sq);
}

template <typename R>
__global__ void model_max_abs_sq(const Cx<R> *__restrict__ x, long n, R *out) {
  __shared__ R red[32];
  R m = (R)0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    const R a = abs_sq<R>(x[i]);
    m = a > m ? a : m;
  }
  m = block_max<R>(m, red);
  if (threadIdx.x == 0) atomic_max_nonneg(out, m);
}

// Reference model layout [T][P..][F] <-> device layout [T][F][P..], one
// window per launch (used at the operator-level C-ABI boundary only).
template <typename R>
__global__ void model_layout(const Cx<R> *__restrict__ src, Cx<R> *dst, int T, int F,
                             long plane, int to_device) {
  const long n = (long)T * F * plane;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    // i indexes the device layout
    const long t = i / ((long)F * plane);
    const long rem = i - t * F * plane;
    const long f = rem / plane;
    const long p = rem - f * plane;
    const long r = (t * plane + p) * F + f;
    if (to_device)
      dst[i] = src[r];
    else
      dst[r] = src[i];
  }
}

}  // namespace agd
