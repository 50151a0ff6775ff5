// Wavelet convolution / correlation of window traces (reference
// src/wavelet.c:239-301) for trace lengths C that split into pairwise
// coprime prime powers of at most 32 (e.g. 2431 = 11 * 13 * 17).
//
// Per trace the reference computes y <- c2r(r2c(y) * S) with S the
// 1/C-scaled phase spectrum (conjugated for the adjoint), or the bare
// transform pair for traces without a spectrum.  Here two traces a, b of a
// window travel as one complex sequence z = a + i b:
//
//  * prime-factor (Good-Thomas) FFT in shared memory: with C = f_0 f_1 ...
//    and s_i = C / f_i, sample t has the coordinates n_i = t mod f_i, and
//    the load copies it to position sum_i n_i g_i of a dense array with
//    extents (f_0, f_1, ...) and strides g_i (qmap, built on the host).  As
//    exp(-2 pi i t k / C) factors over the axes for k = sum_i k_i s_i mod C,
//    a pass along axis i is a plain f_i-point DFT over lines of stride g_i,
//    with no twiddles and no index wrap; after the forward passes frequency
//    k sits at sum_i (k s_i^-1 mod f_i) g_i (kpos), and the inverse passes
//    return the dense array to the sample layout, which the store reads
//    back through qmap.  Consecutive samples lie sum_i g_i apart, an odd
//    stride, so the copies in and out are free of bank conflicts.
//  * between them, with Z' the product spectrum,
//      Z'_k = ((Z_k + conj Z_{C-k}) S_a + (Z_k - conj Z_{C-k}) S_b) / 2,
//    which is Z_k S when both traces use the same spectrum.  The real and
//    imaginary parts of the inverse are the two filtered traces.  Traces
//    without a spectrum use 1/C and are scaled by C when stored, which keeps
//    the two halves of a pair at the same scale.
//
// The adjoint reads its traces straight from the blended record (the blend
// adjoint gather of src/blend.c:1262-1292), so the traces are not written
// and re-read between the two steps.  Loads are cp.async copies (zero-filled
// outside a trace's blended samples), all in flight at once.
#pragma once

#include "fast.cuh"

namespace agd {

constexpr int kPfaMaxFactors = 4;
constexpr int kWavThreads = 256;

struct PfaShape {
  int N;                          // transform length C
  int nf;                         // number of factors (axes)
  int f[kPfaMaxFactors];          // pairwise coprime prime powers, outermost axis first
  int g[kPfaMaxFactors];          // dense stride of each axis (product of the later f)
  float inv_g[kPfaMaxFactors];    // 1 / g (quotients by the float reciprocal)
  float inv_lines[kPfaMaxFactors];  // f / N: 1 / (lines of a pass)
};

template <typename R>
struct WaveletFastJob {
  R *y;                        // window traces [n_traces][C]
  const int *src;              // per trace spectrum index, or -1 (transform pair only)
  const unsigned short *qmap;  // [C] dense position of sample t
  const unsigned short *kpos;  // [C] dense position of frequency k after the forward passes
  const long *blend_rec;       // per trace: flat record start, or -1 (adjoint gather)
  const int *blend_ts;         // per trace: first blended sample
  const int *blend_n;          // per trace: number of blended samples
  int n_traces;
  int pad;
  PfaShape sh;
};

// floor(x / d) for 0 <= x < 2^22 from the rounded reciprocal r = 1 / d:
// (x + 1/2) / d lies at least 1/(2d) from an integer and the product's
// relative error is below 2^-23, so truncation gives the exact quotient.
__device__ __forceinline__ int div_small(int x, float r) {
  return __float2int_rz(((float)x + 0.5f) * r);
}

// One pass along an axis of extent F and stride g over np dense arrays of
// N elements: line l of a pair starts at l + (l / g) (F - 1) g.
template <typename R, int F, bool INV>
__device__ __forceinline__ void pfa_pass(Cx<R> *buf, int np, int N, int g, float inv_g,
                                         float inv_lines) {
  using C = Cx<R>;
  const int lines = N / F;
  const int total = np * lines;
  for (int idx = threadIdx.x; idx < total; idx += kWavThreads) {
    const int pr = div_small(idx, inv_lines);
    const int l = idx - pr * lines;
    const int hi = div_small(l, inv_g);
    C *b = buf + pr * N + l + hi * (F - 1) * g;
    C v[F];
#pragma unroll
    for (int m = 0; m < F; ++m) v[m] = b[m * g];
    dft<R, F, INV>(v);
#pragma unroll
    for (int m = 0; m < F; ++m) b[m * g] = v[m];
  }
}

// Factors above FMAX are compiled out (their register DFTs would raise the
// register demand of every pass); the host picks an instantiation whose
// FMAX covers the shape.
template <typename R, bool INV, int FMAX>
__device__ void pfa_pass_any(int F, Cx<R> *buf, int np, int N, int g, float inv_g,
                             float inv_lines) {
#define AGD_PFA_CASE(n) \
  case n: \
    if constexpr (n <= FMAX) pfa_pass<R, n, INV>(buf, np, N, g, inv_g, inv_lines); \
    break;
  switch (F) {
    AGD_PFA_CASE(2)
    AGD_PFA_CASE(3)
    AGD_PFA_CASE(4)
    AGD_PFA_CASE(5)
    AGD_PFA_CASE(7)
    AGD_PFA_CASE(8)
    AGD_PFA_CASE(9)
    AGD_PFA_CASE(11)
    AGD_PFA_CASE(13)
    AGD_PFA_CASE(16)
    AGD_PFA_CASE(17)
    AGD_PFA_CASE(19)
    AGD_PFA_CASE(23)
    AGD_PFA_CASE(25)
    AGD_PFA_CASE(27)
    AGD_PFA_CASE(32)
    default: break;  // the host only builds shapes from the factors above
  }
#undef AGD_PFA_CASE
}

// Spectrum value for frequency k of a real signal's length-N transform,
// conjugated for the adjoint.  A trace without a spectrum (bare transform
// pair, i.e. N times the trace) gets 1/N here and N when it is stored, so
// that both traces of a pair keep the same scale through the inverse
// transform (a factor N between them would cost the smaller one about
// log10(N) digits).
template <typename R>
__device__ __forceinline__ Cx<R> spectrum_at(const Cx<R> *sp, int k, int N, bool adjoint) {
  using C = Cx<R>;
  if (sp == nullptr) return cmake<C>((R)1 / (R)N, (R)0);
  C w = k <= N / 2 ? sp[k] : cmake<C>(sp[N - k].x, -sp[N - k].y);
  if (adjoint) w.y = -w.y;
  return w;
}

// Each CTA transforms np_max pairs of traces of one window (fewer in the
// window's last CTA).  direction +1: convolution in place on the traces;
// -1: correlation of the traces gathered from `record`, written to y.
// MINB blocks per SM (the register budget of the largest DFT decides which
// is faster; the engine times the candidates); factors up to FMAX.
template <typename R, int MINB, int FMAX>
__global__ void __launch_bounds__(kWavThreads, MINB)
    wavelet_fast(const WaveletFastJob<R> *__restrict__ jobs, const int *__restrict__ cta_job,
                 const int *__restrict__ cta_pair0, int np_max,
                 const Cx<R> *__restrict__ spectra, const long *__restrict__ spec_off,
                 int direction, const R *__restrict__ record) {
  using C = Cx<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  const WaveletFastJob<R> &job = jobs[cta_job[blockIdx.x]];
  const PfaShape &sh = job.sh;  // read per pass (a local copy would sit in local memory)
  const int N = sh.N;
  const int n_tr = job.n_traces;
  const int pair0 = cta_pair0[blockIdx.x];
  const int np = min(np_max, ((n_tr + 1) >> 1) - pair0);
  const unsigned short *__restrict__ qmap = job.qmap;
  const unsigned short *__restrict__ kpos = job.kpos;

  // ---- load: trace a -> real part, trace b -> imaginary part, each sample
  // to its dense position; thread u copies half u & 1 of sample u >> 1, so a
  // warp fills 16 whole complex slots; every copy of the block in flight
  // together
  for (int pr = 0; pr < np; ++pr) {
    const int ta = 2 * (pair0 + pr);
    const int tb = ta + 1 < n_tr ? ta + 1 : -1;
    const int mine = tb >= 0 ? ta + (threadIdx.x & 1) : ta;  // this thread's trace
    R *b = reinterpret_cast<R *>(buf + pr * N) + (threadIdx.x & 1);
    const bool live = tb >= 0 || (threadIdx.x & 1) == 0;
    if (record != nullptr) {
      const long r0 = job.blend_rec[mine];
      const int s0 = job.blend_ts[mine];
      const int n0 = live && r0 >= 0 ? job.blend_n[mine] : 0;
      for (int t = threadIdx.x >> 1; t < N; t += kWavThreads / 2) {
        const bool v = t >= s0 && t < s0 + n0;
        cp_async<sizeof(R)>(b + 2 * __ldg(qmap + t), v ? record + r0 + (t - s0) : record, v);
      }
    } else {
      const R *y0 = job.y + (long)mine * N;
      for (int t = threadIdx.x >> 1; t < N; t += kWavThreads / 2)
        cp_async<sizeof(R)>(b + 2 * __ldg(qmap + t), y0 + t, live);
    }
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();

  for (int i = 0; i < sh.nf; ++i) {
    pfa_pass_any<R, false, FMAX>(sh.f[i], buf, np, N, sh.g[i], sh.inv_g[i], sh.inv_lines[i]);
    __syncthreads();
  }

  // ---- spectrum product (frequencies k and C - k together)
  const bool adjoint = direction < 0;
  const int half = N / 2 + 1;
  for (int pr = 0; pr < np; ++pr) {
    const int ta = 2 * (pair0 + pr);
    const int wa = job.src[ta];
    const int wb = ta + 1 < n_tr ? job.src[ta + 1] : wa;
    const C *spa = wa >= 0 ? spectra + spec_off[wa] : nullptr;
    const C *spb = wb >= 0 ? spectra + spec_off[wb] : nullptr;
    C *b = buf + pr * N;
    for (int k = threadIdx.x; k < half; k += kWavThreads) {
      const int p = __ldg(kpos + k);
      const int q = __ldg(kpos + (k ? N - k : 0));
      const C fa = spectrum_at<R>(spa, k, N, adjoint);
      const C zp = b[p];
      const C zq = b[q];
      if (wa == wb) {
        b[p] = cmul(zp, fa);
        if (q != p) b[q] = cmul(zq, cmake<C>(fa.x, -fa.y));
      } else {
        const C fb = spectrum_at<R>(spb, k, N, adjoint);
        const C u = cmake<C>(zp.x + zq.x, zp.y - zq.y);  // Z_k + conj Z_{C-k}
        const C d = cmake<C>(zp.x - zq.x, zp.y + zq.y);  // Z_k - conj Z_{C-k}
        const C ua = cmul(u, fa);
        const C db = cmul(d, fb);
        b[p] = cmake<C>((R)0.5 * (ua.x + db.x), (R)0.5 * (ua.y + db.y));
        // Z'_{C-k} = conj((u S_a - d S_b) / 2)
        if (q != p) b[q] = cmake<C>((R)0.5 * (ua.x - db.x), (R)-0.5 * (ua.y - db.y));
      }
    }
  }
  __syncthreads();

  for (int i = 0; i < sh.nf; ++i) {
    pfa_pass_any<R, true, FMAX>(sh.f[i], buf, np, N, sh.g[i], sh.inv_g[i], sh.inv_lines[i]);
    __syncthreads();
  }

  // ---- store both traces of each pair
  for (int pr = 0; pr < np; ++pr) {
    const int ta = 2 * (pair0 + pr);
    const bool has_b = ta + 1 < n_tr;
    R *ya = job.y + (long)ta * N;
    const C *b = buf + pr * N;
    const R ka = job.src[ta] < 0 ? (R)N : (R)1;
    const R kb = has_b && job.src[ta + 1] < 0 ? (R)N : (R)1;
    for (int t = threadIdx.x; t < N; t += kWavThreads) {
      const C v = b[__ldg(qmap + t)];
      ya[t] = v.x * ka;
      if (has_b) ya[N + t] = v.y * kb;
    }
  }
}

}  // namespace agd
