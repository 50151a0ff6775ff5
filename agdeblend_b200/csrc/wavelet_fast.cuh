// Wavelet convolution / correlation of window traces (reference
// src/wavelet.c:239-301) for trace lengths C that split into pairwise
// coprime prime powers of at most 32 (e.g. 2431 = 11 * 13 * 17).
//
// Per trace the reference computes y <- c2r(r2c(y) * S) with S the
// 1/C-scaled phase spectrum (conjugated for the adjoint), or the bare
// transform pair for traces without a spectrum.  Here two traces a, b of a
// window travel as one complex sequence z = a + i b:
//
//  * prime-factor (Good-Thomas) FFT in place in shared memory: with
//    C = f_0 f_1 ... and s_i = C / f_i, element (n_0, n_1, ...) sits at
//    position sum_i n_i s_i mod C; a pass along axis i is an f_i-point DFT
//    over the positions c + m s_i (mod C) and writes its outputs back to the
//    same positions, so no twiddles and no second buffer are needed.  After
//    the forward passes position p holds Z[kperm[p]] (kperm from the Chinese
//    remainder map, computed on the host); the inverse passes applied to that
//    layout return the natural order.
//  * between them, with Z' the product spectrum,
//      Z'_p = ((Z_p + conj Z_q) S_a + (Z_p - conj Z_q) S_b) / 2,
//    q the position of frequency C - k (q = C - p mod C), which is Z_p S when
//    both traces use the same spectrum.  The real and imaginary parts of the
//    inverse are the two filtered traces.  Traces without a spectrum use
//    1/C and are scaled by C when stored, which keeps the two halves of a
//    pair at the same scale.
//
// The adjoint reads its traces straight from the blended record (the blend
// adjoint gather of src/blend.c:1262-1292), so the traces are not written
// and re-read between the two steps.
#pragma once

#include "fast.cuh"

namespace agd {

constexpr int kPfaMaxFactors = 4;
constexpr int kWavThreads = 256;

struct PfaShape {
  int N;                      // transform length C
  int nf;                     // number of factors
  int f[kPfaMaxFactors];      // pairwise coprime prime powers, pass order
  int s[kPfaMaxFactors];      // N / f
  int inv[kPfaMaxFactors];    // (N / f)^-1 mod f
};

template <typename R>
struct WaveletFastJob {
  R *y;                  // window traces [n_traces][C]
  const int *src;        // per trace spectrum index, or -1 (transform pair only)
  const int *kperm;      // [C] frequency held at each position after the forward passes
  const long *blend_rec; // per trace: flat record start, or -1 (adjoint gather)
  const int *blend_ts;   // per trace: first blended sample
  const int *blend_n;    // per trace: number of blended samples
  int n_traces;
  int pad;
  PfaShape sh;
};

// One pass along an axis of length F for np sequences of length N.  Line l
// starts at position c = F l, whose index along this axis is 0 (a position
// p holds axis index (p mod F) (N/F)^-1 mod F); as gcd(F, N/F) = 1 these
// starts meet every line once.  Consecutive threads then read positions F
// apart, which for odd F are free of shared-memory bank conflicts.
template <typename R, int F, bool INV>
__device__ __forceinline__ void pfa_pass(Cx<R> *buf, int np, int N, int s) {
  using C = Cx<R>;
  for (int idx = threadIdx.x; idx < np * s; idx += blockDim.x) {
    const int pr = idx / s;
    const int c = F * (idx - pr * s);
    C *b = buf + (long)pr * N;
    C v[F];
    int pos = c;
#pragma unroll
    for (int m = 0; m < F; ++m) {
      v[m] = b[pos];
      pos += s;
      if (pos >= N) pos -= N;
    }
    dft<R, F, INV>(v);
    pos = c;
#pragma unroll
    for (int m = 0; m < F; ++m) {
      b[pos] = v[m];
      pos += s;
      if (pos >= N) pos -= N;
    }
  }
}

template <typename R, bool INV>
__device__ void pfa_pass_any(int F, Cx<R> *buf, int np, int N, int s) {
  switch (F) {
    case 2: pfa_pass<R, 2, INV>(buf, np, N, s); break;
    case 3: pfa_pass<R, 3, INV>(buf, np, N, s); break;
    case 4: pfa_pass<R, 4, INV>(buf, np, N, s); break;
    case 5: pfa_pass<R, 5, INV>(buf, np, N, s); break;
    case 7: pfa_pass<R, 7, INV>(buf, np, N, s); break;
    case 8: pfa_pass<R, 8, INV>(buf, np, N, s); break;
    case 9: pfa_pass<R, 9, INV>(buf, np, N, s); break;
    case 11: pfa_pass<R, 11, INV>(buf, np, N, s); break;
    case 13: pfa_pass<R, 13, INV>(buf, np, N, s); break;
    case 16: pfa_pass<R, 16, INV>(buf, np, N, s); break;
    case 17: pfa_pass<R, 17, INV>(buf, np, N, s); break;
    case 19: pfa_pass<R, 19, INV>(buf, np, N, s); break;
    case 23: pfa_pass<R, 23, INV>(buf, np, N, s); break;
    case 25: pfa_pass<R, 25, INV>(buf, np, N, s); break;
    case 27: pfa_pass<R, 27, INV>(buf, np, N, s); break;
    case 32: pfa_pass<R, 32, INV>(buf, np, N, s); break;
    default: break;  // the host only builds shapes from the factors above
  }
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
// MINB blocks per SM (the register budget of the 17-point DFTs decides
// which is faster; the engine times the candidates).
template <typename R, int MINB>
__global__ void __launch_bounds__(kWavThreads, MINB)
    wavelet_fast(const WaveletFastJob<R> *__restrict__ jobs, const int *__restrict__ cta_job,
                 const int *__restrict__ cta_pair0, int np_max,
                 const Cx<R> *__restrict__ spectra, const long *__restrict__ spec_off,
                 int direction, const R *__restrict__ record) {
  using C = Cx<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  const WaveletFastJob<R> &job = jobs[cta_job[blockIdx.x]];
  const int N = job.sh.N;
  const int nf = job.sh.nf;
  const int n_tr = job.n_traces;
  const int pair0 = cta_pair0[blockIdx.x];
  const int np = min(np_max, ((n_tr + 1) >> 1) - pair0);

  // ---- load: trace a -> real part, trace b -> imaginary part (unrolled so
  // that several global loads are in flight per thread)
  for (int pr = 0; pr < np; ++pr) {
    const int ta = 2 * (pair0 + pr);
    const bool has_b = ta + 1 < n_tr;
    C *b = buf + (long)pr * N;
    if (record != nullptr) {
      const long ra = job.blend_rec[ta];
      const int sa = job.blend_ts[ta];
      const int na = job.blend_n[ta];
      long rb = -1;
      int sb = 0, nb = 0;
      if (has_b) {
        rb = job.blend_rec[ta + 1];
        sb = job.blend_ts[ta + 1];
        nb = job.blend_n[ta + 1];
      }
#pragma unroll 4
      for (int e = threadIdx.x; e < N; e += blockDim.x) {
        const R va = (ra >= 0 && e >= sa && e < sa + na) ? record[ra + (e - sa)] : (R)0;
        const R vb = (rb >= 0 && e >= sb && e < sb + nb) ? record[rb + (e - sb)] : (R)0;
        b[e] = cmake<C>(va, vb);
      }
    } else {
      const R *ya = job.y + (long)ta * N;
#pragma unroll 4
      for (int e = threadIdx.x; e < N; e += blockDim.x)
        b[e] = cmake<C>(ya[e], has_b ? ya[N + e] : (R)0);
    }
  }
  __syncthreads();

  for (int i = 0; i < nf; ++i) {
    pfa_pass_any<R, false>(job.sh.f[i], buf, np, N, job.sh.s[i]);
    __syncthreads();
  }

  // ---- spectrum product (positions p and q = N - p together)
  const bool adjoint = direction < 0;
  for (int pr = 0; pr < np; ++pr) {
    const int ta = 2 * (pair0 + pr);
    const int wa = job.src[ta];
    const int wb = ta + 1 < n_tr ? job.src[ta + 1] : wa;
    const C *spa = wa >= 0 ? spectra + spec_off[wa] : nullptr;
    const C *spb = wb >= 0 ? spectra + spec_off[wb] : nullptr;
    C *b = buf + (long)pr * N;
    for (int p = threadIdx.x; p <= N / 2; p += blockDim.x) {
      const int q = p ? N - p : 0;
      const int k = __ldg(job.kperm + p);
      const C fa = spectrum_at<R>(spa, k, N, adjoint);
      const C zp = b[p];
      const C zq = b[q];
      if (wa == wb) {
        b[p] = cmul(zp, fa);
        if (q != p) b[q] = cmul(zq, cmake<C>(fa.x, -fa.y));
      } else {
        const C fb = spectrum_at<R>(spb, k, N, adjoint);
        const C u = cmake<C>(zp.x + zq.x, zp.y - zq.y);  // Z_p + conj Z_q
        const C d = cmake<C>(zp.x - zq.x, zp.y + zq.y);  // Z_p - conj Z_q
        const C ua = cmul(u, fa);
        const C db = cmul(d, fb);
        b[p] = cmake<C>((R)0.5 * (ua.x + db.x), (R)0.5 * (ua.y + db.y));
        // Z'_q = conj((u S_a - d S_b) / 2)
        if (q != p) b[q] = cmake<C>((R)0.5 * (ua.x - db.x), (R)-0.5 * (ua.y - db.y));
      }
    }
  }
  __syncthreads();

  for (int i = 0; i < nf; ++i) {
    pfa_pass_any<R, true>(job.sh.f[i], buf, np, N, job.sh.s[i]);
    __syncthreads();
  }

  // ---- store both traces of each pair
  for (int pr = 0; pr < np; ++pr) {
    const int ta = 2 * (pair0 + pr);
    const bool has_b = ta + 1 < n_tr;
    R *ya = job.y + (long)ta * N;
    const C *b = buf + (long)pr * N;
    const R ka = job.src[ta] < 0 ? (R)N : (R)1;
    const R kb = has_b && job.src[ta + 1] < 0 ? (R)N : (R)1;
    for (int e = threadIdx.x; e < N; e += blockDim.x) {
      const C v = b[e];
      ya[e] = v.x * ka;
      if (has_b) ya[N + e] = v.y * kb;
    }
  }
}

}  // namespace agd
