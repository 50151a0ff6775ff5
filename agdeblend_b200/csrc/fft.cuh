// Block-cooperative FFTs in shared memory for sm_100a.
//
// A thread block transforms `nl` contiguous sequences of length n held in
// shared memory with a mixed-radix Stockham autosort FFT (the published
// formulation in which a radix-R pass reads elements j + r*(n/R) and writes
// them to (j/ns)*ns*R + j%ns + q*ns).  Radices 2, 3, 4 and 5 have dedicated
// butterflies; any other prime factor uses a direct R-point DFT whose
// twiddles come from the same table.  Twiddles W_n^k = exp(-2 pi i k / n) are
// precomputed in double precision on the host and rounded once.
//
// Convention (FFTW's): forward = exp(-2 pi i ...), inverse = exp(+...), no
// normalisation in either direction.
#pragma once

#include <cuda_runtime.h>

namespace agd {

constexpr int kMaxFactors = 24;

struct FftDesc {
  int n;
  int nf;
  int radix[kMaxFactors];
  long tw_off;  // offset of the length-n twiddle table
};

template <typename R>
struct CxT;
template <>
struct CxT<float> {
  using type = float2;
};
template <>
struct CxT<double> {
  using type = double2;
};
template <typename R>
using Cx = typename CxT<R>::type;

template <typename C>
__device__ __forceinline__ C cmake(decltype(C{}.x) a, decltype(C{}.x) b) {
  C r;
  r.x = a;
  r.y = b;
  return r;
}

template <typename C>
__device__ __forceinline__ C cadd(C a, C b) {
  return cmake<C>(a.x + b.x, a.y + b.y);
}
template <typename C>
__device__ __forceinline__ C csub(C a, C b) {
  return cmake<C>(a.x - b.x, a.y - b.y);
}
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  return cmake<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C>
__device__ __forceinline__ C cscale(C a, decltype(C{}.x) s) {
  return cmake<C>(a.x * s, a.y * s);
}
// multiply by -i (forward) or +i (inverse)
template <typename C>
__device__ __forceinline__ C rot_i(C a, int inverse) {
  return inverse ? cmake<C>(-a.y, a.x) : cmake<C>(a.y, -a.x);
}

template <typename C>
__device__ __forceinline__ C twiddle(const C *__restrict__ tw, long idx, int inverse) {
  C w = tw[idx];
  if (inverse) w.y = -w.y;
  return w;
}

// Transforms nl sequences a[line*n + e]; b is scratch of the same size.
// Returns the buffer holding the result.  Ends with a __syncthreads().
template <typename R>
__device__ Cx<R> *block_fft(Cx<R> *a, Cx<R> *b, int nl, const FftDesc &d,
                            const Cx<R> *__restrict__ tw_all, int inverse) {
  using C = Cx<R>;
  const int n = d.n;
  const C *__restrict__ tw = tw_all + d.tw_off;
  int ns = 1;
  for (int f = 0; f < d.nf; ++f) {
    const int radix = d.radix[f];
    const int m = n / radix;
    const int tws = n / (ns * radix);
    const int work = nl * m;
    for (int idx = threadIdx.x; idx < work; idx += blockDim.x) {
      const int line = idx / m;
      const int j = idx - line * m;
      const C *in = a + (long)line * n;
      C *out = b + (long)line * n;
      const int k = j % ns;
      const int base = (j - k) * radix + k;
      const long tk = (long)k * tws;
      if (radix == 2) {
        C v0 = in[j];
        C v1 = in[j + m];
        if (k) v1 = cmul(v1, twiddle(tw, tk, inverse));
        out[base] = cadd(v0, v1);
        out[base + ns] = csub(v0, v1);
      } else if (radix == 4) {
        C v0 = in[j];
        C v1 = in[j + m];
        C v2 = in[j + 2 * m];
        C v3 = in[j + 3 * m];
        if (k) {
          v1 = cmul(v1, twiddle(tw, tk, inverse));
          v2 = cmul(v2, twiddle(tw, 2 * tk, inverse));
          v3 = cmul(v3, twiddle(tw, 3 * tk, inverse));
        }
        const C s02 = cadd(v0, v2);
        const C d02 = csub(v0, v2);
        const C s13 = cadd(v1, v3);
        const C r13 = rot_i(csub(v1, v3), inverse);
        out[base] = cadd(s02, s13);
        out[base + ns] = cadd(d02, r13);
        out[base + 2 * ns] = csub(s02, s13);
        out[base + 3 * ns] = csub(d02, r13);
      } else if (radix == 3) {
        C v0 = in[j];
        C v1 = in[j + m];
        C v2 = in[j + 2 * m];
        if (k) {
          v1 = cmul(v1, twiddle(tw, tk, inverse));
          v2 = cmul(v2, twiddle(tw, 2 * tk, inverse));
        }
        // X1,2 = v0 - (v1+v2)/2 -/+ i (sqrt(3)/2)(v1 - v2)   (forward)
        const R c = (R)0.86602540378443864676;
        const C t1 = cadd(v1, v2);
        const C t2 = cmake<C>(v0.x - (R)0.5 * t1.x, v0.y - (R)0.5 * t1.y);
        const C t3 = rot_i(cscale(csub(v1, v2), c), inverse);
        out[base] = cadd(v0, t1);
        out[base + ns] = cadd(t2, t3);
        out[base + 2 * ns] = csub(t2, t3);
      } else if (radix == 5) {
        C v0 = in[j];
        C v1 = in[j + m];
        C v2 = in[j + 2 * m];
        C v3 = in[j + 3 * m];
        C v4 = in[j + 4 * m];
        if (k) {
          v1 = cmul(v1, twiddle(tw, tk, inverse));
          v2 = cmul(v2, twiddle(tw, 2 * tk, inverse));
          v3 = cmul(v3, twiddle(tw, 3 * tk, inverse));
          v4 = cmul(v4, twiddle(tw, 4 * tk, inverse));
        }
        // cos/sin of 2 pi/5 and 4 pi/5
        const R c1 = (R)0.30901699437494742410;
        const R c2 = (R)-0.80901699437494742410;
        const R s1 = (R)0.95105651629515357212;
        const R s2 = (R)0.58778525229247312917;
        const C t1 = cadd(v1, v4);
        const C t2 = cadd(v2, v3);
        const C t3 = csub(v1, v4);
        const C t4 = csub(v2, v3);
        const C a1 = cmake<C>(v0.x + c1 * t1.x + c2 * t2.x, v0.y + c1 * t1.y + c2 * t2.y);
        const C a2 = cmake<C>(v0.x + c2 * t1.x + c1 * t2.x, v0.y + c2 * t1.y + c1 * t2.y);
        const C b1 = rot_i(cmake<C>(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y), inverse);
        const C b2 = rot_i(cmake<C>(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y), inverse);
        out[base] = cadd(v0, cadd(t1, t2));
        out[base + ns] = cadd(a1, b1);
        out[base + 4 * ns] = csub(a1, b1);
        out[base + 2 * ns] = cadd(a2, b2);
        out[base + 3 * ns] = csub(a2, b2);
      } else {
        // direct R-point DFT with the twiddle folded in:
        // X_q = sum_r in[j + r m] W_n^{r (k tws + q m)}; the exponent
        // r e mod n advances by e < n per term
        for (int q = 0; q < radix; ++q) {
          const int e = (int)(tk + (long)q * m);
          C acc = in[j];
          int ti = 0;
          for (int r = 1; r < radix; ++r) {
            ti += e;
            if (ti >= n) ti -= n;
            acc = cadd(acc, cmul(in[j + r * m], twiddle(tw, ti, inverse)));
          }
          out[base + q * ns] = acc;
        }
      }
    }
    __syncthreads();
    C *t = a;
    a = b;
    b = t;
    ns *= radix;
  }
  return a;
}

}  // namespace agd
