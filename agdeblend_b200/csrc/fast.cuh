// Shape-specialised kernels of the deblending operator for sm_100a.
//
// Every FFT here runs in registers with a compile-time size: a thread owns a
// whole line (space axes) or one factor of a four-step transform (time axis),
// so the radix schedule, the index arithmetic and the twiddle offsets are
// constants.  Lengths with coprime factors (20 = 4 * 5, 40 = 8 * 5, 10 = 2 * 5)
// use the prime-factor split, which needs no twiddles; the other twiddles
// live in __constant__ memory (filled once per device from double-precision
// values), so they are read as constant-bank operands.
//
//   space_fwd_fast  all space axes of a batch of (t, f) planes: load the
//                   planes into shared memory, inverse FFT along every axis
//                   (cropping P -> L), store the [L..] planes;
//   space_adj_fast  the adjoint: zero-pad L -> P, forward FFT along every
//                   axis, then x <- soft_threshold(x - step * g, lambda);
//   space_adj_pipe  the adjoint with the next batch's input copied into a
//                   dense staging buffer behind the passes, and the update
//                   keeping several model loads in flight;
//   time_fwd_fast   per block of traces, every time window: Hermitian
//                   combine, half-length inverse FFT (four-step in shared
//                   memory), taper, overlap-add with a one-hop carry;
//   time_adj_fast   per block of traces, every time window: gather from the
//                   record, taper, half-length forward FFT, split, double.
//
// Kernels for other sizes are the generic ones in kernels.cuh.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.cuh"

namespace agd {

// ------------------------------------------------------------ twiddle tables

// Transform lengths with a constant twiddle table W_N^k = exp(-2 pi i k / N).
constexpr int kTwSizes[] = {6,  7,  9,  10, 11, 12, 13,  15,  16, 17, 19, 20,
                             23, 24, 25, 27, 32, 40, 48, 64, 80, 160, 320};
constexpr int kNumTw = (int)(sizeof(kTwSizes) / sizeof(int));

__host__ __device__ constexpr int tw_offset(int n) {
  int off = 0;
  for (int i = 0; i < kNumTw; ++i) {
    if (kTwSizes[i] == n) return off;
    off += kTwSizes[i];
  }
  return -1;
}

__host__ __device__ constexpr int tw_total() {
  int off = 0;
  for (int i = 0; i < kNumTw; ++i) off += kTwSizes[i];
  return off;
}

constexpr int kTwTotal = tw_total();

static __constant__ float2 c_tw_f[kTwTotal];
static __constant__ double2 c_tw_d[kTwTotal];

template <typename R>
__device__ __forceinline__ Cx<R> ctw(int idx);
template <>
__device__ __forceinline__ float2 ctw<float>(int idx) {
  return c_tw_f[idx];
}
template <>
__device__ __forceinline__ double2 ctw<double>(int idx) {
  return c_tw_d[idx];
}

// W_N^k (forward) or its conjugate (inverse); N must be in kTwSizes
template <typename R, int N, bool INV>
__device__ __forceinline__ Cx<R> wN(int k) {
  static_assert(tw_offset(N) >= 0, "no twiddle table for this length");
  Cx<R> w = ctw<R>(tw_offset(N) + k % N);
  if (INV) w.y = -w.y;
  return w;
}

// ------------------------------------------------------------ async copies

// global -> shared copies that complete asynchronously (cp.async, grouped
// with commit/wait); `valid == false` fills the destination with zeros
template <int BYTES>
__device__ __forceinline__ void cp_async(void *smem, const void *gmem, bool valid = true) {
  static_assert(BYTES == 4 || BYTES == 8 || BYTES == 16, "cp.async size");
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? BYTES : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(s), "l"(gmem),
               "n"(BYTES), "r"(n)
               : "memory");
}

__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ------------------------------------------------------------ register DFTs

template <bool INV, typename C>
__device__ __forceinline__ C mul_i(C a) {  // -i a (forward) or +i a (inverse)
  return INV ? cmake<C>(-a.y, a.x) : cmake<C>(a.y, -a.x);
}

__host__ __device__ constexpr int small_split(int n) {
  // largest explicit radix that divides n with a nontrivial cofactor
  return (n % 8 == 0 && n > 8) ? 8
         : (n % 5 == 0 && n > 5) ? 5
         : (n % 4 == 0 && n > 4) ? 4
         : (n % 3 == 0 && n > 3) ? 3
         : (n % 2 == 0 && n > 2) ? 2
                                 : 0;
}

template <typename R, int N, bool INV>
__device__ __forceinline__ void dft(Cx<R> (&v)[N]);

// Coprime split N = N1 * (N / N1) for the prime-factor DFT: N1 the largest
// power of two dividing N, or for odd N the power of its smallest prime
// (0 when N is a prime power).
__host__ __device__ constexpr int coprime_split(int n) {
  int p2 = 1;
  while (n % (2 * p2) == 0) p2 *= 2;
  if (p2 > 1) return p2 < n ? p2 : 0;
  int p = 3;
  while (p * p <= n && n % p) p += 2;
  if (n % p) return 0;  // n prime
  int q = 1;
  while (n % (q * p) == 0) q *= p;
  return q < n ? q : 0;
}

// k in [0, N1 N2) with k = k1 (mod N1), k = k2 (mod N2)
__host__ __device__ constexpr int crt_index(int k1, int k2, int N1, int N2) {
  int k = k2;
  while (k % N1 != k1) k += N2;
  return k;
}

// Odd length N with a twiddle table: the outputs k and N-k share the sums
// x_j + x_{N-j} (times cos) and x_j - x_{N-j} (times sin), so
//   X_k = A_k -/+ i B_k,  X_{N-k} = A_k +/- i B_k   (forward / inverse),
//   A_k = x_0 + sum_j (x_j + x_{N-j}) cos(2 pi j k / N),
//   B_k = sum_j (x_j - x_{N-j}) sin(2 pi j k / N),   j = 1 .. (N-1)/2.
template <typename R, int N, bool INV>
__device__ __forceinline__ void dft_odd(Cx<R> (&v)[N]) {
  using C = Cx<R>;
  static_assert(N % 2 == 1, "odd length");
  constexpr int H = (N - 1) / 2;
  constexpr int off = tw_offset(N);
  C sum[H], dif[H];
  C tot = v[0];
#pragma unroll
  for (int j = 1; j <= H; ++j) {
    sum[j - 1] = cadd(v[j], v[N - j]);
    dif[j - 1] = csub(v[j], v[N - j]);
    tot = cadd(tot, sum[j - 1]);
  }
  const C x0 = v[0];
#pragma unroll
  for (int k = 1; k <= H; ++k) {
    C a = x0;
    C b = cmake<C>((R)0, (R)0);
#pragma unroll
    for (int j = 1; j <= H; ++j) {
      const C w = ctw<R>(off + (j * k) % N);  // (cos, -sin) of 2 pi j k / N
      a.x += sum[j - 1].x * w.x;
      a.y += sum[j - 1].y * w.x;
      b.x -= dif[j - 1].x * w.y;
      b.y -= dif[j - 1].y * w.y;
    }
    if (INV) {
      v[k] = cmake<C>(a.x - b.y, a.y + b.x);
      v[N - k] = cmake<C>(a.x + b.y, a.y - b.x);
    } else {
      v[k] = cmake<C>(a.x + b.y, a.y - b.x);
      v[N - k] = cmake<C>(a.x - b.y, a.y + b.x);
    }
  }
  v[0] = tot;
}

// Prime-factor (Good-Thomas) DFT in registers for coprime N1, N2: input
// n = (n1 N2 + n2 N1) mod N, output k with k = k1 (mod N1), k = k2
// (mod N2); as exp(-2 pi i n k / N) = W_N1^(n1 k1) W_N2^(n2 k2) the two
// stages need no twiddle factors, and every index is a compile-time
// register name.
template <typename R, int N1, int N2, bool INV>
__device__ __forceinline__ void dft_pfa(Cx<R> (&v)[N1 * N2]) {
  using C = Cx<R>;
  constexpr int N = N1 * N2;
  C a[N];
#pragma unroll
  for (int n2 = 0; n2 < N2; ++n2) {
    C t[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) t[n1] = v[(n1 * N2 + n2 * N1) % N];
    dft<R, N1, INV>(t);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) a[k1 * N2 + n2] = t[k1];
  }
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1) {
    C t[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) t[n2] = a[k1 * N2 + n2];
    dft<R, N2, INV>(t);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) v[crt_index(k1, k2, N1, N2)] = t[k2];
  }
}

// Four-step in registers: N = N1 * N2, natural order in and out.
template <typename R, int N1, int N2, bool INV>
__device__ __forceinline__ void dft_fourstep(Cx<R> (&v)[N1 * N2]) {
  using C = Cx<R>;
  constexpr int N = N1 * N2;
  C a[N];
#pragma unroll
  for (int n2 = 0; n2 < N2; ++n2) {
    C t[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) t[n1] = v[N2 * n1 + n2];
    dft<R, N1, INV>(t);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1)
      a[N2 * k1 + n2] = (n2 * k1 == 0) ? t[k1] : cmul(t[k1], wN<R, N, INV>(n2 * k1));
  }
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1) {
    C t[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) t[n2] = a[N2 * k1 + n2];
    dft<R, N2, INV>(t);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) v[k1 + N1 * k2] = t[k2];
  }
}

template <typename R, int N, bool INV>
__device__ __forceinline__ void dft(Cx<R> (&v)[N]) {
  using C = Cx<R>;
  if constexpr (N == 1) {
  } else if constexpr (N == 2) {
    const C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (N == 3) {
    const R c = (R)0.86602540378443864676;
    const C t1 = cadd(v[1], v[2]);
    const C t2 = cmake<C>(v[0].x - (R)0.5 * t1.x, v[0].y - (R)0.5 * t1.y);
    const C t3 = mul_i<INV>(cscale(csub(v[1], v[2]), c));
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
  } else if constexpr (N == 4) {
    const C s02 = cadd(v[0], v[2]);
    const C d02 = csub(v[0], v[2]);
    const C s13 = cadd(v[1], v[3]);
    const C r13 = mul_i<INV>(csub(v[1], v[3]));
    v[0] = cadd(s02, s13);
    v[1] = cadd(d02, r13);
    v[2] = csub(s02, s13);
    v[3] = csub(d02, r13);
  } else if constexpr (N == 5) {
    const R c1 = (R)0.30901699437494742410;
    const R c2 = (R)-0.80901699437494742410;
    const R s1 = (R)0.95105651629515357212;
    const R s2 = (R)0.58778525229247312917;
    const C t1 = cadd(v[1], v[4]);
    const C t2 = cadd(v[2], v[3]);
    const C t3 = csub(v[1], v[4]);
    const C t4 = csub(v[2], v[3]);
    const C a1 = cmake<C>(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
    const C a2 = cmake<C>(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
    const C b1 = mul_i<INV>(cmake<C>(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
    const C b2 = mul_i<INV>(cmake<C>(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
    v[0] = cadd(v[0], cadd(t1, t2));
    v[1] = cadd(a1, b1);
    v[4] = csub(a1, b1);
    v[2] = cadd(a2, b2);
    v[3] = csub(a2, b2);
  } else if constexpr (N == 8) {
    // even/odd split into two 4-point DFTs, W_8 = (1 -/+ i) / sqrt(2)
    C e[4] = {v[0], v[2], v[4], v[6]};
    C o[4] = {v[1], v[3], v[5], v[7]};
    dft<R, 4, INV>(e);
    dft<R, 4, INV>(o);
    const R h = (R)0.70710678118654752440;
    const C o1 = INV ? cmake<C>(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y))
                     : cmake<C>(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
    const C o2 = mul_i<INV>(o[2]);
    const C o3 = INV ? cmake<C>(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y))
                     : cmake<C>(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);
    v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);
    v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);
    v[7] = csub(e[3], o3);
  } else if constexpr (coprime_split(N) != 0) {
    constexpr int N1 = coprime_split(N);
    dft_pfa<R, N1, N / N1, INV>(v);
  } else if constexpr (small_split(N) != 0) {
    constexpr int N1 = small_split(N);
    dft_fourstep<R, N1, N / N1, INV>(v);
  } else if constexpr (tw_offset(N) >= 0) {
    dft_odd<R, N, INV>(v);
  } else {
    // prime length without a table: direct DFT (only small primes reach here)
    static_assert(N <= 13, "unsupported register DFT length");
    C out[N];
#pragma unroll
    for (int q = 0; q < N; ++q) {
      C acc = v[0];
#pragma unroll
      for (int r = 1; r < N; ++r) {
        R s, c;
        sincospi((R)(2 * ((r * q) % N)) / (R)N, &s, &c);
        const C w = cmake<C>(c, INV ? s : -s);
        acc = cadd(acc, cmul(v[r], w));
      }
      out[q] = acc;
    }
#pragma unroll
    for (int q = 0; q < N; ++q) v[q] = out[q];
  }
}

// ------------------------------------------------------------ space axes

// One window's planes for the fast space kernels (host-side description,
// cut into PlaneBatch records).
template <typename R>
struct PlaneJob {
  const Cx<R> *src;  // forward: model planes [P..]; adjoint: Z planes [L..]
  Cx<R> *dst;        // forward: Z planes [L..]; adjoint: model planes (update)
  long src_plane;    // complex per input plane
  long dst_plane;    // complex per output plane
  int pid;           // problem of the window
};

// One batch of planes for the persistent space kernels: `count` planes
// starting at src (input planes) and dst (output planes), of the window of
// problem `pid` (independent problems solved together keep their own step
// size and threshold).
template <typename R>
struct PlaneBatch {
  const Cx<R> *src;
  Cx<R> *dst;
  int count;
  int pid;
};

template <typename R>
struct PlaneBatches {
  const PlaneBatch<R> *b;
  int n;
};

// Shape of the (t, f) planes one instantiation handles: D space axes of
// padded length P_d; the window length is L_d = 4 P_d / 5, the only length
// whose padded length ceil(1.25 L) is P_d for the instantiated sizes.
// Shared-memory layout [P0][P1][P2 + pad]: the last axis is padded to an odd
// length so threads walking different rows hit different banks.
template <int D, int P0, int P1, int P2>
struct PlaneShape {
  static constexpr int PL = D == 1 ? P0 : (D == 2 ? P1 : P2);  // last axis
  static constexpr int PLS = PL % 2 ? PL : PL + 1;            // padded
  static constexpr int E0 = D == 1 ? PLS : P0;
  static constexpr int E1 = D == 1 ? 1 : (D == 2 ? PLS : P1);
  static constexpr int E2 = D == 3 ? PLS : 1;
  static constexpr int S0 = E1 * E2;  // smem stride of axis 0 (D >= 2)
  static constexpr int S1 = E2;       // smem stride of axis 1 (D == 3)
  static constexpr int size = E0 * E1 * E2;  // complex per plane in smem
  static constexpr int L0 = P0 * 4 / 5;
  static constexpr int L1 = D >= 2 ? P1 * 4 / 5 : 1;
  static constexpr int L2 = D == 3 ? P2 * 4 / 5 : 1;
  static constexpr int Q1 = D >= 2 ? P1 : 1;
  static constexpr int Q2 = D == 3 ? P2 : 1;
  static constexpr int dense_P = P0 * Q1 * Q2;  // model plane
  static constexpr int dense_L = L0 * L1 * L2;  // cropped plane
};

// smem position of dense element e of a plane with extents (X0, X1, X2)
// (row-major, last axis fastest)
template <int D, int P0, int P1, int P2, int X1, int X2>
__device__ __forceinline__ int plane_pos(int e) {
  using S = PlaneShape<D, P0, P1, P2>;
  if constexpr (D == 1) {
    return e;
  } else if constexpr (D == 2) {
    const int i0 = e / X1;
    return i0 * S::E1 + (e - i0 * X1);
  } else {
    const int i0 = e / (X1 * X2);
    const int r = e - i0 * X1 * X2;
    const int i1 = r / X2;
    return i0 * S::E1 * S::E2 + i1 * S::E2 + (r - i1 * X2);
  }
}

// FFT of length N of the lines along one axis of np planes in smem: lines
// run over EO x EI positions of the other axes (smem strides SO, SI), line
// elements have stride SL; NIN elements are read (zero beyond), NOUT written.
template <typename R, int N, bool INV, int NT, int NP, int PLANE, int EO, int EI, int SO, int SL,
          int SI, int NIN, int NOUT>
__device__ __forceinline__ void lines_fft(Cx<R> *buf, int np) {
  using C = Cx<R>;
  constexpr int PER = EO * EI;
  const int total = np * PER;
  for (int l = threadIdx.x; l < total; l += NT) {
    const int p = l / PER;
    const int r = l - p * PER;
    const int o = r / EI;
    const int i = r - o * EI;
    C *line = buf + p * PLANE + o * SO + i * SI;
    C v[N];
#pragma unroll
    for (int e = 0; e < N; ++e) v[e] = e < NIN ? line[e * SL] : cmake<C>((R)0, (R)0);
    dft<R, N, INV>(v);
#pragma unroll
    for (int e = 0; e < NOUT; ++e) line[e * SL] = v[e];
  }
}

// All space axes of np planes: forward operator direction (inverse FFT with
// cropping, last axis first) or adjoint direction (zero-padding, forward FFT,
// first axis first).
template <typename R, int D, int P0, int P1, int P2, int NT, int NP, bool FWD>
__device__ __forceinline__ void space_axes(Cx<R> *buf, int np) {
  using S = PlaneShape<D, P0, P1, P2>;
  constexpr int Z = S::size;
  if constexpr (FWD) {
    if constexpr (D == 1) {
      lines_fft<R, P0, true, NT, NP, Z, 1, 1, 0, 1, 0, P0, S::L0>(buf, np);
    } else if constexpr (D == 2) {
      lines_fft<R, P1, true, NT, NP, Z, P0, 1, S::S0, 1, 0, P1, S::L1>(buf, np);
      __syncthreads();
      lines_fft<R, P0, true, NT, NP, Z, 1, S::L1, 0, S::S0, 1, P0, S::L0>(buf, np);
    } else {
      lines_fft<R, P2, true, NT, NP, Z, P0 * P1, 1, S::S1, 1, 0, P2, S::L2>(buf, np);
      __syncthreads();
      lines_fft<R, P1, true, NT, NP, Z, P0, S::L2, S::S0, S::S1, 1, P1, S::L1>(buf, np);
      __syncthreads();
      lines_fft<R, P0, true, NT, NP, Z, S::L1, S::L2, S::S1, S::S0, 1, P0, S::L0>(buf, np);
    }
  } else {
    if constexpr (D == 1) {
      lines_fft<R, P0, false, NT, NP, Z, 1, 1, 0, 1, 0, S::L0, P0>(buf, np);
    } else if constexpr (D == 2) {
      lines_fft<R, P0, false, NT, NP, Z, 1, S::L1, 0, S::S0, 1, S::L0, P0>(buf, np);
      __syncthreads();
      lines_fft<R, P1, false, NT, NP, Z, P0, 1, S::S0, 1, 0, S::L1, P1>(buf, np);
    } else {
      lines_fft<R, P0, false, NT, NP, Z, S::L1, S::L2, S::S1, S::S0, 1, S::L0, P0>(buf, np);
      __syncthreads();
      lines_fft<R, P1, false, NT, NP, Z, P0, S::L2, S::S0, S::S1, 1, S::L1, P1>(buf, np);
      __syncthreads();
      lines_fft<R, P2, false, NT, NP, Z, P0 * P1, 1, S::S1, 1, 0, S::L2, P2>(buf, np);
    }
  }
}

// Forward operator, all space axes: Z[L..] = crop(IFFT_space(X[P..])).
// Persistent blocks of NT threads walk batches of NP planes.  STAGES = 2:
// the planes of the next batch are copied into a second shared buffer
// (cp.async) while the current one is transformed (shared memory: 2 NP
// planes, one block per SM).  STAGES = 1: one buffer, refilled after each
// store; MINB blocks share an SM and overlap one another's copies.
template <typename R, int D, int P0, int P1, int P2, int NT, int NP, int STAGES, int MINB>
__global__ void __launch_bounds__(NT, MINB) space_fwd_fast(PlaneBatches<R> batches) {
  static_assert(STAGES == 1 || STAGES == 2, "one or two stages");
  using C = Cx<R>;
  using S = PlaneShape<D, P0, P1, P2>;
  constexpr int PL = S::PL;
  constexpr int PLS = S::PLS;
  constexpr int ROWS = S::dense_P / PL;  // model rows per plane
  static_assert(S::size == ROWS * PLS, "padded rows evenly spaced");
  constexpr int LL = PL * 4 / 5;         // cropped row
  constexpr int ORW = S::dense_L / LL;   // cropped rows per plane
  static_assert(LL % 2 == 0, "cropped rows of column pairs");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *stage[2] = {reinterpret_cast<C *>(smem_raw),
                 reinterpret_cast<C *>(smem_raw) + (STAGES == 2 ? NP * S::size : 0)};
  // copies in: thread -> (row, column) fixed, rows TR apart per sweep (the
  // model rows are dense, the padded rows PLS apart: no index division)
  constexpr int TR = NT / PL;
  const int lc = threadIdx.x % PL;
  const int lr = threadIdx.x / PL;
  auto issue = [&](const PlaneBatch<R> &bt, C *buf) {
    if (lr >= TR) return;
    const int nrows = bt.count * ROWS;
    const C *s = bt.src + lr * PL + lc;
    C *d = buf + lr * PLS + lc;
    for (int r = lr; r < nrows; r += TR, s += TR * PL, d += TR * PLS) cp_async<sizeof(C)>(d, s);
  };
  // copies out: column pairs of the cropped rows, 16-byte stores when the
  // batch's output is 16-byte aligned (float)
  constexpr int CW = LL / 2;
  constexpr int TS = NT / CW;
  const int sc = threadIdx.x % CW;
  const int sr = threadIdx.x / CW;
  const PlaneBatch<R> none{nullptr, nullptr, 0, 0};
  int b = blockIdx.x;
  PlaneBatch<R> cur = b < batches.n ? batches.b[b] : none;
  PlaneBatch<R> nxt = b + gridDim.x < batches.n ? batches.b[b + gridDim.x] : none;
  if (b < batches.n) issue(cur, stage[0]);
  cp_async_commit();
  for (int k = 0; b < batches.n; ++k, b += gridDim.x) {
    // batch records are loaded one batch ahead of their use
    const int b2 = b + 2 * gridDim.x;
    const PlaneBatch<R> after = b2 < batches.n ? batches.b[b2] : none;
    if constexpr (STAGES == 2) {
      if (nxt.count > 0) issue(nxt, stage[(k + 1) & 1]);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    C *buf = stage[STAGES == 2 ? (k & 1) : 0];
    const int np = cur.count;
    space_axes<R, D, P0, P1, P2, NT, NP, true>(buf, np);
    __syncthreads();
    C *dst = cur.dst;
    if (sr < TS) {
      const int nrows = np * ORW;
      const bool vec = sizeof(R) == sizeof(float) && (reinterpret_cast<uintptr_t>(dst) & 15) == 0;
      for (int r = sr; r < nrows; r += TS) {
        const int p = r / ORW;
        const int rem = r - p * ORW;
        int srow = p * ROWS + rem;  // padded row holding cropped row r
        if constexpr (D == 3) {
          const int i0 = rem / S::L1;
          srow = p * ROWS + i0 * P1 + (rem - i0 * S::L1);
        }
        const C g0 = buf[srow * PLS + 2 * sc];
        const C g1 = buf[srow * PLS + 2 * sc + 1];
        C *o = dst + (long)r * LL + 2 * sc;
        if (vec) {
          *reinterpret_cast<float4 *>(o) = make_float4((float)g0.x, (float)g0.y, (float)g1.x,
                                                       (float)g1.y);
        } else {
          o[0] = g0;
          o[1] = g1;
        }
      }
    }
    __syncthreads();
    if constexpr (STAGES == 1) {
      if (nxt.count > 0) issue(nxt, stage[0]);
      cp_async_commit();
    }
    cur = nxt;
    nxt = after;
  }
}

// Adjoint, all space axes, with the ISTA update fused:
// X <- soft_threshold(X - step * FFT_space(pad(G[L..])), lamb)   (epilogue
// kUpdateThreshold), X <- X - step * ..., tracking max |X|^2 (kUpdateMax), or
// X <- FFT_space(pad(G)) (kStore).  Persistent like the forward kernel.
// STAGES = 2: double buffered, and the model planes of the current batch are
// copied into a third buffer while its FFTs run (shared memory: 2 NP padded
// planes and NP dense planes).  STAGES = 1: one padded buffer; the epilogue
// reads the model planes from global memory, and MINB blocks share an SM.
// With step_dev (independent problems solved together) the step, the
// threshold (lamb_dev) and the tracked maximum (max_out) are per problem,
// indexed by the batch's pid.
template <typename R, int D, int P0, int P1, int P2, int NT, int NP, int STAGES, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    space_adj_fast(PlaneBatches<R> batches, int epilogue, R step_arg, R lamb_arg,
                   const R *step_dev, const R *lamb_dev, R *max_out) {
  static_assert(STAGES == 1 || STAGES == 2, "one or two stages");
  using C = Cx<R>;
  using S = PlaneShape<D, P0, P1, P2>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *base = reinterpret_cast<C *>(smem_raw);
  C *stage[2] = {base, base + (STAGES == 2 ? NP * S::size : 0)};
  C *xbuf = base + STAGES * NP * S::size;
  const bool need_x = epilogue != kStore;
  auto issue = [&](const PlaneBatch<R> &bt, C *buf) {
    const int n = bt.count * S::dense_L;
    for (int e = threadIdx.x; e < n; e += NT) {
      const int p = e / S::dense_L;
      cp_async<sizeof(C)>(buf + p * S::size + plane_pos<D, P0, P1, P2, S::L1, S::L2>(
                                                  e - p * S::dense_L),
                          bt.src + e);
    }
  };
  const bool multi = step_dev != nullptr;
  R local_max = (R)0;
  const PlaneBatch<R> none{nullptr, nullptr, 0, 0};
  int b = blockIdx.x;
  PlaneBatch<R> cur = b < batches.n ? batches.b[b] : none;
  PlaneBatch<R> nxt = b + gridDim.x < batches.n ? batches.b[b + gridDim.x] : none;
  if (b < batches.n) issue(cur, stage[0]);
  cp_async_commit();
  for (int k = 0; b < batches.n; ++k, b += gridDim.x) {
    const int b2 = b + 2 * gridDim.x;
    const PlaneBatch<R> after = b2 < batches.n ? batches.b[b2] : none;
    if constexpr (STAGES == 2) {
      if (nxt.count > 0) issue(nxt, stage[(k + 1) & 1]);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const int np = cur.count;
    C *dst = cur.dst;
    const int n_store = np * S::dense_P;
    // lambda from device memory when replayed from a CUDA graph
    const R step = multi ? step_dev[cur.pid] : step_arg;
    const R lamb = lamb_dev != nullptr ? lamb_dev[multi ? cur.pid : 0] : lamb_arg;
    const R lamb_sq = lamb * lamb;
    if constexpr (STAGES == 2) {
      if (need_x) {
        for (int e = threadIdx.x; e < n_store; e += NT) cp_async<sizeof(C)>(xbuf + e, dst + e);
      }
      cp_async_commit();
    }
    C *buf = stage[STAGES == 2 ? (k & 1) : 0];
    space_axes<R, D, P0, P1, P2, NT, NP, false>(buf, np);
    if constexpr (STAGES == 2) cp_async_wait<0>();
    __syncthreads();
    // two consecutive elements per thread in 16-byte vectors when the model
    // is 16-byte aligned (float; rows have even length, so elements 2q and
    // 2q + 1 share a row of the padded plane)
    const bool vec = sizeof(R) == sizeof(float) && (reinterpret_cast<uintptr_t>(dst) & 15) == 0;
    const int n_vec = vec ? n_store / 2 : 0;
#pragma unroll 2
    for (int q = threadIdx.x; q < n_vec; q += NT) {
      const int e = 2 * q;
      const int p = e / S::dense_P;
      const int pos = p * S::size + plane_pos<D, P0, P1, P2, S::Q1, S::Q2>(e - p * S::dense_P);
      const C g0 = buf[pos];
      const C g1 = buf[pos + 1];
      float4 *d4 = reinterpret_cast<float4 *>(dst) + q;
      if (epilogue == kStore) {
        *d4 = make_float4((float)g0.x, (float)g0.y, (float)g1.x, (float)g1.y);
        continue;
      }
      const float4 xv = STAGES == 2 ? reinterpret_cast<const float4 *>(xbuf)[q] : *d4;
      C n0 = cmake<C>(sub_rn<R>((R)xv.x, mul_rn<R>(step, g0.x)),
                      sub_rn<R>((R)xv.y, mul_rn<R>(step, g0.y)));
      C n1 = cmake<C>(sub_rn<R>((R)xv.z, mul_rn<R>(step, g1.x)),
                      sub_rn<R>((R)xv.w, mul_rn<R>(step, g1.y)));
      if (epilogue == kUpdateThreshold) {
        n0 = soft_threshold<R>(n0, lamb, lamb_sq);
        n1 = soft_threshold<R>(n1, lamb, lamb_sq);
      } else {
        const R a0 = abs_sq<R>(n0);
        const R a1 = abs_sq<R>(n1);
        local_max = a0 > local_max ? a0 : local_max;
        local_max = a1 > local_max ? a1 : local_max;
      }
      *d4 = make_float4((float)n0.x, (float)n0.y, (float)n1.x, (float)n1.y);
    }
    for (int e = vec ? n_store : threadIdx.x; e < n_store; e += NT) {
      const int p = e / S::dense_P;
      const C g = buf[p * S::size + plane_pos<D, P0, P1, P2, S::Q1, S::Q2>(e - p * S::dense_P)];
      if (epilogue == kStore) {
        dst[e] = g;
      } else {
        const C x = STAGES == 2 ? xbuf[e] : dst[e];
        C xn = cmake<C>(sub_rn<R>(x.x, mul_rn<R>(step, g.x)),
                        sub_rn<R>(x.y, mul_rn<R>(step, g.y)));
        if (epilogue == kUpdateThreshold) {
          xn = soft_threshold<R>(xn, lamb, lamb_sq);
        } else {
          const R a2 = abs_sq<R>(xn);
          local_max = a2 > local_max ? a2 : local_max;
        }
        dst[e] = xn;
      }
    }
    __syncthreads();
    if (multi && epilogue == kUpdateMax) {  // one maximum per problem
      __shared__ R red_b[32];
      const R m = block_max<R>(local_max, red_b);
      if (threadIdx.x == 0) atomic_max_nonneg(max_out + cur.pid, m);
      local_max = (R)0;
    }
    if constexpr (STAGES == 1) {
      if (nxt.count > 0) issue(nxt, stage[0]);
      cp_async_commit();
    }
    cur = nxt;
    nxt = after;
  }
  if (!multi && epilogue == kUpdateMax) {
    __shared__ R red[32];
    const R m = block_max<R>(local_max, red);
    if (threadIdx.x == 0) atomic_max_nonneg(max_out, m);
  }
}

// ------------------------------------------------------------ row-fused space kernels

// One row of N complex values from global memory, in 16-byte vectors when
// `vec` (float, even N, a 16-byte aligned row; windows of odd model size
// leave the next windows' rows at odd complex offsets).
template <typename R, int N>
__device__ __forceinline__ void load_row(Cx<R> (&v)[N], const Cx<R> *src, bool vec) {
  if (sizeof(R) == sizeof(float) && N % 2 == 0 && vec) {
    const float4 *s4 = reinterpret_cast<const float4 *>(src);
#pragma unroll
    for (int k = 0; k < N / 2; ++k) {
      const float4 q = s4[k];
      v[2 * k] = cmake<Cx<R>>(q.x, q.y);
      v[2 * k + 1] = cmake<Cx<R>>(q.z, q.w);
    }
  } else {
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = src[k];
  }
}

// Forward operator, all space axes, with the first pass (last axis) reading
// each model row straight from global memory into registers: no staging of
// the model planes in shared memory.  The remaining axes and the store of
// the cropped planes are those of space_fwd_fast.  MINB blocks per SM
// overlap one another's loads.
template <typename R, int D, int P0, int P1, int P2, int NT, int NP, int MINB>
__global__ void __launch_bounds__(NT, MINB) space_fwd_rows(PlaneBatches<R> batches) {
  using C = Cx<R>;
  using S = PlaneShape<D, P0, P1, P2>;
  constexpr int Z = S::size;
  constexpr int PL = S::PL;                      // last-axis padded length
  constexpr int LL = PL * 4 / 5;                 // its window length
  constexpr int ROWS = S::dense_P / PL;          // rows per model plane
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  for (int b = blockIdx.x; b < batches.n; b += gridDim.x) {
    const PlaneBatch<R> bt = batches.b[b];
    const int np = bt.count;
    // rows are PL (even) apart within a window: one alignment test per batch
    const bool vec = (reinterpret_cast<uintptr_t>(bt.src) & 15) == 0;
    for (int r = threadIdx.x; r < np * ROWS; r += NT) {
      const int p = r / ROWS;
      const int q = r - p * ROWS;
      C v[PL];
      load_row<R, PL>(v, bt.src + (long)p * S::dense_P + (long)q * PL, vec);
      dft<R, PL, true>(v);
      C *row = buf + p * Z + q * S::PLS;
#pragma unroll
      for (int e = 0; e < LL; ++e) row[e] = v[e];
    }
    __syncthreads();
    if constexpr (D == 2) {
      lines_fft<R, P0, true, NT, NP, Z, 1, S::L1, 0, S::S0, 1, P0, S::L0>(buf, np);
      __syncthreads();
    } else if constexpr (D == 3) {
      lines_fft<R, P1, true, NT, NP, Z, P0, S::L2, S::S0, S::S1, 1, P1, S::L1>(buf, np);
      __syncthreads();
      lines_fft<R, P0, true, NT, NP, Z, S::L1, S::L2, S::S1, S::S0, 1, P0, S::L0>(buf, np);
      __syncthreads();
    }
    C *dst = bt.dst;
    const int n_store = np * S::dense_L;
    for (int e = threadIdx.x; e < n_store; e += NT) {
      const int p = e / S::dense_L;
      dst[e] = buf[p * Z + plane_pos<D, P0, P1, P2, S::L1, S::L2>(e - p * S::dense_L)];
    }
    __syncthreads();
  }
}

// Adjoint, all space axes, with the update fused into the last pass: that
// pass runs along the contiguous axis, so each thread's P outputs are one
// row of the model plane, which it reads, updates (epilogues as
// space_adj_fast) and writes back in 16-byte vectors.  The padded planes of
// the intermediate are staged as in space_adj_fast (STAGES 1 or 2); no model
// staging buffer.
template <typename R, int D, int P0, int P1, int P2, int NT, int NP, int STAGES, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    space_adj_rows(PlaneBatches<R> batches, int epilogue, R step_arg, R lamb_arg,
                   const R *step_dev, const R *lamb_dev, R *max_out) {
  static_assert(STAGES == 1 || STAGES == 2, "one or two stages");
  using C = Cx<R>;
  using S = PlaneShape<D, P0, P1, P2>;
  constexpr int Z = S::size;
  constexpr int PL = S::PL;
  constexpr int LL = PL * 4 / 5;
  constexpr int ROWS = S::dense_P / PL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *base = reinterpret_cast<C *>(smem_raw);
  C *stage[2] = {base, base + (STAGES == 2 ? NP * Z : 0)};
  auto issue = [&](const PlaneBatch<R> &bt, C *buf) {
    const int n = bt.count * S::dense_L;
    for (int e = threadIdx.x; e < n; e += NT) {
      const int p = e / S::dense_L;
      cp_async<sizeof(C)>(buf + p * Z + plane_pos<D, P0, P1, P2, S::L1, S::L2>(
                                            e - p * S::dense_L),
                          bt.src + e);
    }
  };
  const bool multi = step_dev != nullptr;
  R local_max = (R)0;
  const PlaneBatch<R> none{nullptr, nullptr, 0, 0};
  int b = blockIdx.x;
  PlaneBatch<R> cur = b < batches.n ? batches.b[b] : none;
  PlaneBatch<R> nxt = b + gridDim.x < batches.n ? batches.b[b + gridDim.x] : none;
  if (b < batches.n) issue(cur, stage[0]);
  cp_async_commit();
  for (int k = 0; b < batches.n; ++k, b += gridDim.x) {
    const int b2 = b + 2 * gridDim.x;
    const PlaneBatch<R> after = b2 < batches.n ? batches.b[b2] : none;
    if constexpr (STAGES == 2) {
      if (nxt.count > 0) issue(nxt, stage[(k + 1) & 1]);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const int np = cur.count;
    C *buf = stage[STAGES == 2 ? (k & 1) : 0];
    if constexpr (D == 2) {
      lines_fft<R, P0, false, NT, NP, Z, 1, S::L1, 0, S::S0, 1, S::L0, P0>(buf, np);
      __syncthreads();
    } else if constexpr (D == 3) {
      lines_fft<R, P0, false, NT, NP, Z, S::L1, S::L2, S::S1, S::S0, 1, S::L0, P0>(buf, np);
      __syncthreads();
      lines_fft<R, P1, false, NT, NP, Z, P0, S::L2, S::S0, S::S1, 1, S::L1, P1>(buf, np);
      __syncthreads();
    }
    const R step = multi ? step_dev[cur.pid] : step_arg;
    const R lamb = lamb_dev != nullptr ? lamb_dev[multi ? cur.pid : 0] : lamb_arg;
    const R lamb_sq = lamb * lamb;
    // rows are PL (even) apart within a window: one alignment test per batch
    const bool vec = sizeof(R) == sizeof(float) && (reinterpret_cast<uintptr_t>(cur.dst) & 15) == 0;
    for (int r = threadIdx.x; r < np * ROWS; r += NT) {
      const int p = r / ROWS;
      const int q = r - p * ROWS;
      const C *row = buf + p * Z + q * S::PLS;
      C v[PL];
#pragma unroll
      for (int e = 0; e < PL; ++e) v[e] = e < LL ? row[e] : cmake<C>((R)0, (R)0);
      dft<R, PL, false>(v);
      C *xr = cur.dst + (long)p * S::dense_P + (long)q * PL;
      if (epilogue == kStore) {
#pragma unroll
        for (int e = 0; e < PL; ++e) xr[e] = v[e];
        continue;
      }
#pragma unroll
      for (int e = 0; e < PL; e += 2) {
        C x0, x1;
        if (vec) {
          const float4 q4 = *reinterpret_cast<const float4 *>(xr + e);
          x0 = cmake<C>((R)q4.x, (R)q4.y);
          x1 = cmake<C>((R)q4.z, (R)q4.w);
        } else {
          x0 = xr[e];
          x1 = xr[e + 1];
        }
        C n0 = cmake<C>(sub_rn<R>(x0.x, mul_rn<R>(step, v[e].x)),
                        sub_rn<R>(x0.y, mul_rn<R>(step, v[e].y)));
        C n1 = cmake<C>(sub_rn<R>(x1.x, mul_rn<R>(step, v[e + 1].x)),
                        sub_rn<R>(x1.y, mul_rn<R>(step, v[e + 1].y)));
        if (epilogue == kUpdateThreshold) {
          n0 = soft_threshold<R>(n0, lamb, lamb_sq);
          n1 = soft_threshold<R>(n1, lamb, lamb_sq);
        } else {
          const R a0 = abs_sq<R>(n0);
          const R a1 = abs_sq<R>(n1);
          local_max = a0 > local_max ? a0 : local_max;
          local_max = a1 > local_max ? a1 : local_max;
        }
        if (vec) {
          *reinterpret_cast<float4 *>(xr + e) =
              make_float4((float)n0.x, (float)n0.y, (float)n1.x, (float)n1.y);
        } else {
          xr[e] = n0;
          xr[e + 1] = n1;
        }
      }
    }
    __syncthreads();
    if (multi && epilogue == kUpdateMax) {  // one maximum per problem
      __shared__ R red_b[32];
      const R m = block_max<R>(local_max, red_b);
      if (threadIdx.x == 0) atomic_max_nonneg(max_out + cur.pid, m);
      local_max = (R)0;
    }
    if constexpr (STAGES == 1) {
      if (nxt.count > 0) issue(nxt, stage[0]);
      cp_async_commit();
    }
    cur = nxt;
    nxt = after;
  }
  if (!multi && epilogue == kUpdateMax) {
    __shared__ R red[32];
    const R m = block_max<R>(local_max, red);
    if (threadIdx.x == 0) atomic_max_nonneg(max_out, m);
  }
}

// Line FFTs from one buffer into another: lines over EO x EI positions of
// np planes, source strides (plane SPL, outer SSO, line SSL, inner SSI),
// destination strides (DPL, DSO, DSL, DSI); NIN elements read (zero beyond),
// NOUT written.
template <typename R, int N, bool INV, int NT, int EO, int EI, int SPL, int SSO, int SSL,
          int SSI, int DPL, int DSO, int DSL, int DSI, int NIN, int NOUT>
__device__ __forceinline__ void lines_fft_copy(const Cx<R> *src, Cx<R> *dst, int np) {
  using C = Cx<R>;
  constexpr int PER = EO * EI;
  const int total = np * PER;
  for (int l = threadIdx.x; l < total; l += NT) {
    const int p = l / PER;
    const int r = l - p * PER;
    const int o = r / EI;
    const int i = r - o * EI;
    const C *s = src + p * SPL + o * SSO + i * SSI;
    C *d = dst + p * DPL + o * DSO + i * DSI;
    C v[N];
#pragma unroll
    for (int e = 0; e < N; ++e) v[e] = e < NIN ? s[e * SSL] : cmake<C>((R)0, (R)0);
    dft<R, N, INV>(v);
#pragma unroll
    for (int e = 0; e < NOUT; ++e) d[e * DSL] = v[e];
  }
}

// Adjoint, all space axes, with the ISTA update fused (epilogues as
// space_adj_fast), pipelined: the cropped input planes of a batch are copied
// densely (16-byte cp.async where aligned) into a staging buffer; the first
// pass (axis 0, zero-padding L0 -> P0) reads them from there into the padded
// work buffer, after which the staging buffer takes the next batch's copies
// while the remaining passes and the update run.  The update walks the model
// rows (the contiguous axis, PL elements) with a fixed thread -> (row,
// 16-byte column) map: padded rows sit PLS apart in the work buffer and PL
// apart in the model, so no index division is needed.  The model planes
// come either from registers (XS false: each thread keeps U loads in
// flight, the first U issued before the last pass) or from a third shared
// buffer filled by cp.async at the start of the batch, behind all three
// passes (XS true).  Shared memory: NP dense cropped planes, NP padded
// planes (and NP dense model planes).
template <typename R, int D, int P0, int P1, int P2, int NT, int NP, int MINB, bool XS>
__global__ void __launch_bounds__(NT, MINB)
    space_adj_pipe(PlaneBatches<R> batches, int epilogue, R step_arg, R lamb_arg,
                   const R *step_dev, const R *lamb_dev, R *max_out) {
  using C = Cx<R>;
  using S = PlaneShape<D, P0, P1, P2>;
  constexpr int Z = S::size;
  constexpr int PL = S::PL;
  constexpr int PLS = S::PLS;
  constexpr int ROWS = S::dense_P / PL;
  static_assert(Z == ROWS * PLS, "padded rows evenly spaced");
  constexpr int CW = PL / 2;               // 16-byte columns of a row (float)
  constexpr int TR = NT / CW;              // rows per sweep
  // model loads in flight per thread (XS false), and whether the first ones
  // are issued before the last pass, from the register budget
  constexpr int kRegs = 65536 / (NT * MINB);
  constexpr int U = XS ? 1 : (kRegs >= 120 && PL <= 20 ? 8 : 4);
  constexpr bool kEarly = !XS && D > 1 && 2 * PL + 4 * U + 24 <= kRegs;
  constexpr bool kVec = sizeof(R) == sizeof(float) && PL % 2 == 0;
  constexpr int kStg = NP * S::dense_L + (NP * S::dense_L) % 2;  // 16-byte aligned
  constexpr int kWork = NP * Z + (NP * Z) % 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *stg = reinterpret_cast<C *>(smem_raw);
  C *work = stg + kStg;
  C *xbuf = work + kWork;  // XS only
  auto copy_in = [&](C *to, const C *from, int n) {
    if (sizeof(C) == 8 && n % 2 == 0 && (reinterpret_cast<uintptr_t>(from) & 15) == 0) {
      for (int e = threadIdx.x; e < n / 2; e += NT) cp_async<16>(to + 2 * e, from + 2 * e);
    } else {
      for (int e = threadIdx.x; e < n; e += NT) cp_async<sizeof(C)>(to + e, from + e);
    }
  };
  const bool multi = step_dev != nullptr;
  const bool need_x = epilogue != kStore;
  R local_max = (R)0;
  const int col = threadIdx.x % CW;
  const int rr = threadIdx.x / CW;
  const bool lane_on = rr < TR;
  const PlaneBatch<R> none{nullptr, nullptr, 0, 0};
  int b = blockIdx.x;
  PlaneBatch<R> cur = b < batches.n ? batches.b[b] : none;
  PlaneBatch<R> nxt = b + gridDim.x < batches.n ? batches.b[b + gridDim.x] : none;
  if (b < batches.n) copy_in(stg, cur.src, cur.count * S::dense_L);
  cp_async_commit();
  for (; b < batches.n; b += gridDim.x) {
    const int b2 = b + 2 * gridDim.x;
    const PlaneBatch<R> after = b2 < batches.n ? batches.b[b2] : none;
    const int np = cur.count;
    C *dst = cur.dst;
    if constexpr (XS) {
      // model planes of this batch, behind the three passes (group order:
      // staging of this batch, model of this batch, staging of the next)
      if (need_x) copy_in(xbuf, dst, np * S::dense_P);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    // first pass: staging (dense L planes) -> work (padded P planes)
    if constexpr (D == 1) {
      lines_fft_copy<R, P0, false, NT, 1, 1, S::dense_L, 0, 1, 0, Z, 0, 1, 0, S::L0, P0>(
          stg, work, np);
    } else if constexpr (D == 2) {
      lines_fft_copy<R, P0, false, NT, 1, S::L1, S::dense_L, 0, S::L1, 1, Z, 0, S::S0, 1, S::L0,
                     P0>(stg, work, np);
    } else {
      lines_fft_copy<R, P0, false, NT, S::L1, S::L2, S::dense_L, S::L2, S::L1 * S::L2, 1, Z,
                     S::S1, S::S0, 1, S::L0, P0>(stg, work, np);
    }
    __syncthreads();
    if (nxt.count > 0) copy_in(stg, nxt.src, nxt.count * S::dense_L);
    cp_async_commit();
    const R step = multi ? step_dev[cur.pid] : step_arg;
    const R lamb = lamb_dev != nullptr ? lamb_dev[multi ? cur.pid : 0] : lamb_arg;
    const R lamb_sq = lamb * lamb;
    if constexpr (D == 3) {
      lines_fft<R, P1, false, NT, NP, Z, P0, S::L2, S::S0, S::S1, 1, S::L1, P1>(work, np);
      __syncthreads();
    }
    const int nrows = np * ROWS;
    const bool vec = kVec && (reinterpret_cast<uintptr_t>(dst) & 15) == 0;
    float4 xv[U];
    auto load_x = [&](int r0) {
#pragma unroll
      for (int j = 0; j < U; ++j) {
        const int r = r0 + rr + TR * j;
        if (lane_on && r < nrows)
          xv[j] = reinterpret_cast<const float4 *>(XS ? xbuf : dst)[r * CW + col];
      }
    };
    if (kEarly && vec && need_x) load_x(0);
    // last pass (contiguous axis) in the work buffer
    if constexpr (D == 2) {
      lines_fft<R, P1, false, NT, NP, Z, P0, 1, S::S0, 1, 0, S::L1, P1>(work, np);
    } else if constexpr (D == 3) {
      lines_fft<R, P2, false, NT, NP, Z, P0 * P1, 1, S::S1, 1, 0, S::L2, P2>(work, np);
    }
    if constexpr (XS) cp_async_wait<1>();  // this batch's model planes
    __syncthreads();
    if (vec) {
      for (int r0 = 0; r0 < nrows; r0 += TR * U) {
        if ((r0 > 0 || !kEarly) && need_x) load_x(r0);
#pragma unroll
        for (int j = 0; j < U; ++j) {
          const int r = r0 + rr + TR * j;
          if (!lane_on || r >= nrows) continue;
          const C g0 = work[r * PLS + 2 * col];
          const C g1 = work[r * PLS + 2 * col + 1];
          float4 *d4 = reinterpret_cast<float4 *>(dst) + r * CW + col;
          if (!need_x) {
            *d4 = make_float4((float)g0.x, (float)g0.y, (float)g1.x, (float)g1.y);
            continue;
          }
          C n0 = cmake<C>(sub_rn<R>((R)xv[j].x, mul_rn<R>(step, g0.x)),
                          sub_rn<R>((R)xv[j].y, mul_rn<R>(step, g0.y)));
          C n1 = cmake<C>(sub_rn<R>((R)xv[j].z, mul_rn<R>(step, g1.x)),
                          sub_rn<R>((R)xv[j].w, mul_rn<R>(step, g1.y)));
          if (epilogue == kUpdateThreshold) {
            n0 = soft_threshold<R>(n0, lamb, lamb_sq);
            n1 = soft_threshold<R>(n1, lamb, lamb_sq);
          } else {
            const R a0 = abs_sq<R>(n0);
            const R a1 = abs_sq<R>(n1);
            local_max = a0 > local_max ? a0 : local_max;
            local_max = a1 > local_max ? a1 : local_max;
          }
          *d4 = make_float4((float)n0.x, (float)n0.y, (float)n1.x, (float)n1.y);
        }
      }
    } else {
      const int n_store = nrows * PL;
      for (int e = threadIdx.x; e < n_store; e += NT) {
        const int r = e / PL;
        const C g = work[r * PLS + (e - r * PL)];
        if (!need_x) {
          dst[e] = g;
          continue;
        }
        const C x = XS ? xbuf[e] : dst[e];
        C xn = cmake<C>(sub_rn<R>(x.x, mul_rn<R>(step, g.x)),
                        sub_rn<R>(x.y, mul_rn<R>(step, g.y)));
        if (epilogue == kUpdateThreshold) {
          xn = soft_threshold<R>(xn, lamb, lamb_sq);
        } else {
          const R a2 = abs_sq<R>(xn);
          local_max = a2 > local_max ? a2 : local_max;
        }
        dst[e] = xn;
      }
    }
    __syncthreads();
    if (multi && epilogue == kUpdateMax) {  // one maximum per problem
      __shared__ R red_b[32];
      const R m = block_max<R>(local_max, red_b);
      if (threadIdx.x == 0) atomic_max_nonneg(max_out + cur.pid, m);
      local_max = (R)0;
    }
    cur = nxt;
    nxt = after;
  }
  cp_async_wait<0>();
  if (!multi && epilogue == kUpdateMax) {
    __shared__ R red[32];
    const R m = block_max<R>(local_max, red);
    if (threadIdx.x == 0) atomic_max_nonneg(max_out, m);
  }
}

// ------------------------------------------------------------ time axis

// Twiddles W_N^k, k < N, copied to shared memory for lookups whose index
// differs between threads (constant memory serialises such accesses).
template <typename R, int N>
__device__ __forceinline__ void load_twiddles(Cx<R> *tw) {
  for (int k = threadIdx.x; k < N; k += blockDim.x) tw[k] = ctw<R>(tw_offset(N) + k);
}

template <bool INV, typename C>
__device__ __forceinline__ C tw_at(const C *tw, int k) {
  C w = tw[k];
  if (INV) w.y = -w.y;
  return w;
}

// Four-step FFT of length M = M1 * M2 on nl lines of shared memory (line
// stride LS), twiddles W_M from shared memory.  Output X[k1 + M1 k2] is left
// at position M2 k1 + k2.
template <typename R, int M1, int M2, bool INV>
__device__ __forceinline__ void lines_fourstep(Cx<R> *buf, int nl, int LS, const Cx<R> *twM) {
  using C = Cx<R>;
  constexpr int M = M1 * M2;
  for (int w = threadIdx.x; w < nl * M2; w += blockDim.x) {
    const int line = w / M2;
    const int n2 = w - line * M2;
    C *b = buf + line * LS;
    C v[M1];
#pragma unroll
    for (int n1 = 0; n1 < M1; ++n1) v[n1] = b[M2 * n1 + n2];
    dft<R, M1, INV>(v);
#pragma unroll
    for (int k1 = 0; k1 < M1; ++k1)
      b[M2 * k1 + n2] = (k1 == 0) ? v[0] : cmul(v[k1], tw_at<INV>(twM, (n2 * k1) % M));
  }
  __syncthreads();
  for (int w = threadIdx.x; w < nl * M1; w += blockDim.x) {
    const int line = w / M1;
    const int k1 = w - line * M1;
    C *b = buf + line * LS + M2 * k1;
    C v[M2];
#pragma unroll
    for (int n2 = 0; n2 < M2; ++n2) v[n2] = b[n2];
    dft<R, M2, INV>(v);
#pragma unroll
    for (int k2 = 0; k2 < M2; ++k2) b[k2] = v[k2];
  }
  __syncthreads();
}

template <int M1, int M2>
__device__ __forceinline__ int fourstep_pos(int k) {
  return M2 * (k % M1) + k / M1;
}

// Forward time axis for Pt = 2 M (M = M1 M2) and Lt = 2 h with h = 4 M / 5
// (the window length whose padded length is Pt): per trace and time window,
// c2r of the F = M + 1 bins through a length-M complex FFT, then taper and
// overlap-add; segment [t h, (t+1) h) of a trace is final once window t is
// added, so only a one-hop carry stays in shared memory.  Blocks own NB
// traces; the bins of window t + 1 are copied in (cp.async) while window t is
// processed.  Lines of the F = M + 1 bins are LS >= F apart in shared memory
// (a padded stride spreads the four-step accesses over the banks); MINB
// blocks share an SM.
template <typename R, int M1, int M2, int NB, int LS, int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
    time_fwd_fast(const TimeJob<R> *__restrict__ jobs, const int *__restrict__ cta_job,
                  const int *__restrict__ cta_trace0) {
  using C = Cx<R>;
  constexpr int M = M1 * M2;
  constexpr int F = M + 1;  // bins per line
  static_assert(LS >= F, "line stride");
  constexpr int H = 4 * M / 5;
  constexpr int HALF = M / 2 + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ C twM[M];
  __shared__ C tw2M[2 * M];
  __shared__ R taper[2 * H];
  __shared__ R scale[NB];
  load_twiddles<R, M>(twM);
  load_twiddles<R, 2 * M>(tw2M);
  const TimeJob<R> job = jobs[cta_job[blockIdx.x]];
  const int t0 = cta_trace0[blockIdx.x];
  const int nb = min(NB, job.n_traces - t0);
  const long ntr = job.n_traces;
  for (int j = threadIdx.x; j < 2 * H; j += kThreads) taper[j] = job.time_taper[j];
  for (int i = threadIdx.x; i < NB; i += kThreads) scale[i] = i < nb ? job.space_scale[t0 + i] : (R)0;
  C *stage[2] = {reinterpret_cast<C *>(smem_raw), reinterpret_cast<C *>(smem_raw) + NB * LS};
  R *carry = reinterpret_cast<R *>(stage[1] + NB * LS);  // [NB][H]
  auto issue = [&](int t, C *buf) {
    const C *zt = job.z + (long)t * F * ntr + t0;
    for (int idx = threadIdx.x; idx < NB * F; idx += kThreads) {
      const int f = idx / NB;
      const int i = idx - f * NB;
      if (i < nb) cp_async<sizeof(C)>(buf + i * LS + f, zt + f * ntr + i);
    }
  };
  for (int i = threadIdx.x; i < NB * H; i += kThreads) carry[i] = (R)0;
  issue(0, stage[0]);
  cp_async_commit();
  for (int t = 0; t < job.T; ++t) {
    if (t + 1 < job.T) issue(t + 1, stage[(t + 1) & 1]);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    C *buf = stage[t & 1];
    // Hermitian combine into M complex values (pairs k, M - k per thread):
    // Z_k = (X_k + conj X_{M-k}) + i e^{+2 pi i k / Pt} (X_k - conj X_{M-k})
    for (int w = threadIdx.x; w < NB * HALF; w += kThreads) {
      const int i = w / HALF;
      const int k = w - i * HALF;
      C *b = buf + i * LS;
      const int kk = M - k;
      C xa = b[k];
      C xb = b[kk];
      if (k == 0) {
        xa.y = (R)0;
        xb.y = (R)0;
      }
      auto comb = [&](C a, C bc_src, int kidx) {
        const C bc = cmake<C>(bc_src.x, -bc_src.y);
        const C e = cadd(a, bc);
        const C d = csub(a, bc);
        const C o = cmul(d, tw_at<true>(tw2M, kidx));
        return cmake<C>(e.x - o.y, e.y + o.x);
      };
      const C za = comb(xa, xb, k);
      if (k != 0 && k != kk) b[kk] = comb(xb, xa, kk);
      b[k] = za;  // k == 0 pairs with the Nyquist bin, which is then unused
    }
    __syncthreads();
    lines_fourstep<R, M1, M2, true>(buf, NB, LS, twM);
    // taper, overlap-add, write the completed segment of each trace; one
    // thread owns samples j and j + H, so the carry is read then rewritten
    // by the same thread
    for (int idx = threadIdx.x; idx < NB * H; idx += kThreads) {
      const int i = idx / H;
      const int j = idx - i * H;
      if (i < nb) {
        const R sc = scale[i];
        const C z_lo = buf[i * LS + fourstep_pos<M1, M2>(j >> 1)];
        const C z_hi = buf[i * LS + fourstep_pos<M1, M2>((j + H) >> 1)];
        const R u_lo = (j & 1) ? z_lo.y : z_lo.x;
        const R u_hi = ((j + H) & 1) ? z_hi.y : z_hi.x;
        job.y[(long)(t0 + i) * job.C + t * H + j] = carry[idx] + (u_lo * sc) * taper[j];
        carry[idx] = (u_hi * sc) * taper[j + H];
      }
    }
    __syncthreads();
  }
  // last half window and the zero tail up to C
  for (int idx = threadIdx.x; idx < NB * H; idx += kThreads) {
    const int i = idx / H;
    if (i < nb) job.y[(long)(t0 + i) * job.C + job.T * H + (idx - i * H)] = carry[idx];
  }
  const int tail = job.C - (job.T + 1) * H;
  for (int idx = threadIdx.x; idx < nb * tail; idx += kThreads) {
    const int i = idx / tail;
    const int j = idx - i * tail;
    job.y[(long)(t0 + i) * job.C + (job.T + 1) * H + j] = (R)0;
  }
}

// Adjoint time axis for Pt = 2 M and Lt = 2 h, h = 4 M / 5: per trace and
// window, gather Lt samples (record through the blend coordinates, or the
// trace buffer), taper, pack pairs into M complex values, forward FFT, split
// into the M + 1 bins and double bins 1..M-1.  The raw samples of window
// t + 1 are copied in (cp.async, zero-filled outside the blended span) while
// window t is transformed.  Line stride LS >= M + 1 and MINB as in
// time_fwd_fast.
template <typename R, int M1, int M2, int NB, int LS, int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
    time_adj_fast(const TimeJob<R> *__restrict__ jobs, const int *__restrict__ cta_job,
                  const int *__restrict__ cta_trace0, const R *__restrict__ record,
                  int from_record) {
  using C = Cx<R>;
  constexpr int M = M1 * M2;
  constexpr int F = M + 1;  // bins per line
  static_assert(LS >= F, "line stride");
  constexpr int H = 4 * M / 5;
  constexpr int LT = 2 * H;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ C twM[M];
  __shared__ C tw2M[2 * M];
  __shared__ long span_base[NB];  // source index of trace sample 0
  __shared__ int span_lo[NB], span_hi[NB];  // readable trace samples [lo, hi)
  __shared__ R scale[NB];
  __shared__ R taper[LT];
  load_twiddles<R, M>(twM);
  load_twiddles<R, 2 * M>(tw2M);
  const TimeJob<R> job = jobs[cta_job[blockIdx.x]];
  const int t0 = cta_trace0[blockIdx.x];
  const int nb = min(NB, job.n_traces - t0);
  const long ntr = job.n_traces;
  for (int j = threadIdx.x; j < LT; j += kThreads) taper[j] = job.time_taper[j];
  for (int i = threadIdx.x; i < NB; i += kThreads) {
    const int tr = t0 + i;
    span_lo[i] = 0;
    span_hi[i] = 0;
    span_base[i] = 0;
    scale[i] = (R)0;
    if (i >= nb) continue;
    scale[i] = job.space_scale[tr];
    if (from_record) {
      const long rec = job.blend_rec[tr];
      const int ts = job.blend_ts[tr];
      span_base[i] = rec - ts;
      span_lo[i] = rec >= 0 ? ts : 0;
      span_hi[i] = rec >= 0 ? ts + job.blend_n[tr] : 0;
    } else {
      span_base[i] = (long)tr * job.C;
      span_hi[i] = job.C;
    }
  }
  __syncthreads();
  const R *src_base = from_record ? record : job.y;
  C *line = reinterpret_cast<C *>(smem_raw);
  R *raw[2] = {reinterpret_cast<R *>(line + NB * LS), reinterpret_cast<R *>(line + NB * LS) + NB * LT};
  auto issue = [&](int t, R *rb) {
    // four consecutive samples per thread and step
    for (int g = threadIdx.x; g < NB * (LT / 4); g += kThreads) {
      const int i = g / (LT / 4);
      const int j0 = 4 * (g - i * (LT / 4));
      const int s0 = t * H + j0;
      const int lo = span_lo[i];
      const int hi = span_hi[i];
      const R *src = src_base + span_base[i] + s0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const bool valid = s0 + q >= lo && s0 + q < hi;
        cp_async<sizeof(R)>(rb + i * LT + j0 + q, valid ? src + q : src_base, valid);
      }
    }
  };
  issue(0, raw[0]);
  cp_async_commit();
  for (int t = 0; t < job.T; ++t) {
    if (t + 1 < job.T) issue(t + 1, raw[(t + 1) & 1]);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const R *rb = raw[t & 1];
    for (int idx = threadIdx.x; idx < NB * M; idx += kThreads) {
      const int i = idx / M;
      const int m = idx - i * M;
      const int j = 2 * m;
      R v0 = (R)0, v1 = (R)0;
      if (j < LT) {
        v0 = (rb[i * LT + j] * scale[i]) * taper[j];
        v1 = (rb[i * LT + j + 1] * scale[i]) * taper[j + 1];
      }
      line[i * LS + m] = cmake<C>(v0, v1);
    }
    __syncthreads();
    lines_fourstep<R, M1, M2, false>(line, NB, LS, twM);
    // split: X_k = (Z_k + conj Z_{M-k}) / 2 - i e^{-2 pi i k / Pt} (Z_k - conj Z_{M-k}) / 2
    C *zt = job.z + (long)t * F * ntr + t0;
    for (int idx = threadIdx.x; idx < NB * F; idx += kThreads) {
      const int f = idx / NB;
      const int i = idx - f * NB;
      if (i < nb) {
        const C *b = line + i * LS;
        const C zk = b[fourstep_pos<M1, M2>(f % M)];
        const C zm = b[fourstep_pos<M1, M2>((M - f) % M)];
        const C zc = cmake<C>(zm.x, -zm.y);
        const C e = cmake<C>((R)0.5 * (zk.x + zc.x), (R)0.5 * (zk.y + zc.y));
        const C o = cmake<C>((R)0.5 * (zk.y - zc.y), (R)-0.5 * (zk.x - zc.x));
        C x = cadd(e, cmul(tw_at<false>(tw2M, f), o));
        if (f >= 1 && f <= M - 1) x = cmake<C>(x.x * (R)2, x.y * (R)2);
        zt[f * ntr + i] = x;
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------ fused time kernels

// Hermitian combine of the c2r input (bins X of one trace, F = M + 1):
// Z_k = (X_k + conj X_{M-k}) + i e^{+2 pi i k / Pt} (X_k - conj X_{M-k}),
// the imaginary parts of X_0 and X_M dropped (c2r ignores them).
template <typename R, int M>
__device__ __forceinline__ Cx<R> combine_bin(const Cx<R> *x, int k, const Cx<R> *tw2M) {
  using C = Cx<R>;
  C a = x[k];
  C b = x[M - k];
  if (k == 0) {
    a.y = (R)0;
    b.y = (R)0;
  }
  const C bc = cmake<C>(b.x, -b.y);
  const C e = cadd(a, bc);
  const C d = csub(a, bc);
  const C o = cmul(d, tw_at<true>(tw2M, k));
  return cmake<C>(e.x - o.y, e.y + o.x);
}

// Forward time axis, fused: as time_fwd_fast, but the Hermitian combine is
// done while loading the first four-step pass, and the second pass keeps
// its outputs in registers: thread (trace i, k1) holds the samples
// j = 2 (k1 + M1 k2) + c, and as H / 2 = 2 M / 5 = 4 M1 (M2 = 10), the
// samples j < H (k2 < 4) and their successors j + H (k2 + 4) belong to the
// same thread, so taper, overlap-add and the one-hop carry stay in
// registers.  Two barriers per time window.  NB = 256 / M1 traces per block;
// M2 = 10.  Bins lines LSB apart, work groups M2 + 1 apart within lines LSW
// apart (both 10 mod 16, so the passes hit distinct banks).
template <typename R, int M1, int M2, int LSB, int LSW, int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
    time_fwd_fused(const TimeJob<R> *__restrict__ jobs, const int *__restrict__ cta_job,
                   const int *__restrict__ cta_trace0) {
  using C = Cx<R>;
  constexpr int M = M1 * M2;
  constexpr int F = M + 1;
  constexpr int H = 4 * M / 5;
  constexpr int NB = kThreads / M1;
  constexpr int G = M2 + 1;  // work group stride
  static_assert(M2 == 10 && NB * M1 == kThreads, "fused time kernel shape");
  static_assert(LSB >= F && LSW >= M1 * G, "line strides");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ C twM[M];
  __shared__ C tw2M[2 * M];
  load_twiddles<R, M>(twM);
  load_twiddles<R, 2 * M>(tw2M);
  const TimeJob<R> job = jobs[cta_job[blockIdx.x]];
  const int t0 = cta_trace0[blockIdx.x];
  const int nb = min(NB, job.n_traces - t0);
  const long ntr = job.n_traces;
  C *stage[2] = {reinterpret_cast<C *>(smem_raw), reinterpret_cast<C *>(smem_raw) + NB * LSB};
  C *work = stage[1] + NB * LSB;
  // this thread's trace and second-pass line, fixed over the time windows
  const int ti = threadIdx.x / M1;
  const int k1 = threadIdx.x - ti * M1;
  const bool live = ti < nb;
  const R sc = live ? job.space_scale[t0 + ti] : (R)0;
  R tap[8][2];  // tapers of the samples j = 2 (k1 + M1 k2) + c, k2 < 8
#pragma unroll
  for (int k2 = 0; k2 < 8; ++k2)
#pragma unroll
    for (int c = 0; c < 2; ++c) tap[k2][c] = job.time_taper[2 * (k1 + M1 * k2) + c];
  R carry[4][2];
#pragma unroll
  for (int k2 = 0; k2 < 4; ++k2) carry[k2][0] = carry[k2][1] = (R)0;
  R *yrow = job.y + (long)(t0 + (live ? ti : 0)) * job.C;
  auto issue = [&](int t, C *buf) {
    const C *zt = job.z + (long)t * F * ntr + t0;
    for (int idx = threadIdx.x; idx < NB * F; idx += kThreads) {
      const int f = idx / NB;
      const int i = idx - f * NB;
      if (i < nb) cp_async<sizeof(C)>(buf + i * LSB + f, zt + f * ntr + i);
    }
  };
  issue(0, stage[0]);
  cp_async_commit();
  for (int t = 0; t < job.T; ++t) {
    if (t + 1 < job.T) issue(t + 1, stage[(t + 1) & 1]);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const C *bins = stage[t & 1];
    // first pass: lines (trace i, n2) over n1, combined bins as input
    for (int it = threadIdx.x; it < NB * M2; it += kThreads) {
      const int i = it / M2;
      const int n2 = it - i * M2;
      C v[M1];
      if (i < nb) {
#pragma unroll
        for (int n1 = 0; n1 < M1; ++n1) v[n1] = combine_bin<R, M>(bins + i * LSB, M2 * n1 + n2, tw2M);
      } else {
#pragma unroll
        for (int n1 = 0; n1 < M1; ++n1) v[n1] = cmake<C>((R)0, (R)0);
      }
      dft<R, M1, true>(v);
      C *w = work + i * LSW + n2;
#pragma unroll
      for (int q = 0; q < M1; ++q)
        w[G * q] = (q == 0) ? v[0] : cmul(v[q], tw_at<true>(twM, (n2 * q) % M));
    }
    __syncthreads();
    // second pass: line k1 of trace ti; outputs X[k1 + M1 k2] = samples
    // 2 (k1 + M1 k2) + {0, 1}
    C v[M2];
    const C *w = work + ti * LSW + G * k1;
#pragma unroll
    for (int n2 = 0; n2 < M2; ++n2) v[n2] = w[n2];
    dft<R, M2, true>(v);
    if (live) {
      R *yt = yrow + t * H;
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) {
        const int j = 2 * (k1 + M1 * k2);
        yt[j] = carry[k2][0] + (v[k2].x * sc) * tap[k2][0];
        yt[j + 1] = carry[k2][1] + (v[k2].y * sc) * tap[k2][1];
      }
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) {
        carry[k2][0] = (v[k2 + 4].x * sc) * tap[k2 + 4][0];
        carry[k2][1] = (v[k2 + 4].y * sc) * tap[k2 + 4][1];
      }
    }
  }
  // last half window, then zeros up to C
  if (live) {
    R *yt = yrow + job.T * H;
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) {
      const int j = 2 * (k1 + M1 * k2);
      yt[j] = carry[k2][0];
      yt[j + 1] = carry[k2][1];
    }
  }
  const int tail = job.C - (job.T + 1) * H;
  for (int idx = threadIdx.x; idx < nb * tail; idx += kThreads) {
    const int i = idx / tail;
    const int j = idx - i * tail;
    job.y[(long)(t0 + i) * job.C + (job.T + 1) * H + j] = (R)0;
  }
}

// Adjoint time axis, fused: as time_adj_fast, but the scaling, tapering and
// packing of the raw samples is done while loading the first four-step
// pass, and the second pass writes its outputs back into its own group of
// the work buffer (no second buffer).  Three barriers per time window.
template <typename R, int M1, int M2, int LSW, int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
    time_adj_fused(const TimeJob<R> *__restrict__ jobs, const int *__restrict__ cta_job,
                   const int *__restrict__ cta_trace0, const R *__restrict__ record,
                   int from_record) {
  using C = Cx<R>;
  constexpr int M = M1 * M2;
  constexpr int F = M + 1;
  constexpr int H = 4 * M / 5;
  constexpr int LT = 2 * H;
  constexpr int NB = kThreads / M1;
  constexpr int G = M2 + 1;
  // raw sample rows padded to 20 mod 32 floats: the first pass reads sample
  // pairs as 8-byte loads, and a half-warp's pairs then fall in distinct
  // banks
  constexpr int LTP = LT + ((20 - LT % 32) + 32) % 32;
  static_assert(M2 == 10 && NB * M1 == kThreads, "fused time kernel shape");
  static_assert(LSW >= M1 * G, "line stride");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ C twM[M];
  __shared__ C tw2M[2 * M];
  __shared__ long span_base[NB];
  __shared__ int span_lo[NB], span_hi[NB];
  __shared__ R scale[NB];
  __shared__ R taper[LT];
  load_twiddles<R, M>(twM);
  load_twiddles<R, 2 * M>(tw2M);
  const TimeJob<R> job = jobs[cta_job[blockIdx.x]];
  const int t0 = cta_trace0[blockIdx.x];
  const int nb = min(NB, job.n_traces - t0);
  const long ntr = job.n_traces;
  for (int j = threadIdx.x; j < LT; j += kThreads) taper[j] = job.time_taper[j];
  for (int i = threadIdx.x; i < NB; i += kThreads) {
    const int tr = t0 + i;
    span_lo[i] = 0;
    span_hi[i] = 0;
    span_base[i] = 0;
    scale[i] = (R)0;
    if (i >= nb) continue;
    scale[i] = job.space_scale[tr];
    if (from_record) {
      const long rec = job.blend_rec[tr];
      const int ts = job.blend_ts[tr];
      span_base[i] = rec - ts;
      span_lo[i] = rec >= 0 ? ts : 0;
      span_hi[i] = rec >= 0 ? ts + job.blend_n[tr] : 0;
    } else {
      span_base[i] = (long)tr * job.C;
      span_hi[i] = job.C;
    }
  }
  __syncthreads();
  const R *src_base = from_record ? record : job.y;
  C *work = reinterpret_cast<C *>(smem_raw);
  R *raw[2] = {reinterpret_cast<R *>(work + NB * LSW),
               reinterpret_cast<R *>(work + NB * LSW) + NB * LTP};
  auto issue = [&](int t, R *rb) {
    for (int g = threadIdx.x; g < NB * (LT / 4); g += kThreads) {
      const int i = g / (LT / 4);
      const int j0 = 4 * (g - i * (LT / 4));
      const int s0 = t * H + j0;
      const int lo = span_lo[i];
      const int hi = span_hi[i];
      const R *src = src_base + span_base[i] + s0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const bool valid = s0 + q >= lo && s0 + q < hi;
        cp_async<sizeof(R)>(rb + i * LTP + j0 + q, valid ? src + q : src_base, valid);
      }
    }
  };
  const int ti = threadIdx.x / M1;
  const int k1 = threadIdx.x - ti * M1;
  issue(0, raw[0]);
  cp_async_commit();
  for (int t = 0; t < job.T; ++t) {
    if (t + 1 < job.T) issue(t + 1, raw[(t + 1) & 1]);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const R *rb = raw[t & 1];
    // first pass: packed, tapered samples (2 m, 2 m + 1) as input
    for (int it = threadIdx.x; it < NB * M2; it += kThreads) {
      const int i = it / M2;
      const int n2 = it - i * M2;
      const R sc = scale[i];
      C v[M1];
#pragma unroll
      for (int n1 = 0; n1 < M1; ++n1) {
        const int j = 2 * (M2 * n1 + n2);
        R v0 = (R)0, v1 = (R)0;
        if (j < LT) {
          const Cx<R> pr = *reinterpret_cast<const Cx<R> *>(rb + i * LTP + j);
          v0 = (pr.x * sc) * taper[j];
          v1 = (pr.y * sc) * taper[j + 1];
        }
        v[n1] = cmake<C>(v0, v1);
      }
      dft<R, M1, false>(v);
      C *w = work + i * LSW + n2;
#pragma unroll
      for (int q = 0; q < M1; ++q)
        w[G * q] = (q == 0) ? v[0] : cmul(v[q], tw_at<false>(twM, (n2 * q) % M));
    }
    __syncthreads();
    {  // second pass, in place in this thread's group: Z[k1 + M1 k2]
      C v[M2];
      C *w = work + ti * LSW + G * k1;
#pragma unroll
      for (int n2 = 0; n2 < M2; ++n2) v[n2] = w[n2];
      dft<R, M2, false>(v);
#pragma unroll
      for (int k2 = 0; k2 < M2; ++k2) w[k2] = v[k2];
    }
    __syncthreads();
    // split: X_k = (Z_k + conj Z_{M-k}) / 2 - i e^{-2 pi i k / Pt} (Z_k - conj Z_{M-k}) / 2
    C *zt = job.z + (long)t * F * ntr + t0;
    for (int idx = threadIdx.x; idx < NB * F; idx += kThreads) {
      const int f = idx / NB;
      const int i = idx - f * NB;
      if (i < nb) {
        const C *b = work + i * LSW;
        const int fa = f % M;
        const int fb = (M - f) % M;
        const C zk = b[G * (fa % M1) + fa / M1];
        const C zm = b[G * (fb % M1) + fb / M1];
        const C zc = cmake<C>(zm.x, -zm.y);
        const C e = cmake<C>((R)0.5 * (zk.x + zc.x), (R)0.5 * (zk.y + zc.y));
        const C o = cmake<C>((R)0.5 * (zk.y - zc.y), (R)-0.5 * (zk.x - zc.x));
        C x = cadd(e, cmul(tw_at<false>(tw2M, f), o));
        if (f >= 1 && f <= M - 1) x = cmake<C>(x.x * (R)2, x.y * (R)2);
        zt[f * ntr + i] = x;
      }
    }
  }
}

}  // namespace agd
