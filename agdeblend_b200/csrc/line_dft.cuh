// Space transforms of windows with one space axis of any padded length P
// (the reference's per-window FFT along that axis, src/fk.c:307-373 forward,
// src/fk.c:375-443 adjoint), for the lengths without a shape-specialised
// kernel: enlarged edge windows (L = 33, 65, 67, ...), prime P (83, 89) and
// lengths whose factors include large primes (82 = 2 * 41).
//
// A plane of such a window is one line of P complex values, and every line
// of a window has the same P and L, so the DFT of a batch of lines is a
// small matrix product with a real cosine / sine table:
//
//   forward (inverse DFT, P inputs, the first L outputs):
//     y_k = x_0 + (-1)^k x_{P/2} [P even]
//           + sum_{j=1}^{H} (x_j + x_{P-j}) cos(2 pi j k / P)
//                        + i (x_j - x_{P-j}) sin(2 pi j k / P),  H = (P-1)/2
//   adjoint (forward DFT, L inputs zero-padded to P, all P outputs):
//     A_k = sum_{j<L} x_j cos(2 pi j k / P),  B_k = sum_{j<L} x_j sin(...),
//     y_k = A_k - i B_k,  y_{P-k} = A_k + i B_k,  k = 0 .. P/2
//
// so each line costs about 2 P L fused multiply-adds instead of the 4 P^2 of
// a plain DFT, with no index arithmetic in the inner loop.  A block stages
// NL lines (cp.async) and the table (host-computed in double precision,
// rounded once, shared by all blocks of the window through L2) in shared
// memory; each thread accumulates a 4-line x 4-frequency tile in registers,
// the threads of a warp sharing their lines (broadcast loads) and differing
// in frequencies.  Results go through shared memory so that the stores, and
// the model reads of the fused ISTA update, are contiguous runs.
#pragma once

#include "fast.cuh"

namespace agd {

constexpr int kLineThreads = 128;
constexpr int kLineMaxP = 128;    // longest axis served

// One window's lines for the line kernels.
template <typename R>
struct LineJob {
  const Cx<R> *src;  // forward: model lines [lines][P]; adjoint: [lines][L]
  Cx<R> *dst;        // forward: [lines][L]; adjoint: model lines [lines][P]
  const R *tab_c;    // [rows][kpad] cosines (forward rows j = 1..H, adjoint j < L)
  const R *tab_s;    // [rows][kpad] sines
  long lines;
  int P, L;
  int rows;          // forward H = (P - 1) / 2, adjoint L
  int kout;          // forward L, adjoint P / 2 + 1
  int kpad;          // kout rounded up to a multiple of 4
  int nl;            // lines per block (a multiple of 4), chosen per window
  int pid;           // problem of the window
};

// Shared-memory bytes of a block of nl lines (regions rounded to 16 bytes).
// Forward: lines [nl][P] (then results [nl][L]), pair sums and differences
// [H][nl + 1] each (an odd row stride: the transposing writes hit distinct
// banks), x_0 and x_{P/2} [nl] each, tables [H][kpad] each.  Adjoint: lines
// [nl][L], model lines [nl][P] (updated in place, then stored), tables
// [L][kpad] each.
__host__ __device__ inline int line_even(int n) { return n + (n & 1); }
template <typename R>
size_t line_fwd_smem(int P, int H, int kpad, int nl) {
  return (size_t)(line_even(nl * P) + 2 * line_even(H * (nl + 1)) + 2 * nl) * sizeof(Cx<R>) +
         2 * (size_t)H * kpad * sizeof(R);
}
template <typename R>
size_t line_adj_smem(int P, int L, int kpad, int nl) {
  return (size_t)(line_even(nl * L) + line_even(nl * P)) * sizeof(Cx<R>) +
         2 * (size_t)L * kpad * sizeof(R);
}

template <typename R>
__device__ __forceinline__ void line_copy_in(Cx<R> *to, const Cx<R> *from, int n) {
  for (int e = threadIdx.x; e < n; e += kLineThreads) cp_async<sizeof(Cx<R>)>(to + e, from + e);
}

template <typename R>
__device__ __forceinline__ void line_table_in(R *to, const R *from, int n) {
  // tables start 16-byte aligned and hold a multiple of 4 values per row
  constexpr int per = 16 / sizeof(R);
  for (int e = threadIdx.x; e < n / per; e += kLineThreads)
    cp_async<16>(to + e * per, from + e * per);
}

// four consecutive table values (16-byte aligned for float)
template <typename R>
__device__ __forceinline__ void load4(const R *p, R (&v)[4]) {
  if constexpr (sizeof(R) == sizeof(float)) {
    const float4 q = *reinterpret_cast<const float4 *>(p);
    v[0] = q.x;
    v[1] = q.y;
    v[2] = q.z;
    v[3] = q.w;
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = p[i];
  }
}

// floor(x / d) for 0 <= x < 2^22 from r = 1 / d rounded: (x + 1/2) / d is
// at least 1/(2d) from an integer, the product's relative error below 2^-23
__device__ __forceinline__ int line_div(int x, float r) {
  return __float2int_rz(((float)x + 0.5f) * r);
}

// Forward operator: Z[line][0..L) = crop(IDFT_P(X[line][0..P))).
template <typename R>
__global__ void __launch_bounds__(kLineThreads, 3)
    line_dft_fwd(const LineJob<R> *__restrict__ jobs, const int *__restrict__ cta_job,
                 const long *__restrict__ cta_line0) {
  using C = Cx<R>;
  const LineJob<R> job = jobs[cta_job[blockIdx.x]];
  const long l0 = cta_line0[blockIdx.x];
  const int NL = job.nl;
  const int nl = (int)min((long)NL, job.lines - l0);
  const int P = job.P, L = job.L, H = job.rows, kpad = job.kpad;
  const int NS = NL + 1;  // row stride of the pair sums
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);  // [NL][P] in, then [NL][L] out
  C *ssum = buf + line_even(NL * P);         // [H][NS]
  C *sdif = ssum + line_even(H * NS);        // [H][NS]
  C *x0 = sdif + line_even(H * NS);          // [NL]
  C *xh = x0 + NL;                           // [NL]
  R *tc = reinterpret_cast<R *>(xh + NL);    // [H][kpad]
  R *ts = tc + H * kpad;
  line_copy_in<R>(buf, job.src + l0 * P, nl * P);
  line_table_in<R>(tc, job.tab_c, H * kpad);
  line_table_in<R>(ts, job.tab_s, H * kpad);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  // pair sums and differences: reads along each line, writes at the odd
  // stride NS
  const float inv_h = 1.0f / (float)H;
  for (int idx = threadIdx.x; idx < nl * H; idx += kLineThreads) {
    const int l = line_div(idx, inv_h);
    const int j = idx - l * H;
    const C a = buf[l * P + j + 1];
    const C b = buf[l * P + P - 1 - j];
    ssum[j * NS + l] = cadd(a, b);
    sdif[j * NS + l] = csub(a, b);
  }
  for (int l = threadIdx.x; l < NL; l += kLineThreads) {
    x0[l] = l < nl ? buf[l * P] : cmake<C>((R)0, (R)0);
    xh[l] = (l < nl && P % 2 == 0) ? buf[l * P + P / 2] : cmake<C>((R)0, (R)0);
  }
  __syncthreads();
  // 4 lines x 4 outputs per thread; results into buf as [nl][L] (lines past
  // nl of the window's last block are computed from stale values, never
  // stored)
  const int kt_n = kpad / 4;
  const int lt_n = (nl + 3) / 4;
  for (int tile = threadIdx.x; tile < lt_n * kt_n; tile += kLineThreads) {
    const int lt = tile / kt_n;
    const int kt = tile - lt * kt_n;
    R re[4][4], im[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const C a = x0[4 * lt + i];
      const C h = xh[4 * lt + i];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const R sg = ((4 * kt + m) & 1) ? (R)-1 : (R)1;
        re[i][m] = a.x + sg * h.x;
        im[i][m] = a.y + sg * h.y;
      }
    }
    for (int j = 0; j < H; ++j) {
      C sv[4], dv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        sv[i] = ssum[j * NS + 4 * lt + i];
        dv[i] = sdif[j * NS + 4 * lt + i];
      }
      R c[4], sn[4];
      load4<R>(tc + j * kpad + 4 * kt, c);
      load4<R>(ts + j * kpad + 4 * kt, sn);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          re[i][m] += sv[i].x * c[m] - dv[i].y * sn[m];
          im[i][m] += sv[i].y * c[m] + dv[i].x * sn[m];
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const int l = 4 * lt + i, k = 4 * kt + m;
        if (l < nl && k < L) buf[l * L + k] = cmake<C>(re[i][m], im[i][m]);
      }
  }
  __syncthreads();
  C *dst = job.dst + l0 * L;
  for (int e = threadIdx.x; e < nl * L; e += kLineThreads) dst[e] = buf[e];
}

// Adjoint with the ISTA update fused (epilogues as axis_pass):
// G[line][0..P) = DFT_P(pad(Z[line][0..L))), then X <- update(X, G).  The
// block's model lines are copied into shared memory with its input lines,
// behind the transform; each tile updates its outputs there in place, and
// the updated lines are stored as one contiguous run.
template <typename R>
__global__ void __launch_bounds__(kLineThreads, 3)
    line_dft_adj(const LineJob<R> *__restrict__ jobs, const int *__restrict__ cta_job,
                 const long *__restrict__ cta_line0, int epilogue, R step_arg, R lamb_arg,
                 const R *step_dev, const R *lamb_dev, R *max_out) {
  using C = Cx<R>;
  const LineJob<R> job = jobs[cta_job[blockIdx.x]];
  const long l0 = cta_line0[blockIdx.x];
  const int NL = job.nl;
  const int nl = (int)min((long)NL, job.lines - l0);
  const int P = job.P, L = job.L, kpad = job.kpad, KO = job.kout;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *xin = reinterpret_cast<C *>(smem_raw);  // [NL][L]
  C *xm = xin + line_even(NL * L);           // [NL][P] model, updated in place
  R *tc = reinterpret_cast<R *>(xm + line_even(NL * P));  // [L][kpad]
  R *ts = tc + L * kpad;
  C *dst = job.dst + l0 * P;
  const bool need_x = epilogue != kStore;
  line_copy_in<R>(xin, job.src + l0 * L, nl * L);
  line_table_in<R>(tc, job.tab_c, L * kpad);
  line_table_in<R>(ts, job.tab_s, L * kpad);
  if (need_x) line_copy_in<R>(xm, dst, nl * P);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  const bool multi = step_dev != nullptr;
  const R step = multi ? step_dev[job.pid] : step_arg;
  const R lamb = lamb_dev != nullptr ? lamb_dev[multi ? job.pid : 0] : lamb_arg;
  const R lamb_sq = lamb * lamb;
  R local_max = (R)0;
  auto update = [&](C *xp, C g) {
    if (!need_x) {
      *xp = g;
      return;
    }
    const C x = *xp;
    C xn = cmake<C>(sub_rn<R>(x.x, mul_rn<R>(step, g.x)), sub_rn<R>(x.y, mul_rn<R>(step, g.y)));
    if (epilogue == kUpdateThreshold) {
      xn = soft_threshold<R>(xn, lamb, lamb_sq);
    } else {
      const R a2 = abs_sq<R>(xn);
      local_max = a2 > local_max ? a2 : local_max;
    }
    *xp = xn;
  };
  const int kt_n = kpad / 4;
  const int lt_n = (nl + 3) / 4;
  for (int tile = threadIdx.x; tile < lt_n * kt_n; tile += kLineThreads) {
    const int lt = tile / kt_n;
    const int kt = tile - lt * kt_n;
    C a[4][4], bsum[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int m = 0; m < 4; ++m) a[i][m] = bsum[i][m] = cmake<C>((R)0, (R)0);
    for (int j = 0; j < L; ++j) {
      C x[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) x[i] = xin[(4 * lt + i) * L + j];
      R c[4], sn[4];
      load4<R>(tc + j * kpad + 4 * kt, c);
      load4<R>(ts + j * kpad + 4 * kt, sn);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          a[i][m].x += x[i].x * c[m];
          a[i][m].y += x[i].y * c[m];
          bsum[i][m].x += x[i].x * sn[m];
          bsum[i][m].y += x[i].y * sn[m];
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const int l = 4 * lt + i, k = 4 * kt + m;
        if (l >= nl || k >= KO) continue;
        const C A = a[i][m], B = bsum[i][m];
        update(xm + l * P + k, cmake<C>(A.x + B.y, A.y - B.x));  // A - i B
        if (k > 0 && P - k != k) update(xm + l * P + P - k, cmake<C>(A.x - B.y, A.y + B.x));
      }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nl * P; e += kLineThreads) dst[e] = xm[e];
  if (epilogue == kUpdateMax) {
    __shared__ R red[32];
    const R m = block_max<R>(local_max, red);
    if (threadIdx.x == 0) atomic_max_nonneg(max_out + (multi ? job.pid : 0), m);
  }
}

}  // namespace agd
