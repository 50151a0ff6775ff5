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

// lines per block: 32 in float, 16 in double (the blocks of the longest
// axes then still fit in shared memory)
template <typename R>
__host__ __device__ constexpr int line_lines() {
  return sizeof(R) == sizeof(float) ? 32 : 16;
}

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
  int pid;           // problem of the window
};

// Shared-memory bytes of a block (csize / rsize: bytes of a complex / real
// value).  Forward: lines [NL][P], pair sums and differences [H][NL] each,
// x_0 and x_{P/2} [NL] each, tables [H][kpad] each.  Adjoint: lines [NL][L]
// then results [NL][P], transposed lines [L][NL], tables [L][kpad] each.
// Every part is a whole number of 16-byte units (NL a multiple of 16, kpad
// of 4).
template <typename R>
size_t line_fwd_smem(int P, int H, int kpad) {
  constexpr size_t NL = line_lines<R>();
  return (NL * P + 2 * (size_t)H * NL + 2 * NL) * sizeof(Cx<R>) + 2 * (size_t)H * kpad * sizeof(R);
}
template <typename R>
size_t line_adj_smem(int P, int L, int kpad) {
  constexpr size_t NL = line_lines<R>();
  return (NL * P + (size_t)L * NL) * sizeof(Cx<R>) + 2 * (size_t)L * kpad * sizeof(R);
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

// Forward operator: Z[line][0..L) = crop(IDFT_P(X[line][0..P))).
template <typename R>
__global__ void __launch_bounds__(kLineThreads, 3)
    line_dft_fwd(const LineJob<R> *__restrict__ jobs, const int *__restrict__ cta_job,
                 const long *__restrict__ cta_line0) {
  using C = Cx<R>;
  constexpr int NL = line_lines<R>();
  const LineJob<R> job = jobs[cta_job[blockIdx.x]];
  const long l0 = cta_line0[blockIdx.x];
  const int nl = (int)min((long)NL, job.lines - l0);
  const int P = job.P, L = job.L, H = job.rows, kpad = job.kpad;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);  // [NL][P] in, then [NL][L] out
  C *ssum = buf + NL * P;                    // [H][NL]
  C *sdif = ssum + H * NL;                   // [H][NL]
  C *x0 = sdif + H * NL;                     // [NL]
  C *xh = x0 + NL;                           // [NL]
  R *tc = reinterpret_cast<R *>(xh + NL);    // [H][kpad]
  R *ts = tc + H * kpad;
  line_copy_in<R>(buf, job.src + l0 * P, nl * P);
  line_table_in<R>(tc, job.tab_c, H * kpad);
  line_table_in<R>(ts, job.tab_s, H * kpad);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  // pair sums and differences, lines fastest
  for (int idx = threadIdx.x; idx < H * NL; idx += kLineThreads) {
    const int j = idx / NL;
    const int l = idx - j * NL;
    C s = cmake<C>((R)0, (R)0), d = s;
    if (l < nl) {
      const C a = buf[l * P + j + 1];
      const C b = buf[l * P + P - 1 - j];
      s = cadd(a, b);
      d = csub(a, b);
    }
    ssum[idx] = s;
    sdif[idx] = d;
  }
  for (int l = threadIdx.x; l < NL; l += kLineThreads) {
    x0[l] = l < nl ? buf[l * P] : cmake<C>((R)0, (R)0);
    xh[l] = (l < nl && P % 2 == 0) ? buf[l * P + P / 2] : cmake<C>((R)0, (R)0);
  }
  __syncthreads();
  // 4 lines x 4 outputs per thread; results into buf as [nl][L]
  const int kt_n = kpad / 4;
  for (int tile = threadIdx.x; tile < (NL / 4) * kt_n; tile += kLineThreads) {
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
      C s[4], d[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        s[i] = ssum[j * NL + 4 * lt + i];
        d[i] = sdif[j * NL + 4 * lt + i];
      }
      R c[4], sn[4];
      load4<R>(tc + j * kpad + 4 * kt, c);
      load4<R>(ts + j * kpad + 4 * kt, sn);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          re[i][m] += s[i].x * c[m] - d[i].y * sn[m];
          im[i][m] += s[i].y * c[m] + d[i].x * sn[m];
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
// G[line][0..P) = DFT_P(pad(Z[line][0..L))), then X <- update(X, G).
template <typename R>
__global__ void __launch_bounds__(kLineThreads, 3)
    line_dft_adj(const LineJob<R> *__restrict__ jobs, const int *__restrict__ cta_job,
                 const long *__restrict__ cta_line0, int epilogue, R step_arg, R lamb_arg,
                 const R *step_dev, const R *lamb_dev, R *max_out) {
  using C = Cx<R>;
  constexpr int NL = line_lines<R>();
  const LineJob<R> job = jobs[cta_job[blockIdx.x]];
  const long l0 = cta_line0[blockIdx.x];
  const int nl = (int)min((long)NL, job.lines - l0);
  const int P = job.P, L = job.L, kpad = job.kpad, KO = job.kout;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);  // [NL][L] in, then [NL][P] results
  C *xt = buf + NL * P;                      // [L][NL]
  R *tc = reinterpret_cast<R *>(xt + L * NL);  // [L][kpad]
  R *ts = tc + L * kpad;
  line_copy_in<R>(buf, job.src + l0 * L, nl * L);
  line_table_in<R>(tc, job.tab_c, L * kpad);
  line_table_in<R>(ts, job.tab_s, L * kpad);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  for (int idx = threadIdx.x; idx < L * NL; idx += kLineThreads) {
    const int j = idx / NL;
    const int l = idx - j * NL;
    xt[idx] = l < nl ? buf[l * L + j] : cmake<C>((R)0, (R)0);
  }
  __syncthreads();
  const int kt_n = kpad / 4;
  for (int tile = threadIdx.x; tile < (NL / 4) * kt_n; tile += kLineThreads) {
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
      for (int i = 0; i < 4; ++i) x[i] = xt[j * NL + 4 * lt + i];
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
        buf[l * P + k] = cmake<C>(A.x + B.y, A.y - B.x);  // A - i B
        if (k > 0 && P - k != k) buf[l * P + P - k] = cmake<C>(A.x - B.y, A.y + B.x);
      }
  }
  __syncthreads();
  // update the model lines (contiguous over the block's lines)
  const bool multi = step_dev != nullptr;
  const R step = multi ? step_dev[job.pid] : step_arg;
  const R lamb = lamb_dev != nullptr ? lamb_dev[multi ? job.pid : 0] : lamb_arg;
  const R lamb_sq = lamb * lamb;
  R local_max = (R)0;
  C *dst = job.dst + l0 * P;
  for (int e = threadIdx.x; e < nl * P; e += kLineThreads) {
    const C g = buf[e];
    if (epilogue == kStore) {
      dst[e] = g;
      continue;
    }
    const C x = dst[e];
    C xn = cmake<C>(sub_rn<R>(x.x, mul_rn<R>(step, g.x)), sub_rn<R>(x.y, mul_rn<R>(step, g.y)));
    if (epilogue == kUpdateThreshold) {
      xn = soft_threshold<R>(xn, lamb, lamb_sq);
    } else {
      const R a2 = abs_sq<R>(xn);
      local_max = a2 > local_max ? a2 : local_max;
    }
    dst[e] = xn;
  }
  if (epilogue == kUpdateMax) {
    __shared__ R red[32];
    const R m = block_max<R>(local_max, red);
    if (threadIdx.x == 0) atomic_max_nonneg(max_out + (multi ? job.pid : 0), m);
  }
}

}  // namespace agd
