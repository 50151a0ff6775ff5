// Element-wise and data-movement kernels of the warm-start network (the
// convolutions themselves are tensor-core GEMMs, tc_gemm.cuh).  Activations
// are NHWC: pixel p = (n * H + y) * W + x, channel fastest, with a channel
// stride C_s (channels padded to a multiple of 8 so that GEMM rows are
// 16-byte aligned).  Values fed to the tensor cores are BF16; GEMM outputs,
// gradients and the optimiser state are FP32.
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

namespace agd {
namespace nn {

constexpr int kNnThreads = 256;

__device__ __forceinline__ uint16_t to_bf16(float v) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(v));
}
__device__ __forceinline__ float from_bf16(uint16_t h) {
  return __bfloat162float(__ushort_as_bfloat16(h));
}

// col[p][k], k = (ky * 3 + kx) * Cin + ci (k < 9 Cin; zero for k >= 9 Cin up
// to the row stride Kp): the 3 x 3, padding 1 neighbourhood of pixel p.
__global__ void im2col3x3(const uint16_t *__restrict__ x, int N, int H, int W, int Cin, int Cs,
                          int Kp, uint16_t *__restrict__ col) {
  const long total = (long)N * H * W * Kp;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const long p = i / Kp;
    const int k = (int)(i - p * Kp);
    uint16_t v = 0;
    if (k < 9 * Cin) {
      const int tap = k / Cin, ci = k - tap * Cin;
      const int ky = tap / 3, kx = tap - 3 * ky;
      const int xx = (int)(p % W);
      const long r = p / W;
      const int yy = (int)(r % H);
      const long n = r / H;
      const int sy = yy + ky - 1, sx = xx + kx - 1;
      if (sy >= 0 && sy < H && sx >= 0 && sx < W)
        v = x[((n * H + sy) * W + sx) * Cs + ci];
    }
    col[i] = v;
  }
}

// dx[p][ci] (+)= sum over the 3 x 3 taps of dcol[p'][k] with p' the pixel
// whose neighbourhood holds p at tap (ky, kx): the transpose of im2col3x3,
// as a gather (no atomics).
__global__ void col2im3x3(const float *__restrict__ dcol, int N, int H, int W, int Cin, int Kp,
                          float *__restrict__ dx, int Cs, int accumulate) {
  const long total = (long)N * H * W * Cin;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const long p = i / Cin;
    const int ci = (int)(i - p * Cin);
    const int xx = (int)(p % W);
    const long r = p / W;
    const int yy = (int)(r % H);
    const long n = r / H;
    float s = 0.f;
#pragma unroll
    for (int ky = 0; ky < 3; ++ky)
#pragma unroll
      for (int kx = 0; kx < 3; ++kx) {
        const int oy = yy - ky + 1, ox = xx - kx + 1;  // pixel whose tap (ky, kx) is p
        if (oy >= 0 && oy < H && ox >= 0 && ox < W)
          s += dcol[((n * H + oy) * W + ox) * Kp + (ky * 3 + kx) * Cin + ci];
      }
    float *d = dx + p * Cs + ci;
    *d = accumulate ? *d + s : s;
  }
}

// y = act(z + b) per channel (act: ReLU when relu, identity otherwise),
// written as BF16 (the next layer's operand) and optionally as FP32.
__global__ void bias_act(const float *__restrict__ z, const float *__restrict__ b, long P, int C,
                         int Cs, int relu, uint16_t *__restrict__ y, float *__restrict__ yf) {
  const long total = P * Cs;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i % Cs);
    float v = 0.f;
    if (c < C) {
      v = z[i] + b[c];
      if (relu && v < 0.f) v = 0.f;
    }
    y[i] = to_bf16(v);
    if (yf) yf[i] = v;
  }
}

// dz = dy where the ReLU was active (y > 0) or everywhere (linear layer), as
// BF16 (a GEMM operand); padded channels zero.
__global__ void act_backward(const float *__restrict__ dy, const uint16_t *__restrict__ y,
                             long P, int C, int Cs, int relu, uint16_t *__restrict__ dz) {
  const long total = P * Cs;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i % Cs);
    float v = 0.f;
    if (c < C) {
      v = dy[i];
      if (relu && !(from_bf16(y[i]) > 0.f)) v = 0.f;
    }
    dz[i] = to_bf16(v);
  }
}

// db[c] = sum_p dz[p][c] (block per channel group; dz BF16)
__global__ void bias_grad(const uint16_t *__restrict__ dz, long P, int C, int Cs,
                          float *__restrict__ db) {
  const int c = blockIdx.x;
  if (c >= C) return;
  float s = 0.f;
  for (long p = threadIdx.x; p < P; p += blockDim.x) s += from_bf16(dz[p * Cs + c]);
  __shared__ float red[kNnThreads];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[c] += red[0];
}

// out[c][r] = in[r][c] for an R x Cn BF16 matrix (rows of `in` stride ld_in,
// rows of `out` stride ld_out), 32 x 32 tiles through shared memory.
__global__ void transpose_bf16(const uint16_t *__restrict__ in, long R, int Cn, long ld_in,
                               uint16_t *__restrict__ out, long ld_out) {
  __shared__ uint16_t t[32][33];
  const long r0 = (long)blockIdx.x * 32;
  const int c0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const long r = r0 + k;
    const int c = c0 + threadIdx.x;
    t[k][threadIdx.x] = (r < R && c < Cn) ? in[r * ld_in + c] : (uint16_t)0;
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = c0 + k;
    const long r = r0 + threadIdx.x;
    if (c < Cn && r < R) out[(long)c * ld_out + r] = t[threadIdx.x][k];
  }
}

// 2 x 2 average pooling of BF16 NHWC (H, W even); backward spreads a quarter
// of each gradient to the four inputs (accumulating).
__global__ void avgpool2(const uint16_t *__restrict__ x, int N, int H, int W, int Cs,
                         uint16_t *__restrict__ y) {
  const int Ho = H / 2, Wo = W / 2;
  const long total = (long)N * Ho * Wo * Cs;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i % Cs);
    const long q = i / Cs;
    const int xo = (int)(q % Wo);
    const long r = q / Wo;
    const int yo = (int)(r % Ho);
    const long n = r / Ho;
    const long b = ((n * H + 2 * yo) * W + 2 * xo) * Cs + c;
    const float s = from_bf16(x[b]) + from_bf16(x[b + Cs]) + from_bf16(x[b + (long)W * Cs]) +
                    from_bf16(x[b + (long)W * Cs + Cs]);
    y[i] = to_bf16(0.25f * s);
  }
}

__global__ void avgpool2_backward(const float *__restrict__ dy, int N, int H, int W, int Cs,
                                  float *__restrict__ dx) {
  const long total = (long)N * H * W * Cs;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i % Cs);
    const long q = i / Cs;
    const int xx = (int)(q % W);
    const long r = q / W;
    const int yy = (int)(r % H);
    const long n = r / H;
    dx[i] += 0.25f * dy[((n * (H / 2) + yy / 2) * (W / 2) + xx / 2) * Cs + c];
  }
}

// y = nearest 2x upsampling of a (N, H/2, W/2) tensor + skip (both BF16;
// H, W of the output); backward: dlow[q] += sum of the four dy it fed.
__global__ void upsample2_add(const uint16_t *__restrict__ low, const uint16_t *__restrict__ skip,
                              int N, int H, int W, int Cs, uint16_t *__restrict__ y) {
  const long total = (long)N * H * W * Cs;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i % Cs);
    const long q = i / Cs;
    const int xx = (int)(q % W);
    const long r = q / W;
    const int yy = (int)(r % H);
    const long n = r / H;
    const float v = from_bf16(low[((n * (H / 2) + yy / 2) * (W / 2) + xx / 2) * Cs + c]) +
                    from_bf16(skip[i]);
    y[i] = to_bf16(v);
  }
}

__global__ void upsample2_backward(const float *__restrict__ dy, int N, int H, int W, int Cs,
                                   float *__restrict__ dlow) {
  const int Ho = H / 2, Wo = W / 2;
  const long total = (long)N * Ho * Wo * Cs;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i % Cs);
    const long q = i / Cs;
    const int xo = (int)(q % Wo);
    const long r = q / Wo;
    const int yo = (int)(r % Ho);
    const long n = r / Ho;
    const long b = ((n * H + 2 * yo) * W + 2 * xo) * Cs + c;
    dlow[i] += dy[b] + dy[b + Cs] + dy[b + (long)W * Cs] + dy[b + (long)W * Cs + Cs];
  }
}

// out = in + r (the residual output, channel 0 of a Cs-strided tensor)
__global__ void residual_out(const float *__restrict__ in, int in_ch, const float *__restrict__ r,
                             long P, int Cs, float *__restrict__ out) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < P;
       p += (long)gridDim.x * blockDim.x)
    out[p] = in[p * in_ch] + r[p * Cs];
}

// Mean squared error over P values and its gradient with respect to the
// residual (Cs-strided channel 0): d[p * Cs] = 2 (out - target) / P.
__global__ void mse_grad(const float *__restrict__ out, const float *__restrict__ target, long P,
                         int Cs, float *__restrict__ d, double *__restrict__ loss) {
  __shared__ double red[kNnThreads];
  double s = 0.0;
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < P;
       p += (long)gridDim.x * blockDim.x) {
    const float e = out[p] - target[p];
    s += (double)e * e;
    d[p * Cs] = 2.f * e / (float)P;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0] / (double)P);
}

// Adam on FP32 master parameters; refreshes their BF16 copies.
__global__ void adam_step(float *__restrict__ w, const float *__restrict__ g,
                          float *__restrict__ m, float *__restrict__ v, long n, float lr,
                          float b1, float b2, float eps, float c1, float c2,
                          uint16_t *__restrict__ w_bf16) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (w_bf16) w_bf16[i] = to_bf16(wi);
  }
}

__global__ void to_bf16_kernel(const float *__restrict__ x, long n, uint16_t *__restrict__ y) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    y[i] = to_bf16(x[i]);
}

__global__ void pack_kernel(const float *__restrict__ wsrc, int cout, int k9,
                                   int cout_s, int kp, uint16_t *__restrict__ out,
                                   uint16_t *__restrict__ outT) {
  const long total = (long)cout_s * kp;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int co = (int)(i / kp), k = (int)(i - (long)co * kp);
    const uint16_t b = (co < cout && k < k9) ? to_bf16(wsrc[(long)co * k9 + k]) : (uint16_t)0;
    out[i] = b;
    outT[(long)k * cout_s + co] = b;
  }
}

// dW[co][k] (+)= dWp[co][k] for the layer's real rows and columns
__global__ void unpack_grad(const float *__restrict__ dwp, int cout, int k9, int kp,
                                   float *__restrict__ g) {
  const long total = (long)cout * k9;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int co = (int)(i / k9), k = (int)(i - (long)co * k9);
    g[i] += dwp[(long)co * kp + k];
  }
}

// input images (fp32 [n][h][w]) into the first tensor (BF16, channel 0)
__global__ void load_input(const float *__restrict__ x, int in_ch, long P, int Cs,
                                  uint16_t *__restrict__ y) {
  const long total = P * Cs;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i % Cs);
    y[i] = c < in_ch ? to_bf16(x[i / Cs * in_ch + c]) : (uint16_t)0;
  }
}

// batch b of a device dataset: samples idx[0..n) of [count][hw] arrays
__global__ void gather_samples(const float *__restrict__ src, const int *__restrict__ idx,
                                      int n, long hw, float *__restrict__ dst) {
  const long total = (long)n * hw;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const long j = i / hw;
    dst[i] = src[(long)idx[j] * hw + (i - j * hw)];
  }
}

__global__ void axpy1(const float *__restrict__ x, long n, float *__restrict__ y) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    y[i] += x[i];
}


// Images of an ImageGroup (nn_api.hpp) gathered into [n][hp][wp][in_ch]
// (zero padding; channel c > 0 from the start nbr[i (in_ch - 1) + c - 1]),
// and the RMS of channel 0 over its real rows x cols samples: one block per
// image; the image is divided by that RMS (1 for a zero image), which is
// kept for scatter_images.
__global__ void gather_images(const float *__restrict__ data, const long *__restrict__ base,
                              const long *__restrict__ nbr, int in_ch, int rows, int cols,
                              long row_stride, int hp, int wp, float *__restrict__ out,
                              float *__restrict__ rms) {
  const int i = blockIdx.x;
  const long n_px = (long)hp * wp;
  float *dst = out + (long)i * n_px * in_ch;
  float s = 0.f;
  for (int ch = 0; ch < in_ch; ++ch) {
    const float *src = data + (ch == 0 ? base[i] : nbr[(long)i * (in_ch - 1) + ch - 1]);
    for (long e = threadIdx.x; e < n_px; e += blockDim.x) {
      const int r = (int)(e / wp), c = (int)(e - (long)r * wp);
      const float v = (r < rows && c < cols) ? src[(long)r * row_stride + c] : 0.f;
      dst[e * in_ch + ch] = v;
      if (ch == 0) s += v * v;
    }
  }
  __shared__ float red[kNnThreads];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  const float rm = sqrtf(red[0] / (float)((long)rows * cols));
  const float r = rm > 0.f ? rm : 1.f;
  const float inv = 1.f / r;
  for (long e = threadIdx.x; e < n_px * in_ch; e += blockDim.x) dst[e] *= inv;
  if (threadIdx.x == 0) rms[i] = r;
}

// data[image i, row r, col c] = est[i][r][c] * rms[i] (real rows and cols)
__global__ void scatter_images(const float *__restrict__ est, const long *__restrict__ base,
                               int rows, int cols, long row_stride, int hp, int wp,
                               const float *__restrict__ rms, float *__restrict__ data) {
  const int i = blockIdx.x;
  float *dst = data + base[i];
  const float *src = est + (long)i * hp * wp;
  const float r = rms[i];
  for (long e = threadIdx.x; e < (long)rows * cols; e += blockDim.x) {
    const int rr = (int)(e / cols), c = (int)(e - (long)rr * cols);
    dst[(long)rr * row_stride + c] = src[(long)rr * wp + c] * r;
  }
}

// ------------------------------------------------ 16-byte forms (inference)
//
// Eight BF16 channels per thread and one row of pixels per block iteration,
// so that the index arithmetic (divisions by H and W) happens once per row,
// not per element.  Channel strides are powers of two times 8 (c8s = log2 of
// the 16-byte chunks per pixel).

__device__ __forceinline__ void unpack8(uint4 v, float (&f)[8]) {
  const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    f[2 * i] = __uint_as_float(w[i] << 16);
    f[2 * i + 1] = __uint_as_float(w[i] & 0xFFFF0000u);
  }
}

__device__ __forceinline__ uint4 pack8(const float (&f)[8]) {
  uint32_t w[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const __nv_bfloat162 h2 = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
    w[i] = *reinterpret_cast<const uint32_t *>(&h2);
  }
  return make_uint4(w[0], w[1], w[2], w[3]);
}

// y = nearest 2x upsampling of low (N, H/2, W/2) + skip (N, H, W)
__global__ void upsample2_add_v(const uint4 *__restrict__ low, const uint4 *__restrict__ skip,
                                int N, int H, int W, int c8s, uint4 *__restrict__ y) {
  const int C8 = 1 << c8s, per_row = W << c8s;
  const long rows = (long)N * H;
  for (long r = blockIdx.x; r < rows; r += gridDim.x) {
    const long n = r / H;
    const int yy = (int)(r - n * H);
    const uint4 *lrow = low + ((n * (H / 2) + yy / 2) * (W / 2) << c8s);
    const uint4 *srow = skip + (r * W << c8s);
    uint4 *yrow = y + (r * W << c8s);
    for (int e = threadIdx.x; e < per_row; e += blockDim.x) {
      float a[8], b[8];
      unpack8(lrow[((e >> c8s) >> 1 << c8s) + (e & (C8 - 1))], a);
      unpack8(srow[e], b);
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] += b[i];
      yrow[e] = pack8(a);
    }
  }
}

// y (N, H/2, W/2) = 2 x 2 average of x (N, H, W)
__global__ void avgpool2_v(const uint4 *__restrict__ x, int N, int H, int W, int c8s,
                           uint4 *__restrict__ y) {
  const int C8 = 1 << c8s, Ho = H / 2, Wo = W / 2, per_row = Wo << c8s;
  const long rows = (long)N * Ho;
  for (long r = blockIdx.x; r < rows; r += gridDim.x) {
    const long n = r / Ho;
    const int yo = (int)(r - n * Ho);
    const uint4 *r0 = x + ((n * H + 2 * yo) * W << c8s);
    const uint4 *r1 = r0 + ((long)W << c8s);
    uint4 *yrow = y + (r * Wo << c8s);
    for (int e = threadIdx.x; e < per_row; e += blockDim.x) {
      const int xo = e >> c8s, c = e & (C8 - 1);
      const int i0 = (2 * xo << c8s) + c, i1 = i0 + C8;
      float a[8], b[8], c2[8], d[8];
      unpack8(r0[i0], a);
      unpack8(r0[i1], b);
      unpack8(r1[i0], c2);
      unpack8(r1[i1], d);
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = 0.25f * (a[i] + b[i] + c2[i] + d[i]);
      yrow[e] = pack8(a);
    }
  }
}

// First layer (in_ch <= kFirstMaxIn input channels, interleaved per pixel):
// y[p][co] = bf16(act(bias[co] + sum over the 3 x 3 neighbourhood and the
// channels of bf16(x) * bf16(w[co][ky][kx][ci]))) for co < cout, zero for
// cout <= co < cout_s (a multiple of 8, at most 64), on the CUDA cores: 9
// in_ch products per output do not pay for an im2col copy.  One thread per
// pixel; products exact in FP32 (BF16 operands), FP32 sums.
constexpr int kFirstMaxIn = 4;

__global__ void conv_first(const float *__restrict__ x, int in_ch, int N, int H, int W,
                           const float *__restrict__ w, const float *__restrict__ bias, int cout,
                           int cout_s, int relu, uint4 *__restrict__ y) {
  __shared__ float ws[9 * kFirstMaxIn * 64], bs[64];
  const int K = 9 * in_ch;  // k = (ky * 3 + kx) * in_ch + ci, as the weight layout
  for (int i = threadIdx.x; i < K * cout_s; i += blockDim.x) {
    const int co = i / K, k = i - K * co;
    ws[k * 64 + co] = co < cout ? from_bf16(to_bf16(w[co * K + k])) : 0.f;
  }
  for (int i = threadIdx.x; i < cout_s; i += blockDim.x) bs[i] = i < cout ? bias[i] : 0.f;
  __syncthreads();
  const long P = (long)N * H * W;
  const int c8 = cout_s / 8;
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < P;
       p += (long)gridDim.x * blockDim.x) {
    const long r = p / W;
    const int xx = (int)(p - r * W), yy = (int)(r % H);
    float v[9 * kFirstMaxIn];
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const int dy = tap / 3 - 1, dx = tap % 3 - 1;
      const bool in = (unsigned)(yy + dy) < (unsigned)H && (unsigned)(xx + dx) < (unsigned)W;
      const float *src = x + (p + (long)dy * W + dx) * in_ch;
#pragma unroll
      for (int ci = 0; ci < kFirstMaxIn; ++ci)
        v[tap * kFirstMaxIn + ci] = in && ci < in_ch ? from_bf16(to_bf16(src[ci])) : 0.f;
    }
    for (int c = 0; c < c8; ++c) {
      float o[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        float acc = 0.f;
#pragma unroll
        for (int tap = 0; tap < 9; ++tap)
#pragma unroll
          for (int ci = 0; ci < kFirstMaxIn; ++ci)
            if (ci < in_ch)
              acc = fmaf(v[tap * kFirstMaxIn + ci], ws[(tap * in_ch + ci) * 64 + 8 * c + i], acc);
        acc += bs[8 * c + i];
        o[i] = (relu && acc < 0.f) || 8 * c + i >= cout ? 0.f : acc;
      }
      y[p * c8 + c] = pack8(o);
    }
  }
}

// x (P x in_ch, in_ch <= 8) -> channels 0 .. in_ch - 1 of y (P x 8 BF16, the
// other channels zero)
__global__ void load_input_v(const float *__restrict__ x, int in_ch, long P,
                             uint4 *__restrict__ y) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < P;
       p += (long)gridDim.x * blockDim.x) {
    uint32_t w[4] = {0u, 0u, 0u, 0u};
    for (int c = 0; c < in_ch; ++c) w[c >> 1] |= (uint32_t)to_bf16(x[p * in_ch + c]) << (16 * (c & 1));
    y[p] = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

}  // namespace nn
}  // namespace agd
