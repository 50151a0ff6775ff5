// BF16 GEMM on the tcgen05 tensor cores with FP32 accumulation in TMEM:
//   C[m][n] = alpha * sum_k A[m][k] B[n][k] + beta * C[m][n]
// A (M x K) and B (N x K) row-major BF16 with row strides lda, ldb (elements,
// multiples of 8, 16-byte aligned rows), K a multiple of 8; C row-major FP32.
//
// Split K (gridDim.z > 1): CTA z sums k in [z * k_split, (z + 1) * k_split)
// and adds alpha times its partial tile into C with atomics (C holds beta C
// beforehand; the caller scales or zeroes it).
//
// One CTA of 128 threads computes a 128 x BN tile: K is walked in 64-wide
// steps through two shared-memory stages filled by 16-byte cp.async copies
// (rows and k chunks past the matrix edges are zero-filled); thread 0 issues
// the four K = 16 MMAs of a stage and commits them to that stage's
// mbarrier, which the copies into the stage wait for before reusing it.  The
// epilogue reads the accumulator from TMEM (warp w holds rows 32w..32w+31).
#pragma once

#include <cstdint>

#include "umma.cuh"

namespace agd {

constexpr int kTcBM = 128;
constexpr int kTcBK = 64;
// stage layout: [row group][k chunk][8 rows][16 bytes], k chunks adjacent
constexpr uint32_t kTcLbo = 128;
constexpr uint32_t kTcSbo = (kTcBK / 8) * 128;

template <int BN>
struct TcGemmSmem {
  static constexpr int kABytes = kTcBM * kTcBK * 2;
  static constexpr int kBBytes = BN * kTcBK * 2;
  static constexpr int kStage = kABytes + kBBytes;
  static constexpr int kBytes = 2 * kStage + 64;  // two stages + barriers + TMEM slot
};

__device__ __forceinline__ void cp_async16_zfill(uint32_t saddr, const void *g, bool valid) {
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(saddr), "l"(g), "r"(n)
               : "memory");
}

// Copies rows [r0, r0 + rows) x k [k0, k0 + 64) of a row-major BF16 matrix
// (n_rows x K, row stride ld) into a stage in the K-major layout.
template <int ROWS>
__device__ __forceinline__ void tc_load_tile(uint32_t sbase, const uint16_t *g, int n_rows,
                                             int K, int ld, int r0, int k0) {
  constexpr int kChunks = ROWS * (kTcBK / 8);
  for (int q = threadIdx.x; q < kChunks; q += blockDim.x) {
    const int row = q >> 3, c = q & 7;
    const int gr = r0 + row, gk = k0 + 8 * c;
    const bool valid = gr < n_rows && gk < K;
    const uint16_t *src = valid ? g + (long)gr * ld + gk : g;
    const uint32_t dst = sbase + (uint32_t)(row >> 3) * kTcSbo + (uint32_t)c * kTcLbo +
                         (uint32_t)(row & 7) * 16u;
    cp_async16_zfill(dst, src, valid);
  }
}

// Implicit GEMM of a 3 x 3, padding 1 convolution: A[p][k] is read straight
// from NHWC BF16 activations x (n, h, w, channel stride cs) - row p a pixel,
// k = (ky * 3 + kx) * cin + ci - instead of from an im2col matrix.  Needs cin
// and cs multiples of 8 (a 16-byte chunk holds 8 channels of one tap).
struct ConvGeom {
  const uint16_t *x;  // nullptr: A is a plain matrix
  int n, h, w, cin, cs;
};

// Epilogue that writes BF16 activations instead of FP32 C: y[m][n] =
// bf16(act(acc + bias[n])) for n < n_real (ReLU when relu), 0 for the padded
// columns n_real <= n < N; y rows ldy apart.
struct BiasActOut {
  uint16_t *y;  // nullptr: the FP32 epilogue
  const float *bias;
  int n_real, ldy, relu;
};

template <int BN>
__global__ void __launch_bounds__(128) tc_gemm_bf16(const uint16_t *__restrict__ A,
                                                    const uint16_t *__restrict__ B,
                                                    float *__restrict__ C, int M, int N, int K,
                                                    int lda, int ldb, int ldc, float alpha,
                                                    float beta, int k_split, ConvGeom conv,
                                                    BiasActOut act, int *err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  using L = TcGemmSmem<BN>;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + 2 * L::kStage);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(smem + 2 * L::kStage + 32);
  constexpr uint32_t kCols = BN < 32 ? 32 : BN;
  const int m0 = blockIdx.x * kTcBM, n0 = blockIdx.y * BN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    umma::bar_init(&bars[0], 1);
    umma::bar_init(&bars[1], 1);
    umma::bar_init_fence();
  }
  if (warp == 0) umma::tmem_alloc(tslot, kCols);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = *tslot;
  const uint32_t s0 = umma::smem_u32(smem);
  constexpr uint32_t idesc = umma::idesc_bf16(kTcBM, BN);

  // this CTA's K range (split K: a slice of k_split, a multiple of kTcBK)
  const int kz0 = gridDim.z > 1 ? blockIdx.z * k_split : 0;
  const int kz1 = gridDim.z > 1 ? min(K, kz0 + k_split) : K;
  // (implicit convolutions are not split: kz0 = 0 for them)
  A += kz0;
  B += kz0;
  K = kz1 > kz0 ? kz1 - kz0 : 0;
  // implicit convolution: thread t always loads k chunk t & 7 of the rows
  // (t >> 3) + 16 i, i < 8 - their pixel coordinates are fixed for the tile
  constexpr int kRowsPerThread = kTcBM * (kTcBK / 8) / 128;
  long pix[kRowsPerThread];
  int py[kRowsPerThread], px[kRowsPerThread];
  if (conv.x != nullptr) {
#pragma unroll
    for (int i = 0; i < kRowsPerThread; ++i) {
      const int p = m0 + (int)(threadIdx.x >> 3) + 16 * i;
      const int xx = p % conv.w, t = p / conv.w;
      const int yy = t % conv.h, n = t / conv.h;
      py[i] = p < M ? yy : -(1 << 20);  // rows past M never pass the bounds test
      px[i] = xx;
      pix[i] = ((long)(n * conv.h + yy) * conv.w + xx) * conv.cs;
    }
  }
  auto load_a = [&](uint32_t sbase, int k0) {
    if (conv.x != nullptr) {
      const int c = threadIdx.x & 7;
      const int k = k0 + 8 * c;
      int dy = 0, dx = 0;
      long off = 0;
      const bool kv = k < K;
      if (kv) {
        const int tap = k / conv.cin, ci = k - tap * conv.cin;
        const int ky = tap / 3;
        dy = ky - 1;
        dx = tap - 3 * ky - 1;
        off = ((long)dy * conv.w + dx) * conv.cs + ci;
      }
#pragma unroll
      for (int i = 0; i < kRowsPerThread; ++i) {
        const int row = (int)(threadIdx.x >> 3) + 16 * i;
        const int sy = py[i] + dy, sx = px[i] + dx;
        const bool valid = kv && (unsigned)sy < (unsigned)conv.h && (unsigned)sx < (unsigned)conv.w;
        const uint32_t dst = sbase + (uint32_t)(row >> 3) * kTcSbo + (uint32_t)c * kTcLbo +
                             (uint32_t)(row & 7) * 16u;
        cp_async16_zfill(dst, valid ? conv.x + pix[i] + off : conv.x, valid);
      }
    } else {
      tc_load_tile<kTcBM>(sbase, A, M, K, lda, m0, k0);
    }
  };
  const bool split = gridDim.z > 1;
  const int nk = (K + kTcBK - 1) / kTcBK;
  bool ok = true;
  auto stage_a = [&](int s) { return s0 + (uint32_t)s * L::kStage; };
  auto stage_b = [&](int s) { return s0 + (uint32_t)s * L::kStage + L::kABytes; };
  load_a(stage_a(0), 0);
  tc_load_tile<BN>(stage_b(0), B, N, K, ldb, n0, 0);
  asm volatile("cp.async.commit_group;" ::: "memory");
  for (int kt = 0; kt < nk && ok; ++kt) {
    const int s = kt & 1;
    if (kt + 1 < nk) {
      // stage s^1 was read by the MMAs of step kt - 1
      if (kt >= 1) ok = umma::bar_wait(&bars[s ^ 1], ((kt - 1) >> 1) & 1);
      if (ok) {
        load_a(stage_a(s ^ 1), (kt + 1) * kTcBK);
        tc_load_tile<BN>(stage_b(s ^ 1), B, N, K, ldb, n0, (kt + 1) * kTcBK);
      }
      asm volatile("cp.async.commit_group;" ::: "memory");
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    umma::fence_async_smem();
    ok = __syncthreads_and(ok);  // every thread takes the same branch
    if (!ok) break;
    if (threadIdx.x == 0) {
      umma::fence_after_sync();
#pragma unroll
      for (int j = 0; j < kTcBK / 16; ++j) {
        const uint64_t ad = umma::desc_kmajor(stage_a(s) + 2 * j * kTcLbo, kTcLbo, kTcSbo);
        const uint64_t bd = umma::desc_kmajor(stage_b(s) + 2 * j * kTcLbo, kTcLbo, kTcSbo);
        umma::mma_bf16(tbase, ad, bd, idesc, (kt > 0 || j > 0) ? 1u : 0u);
      }
      umma::commit(&bars[s]);
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  if (ok && nk > 0) ok = umma::bar_wait(&bars[(nk - 1) & 1], ((nk - 1) >> 1) & 1);
  ok = __syncthreads_and(ok);
  umma::fence_after_sync();
  if (!ok) {
    if (lane == 0) atomicExch(err, 1);
  } else {
    const int row = m0 + 32 * (warp & 3) + lane;
    const uint32_t taddr = tbase + ((uint32_t)(32 * (warp & 3)) << 16);
#pragma unroll 1
    for (int cc = 0; cc < BN / 16; ++cc) {
      float v[16];
      if (nk > 0) {
        umma::tmem_ld16(taddr + cc * 16, v);
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = 0.f;
      }
      if (row < M && act.y != nullptr) {
        uint32_t packed[8];
#pragma unroll
        for (int i = 0; i < 16; i += 2) {
          const int n = n0 + cc * 16 + i;
          float a = n < act.n_real ? v[i] + act.bias[n] : 0.f;
          float b = n + 1 < act.n_real ? v[i + 1] + act.bias[n + 1] : 0.f;
          if (act.relu) {
            a = fmaxf(a, 0.f);
            b = fmaxf(b, 0.f);
          }
          const __nv_bfloat162 h2 = __floats2bfloat162_rn(a, b);
          packed[i / 2] = *reinterpret_cast<const uint32_t *>(&h2);
        }
        uint16_t *y = act.y + (long)row * act.ldy + n0 + cc * 16;
        if (n0 + cc * 16 + 16 <= N) {  // 16 columns: two 16-byte stores
          reinterpret_cast<uint4 *>(y)[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
          reinterpret_cast<uint4 *>(y)[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
        } else {
#pragma unroll
          for (int i = 0; i < 16; ++i)
            if (n0 + cc * 16 + i < N)
              y[i] = (uint16_t)(packed[i / 2] >> (16 * (i & 1)));
        }
      } else if (row < M) {
        float *c = C + (long)row * ldc + n0 + cc * 16;
        if (split) {
#pragma unroll
          for (int i = 0; i < 16; ++i)
            if (n0 + cc * 16 + i < N && nk > 0) atomicAdd(c + i, alpha * v[i]);
        } else {
#pragma unroll
          for (int i = 0; i < 16; ++i)
            if (n0 + cc * 16 + i < N) c[i] = alpha * v[i] + (beta != 0.f ? beta * c[i] : 0.f);
        }
      }
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tbase, kCols);
}

}  // namespace agd
