// BF16 GEMM on the tcgen05 tensor cores with FP32 accumulation in TMEM:
//   C[m][n] = alpha * sum_k A[m][k] B[n][k] + beta * C[m][n]
// A (M x K) and B (N x K) row-major BF16 with row strides lda, ldb (elements,
// multiples of 8, 16-byte aligned rows), K a multiple of 8; C row-major FP32.
//
// Split K (gridDim.z > 1): CTA z sums k in [z * k_split, (z + 1) * k_split)
// and either stores alpha times its partial tile into the slice C + z *
// split_stride (split_stride > 0; split_reduce then sums the slices in a
// fixed order, so the result does not depend on the CTAs' timing) or adds
// it into C with atomics (C holds beta C beforehand; the caller scales or
// zeroes it).
//
// One CTA of 128 threads computes a 128 x BN tile: K is walked in 64-wide
// steps through two shared-memory stages filled by 16-byte cp.async copies
// (rows and k chunks past the matrix edges are zero-filled); thread 0 issues
// the four K = 16 MMAs of a stage and commits them to that stage's
// mbarrier, which the copies into the stage wait for before reusing it.  The
// epilogue reads the accumulator from TMEM (warp w holds rows 32w..32w+31).
#pragma once

#include <cstdint>

#include <cuda.h>

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
                                                    float beta, int k_split, long split_stride,
                                                    ConvGeom conv,
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
        if (split && split_stride > 0) {
          float *cz = c + (long)blockIdx.z * split_stride;
#pragma unroll
          for (int i = 0; i < 16; ++i)
            if (n0 + cc * 16 + i < N) cz[i] = alpha * v[i];  // v is 0 for an empty slice
        } else if (split) {
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

// C[r][c] = beta C[r][c] + sum over z < splits (in order) of the slices
// ws[z * slice + r * ldc + c], r < M, c < N.
__global__ void split_reduce(const float *__restrict__ ws, int splits, long slice, int M, int N,
                             int ldc, float *__restrict__ C, float beta) {
  const long total = (long)M * N;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int r = (int)(i / N), c = (int)(i - (long)r * N);
    const long o = (long)r * ldc + c;
    float s = beta != 0.f ? beta * C[o] : 0.f;
    for (int z = 0; z < splits; ++z) s += ws[z * slice + o];
    C[o] = s;
  }
}

}  // namespace agd

namespace agd {

// ------------------------------------------------------------ persistent GEMM
//
// The same product (no split K) by persistent CTAs of 256 threads, two per
// SM, that walk the output tiles blockIdx.x, blockIdx.x + gridDim.x, ...
// (all M tiles of an N tile before the next N tile, so the B tile stays in
// L2).  The K steps of every tile form one sequence per CTA, streamed
// through S shared-memory stages by cp.async S - 1 steps ahead of the MMAs
// (S = 4, or 3 for BN = 128 so that two CTAs fit an SM); the accumulator has
// two TMEM buffers, so the epilogue of tile j - 1 runs while the tensor core
// works on tile j and the copies for tile j + 1 are in flight.  Iteration g
// of the sequence: wait for step g's copies, thread 0 issues its four MMAs
// (and commits them to the stage's mbarrier, and at a tile's last step to
// the accumulator's), then every thread waits for step g - 1's MMAs and
// refills their stage with step g + S - 1.
//
// Copies: thread t fills k chunk (t >> 3) & 7 of rows (t & 7) + 8 (t >> 6)
// + 32 i, so the eight threads of a shared-memory wavefront write the eight
// rows of one core matrix (no bank conflicts) and a warp reads eight
// consecutive rows x 64 bytes.  For implicit convolutions the tap of every
// k chunk (its offset in the activations and its (dy, dx)) comes from a
// table the CTA builds once, and the pixel coordinates of a thread's rows
// are derived once per tile.  Needs K > 0 and, for convolutions,
// K / 8 <= kPipeMaxChunks.
constexpr int kPipeThreads = 256;
constexpr int kPipeMaxChunks = 512;

template <int BN>
struct TcPipeSmem {
  static constexpr int kStages = BN >= 128 ? 3 : 4;
  static constexpr int kABytes = kTcBM * kTcBK * 2;
  static constexpr int kBBytes = BN * kTcBK * 2;
  static constexpr int kStage = kABytes + kBBytes;
  static constexpr int kTab = kStages * kStage;             // int2 per k chunk
  static constexpr int kBar = kTab + 8 * kPipeMaxChunks;    // stage, accumulator barriers
  static constexpr int kBytes = kBar + 8 * (kStages + 2) + 16;
  static constexpr uint32_t kCols = 2 * BN < 32 ? 32 : 2 * BN;  // power of two for BN 16..128
  static constexpr int kPerSm = 2;
  static_assert(kPerSm * (kBytes + 1024) <= 233472, "two CTAs per SM");
};

template <int BN>
__global__ void __launch_bounds__(kPipeThreads, 2)
    tc_gemm_pipe(const uint16_t *__restrict__ A, const uint16_t *__restrict__ B,
                 float *__restrict__ C, int M, int N, int K, int lda, int ldb, int ldc,
                 float alpha, float beta, ConvGeom conv, BiasActOut act, int *err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  using L = TcPipeSmem<BN>;
  constexpr int S = L::kStages;
  int2 *tab = reinterpret_cast<int2 *>(smem + L::kTab);
  uint64_t *sbar = reinterpret_cast<uint64_t *>(smem + L::kBar);  // [S] stages
  uint64_t *abar = sbar + S;                                       // [2] accumulators
  uint32_t *tslot = reinterpret_cast<uint32_t *>(abar + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nk = (K + kTcBK - 1) / kTcBK;
  if (tid == 0) {
    for (int i = 0; i < S + 2; ++i) umma::bar_init(&sbar[i], 1);
    umma::bar_init_fence();
  }
  if (conv.x != nullptr) {
    // k chunk j: tap (ky, kx), channel ci; .x the offset of (dy, dx, ci) in
    // the activations, .y = (dy + 1) | (dx + 1) << 2, or -1 past K
    for (int j = tid; j < nk * (kTcBK / 8); j += kPipeThreads) {
      const int k = 8 * j;
      int2 e = make_int2(0, -1);
      if (k < K) {
        const int tap = k / conv.cin, ci = k - tap * conv.cin;
        const int ky = tap / 3, kx = tap - 3 * ky;
        e.x = ((ky - 1) * conv.w + (kx - 1)) * conv.cs + ci;
        e.y = ky | (kx << 2);
      }
      tab[j] = e;
    }
  }
  if (warp == 0) umma::tmem_alloc(tslot, L::kCols);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = *tslot;
  const uint32_t s0 = umma::smem_u32(smem);
  constexpr uint32_t idesc = umma::idesc_bf16(kTcBM, BN);
  const int n_m = (M + kTcBM - 1) / kTcBM;
  const int total = n_m * ((N + BN - 1) / BN);
  const int n_local = (int)blockIdx.x < total ? (total - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int G = n_local * nk;
  auto tile_of = [&](int lt, int &m0, int &n0) {
    const int t = (int)blockIdx.x + lt * (int)gridDim.x;
    const int nt = t / n_m;
    m0 = (t - nt * n_m) * kTcBM;
    n0 = nt * BN;
  };
  // this thread's copy slots
  const int ck = (tid >> 3) & 7;                  // k chunk
  const int rb = (tid & 7) + 8 * (tid >> 6);      // first row; rows rb + 32 i
  const uint32_t slot = (uint32_t)(rb >> 3) * kTcSbo + (uint32_t)ck * kTcLbo + (uint32_t)(rb & 7) * 16u;
  constexpr uint32_t kRowStep = 4 * kTcSbo;       // 32 rows
  constexpr int kRowsA = kTcBM / 32, kRowsB = BN / 32 > 0 ? BN / 32 : 1;
  // loader state: the step it copies next
  int ld_lt = 0, ld_kt = 0, ld_st = 0, m0l = 0, n0l = 0;
  long pix[kRowsA];
  int py[kRowsA], px[kRowsA];
  auto load_next = [&]() {
    if (ld_lt < n_local) {
      if (ld_kt == 0) {
        tile_of(ld_lt, m0l, n0l);
        if (conv.x != nullptr) {
          int p = m0l + rb;
          int x = p % conv.w, y = (p / conv.w) % conv.h;
#pragma unroll
          for (int i = 0; i < kRowsA; ++i) {
            py[i] = p < M ? y : -(1 << 20);  // rows past M never pass the bounds test
            px[i] = x;
            pix[i] = (long)p * conv.cs;
            p += 32;
            x += 32;
            while (x >= conv.w) {
              x -= conv.w;
              if (++y == conv.h) y = 0;
            }
          }
        }
      }
      const uint32_t sa = s0 + (uint32_t)ld_st * L::kStage, sb = sa + L::kABytes;
      const int k0 = ld_kt * kTcBK, k = k0 + 8 * ck;
      if (conv.x != nullptr) {
        const int2 e = tab[ld_kt * (kTcBK / 8) + ck];
        const int dy = (e.y & 3) - 1, dx = ((e.y >> 2) & 3) - 1;
#pragma unroll
        for (int i = 0; i < kRowsA; ++i) {
          const int sy = py[i] + dy, sx = px[i] + dx;
          const bool valid =
              e.y >= 0 && (unsigned)sy < (unsigned)conv.h && (unsigned)sx < (unsigned)conv.w;
          cp_async16_zfill(sa + slot + i * kRowStep, valid ? conv.x + pix[i] + e.x : conv.x,
                           valid);
        }
      } else {
#pragma unroll
        for (int i = 0; i < kRowsA; ++i) {
          const int gr = m0l + rb + 32 * i;
          const bool valid = gr < M && k < K;
          cp_async16_zfill(sa + slot + i * kRowStep, valid ? A + (long)gr * lda + k : A, valid);
        }
      }
#pragma unroll
      for (int i = 0; i < kRowsB; ++i) {
        const int gr = n0l + rb + 32 * i;
        const bool valid = rb + 32 * i < BN && gr < N && k < K;
        if (rb + 32 * i < BN)
          cp_async16_zfill(sb + slot + i * kRowStep, valid ? B + (long)gr * ldb + k : B, valid);
      }
      ld_st = ld_st + 1 == S ? 0 : ld_st + 1;
      if (++ld_kt == nk) {
        ld_kt = 0;
        ++ld_lt;
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  bool ok = true;
  // epilogue: warp w reads TMEM lanes 32 (w % 4) .., columns of half w / 4
  auto epilogue = [&](int lt) {
    ok = umma::bar_wait(&abar[lt & 1], (lt >> 1) & 1) && ok;
    ok = __syncthreads_and(ok);
    umma::fence_after_sync();
    if (!ok) return;
    int m0, n0;
    tile_of(lt, m0, n0);
    const int row = m0 + 32 * (warp & 3) + lane;
    const int c0 = (warp >> 2) * (BN / 2);
    const uint32_t taddr = tbase + ((uint32_t)(32 * (warp & 3)) << 16) +
                           (uint32_t)((lt & 1) * BN + c0);
#pragma unroll 1
    for (int cc = 0; cc < BN / 32; ++cc) {
      float v[16];
      umma::tmem_ld16(taddr + cc * 16, v);
      if (row >= M) continue;
      const int nb = n0 + c0 + cc * 16;
      if (act.y != nullptr) {
        uint32_t packed[8];
#pragma unroll
        for (int i = 0; i < 16; i += 2) {
          const int n = nb + i;
          float a = n < act.n_real ? v[i] + act.bias[n] : 0.f;
          float b = n + 1 < act.n_real ? v[i + 1] + act.bias[n + 1] : 0.f;
          if (act.relu) {
            a = fmaxf(a, 0.f);
            b = fmaxf(b, 0.f);
          }
          const __nv_bfloat162 h2 = __floats2bfloat162_rn(a, b);
          packed[i / 2] = *reinterpret_cast<const uint32_t *>(&h2);
        }
        uint16_t *y = act.y + (long)row * act.ldy + nb;
        if (nb + 16 <= N) {
          reinterpret_cast<uint4 *>(y)[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
          reinterpret_cast<uint4 *>(y)[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
        } else {
#pragma unroll
          for (int i = 0; i < 16; ++i)
            if (nb + i < N) y[i] = (uint16_t)(packed[i / 2] >> (16 * (i & 1)));
        }
      } else {
        float *c = C + (long)row * ldc + nb;
#pragma unroll
        for (int i = 0; i < 16; ++i)
          if (nb + i < N) c[i] = alpha * v[i] + (beta != 0.f ? beta * c[i] : 0.f);
      }
    }
    umma::fence_before_sync();  // TMEM reads done before the buffer is reused
  };

  for (int g = 0; g < S - 1; ++g) load_next();  // steps 0 .. S - 2 in flight
  int lt = 0, kt = 0, st = 0, ph = 0;            // the step the MMAs take next
  int pst = 0, pph = 0;                           // the previous step's stage, phase
  for (int g = 0; g < G; ++g) {
    asm volatile("cp.async.wait_group %0;" ::"n"(S - 2) : "memory");  // step g landed
    umma::fence_async_smem();
    ok = __syncthreads_and(ok);  // every thread takes the same branch
    if (!ok) break;
    if (tid == 0) {
      umma::fence_after_sync();
      const uint32_t sa = s0 + (uint32_t)st * L::kStage, sb = sa + L::kABytes;
      const uint32_t d = tbase + (uint32_t)((lt & 1) * BN);
      const uint64_t a0 = umma::desc_kmajor(sa, kTcLbo, kTcSbo);
      const uint64_t b0 = umma::desc_kmajor(sb, kTcLbo, kTcSbo);
#pragma unroll
      for (int j = 0; j < kTcBK / 16; ++j)  // K = 16: two chunks, 2 * 128 bytes
        umma::mma_bf16(d, a0 + 16u * j, b0 + 16u * j, idesc, (kt > 0 || j > 0) ? 1u : 0u);
      umma::commit(&sbar[st]);
      if (kt == nk - 1) umma::commit(&abar[lt & 1]);
    }
    // step g - 1's MMAs done: its stage takes step g + S - 1
    if (g >= 1) ok = umma::bar_wait(&sbar[pst], pph) && ok;
    load_next();
    if (kt == nk - 1 && lt >= 1) epilogue(lt - 1);
    pst = st;
    pph = ph;
    if (++st == S) {
      st = 0;
      ph ^= 1;
    }
    if (++kt == nk) {
      kt = 0;
      ++lt;
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  ok = __syncthreads_and(ok);
  if (ok && n_local > 0) epilogue(n_local - 1);
  if (!ok && tid == 0) atomicExch(err, 1);
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tbase, L::kCols);
}

}  // namespace agd

namespace agd {

// ------------------------------------------------ 3 x 3 convolution, halo tiles
//
// Y = conv3x3(X) (padding 1) with the weight rows [n0, n0 + BN) of the
// layer (B, N x 9 cin, k = tap * cin + ci) held in shared memory for the
// life of the CTA: blockIdx.y selects the group of BN output channels.  An
// output tile is 128 consecutive pixels of one image row (w a multiple of
// 128); for each block of 32 input channels the tile's halo - 3 rows x 130
// pixels of each 8-channel chunk, zero outside the image - arrives by four
// TMA box loads (box 8 channels x 130 pixels x 3 rows of the NHWC tensor
// map, corner at (channel, x0 - 1, y - 1, image); the tensor map's bounds
// give the zero padding), one plane per chunk, and the nine taps read it
// through shifted shared-memory descriptors: tap (ky, kx) of chunk c starts
// at plane c, row ky, pixel kx, with 8 pixels (16 bytes each) per core
// matrix.  So each input value crosses L2 about 3 times per layer and
// channel group instead of 9 (the implicit-GEMM loader), and B once per
// CTA.  Persistent CTAs (PER_SM per SM: two with at most 36 KB of B, one
// with up to 144 KB) walk the tiles.
//
// Roles, linked only by mbarriers: lane 0 of warp 8 issues the TMA loads of
// step g + 2 into the 3-stage ring (after the MMAs of step g - 1 released
// it: `empty`) and then the 18 MMAs of step g (after its loads landed:
// `full`; at a tile's first step also after the epilogue of the tile that
// last used the accumulator: `acc_empty`), committed to `empty` (and at a
// tile's last step to `acc_full`).  Warps 0-7 run the epilogues (TMEM ->
// bias, ReLU, BF16 or FP32 -> global) and arrive on `acc_empty`.  Two TMEM
// accumulators, so the tensor core runs tile j while the epilogue of tile
// j - 1 drains.  Every wait is bounded; a timeout sets *err.
constexpr int kHaloPix = 130;                       // pixels of a halo row (the TMA box)
constexpr int kHaloBox = 3 * kHaloPix * 16;         // bytes of one chunk's box
constexpr int kHaloPlane = 6528;                    // plane stride: the box, 128-byte aligned
constexpr int kHaloStage = 4 * kHaloPlane;          // 32 channels
constexpr int kHaloStages = 3;
constexpr int kHaloThreads = kPipeThreads + 32;     // 8 epilogue warps + the control warp
static_assert(kHaloPlane % 128 == 0 && kHaloPlane >= kHaloBox, "TMA destinations");

template <int PER_SM>
struct TcHaloSmem {
  static constexpr int kMaxB = PER_SM == 2 ? 36864 : 147456;  // bytes of B (BN x K bf16)
  static constexpr int kB = kHaloStages * kHaloStage;
  static constexpr int kBias = kB + kMaxB;                     // BN floats
  static constexpr int kBar = kBias + (PER_SM == 2 ? 256 : 512);
  static constexpr int kBytes = kBar + 8 * (2 * kHaloStages + 4) + 16;
  static_assert(PER_SM * (kBytes + 1024) <= 233472, "CTAs per SM");
};

template <int BN, int PER_SM>
__global__ void __launch_bounds__(kHaloThreads, PER_SM)
    tc_conv_halo(const __grid_constant__ CUtensorMap xmap, const uint16_t *__restrict__ B,
                 float *__restrict__ C, int M, int N, int ldc, ConvGeom conv, BiasActOut act,
                 int *err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  using L = TcHaloSmem<PER_SM>;
  constexpr int S = kHaloStages;
  constexpr int P = kPipeThreads;  // epilogue threads
  static_assert(BN * 4 <= L::kBar - L::kBias, "bias buffer");
  float *bias_s = reinterpret_cast<float *>(smem + L::kBias);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + L::kBar);
  uint64_t *empty = full + S;
  uint64_t *acc_full = empty + S;
  uint64_t *acc_empty = acc_full + 2;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(acc_empty + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int K = 9 * conv.cin;           // B row length (cin == cs, a multiple of 32)
  const int nkb = conv.cin / 32;        // channel blocks per tile
  const uint32_t s0 = umma::smem_u32(smem);
  const uint32_t sB = s0 + L::kB;
  const uint32_t b_sbo = (uint32_t)(K / 8) * 128u;  // B: [row group][k chunk][8 rows][16 B]
  const int n0 = (int)blockIdx.y * BN;
  if ((s0 & 127u) != 0) {  // TMA destinations must be 128-byte aligned
    if (tid == 0) atomicExch(err, 1);
    return;
  }
  if (tid == 0) {
    for (int i = 0; i < S; ++i) {
      umma::bar_init(&full[i], 1);
      umma::bar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      umma::bar_init(&acc_full[i], 1);
      umma::bar_init(&acc_empty[i], P);
    }
    umma::bar_init_fence();
  }
  // this CTA's weight rows (rows >= N zero) and biases, once
  for (int q = tid; q < BN * (K / 8); q += kHaloThreads) {
    const int row = q / (K / 8), c = q - row * (K / 8);
    const bool valid = n0 + row < N;
    cp_async16_zfill(sB + (uint32_t)(row >> 3) * b_sbo + (uint32_t)c * 128u +
                         (uint32_t)(row & 7) * 16u,
                     valid ? B + (long)(n0 + row) * K + 8 * c : B, valid);
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
  if (tid < BN)
    bias_s[tid] = act.bias != nullptr && n0 + tid < act.n_real ? act.bias[n0 + tid] : 0.f;
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  umma::fence_async_smem();
  if (warp == 0) umma::tmem_alloc(tslot, 2 * BN);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = *tslot;
  const int total = M / kTcBM;
  const int n_local =
      (int)blockIdx.x < total ? (total - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int G = n_local * nkb;
  bool ok = true;

  if (warp == P / 32) {
    // ------------------------------------------------- TMA loads and MMAs
    if (lane == 0) {
      constexpr uint32_t idesc = umma::idesc_bf16(kTcBM, BN);
      const uint32_t tap_chunks = (uint32_t)(conv.cin / 8);
      const long hw = (long)conv.h * conv.w;
      int ld_lt = 0, ld_kb = 0, ld_n = 0, ld_y = 0, ld_x0 = 0, issued = 0, consumed = 0;
      auto load = [&](int g) {  // step g (in order) into stage g % S
        const int st = g % S;
        if (g >= S) ok = umma::bar_wait(&empty[st], ((g / S) - 1) & 1) && ok;
        if (!ok) return;
        if (ld_kb == 0) {
          const long p0 = (long)((int)blockIdx.x + ld_lt * (int)gridDim.x) * kTcBM;
          ld_n = (int)(p0 / hw);
          const long r = p0 - (long)ld_n * hw;
          ld_y = (int)(r / conv.w);
          ld_x0 = (int)(r - (long)ld_y * conv.w);
        }
        umma::bar_arrive_expect_tx(&full[st], 4 * kHaloBox);
        const uint32_t dst = s0 + (uint32_t)st * kHaloStage;
#pragma unroll
        for (int c = 0; c < 4; ++c)
          umma::tma_load_4d(dst + (uint32_t)c * kHaloPlane, &xmap, 32 * ld_kb + 8 * c, ld_x0 - 1,
                            ld_y - 1, ld_n, &full[st]);
        issued = g + 1;
        if (++ld_kb == nkb) {
          ld_kb = 0;
          ++ld_lt;
        }
      };
      for (int g = 0; g < S - 1 && g < G; ++g) load(g);
      int lt = 0, kb = 0, st = 0, ph = 0;
      for (int g = 0; g < G && ok; ++g) {
        if (g + S - 1 < G) load(g + S - 1);
        // the epilogue of tile lt - 2 has read this accumulator
        if (ok && kb == 0 && lt >= 2)
          ok = umma::bar_wait(&acc_empty[lt & 1], ((lt >> 1) - 1) & 1);
        if (ok) ok = umma::bar_wait(&full[st], ph);
        if (!ok) break;
        consumed = g + 1;
        umma::fence_after_sync();
        // descriptors as base + start offset (16-byte units; shared-memory
        // addresses stay below 2^18, so the 14-bit start field cannot carry)
        const uint64_t a0 = umma::desc_kmajor(s0 + (uint32_t)st * kHaloStage, kHaloPlane, 128u);
        const uint64_t b0 = umma::desc_kmajor(sB, 128u, b_sbo) + (uint64_t)(4 * kb) * 8u;
        const uint32_t d = tbase + (uint32_t)((lt & 1) * BN);
#pragma unroll
        for (int tap = 0; tap < 9; ++tap) {
          const int ky = tap / 3, kx = tap - 3 * ky;
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const uint64_t ad =
                a0 + (uint64_t)((2 * q * kHaloPlane + (ky * kHaloPix + kx) * 16) >> 4);
            const uint64_t bd = b0 + (uint64_t)(tap * tap_chunks + 2 * q) * 8u;
            umma::mma_bf16(d, ad, bd, idesc, (kb > 0 || tap > 0 || q > 0) ? 1u : 0u);
          }
        }
        umma::commit(&empty[st]);
        if (kb == nkb - 1) umma::commit(&acc_full[lt & 1]);
        if (++st == S) {
          st = 0;
          ph ^= 1;
        }
        if (++kb == nkb) {
          kb = 0;
          ++lt;
        }
      }
      // after an error: loads still in flight land before the CTA's shared
      // memory goes away (bounded waits)
      for (int g = consumed; g < issued; ++g) umma::bar_wait(&full[g % S], (g / S) & 1);
    }
  } else {
    // -------------------------------------------------------- epilogues
    for (int lt = 0; lt < n_local && ok; ++lt) {
      ok = umma::bar_wait(&acc_full[lt & 1], (lt >> 1) & 1);
      if (!ok) break;
      umma::fence_after_sync();
      const int row = ((int)blockIdx.x + lt * (int)gridDim.x) * kTcBM + 32 * (warp & 3) + lane;
      const int c0 = (warp >> 2) * (BN / 2);
      const uint32_t taddr = tbase + ((uint32_t)(32 * (warp & 3)) << 16) +
                             (uint32_t)((lt & 1) * BN + c0);
#pragma unroll 1
      for (int cc = 0; cc < BN / 32; ++cc) {
        float v[16];
        umma::tmem_ld16(taddr + cc * 16, v);
        const int nl = c0 + cc * 16, nb = n0 + nl;
        if (nb >= N) continue;
        if (act.y != nullptr) {
          uint32_t packed[8];
#pragma unroll
          for (int i = 0; i < 16; i += 2) {
            float a = nb + i < act.n_real ? v[i] + bias_s[nl + i] : 0.f;
            float b = nb + i + 1 < act.n_real ? v[i + 1] + bias_s[nl + i + 1] : 0.f;
            if (act.relu) {
              a = fmaxf(a, 0.f);
              b = fmaxf(b, 0.f);
            }
            const __nv_bfloat162 h2 = __floats2bfloat162_rn(a, b);
            packed[i / 2] = *reinterpret_cast<const uint32_t *>(&h2);
          }
          uint16_t *y = act.y + (long)row * act.ldy + nb;
          if (nb + 16 <= N) {
            reinterpret_cast<uint4 *>(y)[0] =
                make_uint4(packed[0], packed[1], packed[2], packed[3]);
            reinterpret_cast<uint4 *>(y)[1] =
                make_uint4(packed[4], packed[5], packed[6], packed[7]);
          } else {
#pragma unroll
            for (int i = 0; i < 16; ++i)
              if (nb + i < N) y[i] = (uint16_t)(packed[i / 2] >> (16 * (i & 1)));
          }
        } else {
          float *c = C + (long)row * ldc + nb;
#pragma unroll
          for (int i = 0; i < 16; ++i)
            if (nb + i < N) c[i] = v[i];
        }
      }
      umma::fence_before_sync();  // TMEM reads done before the MMAs reuse the buffer
      umma::bar_arrive(&acc_empty[lt & 1]);
    }
  }
  if (!ok) atomicExch(err, 1);
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tbase, 2 * BN);
}

}  // namespace agd
