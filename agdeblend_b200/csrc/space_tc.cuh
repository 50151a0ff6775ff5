// Space axes of the FK operator as split-BF16 tensor-core contractions
// (tcgen05, FP32 accumulation in TMEM) for windows with three space axes of
// padded length P and window length L (the forward crops P -> L, the adjoint
// zero-pads L -> P): the precision variant of space_fwd_fast /
// space_adj_fast (reference fk_forward / fk_adjoint, src/fk.c:307-452, whose
// space part is the FFTW c2r / r2c over the padded space axes).
//
// The DFT along one axis of a plane is a product with a small complex
// matrix, written as a real matrix on interleaved (re, im) values:
//   forward  y_n = sum_k exp(+2 pi i n k / P) x_k   (n < L, k < P)
//   adjoint  y_k = sum_n exp(-2 pi i n k / P) x_n   (k < P, n < L)
// Operands and matrices are split into hi + lo BF16 parts and each product
// is A_hi B_hi + A_hi B_lo + A_lo B_hi (three MMAs per K = 16 step, "3-pass"
// split-BF16): about 16 significant bits per operand, FP32 sums.
//
// One plane per step of a persistent CTA (256 threads, one CTA per SM):
//   1. the plane (staged in shared memory by cp.async one plane ahead) is
//      split into the A operand of the first axis: rows = the lines of that
//      axis, k = 2 * index + (re, im);
//   2. for each axis: thread 0 issues the MMAs of every 128-row tile (D = A
//      B^T, N = 2 * outputs) and commits them to an mbarrier; after the
//      wait, the epilogue reads D from TMEM (warp w: lanes 32 (w % 4).. of
//      the tile, column half w / 4) and writes the next axis's A operand,
//      transposed so that the next axis's index becomes k;
//   3. the last epilogue stores the cropped plane (forward) or applies the
//      ISTA update to the model plane (adjoint, model staged by cp.async).
// Operand layout: K-major 8 x 16-byte core matrices with k chunks 144 bytes
// apart (128 + 16: the transposing stores of a warp spread over the banks).
#pragma once

#include <cstdint>

#include "fast.cuh"
#include "kernels.cuh"
#include "umma.cuh"

namespace agd {

constexpr int kTcThreads = 256;
constexpr uint32_t kTcChunkStride = 144;  // bytes between the k chunks of a row group
constexpr int kTcTileCols = 64;           // TMEM columns between the accumulators of two tiles

// K-major operand of KCH k chunks (8 BF16 each): row groups SBO bytes apart.
template <int KCH>
struct TcOp {
  static constexpr uint32_t kLbo = kTcChunkStride;
  static constexpr uint32_t kSbo = (KCH - 1) * kTcChunkStride + 128;
  static_assert(kSbo % 16 == 0, "16-byte strides");
  __host__ __device__ static constexpr uint32_t bytes(int rows) {
    return (uint32_t)(rows / 8) * kSbo;
  }
  __device__ static uint32_t offset(int row, int k) {
    return (uint32_t)(row >> 3) * kSbo + (uint32_t)(k >> 3) * kLbo + (uint32_t)(row & 7) * 16u +
           (uint32_t)(k & 7) * 2u;
  }
};

// Shapes of one kernel: P padded, L window length, three space axes.
template <int P, int L>
struct TcDft3 {
  static_assert(L <= P && 2 * L % 16 == 0, "window columns in 16-column groups");
  // forward: contraction over P (K = 2P padded to a multiple of 16), L outputs
  static constexpr int kFwdK = (2 * P + 15) / 16 * 16;
  static constexpr int kFwdKch = kFwdK / 8;
  static constexpr int kFwdN = 2 * L;
  // adjoint: contraction over L, P outputs (N padded to a multiple of 16)
  static constexpr int kAdjK = (2 * L + 15) / 16 * 16;
  static constexpr int kAdjKch = kAdjK / 8;
  static constexpr int kAdjN = (2 * P + 15) / 16 * 16;
  // rows of the three passes (lines of the remaining axes)
  static constexpr int kRowsMax = P * P;
  static constexpr int kTilesMax = (kRowsMax + 127) / 128;
  static constexpr int kRowsPad = kTilesMax * 128;
  static constexpr int kPlaneP = P * P * P;  // model plane, complex
  static constexpr int kPlaneL = L * L * L;  // cropped plane, complex
  using FwdOp = TcOp<kFwdKch>;
  using AdjOp = TcOp<kAdjKch>;
  // shared memory: A hi, A lo (largest pass), B hi, B lo, staging, barriers
  static constexpr uint32_t kFwdA = FwdOp::bytes(kRowsPad);
  static constexpr uint32_t kFwdB = FwdOp::bytes(kFwdN);
  static constexpr uint32_t kFwdStage = kPlaneP * 8;
  static constexpr uint32_t kFwdSmem = 2 * kFwdA + 2 * kFwdB + kFwdStage + 64;
  static constexpr uint32_t kAdjA = AdjOp::bytes(kRowsPad);
  static constexpr uint32_t kAdjB = AdjOp::bytes(kAdjN);
  static constexpr uint32_t kAdjStageG = kPlaneL * 8;
  static constexpr uint32_t kAdjStageX = kPlaneP * 8;
  static constexpr uint32_t kAdjSmem = 2 * kAdjA + 2 * kAdjB + kAdjStageG + kAdjStageX + 64;
  static constexpr uint32_t kFwdCols = 256;  // TMEM columns (power of two >= tiles * N)
  static constexpr uint32_t kAdjCols = 256;
  static_assert(kFwdN <= kTcTileCols && kAdjN <= kTcTileCols &&
                    kTilesMax * kTcTileCols <= (int)kFwdCols &&
                    kTilesMax * kTcTileCols <= (int)kAdjCols,
                "accumulators fit the TMEM allocation");
};

// DFT matrices of one kernel in global memory: B[n][k] (N rows x K, row-major
// BF16), hi and lo parts (built on the host in double precision).
struct TcMatrices {
  const uint16_t *hi;
  const uint16_t *lo;
};

// Copies a row-major N x K BF16 matrix into the K-major operand layout.
template <int N, int K, typename Op>
__device__ __forceinline__ void tc_stage_matrix(unsigned char *dst, const uint16_t *src) {
  constexpr int kChunks = N * (K / 8);
  for (int q = threadIdx.x; q < kChunks; q += blockDim.x) {
    const int n = q / (K / 8), c = q - n * (K / 8);
    const uint4 v = reinterpret_cast<const uint4 *>(src)[q];
    *reinterpret_cast<uint4 *>(dst + Op::offset(n, 8 * c)) = v;
  }
}

// Zeroes the k columns [k0, K) of rows [0, rows) of an operand (padding that
// the MMAs read but no epilogue writes).
template <int K, typename Op>
__device__ __forceinline__ void tc_zero_columns(unsigned char *a, int rows, int k0) {
  const int w = (K - k0) / 2;  // 4-byte words per row
  for (int q = threadIdx.x; q < rows * w; q += blockDim.x) {
    const int r = q / w, k = k0 + 2 * (q - r * w);
    *reinterpret_cast<uint32_t *>(a + Op::offset(r, k)) = 0u;
  }
}

// One (re, im) pair split into hi and lo BF16 pairs at operand position
// (row, k = 2 * index).
template <typename Op>
__device__ __forceinline__ void tc_put(unsigned char *ahi, unsigned char *alo, int row, int k,
                                       float re, float im) {
  uint16_t rh, rl, ih, il;
  umma::split_bf16(re, rh, rl);
  umma::split_bf16(im, ih, il);
  const uint32_t o = Op::offset(row, k);
  *reinterpret_cast<uint32_t *>(ahi + o) = (uint32_t)rh | ((uint32_t)ih << 16);
  *reinterpret_cast<uint32_t *>(alo + o) = (uint32_t)rl | ((uint32_t)il << 16);
}

// The MMAs of one pass: every tile t of 128 rows, D[t] (+)= A_t B^T in the
// three split products.
template <int KSTEPS, int N, typename Op>
__device__ __forceinline__ void tc_issue_pass(uint32_t tmem, uint32_t a_hi, uint32_t a_lo,
                                              uint32_t b_hi, uint32_t b_lo, int tiles) {
  constexpr uint32_t idesc = umma::idesc_bf16(128, N);
  for (int t = 0; t < tiles; ++t) {
    const uint32_t d = tmem + (uint32_t)(t * kTcTileCols);
    const uint32_t at = (uint32_t)t * 16u * Op::kSbo;
#pragma unroll
    for (int s = 0; s < KSTEPS; ++s) {
      const uint32_t ko = (uint32_t)s * 2u * Op::kLbo;
      const uint64_t ah = umma::desc_kmajor(a_hi + at + ko, Op::kLbo, Op::kSbo);
      const uint64_t al = umma::desc_kmajor(a_lo + at + ko, Op::kLbo, Op::kSbo);
      const uint64_t bh = umma::desc_kmajor(b_hi + ko, Op::kLbo, Op::kSbo);
      const uint64_t bl = umma::desc_kmajor(b_lo + ko, Op::kLbo, Op::kSbo);
      umma::mma_bf16(d, al, bh, idesc, s > 0 ? 1u : 0u);
      umma::mma_bf16(d, ah, bl, idesc, 1u);
      umma::mma_bf16(d, ah, bh, idesc, 1u);
    }
  }
}

// 8 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// Runs the MMAs of a pass and waits for them (block-uniform result: false if
// a wait gave up).  Called by every thread after the operand is written.
template <int KSTEPS, int N, typename Op>
__device__ __forceinline__ bool tc_pass(uint32_t tmem, uint32_t a_hi, uint32_t a_lo,
                                        uint32_t b_hi, uint32_t b_lo, int tiles, uint64_t *bar,
                                        unsigned &phase) {
  umma::fence_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  if (threadIdx.x == 0) {
    umma::fence_after_sync();
    tc_issue_pass<KSTEPS, N, Op>(tmem, a_hi, a_lo, b_hi, b_lo, tiles);
    umma::commit(bar);
  }
  const bool ok = umma::bar_wait(bar, phase & 1u);
  phase++;
  umma::fence_after_sync();
  return __syncthreads_and(ok);
}

// Columns [c0, c0 + 8 * n8) of this thread's row of tile t, in groups of 8,
// handed to f(column, v[8]).  Warp w reads the lanes 32 (w % 4).. of the
// tile; the two warp halves (w / 4) take alternate groups.
template <typename F>
__device__ __forceinline__ void tc_row_groups(uint32_t tmem, int t, int N, int n8, F &&f) {
  const int warp = threadIdx.x >> 5;
  const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
  for (int g = warp >> 2; g < n8; g += 2) {
    float v[8];
    tmem_ld8(tmem + lane_base + (uint32_t)(t * kTcTileCols + 8 * g), v);
    f(8 * g, v);
  }
}

// ---------------------------------------------------------------- forward

// Z[n0][n1][n2] = sum_{a,b,c} W[n0][a] W[n1][b] W[n2][c] X[a][b][c] for
// every plane of the batches (X planes P^3, Z planes L^3 complex).
template <int P, int L>
__global__ void __launch_bounds__(kTcThreads, 1)
    space_fwd_tc(PlaneBatches<float> batches, TcMatrices mats, int *err) {
  using S = TcDft3<P, L>;
  using Op = typename S::FwdOp;
  constexpr int K = S::kFwdK, N = S::kFwdN, KSTEPS = K / 16;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *a_hi = smem;
  unsigned char *a_lo = a_hi + S::kFwdA;
  unsigned char *b_hi = a_lo + S::kFwdA;
  unsigned char *b_lo = b_hi + S::kFwdB;
  float2 *stage = reinterpret_cast<float2 *>(b_lo + S::kFwdB);
  uint64_t *bar = reinterpret_cast<uint64_t *>(b_lo + S::kFwdB + S::kFwdStage);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    umma::bar_init(bar, 1);
    umma::bar_init_fence();
  }
  if (warp == 0) umma::tmem_alloc(tslot, S::kFwdCols);
  tc_stage_matrix<N, K, Op>(b_hi, mats.hi);
  tc_stage_matrix<N, K, Op>(b_lo, mats.lo);
  if (K > 2 * P) {
    tc_zero_columns<K, Op>(a_hi, S::kRowsPad, 2 * P);
    tc_zero_columns<K, Op>(a_lo, S::kRowsPad, 2 * P);
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t sa_hi = umma::smem_u32(a_hi), sa_lo = umma::smem_u32(a_lo);
  const uint32_t sb_hi = umma::smem_u32(b_hi), sb_lo = umma::smem_u32(b_lo);
  unsigned phase = 0;
  bool ok = true;

  // planes of this CTA: batch b, plane j, in order
  auto issue = [&](const PlaneBatch<float> &bt, int j) {
    const float4 *src = reinterpret_cast<const float4 *>(bt.src + (long)j * S::kPlaneP);
    float4 *dst = reinterpret_cast<float4 *>(stage);
    const bool al = (reinterpret_cast<uintptr_t>(src) & 15) == 0;
    if (al) {
      for (int q = threadIdx.x; q < S::kPlaneP / 2; q += blockDim.x) cp_async<16>(dst + q, src + q);
    } else {
      const float2 *s2 = bt.src + (long)j * S::kPlaneP;
      for (int q = threadIdx.x; q < S::kPlaneP; q += blockDim.x) cp_async<8>(stage + q, s2 + q);
    }
    cp_async_commit();
  };
  int b = blockIdx.x, j = 0;
  PlaneBatch<float> cur = b < batches.n ? batches.b[b] : PlaneBatch<float>{nullptr, nullptr, 0, 0};
  if (b < batches.n && cur.count > 0) issue(cur, 0);
  while (ok && b < batches.n) {
    // the plane after this one
    int nb = b, nj = j + 1;
    PlaneBatch<float> nxt = cur;
    if (nj >= cur.count) {
      nb = b + gridDim.x;
      nj = 0;
      nxt = nb < batches.n ? batches.b[nb] : PlaneBatch<float>{nullptr, nullptr, 0, 0};
    }
    cp_async_wait<0>();
    __syncthreads();
    // pass 1 operand: rows (a, b) = a P + b, k = 2 c
    for (int e = threadIdx.x; e < S::kPlaneP; e += blockDim.x) {
      const float2 x = stage[e];
      const int r = e / P, c = e - r * P;
      tc_put<Op>(a_hi, a_lo, r, 2 * c, x.x, x.y);
    }
    __syncthreads();
    if (nb < batches.n && nxt.count > 0) issue(nxt, nj);
    // axis 2: rows (a, b), outputs n2 -> rows (n2, a), k = 2 b
    ok = tc_pass<KSTEPS, N, Op>(tmem, sa_hi, sa_lo, sb_hi, sb_lo, (P * P + 127) / 128, bar,
                                phase);
    if (!ok) break;
    for (int t = 0; t < (P * P + 127) / 128; ++t) {
      const int r = 128 * t + 32 * (warp & 3) + lane;
      const int ra = r / P, rb = r - ra * P;
      tc_row_groups(tmem, t, N, N / 8, [&](int col, const float (&v)[8]) {
        if (r < P * P) {
#pragma unroll
          for (int q = 0; q < 4; ++q)
            tc_put<Op>(a_hi, a_lo, (col / 2 + q) * P + ra, 2 * rb, v[2 * q], v[2 * q + 1]);
        }
      });
    }
    // axis 1: rows (n2, a), outputs n1 -> rows (n1, n2), k = 2 a
    ok = tc_pass<KSTEPS, N, Op>(tmem, sa_hi, sa_lo, sb_hi, sb_lo, (L * P + 127) / 128, bar,
                                phase);
    if (!ok) break;
    for (int t = 0; t < (L * P + 127) / 128; ++t) {
      const int r = 128 * t + 32 * (warp & 3) + lane;
      const int rn2 = r / P, ra = r - rn2 * P;
      tc_row_groups(tmem, t, N, N / 8, [&](int col, const float (&v)[8]) {
        if (r < L * P) {
#pragma unroll
          for (int q = 0; q < 4; ++q)
            tc_put<Op>(a_hi, a_lo, (col / 2 + q) * L + rn2, 2 * ra, v[2 * q], v[2 * q + 1]);
        }
      });
    }
    // axis 0: rows (n1, n2), outputs n0 -> Z[n0][n1][n2]
    ok = tc_pass<KSTEPS, N, Op>(tmem, sa_hi, sa_lo, sb_hi, sb_lo, (L * L + 127) / 128, bar,
                                phase);
    if (!ok) break;
    float2 *z = cur.dst + (long)j * S::kPlaneL;
    for (int t = 0; t < (L * L + 127) / 128; ++t) {
      const int r = 128 * t + 32 * (warp & 3) + lane;
      tc_row_groups(tmem, t, N, N / 8, [&](int col, const float (&v)[8]) {
        if (r < L * L) {
#pragma unroll
          for (int q = 0; q < 4; ++q) z[(col / 2 + q) * L * L + r] = make_float2(v[2 * q], v[2 * q + 1]);
        }
      });
    }
    umma::fence_before_sync();
    b = nb;
    j = nj;
    cur = nxt;
  }
  cp_async_wait<0>();
  if (!ok && threadIdx.x == 0) atomicExch(err, 1);
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tmem, S::kFwdCols);
}

// ---------------------------------------------------------------- adjoint

// G' = sum over the zero-padded space DFT of the G planes (L^3 -> P^3), then
// the epilogue of space_adj_fast on the model planes: kStore (X = G'),
// kUpdateThreshold (X = soft_threshold(X - step G', lamb)), kUpdateMax (X = X
// - step G', tracking max |X|^2).
template <int P, int L>
__global__ void __launch_bounds__(kTcThreads, 1)
    space_adj_tc(PlaneBatches<float> batches, TcMatrices mats, int epilogue, float step_arg,
                 float lamb_arg, const float *step_dev, const float *lamb_dev, float *max_out,
                 int *err) {
  using S = TcDft3<P, L>;
  using Op = typename S::AdjOp;
  constexpr int K = S::kAdjK, N = S::kAdjN, KSTEPS = K / 16;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *a_hi = smem;
  unsigned char *a_lo = a_hi + S::kAdjA;
  unsigned char *b_hi = a_lo + S::kAdjA;
  unsigned char *b_lo = b_hi + S::kAdjB;
  float2 *gst = reinterpret_cast<float2 *>(b_lo + S::kAdjB);
  float2 *xst = gst + S::kPlaneL;
  uint64_t *bar = reinterpret_cast<uint64_t *>(reinterpret_cast<unsigned char *>(xst) +
                                               S::kAdjStageX);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    umma::bar_init(bar, 1);
    umma::bar_init_fence();
  }
  if (warp == 0) umma::tmem_alloc(tslot, S::kAdjCols);
  tc_stage_matrix<N, K, Op>(b_hi, mats.hi);
  tc_stage_matrix<N, K, Op>(b_lo, mats.lo);
  if (K > 2 * L) {
    tc_zero_columns<K, Op>(a_hi, S::kRowsPad, 2 * L);
    tc_zero_columns<K, Op>(a_lo, S::kRowsPad, 2 * L);
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t sa_hi = umma::smem_u32(a_hi), sa_lo = umma::smem_u32(a_lo);
  const uint32_t sb_hi = umma::smem_u32(b_hi), sb_lo = umma::smem_u32(b_lo);
  const bool multi = step_dev != nullptr;
  const bool need_x = epilogue != kStore;
  unsigned phase = 0;
  bool ok = true;
  float local_max = 0.f;

  auto issue = [&](const float2 *src, float2 *dst, int n) {
    if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
      const float4 *s4 = reinterpret_cast<const float4 *>(src);
      float4 *d4 = reinterpret_cast<float4 *>(dst);
      for (int q = threadIdx.x; q < n / 2; q += blockDim.x) cp_async<16>(d4 + q, s4 + q);
    } else {
      for (int q = threadIdx.x; q < n; q += blockDim.x) cp_async<8>(dst + q, src + q);
    }
  };
  int b = blockIdx.x, j = 0;
  PlaneBatch<float> cur = b < batches.n ? batches.b[b] : PlaneBatch<float>{nullptr, nullptr, 0, 0};
  if (b < batches.n && cur.count > 0) issue(cur.src, gst, S::kPlaneL);
  cp_async_commit();
  while (ok && b < batches.n) {
    int nb = b, nj = j + 1;
    PlaneBatch<float> nxt = cur;
    if (nj >= cur.count) {
      nb = b + gridDim.x;
      nj = 0;
      nxt = nb < batches.n ? batches.b[nb] : PlaneBatch<float>{nullptr, nullptr, 0, 0};
    }
    cp_async_wait<0>();
    __syncthreads();
    // pass 1 operand: rows (n0, n1) = n0 L + n1, k = 2 n2
    for (int e = threadIdx.x; e < S::kPlaneL; e += blockDim.x) {
      const float2 g = gst[e];
      const int r = e / L, c = e - r * L;
      tc_put<Op>(a_hi, a_lo, r, 2 * c, g.x, g.y);
    }
    __syncthreads();
    float2 *xg = cur.dst + (long)j * S::kPlaneP;
    if (need_x) issue(xg, xst, S::kPlaneP);
    if (nb < batches.n && nxt.count > 0) issue(nxt.src + (long)nj * S::kPlaneL, gst, S::kPlaneL);
    cp_async_commit();
    // axis 2: rows (n0, n1), outputs c -> rows (c, n0), k = 2 n1
    ok = tc_pass<KSTEPS, N, Op>(tmem, sa_hi, sa_lo, sb_hi, sb_lo, (L * L + 127) / 128, bar,
                                phase);
    if (!ok) break;
    for (int t = 0; t < (L * L + 127) / 128; ++t) {
      const int r = 128 * t + 32 * (warp & 3) + lane;
      const int rn0 = r / L, rn1 = r - rn0 * L;
      tc_row_groups(tmem, t, N, 2 * P / 8 + (2 * P % 8 ? 1 : 0), [&](int col, const float (&v)[8]) {
        if (r < L * L) {
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (col / 2 + q < P)
              tc_put<Op>(a_hi, a_lo, (col / 2 + q) * L + rn0, 2 * rn1, v[2 * q], v[2 * q + 1]);
        }
      });
    }
    // axis 1: rows (c, n0), outputs b -> rows (b, c), k = 2 n0
    ok = tc_pass<KSTEPS, N, Op>(tmem, sa_hi, sa_lo, sb_hi, sb_lo, (P * L + 127) / 128, bar,
                                phase);
    if (!ok) break;
    for (int t = 0; t < (P * L + 127) / 128; ++t) {
      const int r = 128 * t + 32 * (warp & 3) + lane;
      const int rc = r / L, rn0 = r - rc * L;
      tc_row_groups(tmem, t, N, 2 * P / 8 + (2 * P % 8 ? 1 : 0), [&](int col, const float (&v)[8]) {
        if (r < P * L) {
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (col / 2 + q < P)
              tc_put<Op>(a_hi, a_lo, (col / 2 + q) * P + rc, 2 * rn0, v[2 * q], v[2 * q + 1]);
        }
      });
    }
    // axis 0: rows (b, c), outputs a -> X[a][b][c]
    ok = tc_pass<KSTEPS, N, Op>(tmem, sa_hi, sa_lo, sb_hi, sb_lo, (P * P + 127) / 128, bar,
                                phase);
    if (!ok) break;
    cp_async_wait<0>();
    __syncthreads();
    const float step = multi ? step_dev[cur.pid] : step_arg;
    const float lamb = lamb_dev != nullptr ? lamb_dev[multi ? cur.pid : 0] : lamb_arg;
    const float lamb_sq = lamb * lamb;
    for (int t = 0; t < (P * P + 127) / 128; ++t) {
      const int r = 128 * t + 32 * (warp & 3) + lane;
      tc_row_groups(tmem, t, N, 2 * P / 8 + (2 * P % 8 ? 1 : 0), [&](int col, const float (&v)[8]) {
        if (r < P * P) {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int a = col / 2 + q;
            if (a < P) {
              const int e = a * P * P + r;
              const float2 g = make_float2(v[2 * q], v[2 * q + 1]);
              if (epilogue == kStore) {
                xg[e] = g;
              } else {
                const float2 x = xst[e];
                float2 xn = make_float2(__fsub_rn(x.x, __fmul_rn(step, g.x)),
                                        __fsub_rn(x.y, __fmul_rn(step, g.y)));
                if (epilogue == kUpdateThreshold) {
                  xn = soft_threshold<float>(xn, lamb, lamb_sq);
                } else {
                  const float a2 = abs_sq<float>(xn);
                  local_max = a2 > local_max ? a2 : local_max;
                }
                xg[e] = xn;
              }
            }
          }
        }
      });
    }
    if (multi && epilogue == kUpdateMax && (nb != b || nxt.pid != cur.pid || nb >= batches.n)) {
      __shared__ float red_b[32];
      const float m = block_max<float>(local_max, red_b);
      if (threadIdx.x == 0) atomic_max_nonneg(max_out + cur.pid, m);
      local_max = 0.f;
    }
    umma::fence_before_sync();
    b = nb;
    j = nj;
    cur = nxt;
  }
  cp_async_wait<0>();
  if (!ok && threadIdx.x == 0) atomicExch(err, 1);
  if (!multi && epilogue == kUpdateMax) {
    __shared__ float red[32];
    const float m = block_max<float>(local_max, red);
    if (threadIdx.x == 0) atomic_max_nonneg(max_out, m);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tmem, S::kAdjCols);
}

}  // namespace agd
