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
// One plane per step of a persistent CTA (256 threads, two CTAs per SM, so
// that one CTA's MMAs overlap the other's loads and epilogues):
//   1. the plane is read from global memory and split into the A operand of
//      the first axis: rows = the lines of that axis, k = 2 * index + (re,
//      im);
//   2. for each axis: thread 0 issues the MMAs of every 128-row tile (D = A
//      B^T, N = 2 * outputs) and commits them to an mbarrier; after the
//      wait, the epilogue reads D from TMEM (warp w: lanes 32 (w % 4).. of
//      the tile, column half w / 4) and writes the next axis's A operand,
//      transposed so that the next axis's index becomes k;
//   3. the last epilogue stores the cropped plane (forward) or applies the
//      ISTA update to the model plane (adjoint: the model plane is copied by
//      cp.async into the operand area, free once the last MMAs are done).
// Operand layout: K-major 8 x 16-byte core matrices with k chunks 144 bytes
// apart (128 + 16: the transposing stores of a warp spread over the banks).
// An operand holds the P * P rows of the largest pass; the MMAs of the last
// 128-row tile also read the rows past them, which lie over the next
// buffers in shared memory (still inside the CTA's allocation): those
// accumulator rows are never read.
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
  // rows of the largest pass (lines of two padded axes)
  static constexpr int kRows = P * P;
  static_assert(kRows % 8 == 0, "whole row groups");
  static constexpr int kTilesMax = (kRows + 127) / 128;
  static constexpr int kRowsPad = kTilesMax * 128;
  static constexpr int kPlaneP = P * P * P;  // model plane, complex
  static constexpr int kPlaneL = L * L * L;  // cropped plane, complex
  using FwdOp = TcOp<kFwdKch>;
  using AdjOp = TcOp<kAdjKch>;
  // forward shared memory: A hi | A lo | B hi | B lo (the B matrices inside
  // the rows the last tile of A lo reads past its end) | barrier, TMEM slot
  static constexpr uint32_t kFwdA = FwdOp::bytes(kRows);
  static constexpr uint32_t kFwdB = FwdOp::bytes(kFwdN);
  static constexpr uint32_t kFwdBOff = 2 * kFwdA;
  static constexpr uint32_t kFwdEnd = kFwdA + FwdOp::bytes(kRowsPad);  // A lo + last tile
  static constexpr uint32_t kFwdBar = (kFwdEnd > kFwdBOff + 2 * kFwdB ? kFwdEnd
                                                                      : kFwdBOff + 2 * kFwdB);
  static constexpr uint32_t kFwdSmem = kFwdBar + 64;
  // adjoint: A hi | A lo | (last-tile overrun) up to the model plane's size,
  // where the model plane is staged after the last MMAs | B hi | B lo | bar
  static constexpr uint32_t kAdjA = AdjOp::bytes(kRows);
  static constexpr uint32_t kAdjB = AdjOp::bytes(kAdjN);
  static constexpr uint32_t kAdjX = kPlaneP * 8;
  static constexpr uint32_t kAdjEnd = kAdjA + AdjOp::bytes(kRowsPad);
  static constexpr uint32_t kAdjBOff = ((kAdjEnd > kAdjX ? kAdjEnd : kAdjX) + 127) / 128 * 128;
  static constexpr uint32_t kAdjBar = kAdjBOff + 2 * kAdjB;
  // at least 77 KB, so that no third CTA (whose TMEM would not fit) joins
  // two on an SM
  static constexpr uint32_t kAdjSmem = kAdjBar + 64 > 78848 ? kAdjBar + 64 : 78848;
  static constexpr uint32_t kFwdCols = 256;  // TMEM columns: tiles x kTcTileCols
  static constexpr uint32_t kAdjCols = 256;
  static_assert(kFwdN <= kTcTileCols && kAdjN <= kTcTileCols &&
                    kTilesMax * kTcTileCols <= (int)kFwdCols &&
                    kTilesMax * kTcTileCols <= (int)kAdjCols,
                "accumulators fit the TMEM allocation");
  static_assert(2 * (kFwdSmem + 1024) <= 233472 && 2 * (kAdjSmem + 1024) <= 233472,
                "two CTAs per SM");
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

// (re, im) split into packed hi and lo BF16 pairs (re in the low half).
__device__ __forceinline__ void tc_split_pair(float re, float im, uint32_t &hi, uint32_t &lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(re, im);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(re - hf.x, im - hf.y);
  hi = *reinterpret_cast<const uint32_t *>(&h);
  lo = *reinterpret_cast<const uint32_t *>(&l);
}

// One (re, im) pair at operand byte offset o (row, k = 2 * index).
__device__ __forceinline__ void tc_put(unsigned char *ahi, unsigned char *alo, uint32_t o,
                                       float re, float im) {
  uint32_t h, l;
  tc_split_pair(re, im, h, l);
  *reinterpret_cast<uint32_t *>(ahi + o) = h;
  *reinterpret_cast<uint32_t *>(alo + o) = l;
}

// The MMAs of one pass: every tile t of 128 rows, D[t] (+)= A_t B^T in the
// three split products.  Descriptors are built once and advanced by adding
// to their start-address field (byte offset / 16).
template <int KSTEPS, int N, typename Op>
__device__ __forceinline__ void tc_issue_pass(uint32_t tmem, uint32_t a_hi, uint32_t a_lo,
                                              uint32_t b_hi, uint32_t b_lo, int tiles) {
  constexpr uint32_t idesc = umma::idesc_bf16(128, N);
  const uint64_t ah0 = umma::desc_kmajor(a_hi, Op::kLbo, Op::kSbo);
  const uint64_t al0 = umma::desc_kmajor(a_lo, Op::kLbo, Op::kSbo);
  const uint64_t bh0 = umma::desc_kmajor(b_hi, Op::kLbo, Op::kSbo);
  const uint64_t bl0 = umma::desc_kmajor(b_lo, Op::kLbo, Op::kSbo);
  for (int t = 0; t < tiles; ++t) {
    const uint32_t d = tmem + (uint32_t)(t * kTcTileCols);
    const uint64_t at = (uint64_t)(t * 16 * Op::kSbo >> 4);
#pragma unroll
    for (int s = 0; s < KSTEPS; ++s) {
      const uint64_t ko = (uint64_t)(s * 2 * Op::kLbo >> 4);
      umma::mma_bf16(d, al0 + at + ko, bh0 + ko, idesc, s > 0 ? 1u : 0u);
      umma::mma_bf16(d, ah0 + at + ko, bl0 + ko, idesc, 1u);
      umma::mma_bf16(d, ah0 + at + ko, bh0 + ko, idesc, 1u);
    }
  }
}

__device__ __forceinline__ void tmem_ld8_issue(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
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

// This thread's row of tile t: groups of 8 columns [8g, 8g + 8), g < N8, the
// two warp halves (w / 4) taking alternate groups; every load of the tile is
// issued before the one wait, then f(column, v[8]) runs per group.  Warp w
// reads the lanes 32 (w % 4) .. + 31 of the tile.
template <int N8, typename F>
__device__ __forceinline__ void tc_tile_groups(uint32_t tmem, int t, F &&f) {
  constexpr int NG = (N8 + 1) / 2;
  const int warp = threadIdx.x >> 5;
  const int h = warp >> 2;
  const uint32_t base =
      tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(t * kTcTileCols);
  uint32_t r[NG][8];
#pragma unroll
  for (int i = 0; i < NG; ++i)
    if (h + 2 * i < N8) tmem_ld8_issue(base + (uint32_t)(8 * (h + 2 * i)), r[i]);
  tmem_ld_wait();
#pragma unroll
  for (int i = 0; i < NG; ++i) {
    if (h + 2 * i < N8) {
      float v[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) v[q] = __uint_as_float(r[i][q]);
      f(8 * (h + 2 * i), v);
    }
  }
}

// Byte offset of row `row` in an operand (the k part added separately).
template <typename Op>
__device__ __forceinline__ uint32_t tc_row_off(int row) {
  return (uint32_t)(row >> 3) * Op::kSbo + (uint32_t)(row & 7) * 16u;
}
template <typename Op>
__device__ __forceinline__ uint32_t tc_k_off(int k) {
  return (uint32_t)(k >> 3) * Op::kLbo + (uint32_t)(k & 7) * 2u;
}

// ---------------------------------------------------------------- forward

// Z[n0][n1][n2] = sum_{a,b,c} W[n0][a] W[n1][b] W[n2][c] X[a][b][c] for
// every plane of the batches (X planes P^3, Z planes L^3 complex).
template <int P, int L>
__global__ void __launch_bounds__(kTcThreads, 2)
    space_fwd_tc(PlaneBatches<float> batches, TcMatrices mats, int *err) {
  using S = TcDft3<P, L>;
  using Op = typename S::FwdOp;
  constexpr int K = S::kFwdK, N = S::kFwdN, KSTEPS = K / 16;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *a_hi = smem;
  unsigned char *a_lo = smem + S::kFwdA;
  unsigned char *b_hi = smem + S::kFwdBOff;
  unsigned char *b_lo = b_hi + S::kFwdB;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + S::kFwdBar);
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
    tc_zero_columns<K, Op>(a_hi, S::kRows, 2 * P);
    tc_zero_columns<K, Op>(a_lo, S::kRows, 2 * P);
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t sa_hi = umma::smem_u32(a_hi), sa_lo = umma::smem_u32(a_lo);
  const uint32_t sb_hi = umma::smem_u32(b_hi), sb_lo = umma::smem_u32(b_lo);
  unsigned phase = 0;
  bool ok = true;
  constexpr int kU = 8;                  // model loads in flight per thread
  constexpr int kCR = kTcThreads / P;    // rows per sweep of the conversion
  constexpr int kCT = kCR * P;           // threads of the conversion

  for (int b = blockIdx.x; ok && b < batches.n; b += gridDim.x) {
    const PlaneBatch<float> bt = batches.b[b];
    for (int j = 0; ok && j < bt.count; ++j) {
      const float2 *x = bt.src + (long)j * S::kPlaneP;
      // pass 1 operand: rows (a, b) = a P + b, k = 2 c.  Thread t < kCT takes
      // column c = t % P of rows t / P + kCR i (element t + kCT i: coalesced)
      if (threadIdx.x < kCT) {
        const int c = threadIdx.x % P, r0 = threadIdx.x / P;
        const uint32_t ko = tc_k_off<Op>(2 * c);
        for (int i0 = 0; i0 * kCR < S::kRows; i0 += kU) {
          float2 v[kU];
#pragma unroll
          for (int u = 0; u < kU; ++u) {
            const int r = r0 + (i0 + u) * kCR;
            v[u] = r < S::kRows ? __ldcs(x + threadIdx.x + (i0 + u) * kCT) : make_float2(0.f, 0.f);
          }
#pragma unroll
          for (int u = 0; u < kU; ++u) {
            const int r = r0 + (i0 + u) * kCR;
            if (r < S::kRows) tc_put(a_hi, a_lo, tc_row_off<Op>(r) + ko, v[u].x, v[u].y);
          }
        }
      }
      // axis 2: rows (a, b), outputs n2 -> rows (n2, a), k = 2 b
      ok = tc_pass<KSTEPS, N, Op>(tmem, sa_hi, sa_lo, sb_hi, sb_lo, (P * P + 127) / 128, bar,
                                  phase);
      if (!ok) break;
      for (int t = 0; t < (P * P + 127) / 128; ++t) {
        const int r = 128 * t + 32 * (warp & 3) + lane;
        const int ra = r / P, rb = r - ra * P;
        const uint32_t ko = tc_k_off<Op>(2 * rb);
        tc_tile_groups<N / 8>(tmem, t, [&](int col, const float (&v)[8]) {
          if (r < P * P) {
#pragma unroll
            for (int q = 0; q < 4; ++q)
              tc_put(a_hi, a_lo, tc_row_off<Op>((col / 2 + q) * P + ra) + ko, v[2 * q],
                     v[2 * q + 1]);
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
        const uint32_t ko = tc_k_off<Op>(2 * ra);
        tc_tile_groups<N / 8>(tmem, t, [&](int col, const float (&v)[8]) {
          if (r < L * P) {
#pragma unroll
            for (int q = 0; q < 4; ++q)
              tc_put(a_hi, a_lo, tc_row_off<Op>((col / 2 + q) * L + rn2) + ko, v[2 * q],
                     v[2 * q + 1]);
          }
        });
      }
      // axis 0: rows (n1, n2), outputs n0 -> Z[n0][n1][n2]
      ok = tc_pass<KSTEPS, N, Op>(tmem, sa_hi, sa_lo, sb_hi, sb_lo, (L * L + 127) / 128, bar,
                                  phase);
      if (!ok) break;
      float2 *z = bt.dst + (long)j * S::kPlaneL;
      for (int t = 0; t < (L * L + 127) / 128; ++t) {
        const int r = 128 * t + 32 * (warp & 3) + lane;
        tc_tile_groups<N / 8>(tmem, t, [&](int col, const float (&v)[8]) {
          if (r < L * L) {
#pragma unroll
            for (int q = 0; q < 4; ++q)
              __stcs(z + (col / 2 + q) * L * L + r, make_float2(v[2 * q], v[2 * q + 1]));
          }
        });
      }
      umma::fence_before_sync();
    }
  }
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
__global__ void __launch_bounds__(kTcThreads, 2)
    space_adj_tc(PlaneBatches<float> batches, TcMatrices mats, int epilogue, float step_arg,
                 float lamb_arg, const float *step_dev, const float *lamb_dev, float *max_out,
                 int *err) {
  using S = TcDft3<P, L>;
  using Op = typename S::AdjOp;
  constexpr int K = S::kAdjK, N = S::kAdjN, KSTEPS = K / 16;
  constexpr int N8 = (2 * P + 7) / 8;  // column groups holding the P outputs
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *a_hi = smem;
  unsigned char *a_lo = smem + S::kAdjA;
  float2 *xst = reinterpret_cast<float2 *>(smem);  // model plane, after the last MMAs
  unsigned char *b_hi = smem + S::kAdjBOff;
  unsigned char *b_lo = b_hi + S::kAdjB;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + S::kAdjBar);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    umma::bar_init(bar, 1);
    umma::bar_init_fence();
  }
  if (warp == 0) umma::tmem_alloc(tslot, S::kAdjCols);
  tc_stage_matrix<N, K, Op>(b_hi, mats.hi);
  tc_stage_matrix<N, K, Op>(b_lo, mats.lo);
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
  constexpr int kU = 8;
  constexpr int kCR = kTcThreads / L;  // rows per sweep of the conversion
  constexpr int kCT = kCR * L;         // threads of the conversion

  for (int b = blockIdx.x; ok && b < batches.n; b += gridDim.x) {
    const PlaneBatch<float> bt = batches.b[b];
    const float step = multi ? step_dev[bt.pid] : step_arg;
    const float lamb = lamb_dev != nullptr ? lamb_dev[multi ? bt.pid : 0] : lamb_arg;
    const float lamb_sq = lamb * lamb;
    for (int j = 0; ok && j < bt.count; ++j) {
      const float2 *g = bt.src + (long)j * S::kPlaneL;
      // pass 1 operand: rows (n0, n1) = n0 L + n1, k = 2 n2 (thread t < kCT:
      // column t % L of rows t / L + kCR i)
      if (threadIdx.x < kCT) {
        const int c = threadIdx.x % L, r0 = threadIdx.x / L;
        const uint32_t ko = tc_k_off<Op>(2 * c);
        for (int i0 = 0; i0 * kCR < L * L; i0 += kU) {
          float2 v[kU];
#pragma unroll
          for (int u = 0; u < kU; ++u) {
            const int r = r0 + (i0 + u) * kCR;
            v[u] = r < L * L ? __ldcs(g + threadIdx.x + (i0 + u) * kCT) : make_float2(0.f, 0.f);
          }
#pragma unroll
          for (int u = 0; u < kU; ++u) {
            const int r = r0 + (i0 + u) * kCR;
            if (r < L * L) tc_put(a_hi, a_lo, tc_row_off<Op>(r) + ko, v[u].x, v[u].y);
          }
        }
      }
      // axis 2: rows (n0, n1), outputs c -> rows (c, n0), k = 2 n1
      ok = tc_pass<KSTEPS, N, Op>(tmem, sa_hi, sa_lo, sb_hi, sb_lo, (L * L + 127) / 128, bar,
                                  phase);
      if (!ok) break;
      for (int t = 0; t < (L * L + 127) / 128; ++t) {
        const int r = 128 * t + 32 * (warp & 3) + lane;
        const int rn0 = r / L, rn1 = r - rn0 * L;
        const uint32_t ko = tc_k_off<Op>(2 * rn1);
        tc_tile_groups<N8>(tmem, t, [&](int col, const float (&v)[8]) {
          if (r < L * L) {
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (col / 2 + q < P)
                tc_put(a_hi, a_lo, tc_row_off<Op>((col / 2 + q) * L + rn0) + ko, v[2 * q],
                       v[2 * q + 1]);
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
        const uint32_t ko = tc_k_off<Op>(2 * rn0);
        tc_tile_groups<N8>(tmem, t, [&](int col, const float (&v)[8]) {
          if (r < P * L) {
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (col / 2 + q < P)
                tc_put(a_hi, a_lo, tc_row_off<Op>((col / 2 + q) * P + rc) + ko, v[2 * q],
                       v[2 * q + 1]);
          }
        });
      }
      // axis 0: rows (b, c), outputs a -> X[a][b][c]
      ok = tc_pass<KSTEPS, N, Op>(tmem, sa_hi, sa_lo, sb_hi, sb_lo, (P * P + 127) / 128, bar,
                                  phase);
      if (!ok) break;
      float2 *xg = bt.dst + (long)j * S::kPlaneP;
      if (need_x) {  // the model plane into the operand area, free now
        if ((reinterpret_cast<uintptr_t>(xg) & 15) == 0) {
          const float4 *s4 = reinterpret_cast<const float4 *>(xg);
          float4 *d4 = reinterpret_cast<float4 *>(xst);
          for (int q = threadIdx.x; q < S::kPlaneP / 2; q += kTcThreads) cp_async<16>(d4 + q, s4 + q);
        } else {
          for (int q = threadIdx.x; q < S::kPlaneP; q += kTcThreads) cp_async<8>(xst + q, xg + q);
        }
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
      }
      for (int t = 0; t < (P * P + 127) / 128; ++t) {
        const int r = 128 * t + 32 * (warp & 3) + lane;
        tc_tile_groups<N8>(tmem, t, [&](int col, const float (&v)[8]) {
          if (r < P * P) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int a = col / 2 + q;
              if (a < P) {
                const int e = a * P * P + r;
                const float2 gv = make_float2(v[2 * q], v[2 * q + 1]);
                if (epilogue == kStore) {
                  xg[e] = gv;
                } else {
                  const float2 xv = xst[e];
                  float2 xn = make_float2(__fsub_rn(xv.x, __fmul_rn(step, gv.x)),
                                          __fsub_rn(xv.y, __fmul_rn(step, gv.y)));
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
      // the next plane's operand overwrites the staged model plane
      umma::fence_before_sync();
      __syncthreads();
    }
    if (multi && epilogue == kUpdateMax) {  // one maximum per batch (one problem)
      __shared__ float red_b[32];
      const float m = block_max<float>(local_max, red_b);
      if (threadIdx.x == 0) atomic_max_nonneg(max_out + bt.pid, m);
      local_max = 0.f;
    }
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
