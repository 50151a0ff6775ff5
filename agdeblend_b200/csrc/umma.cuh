// Blackwell (sm_100a) tensor-core primitives in inline PTX: shared-memory
// matrix descriptors, the BF16 instruction descriptor, tcgen05.mma issue and
// commit, tensor-memory (TMEM) allocation and loads, and mbarrier waits that
// give up after a bounded number of polls.
//
// Operand layout ("K-major, no swizzle"): a tile of R rows x K bf16 values is
// stored as 8-row x 16-byte core matrices (8 rows of 8 consecutive k values,
// 128 contiguous bytes).  The core matrix of row group g and k chunk c sits at
// g * sbo + c * lbo bytes from the tile base; one MMA step covers K = 16, the
// two chunks c and c + 1.  D = A B^T with A (M x K) and B (N x K) both stored
// this way; D is FP32 in TMEM, row i of D in lane i (M = 128, one CTA).
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

namespace agd {
namespace umma {

// An mbarrier wait gives up after kMaxPolls polls or kMaxWaitNs nanoseconds
// of the global timer, whichever comes first: both far beyond the time any
// group of MMAs or copies takes.
constexpr unsigned kMaxPolls = 1u << 22;
constexpr unsigned long long kMaxWaitNs = 1000000000ull;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor of a K-major tile without swizzle:
// start address, leading-dimension byte offset (between the two k chunks of
// one MMA step), stride-dimension byte offset (between 8-row groups), all
// in 16-byte units; bit 46 = descriptor version 1 (tcgen05); base offset 0,
// relative leading offsets, layout type 0 (no swizzle).
__host__ __device__ constexpr uint64_t desc_kmajor(uint32_t saddr, uint32_t lbo_bytes,
                                                   uint32_t sbo_bytes) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16 with BF16 A and B, FP32 D, both
// operands K-major, dense: D format bits 4-5 = 1 (F32), A format bits 7-9 =
// 1 (BF16), B format bits 10-12 = 1 (BF16), N / 8 in bits 17-22, M / 16 in
// bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// D (+)= A B^T for one K = 16 step; issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a_desc, uint64_t b_desc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrive once on the mbarrier when every tcgen05 operation this thread
// issued before has completed.
__device__ __forceinline__ void commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void bar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void bar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One arrival on the mbarrier (release at CTA scope).
__device__ __forceinline__ void bar_arrive(uint64_t *bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(
                   smem_u32(bar))
               : "memory");
}

// Arrival that also expects `bytes` of asynchronous (TMA) transfers on the
// mbarrier before its phase can complete.
__device__ __forceinline__ void bar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(
          smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

// Tiled TMA load of a 4-D box at coordinates (c0 innermost .. c3) of the
// tensor map into shared memory (128-byte aligned), completing `bytes` on
// the mbarrier.  c0 times the element size must be a multiple of 16 bytes;
// the other coordinates may lie outside the tensor (zero fill).  No
// multicast.
__device__ __forceinline__ void tma_load_4d(uint32_t sdst, const void *tmap, int c0, int c1,
                                            int c2, int c3, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(sdst),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
      "r"(smem_u32(bar))
      : "memory");
}

// Waits for the completion of the mbarrier phase of the given parity; false
// if it did not complete within the limits above.
__device__ __forceinline__ bool bar_wait(uint64_t *bar, unsigned parity) {
  const uint32_t a = smem_u32(bar);
  const unsigned long long t0 = global_ns();
  for (unsigned i = 0; i < kMaxPolls; ++i) {
    if ((i & 255u) == 255u && global_ns() - t0 > kMaxWaitNs) return false;
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Generic-proxy writes to shared memory become visible to the tensor core
// (async proxy) after this fence and a barrier.
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// TMEM allocation by one whole warp: writes the base address into *slot.
// ncols is a power of two >= 32.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (warp w reads
// lanes 32 (w % 4) .. + 31; taddr carries the lane in bits 16-31).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Byte offset of element (row, k) in a K-major tile whose row groups are
// sbo bytes apart and whose k chunks are lbo bytes apart.
__host__ __device__ constexpr uint32_t kmajor_offset(int row, int k, uint32_t lbo,
                                                     uint32_t sbo) {
  return (uint32_t)(row >> 3) * sbo + (uint32_t)(k >> 3) * lbo + (uint32_t)(row & 7) * 16u +
         (uint32_t)(k & 7) * 2u;
}

// Split of an FP32 value into hi + lo BF16 (round to nearest even each):
// hi + lo carries about 16 significant bits.
__device__ __forceinline__ void split_bf16(float v, uint16_t &hi, uint16_t &lo) {
  const __nv_bfloat16 h = __float2bfloat16_rn(v);
  const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
  hi = __bfloat16_as_ushort(h);
  lo = __bfloat16_as_ushort(l);
}

}  // namespace umma
}  // namespace agd
