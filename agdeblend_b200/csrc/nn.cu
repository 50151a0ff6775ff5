// Learned warm start: the tensor-core building blocks (BF16 GEMM on tcgen05)
// and their C entry points.  No counterpart in the reference, whose solver
// always starts from a zero model (src/model.c:1160-1185).
#include <cuda_runtime.h>

#include <cstdio>

#include "agdeblend_gpu.h"
#include "tc_gemm.cuh"

namespace {

template <int BN>
cudaError_t launch_gemm(const uint16_t *A, const uint16_t *B, float *C, int M, int N, int K,
                        int lda, int ldb, int ldc, float alpha, float beta, int *err,
                        cudaStream_t s) {
  using L = agd::TcGemmSmem<BN>;
  static bool configured = false;  // the attribute is per function, set once
  if (!configured) {
    const cudaError_t e = cudaFuncSetAttribute(
        agd::tc_gemm_bf16<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::kBytes);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  const dim3 grid((M + agd::kTcBM - 1) / agd::kTcBM, (N + BN - 1) / BN);
  agd::tc_gemm_bf16<BN><<<grid, 128, L::kBytes, s>>>(A, B, C, M, N, K, lda, ldb, ldc, alpha,
                                                      beta, err);
  return cudaGetLastError();
}

}  // namespace

namespace agd {

// C = alpha A B^T + beta C on the tensor cores (see tc_gemm.cuh for the
// operand rules); err receives 1 if an MMA wait gave up.
cudaError_t tc_gemm(const uint16_t *A, const uint16_t *B, float *C, int M, int N, int K,
                    int lda, int ldb, int ldc, float alpha, float beta, int *err,
                    cudaStream_t s) {
  if (M <= 0 || N <= 0) return cudaSuccess;
  if (N <= 64) return launch_gemm<64>(A, B, C, M, N, K, lda, ldb, ldc, alpha, beta, err, s);
  return launch_gemm<128>(A, B, C, M, N, K, lda, ldb, ldc, alpha, beta, err, s);
}

}  // namespace agd

extern "C" int agd_nn_gemm_bf16(const void *A, const void *B, float *C, int M, int N, int K,
                                int lda, int ldb, int ldc, float alpha, float beta,
                                void *stream) {
  if (A == nullptr || B == nullptr || C == nullptr || M < 0 || N < 0 || K < 0 || K % 8 ||
      lda % 8 || ldb % 8 || lda < K || ldb < K || ldc < N ||
      (reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) % 16) {
    std::fprintf(stderr,
                 "ERROR: agd_nn_gemm_bf16: need K, lda, ldb multiples of 8, lda, ldb >= K, "
                 "ldc >= N and 16-byte aligned A, B\n");
    return 1;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int *err = nullptr;
  cudaError_t e = cudaMalloc(&err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), s);
  if (e == cudaSuccess)
    e = agd::tc_gemm(static_cast<const uint16_t *>(A), static_cast<const uint16_t *>(B), C, M,
                     N, K, lda, ldb, ldc, alpha, beta, err, s);
  int h_err = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (err) cudaFree(err);
  if (e != cudaSuccess || h_err) {
    std::fprintf(stderr, "ERROR: agd_nn_gemm_bf16: %s\n",
                 e != cudaSuccess ? cudaGetErrorString(e) : "tensor-core wait timed out");
    return 1;
  }
  return 0;
}
