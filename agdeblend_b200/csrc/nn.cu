// Learned warm start: the tensor-core building blocks (BF16 GEMM on tcgen05)
// and their C entry points.  No counterpart in the reference, whose solver
// always starts from a zero model (src/model.c:1160-1185).
#include <cuda.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cstdio>

#include "agdeblend_gpu.h"
#include "tc_gemm.cuh"

namespace {

// The persistent kernel: two CTAs per SM (at most one per output tile).
template <int BN>
cudaError_t launch_pipe(const uint16_t *A, const uint16_t *B, float *C, int M, int N, int K,
                        int lda, int ldb, int ldc, float alpha, float beta,
                        const agd::ConvGeom &conv, const agd::BiasActOut &act, int *err,
                        cudaStream_t s) {
  using L = agd::TcPipeSmem<BN>;
  static int n_sms[64] = {};  // per device, per instantiation (attributes set)
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (n_sms[dev] == 0) {
    e = cudaFuncSetAttribute(agd::tc_gemm_pipe<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             L::kBytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(agd::tc_gemm_pipe<BN>,
                               cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    int n_sm = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    n_sms[dev] = std::max(1, n_sm);
  }
  const long tiles =
      (long)((M + agd::kTcBM - 1) / agd::kTcBM) * (long)((N + BN - 1) / BN);
  const int grid = (int)std::min<long>(tiles, (long)n_sms[dev] * L::kPerSm);
  agd::tc_gemm_pipe<BN><<<grid, agd::kPipeThreads, L::kBytes, s>>>(
      A, B, C, M, N, K, lda, ldb, ldc, alpha, beta, conv, act, err);
  return cudaGetLastError();
}

// cuTensorMapEncodeTiled, from the driver through the runtime (no link
// against libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                   const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                   const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// Tensor map of NHWC BF16 activations (channel stride cs) for the halo
// loads: box 8 channels x kHaloPix pixels x 3 rows x 1 image, zero fill
// outside the tensor.
cudaError_t halo_tensor_map(const agd::ConvGeom &conv, CUtensorMap *map) {
  static EncodeTiledFn encode = nullptr;
  if (encode == nullptr) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    const cudaError_t e =
        cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || fn == nullptr)
      return cudaErrorNotSupported;
    encode = reinterpret_cast<EncodeTiledFn>(fn);
  }
  const cuuint64_t cs = (cuuint64_t)conv.cs, w = (cuuint64_t)conv.w, h = (cuuint64_t)conv.h;
  const cuuint64_t dims[4] = {cs, w, h, (cuuint64_t)conv.n};
  const cuuint64_t strides[3] = {2 * cs, 2 * cs * w, 2 * cs * w * h};  // bytes
  const cuuint32_t box[4] = {8, agd::kHaloPix, 3, 1};
  const cuuint32_t unit[4] = {1, 1, 1, 1};
  const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT16, 4,
                            const_cast<uint16_t *>(conv.x), dims, strides, box, unit,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// The halo-tile convolution: PER_SM CTAs per SM over the output tiles of
// each of `groups` groups of BN output channels.
template <int BN, int PER_SM>
cudaError_t launch_halo(const uint16_t *B, float *C, int M, int N, int ldc, int groups,
                        const agd::ConvGeom &conv, const agd::BiasActOut &act, int *err,
                        cudaStream_t s) {
  using L = agd::TcHaloSmem<PER_SM>;
  static int n_sms[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (n_sms[dev] == 0) {
    e = cudaFuncSetAttribute(agd::tc_conv_halo<BN, PER_SM>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, L::kBytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(agd::tc_conv_halo<BN, PER_SM>,
                               cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    int n_sm = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    n_sms[dev] = std::max(1, n_sm);
  }
  CUtensorMap xmap;
  e = halo_tensor_map(conv, &xmap);
  if (e != cudaSuccess) return e;
  const int tiles = M / agd::kTcBM;
  const int per_group = std::max(1, n_sms[dev] * PER_SM / groups);
  const dim3 grid(std::min(tiles, per_group), groups);
  agd::tc_conv_halo<BN, PER_SM><<<grid, agd::kHaloThreads, L::kBytes, s>>>(xmap, B, C, M, N, ldc,
                                                                           conv, act, err);
  return cudaGetLastError();
}

template <int BN>
cudaError_t launch_gemm(const uint16_t *A, const uint16_t *B, float *C, int M, int N, int K,
                        int lda, int ldb, int ldc, float alpha, float beta, int splits,
                        const agd::ConvGeom &conv, const agd::BiasActOut &act, int *err,
                        cudaStream_t s, float *ws, size_t ws_elems) {
  using L = agd::TcGemmSmem<BN>;
  // per function and device; cheap enough to set on every launch
  const cudaError_t e = cudaFuncSetAttribute(
      agd::tc_gemm_bf16<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::kBytes);
  if (e != cudaSuccess) return e;
  // split K: slices of whole 64-wide steps
  const int steps = (K + agd::kTcBK - 1) / agd::kTcBK;
  splits = std::max(1, std::min(splits, steps));
  const int k_split = (steps + splits - 1) / splits * agd::kTcBK;
  splits = (K + k_split - 1) / k_split;
  const bool table_fits = conv.x == nullptr || steps * (agd::kTcBK / 8) <= agd::kPipeMaxChunks;
  if (splits == 1 && K > 0 && table_fits)
    return launch_pipe<BN>(A, B, C, M, N, K, lda, ldb, ldc, alpha, beta, conv, act, err, s);
  const dim3 grid((M + agd::kTcBM - 1) / agd::kTcBM, (N + BN - 1) / BN, std::max(1, splits));
  const long slice = (long)M * ldc;
  if (splits > 1 && ws != nullptr && (size_t)splits * slice <= ws_elems) {
    // partial products in the workspace, summed in a fixed order
    agd::tc_gemm_bf16<BN><<<grid, 128, L::kBytes, s>>>(A, B, ws, M, N, K, lda, ldb, ldc, alpha,
                                                        0.f, k_split, slice, conv, act, err);
    const long total = (long)M * N;
    const unsigned g = (unsigned)std::max<long>(1, std::min<long>((total + 255) / 256, 148L * 8));
    agd::split_reduce<<<g, 256, 0, s>>>(ws, splits, slice, M, N, ldc, C, beta);
    return cudaGetLastError();
  }
  agd::tc_gemm_bf16<BN><<<grid, 128, L::kBytes, s>>>(A, B, C, M, N, K, lda, ldb, ldc, alpha,
                                                      beta, k_split, 0L, conv, act, err);
  return cudaGetLastError();
}

}  // namespace

namespace agd {

// How a 3 x 3 convolution (implicit GEMM geometry conv, N output channels,
// weights N x K) runs on tc_conv_halo: channels a multiple of 32 without
// padding, image rows a multiple of 128 pixels, and the weights of one
// group of BN output channels in shared memory - two CTAs per SM when they
// fit 36 KB, else one with up to 144 KB, in at most two groups of at least
// 64 channels.  bn == 0: not eligible (the implicit GEMM runs it).
struct HaloPlan {
  int bn = 0, per_sm = 0, groups = 0;
};

HaloPlan halo_plan(const ConvGeom &conv, int N, int K) {
  HaloPlan h;
  if (conv.x == nullptr || conv.cin % 32 || conv.cs != conv.cin || conv.w % 128 ||
      K != 9 * conv.cin || N <= 0)
    return h;
  const long row = 2L * K;  // bytes of one weight row
  const int small = N <= 32 ? 32 : 64;
  if (N <= 64 && small * row <= TcHaloSmem<2>::kMaxB) return HaloPlan{small, 2, 1};
  for (int bn : {128, 64}) {
    const int groups = (N + bn - 1) / bn;
    if (bn * row <= TcHaloSmem<1>::kMaxB && groups <= 2 && (bn == 64 || N > 64))
      return HaloPlan{bn, 1, groups};
  }
  return h;
}

// Y = conv3x3(X) on tc_conv_halo with a plan from halo_plan: the epilogue
// act, or FP32 into C (row stride ldc) when act.y is null.
cudaError_t tc_conv(const uint16_t *B, float *C, long M, int N, int ldc, const ConvGeom &conv,
                    const HaloPlan &h, const BiasActOut &act, int *err, cudaStream_t s) {
  if (M <= 0) return cudaSuccess;
  if (M % kTcBM || M > INT32_MAX || h.bn == 0) return cudaErrorInvalidValue;
  const int m = (int)M;
  if (h.per_sm == 2)
    return h.bn == 32 ? launch_halo<32, 2>(B, C, m, N, ldc, 1, conv, act, err, s)
                      : launch_halo<64, 2>(B, C, m, N, ldc, 1, conv, act, err, s);
  return h.bn == 128 ? launch_halo<128, 1>(B, C, m, N, ldc, h.groups, conv, act, err, s)
                     : launch_halo<64, 1>(B, C, m, N, ldc, h.groups, conv, act, err, s);
}

// C = alpha A B^T + beta C on the tensor cores (see tc_gemm.cuh for the
// operand rules); err receives 1 if an MMA wait gave up.
// With splits > 1 the K range is cut into slices: with a workspace of at
// least (splits actually used) x M x ldc floats their partial products are
// summed in a fixed order (deterministic), else added into C with atomics
// (C must then hold beta C already; beta is ignored).
cudaError_t tc_gemm(const uint16_t *A, const uint16_t *B, float *C, int M, int N, int K,
                    int lda, int ldb, int ldc, float alpha, float beta, int *err,
                    cudaStream_t s, int splits = 1,
                    const ConvGeom &conv = ConvGeom{nullptr, 0, 0, 0, 0, 0},
                    const BiasActOut &act = BiasActOut{nullptr, nullptr, 0, 0, 0},
                    float *ws = nullptr, size_t ws_elems = 0) {
  if (M <= 0 || N <= 0) return cudaSuccess;
  if (conv.x != nullptr || act.y != nullptr) splits = 1;
  if (N <= 32)
    return launch_gemm<32>(A, B, C, M, N, K, lda, ldb, ldc, alpha, beta, splits, conv, act, err,
                           s, ws, ws_elems);
  if (N <= 64)
    return launch_gemm<64>(A, B, C, M, N, K, lda, ldb, ldc, alpha, beta, splits, conv, act, err,
                           s, ws, ws_elems);
  return launch_gemm<128>(A, B, C, M, N, K, lda, ldb, ldc, alpha, beta, splits, conv, act, err,
                          s, ws, ws_elems);
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

extern "C" int agd_nn_conv3x3_bf16(const void *x, int n, int h, int w, int cin,
                                   const void *weights, int cout, float *y, void *stream) {
  const long P = (long)n * h * w;
  if (x == nullptr || weights == nullptr || y == nullptr || n <= 0 || h <= 0 || w <= 0 ||
      cin <= 0 || cin % 8 || cout <= 0 || P > INT32_MAX || 9L * cin > INT32_MAX ||
      (reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(weights)) % 16) {
    std::fprintf(stderr,
                 "ERROR: agd_nn_conv3x3_bf16: need positive sizes, cin a multiple of 8 and "
                 "16-byte aligned x, weights\n");
    return 1;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const agd::ConvGeom geom{static_cast<const uint16_t *>(x), n, h, w, cin, cin};
  const agd::BiasActOut none{nullptr, nullptr, 0, 0, 0};
  const auto *wts = static_cast<const uint16_t *>(weights);
  int *err = nullptr;
  cudaError_t e = cudaMalloc(&err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), s);
  if (e == cudaSuccess)
    e = agd::halo_plan(geom, cout, 9 * cin).bn > 0
            ? agd::tc_conv(wts, y, P, cout, cout, geom, agd::halo_plan(geom, cout, 9 * cin),
                           none, err, s)
            : agd::tc_gemm(nullptr, wts, y, (int)P, cout, 9 * cin, 9 * cin, 9 * cin, cout, 1.f,
                           0.f, err, s, 1, geom);
  int h_err = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (err) cudaFree(err);
  if (e != cudaSuccess || h_err) {
    std::fprintf(stderr, "ERROR: agd_nn_conv3x3_bf16: %s\n",
                 e != cudaSuccess ? cudaGetErrorString(e) : "tensor-core wait timed out");
    return 1;
  }
  return 0;
}

// ============================================================== the network
//
// A 4-level 2-D convolutional encoder-decoder on (n, h, w) images (traces x
// time samples of a pseudo-deblended gather; h, w multiples of 8).  Level
// channels c, 2c, 4c, 8c for base c (32: 1,162,945 parameters):
//   enc  conv(1,c) conv(c,c) | pool | conv(c,2c) conv(2c,2c) | pool |
//        conv(2c,4c) conv(4c,4c) | pool | conv(4c,8c) conv(8c,4c)
//   dec  up + skip | conv(4c,4c) conv(4c,2c) | up + skip | conv(2c,2c)
//        conv(2c,c) | up + skip | conv(c,c) conv(c,1, linear)
//   output = input + last conv (the network predicts a correction)
// 3 x 3 convolutions with padding 1 and ReLU, 2 x 2 average pooling, nearest
// 2x upsampling, additive skips.  Forward convolutions run on the tensor
// cores with FP32 accumulation and the bias / ReLU / BF16 store in the
// epilogue: the halo-tile kernel where halo_plan allows it, else the
// implicit GEMM; the first layer (one input channel) on the CUDA cores.  The
// backward pass computes weight gradients as split-K GEMMs over the pixels
// and input gradients as GEMMs followed by the transpose of im2col.
// Parameters: per layer the
// weights [cout][ky][kx][cin] then the biases [cout], FP32 masters updated
// by Adam, BF16 copies for the GEMMs.
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "nn_api.hpp"
#include "nn_kernels.cuh"

namespace agd {
namespace nn {

struct NnError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline void ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw NnError(std::string(what) + ": " + cudaGetErrorString(e));
}
#define NCK(x) ck((x), #x)

template <typename T>
struct Buf {
  T *p = nullptr;
  size_t n = 0;
  Buf() = default;
  Buf(const Buf &) = delete;
  Buf &operator=(const Buf &) = delete;
  Buf(Buf &&o) noexcept : p(o.p), n(o.n) {
    o.p = nullptr;
    o.n = 0;
  }
  Buf &operator=(Buf &&o) noexcept {
    if (this != &o) {
      reset();
      p = o.p;
      n = o.n;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~Buf() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void ensure(size_t count) {
    if (count <= n) return;
    reset();
    NCK(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
    n = count;
  }
  T *get() const { return p; }
};

inline unsigned grid_of(long n) {
  return (unsigned)std::max<long>(1, std::min<long>((n + kNnThreads - 1) / kNnThreads, 148L * 16));
}
inline int pad8(int c) { return (c + 7) / 8 * 8; }

class Net {
 public:
  struct Layer {
    int in, out;      // tensor indices
    int cin, cout;
    int relu;
    long w_off, b_off;  // offsets in the parameter vector
    int cin_s, cout_s, kp;
  };
  enum OpKind { kConv, kPool, kUpAdd };
  struct Op {
    OpKind kind;
    int a, b, out;  // conv: layer a; pool: in a; up-add: low a, skip b
  };
  struct Tensor {
    int level, C, Cs;
    Buf<uint16_t> v;
    Buf<float> g;
  };

  int base;
  int in_ch = 1;  // input channels: the line and in_ch - 1 neighbouring lines
  long n_params = 0;
  std::vector<Layer> layers;
  std::vector<Op> ops;
  std::vector<Tensor> t;
  // parameters and optimiser state
  Buf<float> w, grad, m, v;
  std::vector<Buf<uint16_t>> wp, wpt;  // per layer: [cout_s][kp], [kp][cout_s] BF16
  Buf<float> dwp;                      // weight-gradient GEMM output
  Buf<float> split_ws;                 // its split-K partial products
  // scratch
  Buf<uint16_t> col, colT, dz, dzT;
  Buf<float> z, dcol, in_f, out_f, tgt_f, last_f;
  Buf<double> loss_d;
  Buf<int> err;
  // image RMS values, image and neighbour offsets of estimate_images (grow only)
  Buf<float> rms_buf;
  Buf<long> base_buf, nbr_buf;
  cudaStream_t s = nullptr;
  long adam_t = 0;
  int cur_n = 0, cur_h = 0, cur_w = 0;

  Net(int base_c, unsigned seed, int in_channels = 1) : base(base_c), in_ch(in_channels) {
    NCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    const int c = base;
    auto tensor = [&](int level, int C) {
      Tensor x;
      x.level = level;
      x.C = C;
      x.Cs = pad8(C);
      t.push_back(std::move(x));
      return (int)t.size() - 1;
    };
    auto conv = [&](int in, int cout, int relu) {
      Layer L{};
      L.in = in;
      L.cin = t[in].C;
      L.cout = cout;
      L.relu = relu;
      L.out = tensor(t[in].level, cout);
      L.cin_s = t[in].Cs;
      L.cout_s = pad8(cout);
      L.kp = (9 * L.cin + 15) / 16 * 16;
      L.w_off = n_params;
      n_params += 9L * L.cin * L.cout;
      L.b_off = n_params;
      n_params += L.cout;
      layers.push_back(L);
      ops.push_back(Op{kConv, (int)layers.size() - 1, 0, L.out});
      return L.out;
    };
    auto pool = [&](int in) {
      const int o = tensor(t[in].level + 1, t[in].C);
      ops.push_back(Op{kPool, in, 0, o});
      return o;
    };
    auto upadd = [&](int low, int skip) {
      const int o = tensor(t[skip].level, t[skip].C);
      ops.push_back(Op{kUpAdd, low, skip, o});
      return o;
    };
    const int x0 = tensor(0, in_ch);
    const int s1 = conv(conv(x0, c, 1), c, 1);
    const int s2 = conv(conv(pool(s1), 2 * c, 1), 2 * c, 1);
    const int s3 = conv(conv(pool(s2), 4 * c, 1), 4 * c, 1);
    const int bn = conv(conv(pool(s3), 8 * c, 1), 4 * c, 1);
    const int d3 = conv(conv(upadd(bn, s3), 4 * c, 1), 2 * c, 1);
    const int d2 = conv(conv(upadd(d3, s2), 2 * c, 1), c, 1);
    conv(conv(upadd(d2, s1), c, 1), 1, 0);
    // He-normal weights (the last layer scaled down: the network starts
    // near the identity), zero biases
    std::vector<float> h(n_params, 0.f);
    std::mt19937 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    for (size_t li = 0; li < layers.size(); ++li) {
      const Layer &L = layers[li];
      const float sd = std::sqrt(2.f / (9.f * L.cin)) * (li + 1 == layers.size() ? 0.1f : 1.f);
      for (long i = 0; i < 9L * L.cin * L.cout; ++i) h[L.w_off + i] = sd * nd(rng);
    }
    w.ensure(n_params);
    grad.ensure(n_params);
    m.ensure(n_params);
    v.ensure(n_params);
    NCK(cudaMemcpy(w.get(), h.data(), n_params * sizeof(float), cudaMemcpyHostToDevice));
    NCK(cudaMemset(m.get(), 0, n_params * sizeof(float)));
    NCK(cudaMemset(v.get(), 0, n_params * sizeof(float)));
    wp.resize(layers.size());
    wpt.resize(layers.size());
    size_t dwp_max = 0;
    for (size_t li = 0; li < layers.size(); ++li) {
      const Layer &L = layers[li];
      wp[li].ensure((size_t)L.cout_s * L.kp);
      wpt[li].ensure((size_t)L.kp * L.cout_s);
      dwp_max = std::max(dwp_max, (size_t)L.cout_s * L.kp);
    }
    dwp.ensure(dwp_max);
    loss_d.ensure(1);
    err.ensure(1);
    NCK(cudaMemset(err.get(), 0, sizeof(int)));
    pack_weights();
  }

  ~Net() {
    if (s) cudaStreamDestroy(s);
  }

  // BF16 GEMM copies of the weights: Wp[co][k] and WpT[k][co], zero-padded
  void pack_weights() {
    for (size_t li = 0; li < layers.size(); ++li) {
      const Layer &L = layers[li];
      pack_kernel<<<grid_of((long)L.cout_s * L.kp), kNnThreads, 0, s>>>(
          w.get() + L.w_off, L.cout, 9 * L.cin, L.cout_s, L.kp, wp[li].get(), wpt[li].get());
      NCK(cudaGetLastError());
    }
  }






  long pixels(int level) const {
    return (long)cur_n * (cur_h >> level) * (cur_w >> level);
  }

  // buffers for n images of h x w (training: also the backward buffers)
  void shape(int n, int h, int wd, bool training = true) {
    if (h % 8 || wd % 8 || n <= 0) throw NnError("image sides must be multiples of 8");
    cur_n = n;
    cur_h = h;
    cur_w = wd;
    size_t col_max = 0, z_max = 0;
    for (Tensor &x : t) {
      const long P = pixels(x.level);
      x.v.ensure((size_t)P * x.Cs);
      if (training) x.g.ensure((size_t)P * x.Cs);
    }
    size_t col_fwd = 0;  // im2col of the layers that are not implicit GEMMs
    for (const Layer &L : layers) {
      const long P = pixels(t[L.in].level);
      col_max = std::max(col_max, (size_t)P * L.kp);
      if (L.cin % 8) col_fwd = std::max(col_fwd, (size_t)P * L.kp);
      z_max = std::max(z_max, (size_t)P * L.cout_s);
    }
    col.ensure(training ? col_max : col_fwd);
    // FP32 GEMM output: the last layer's in the forward pass (the others go
    // to BF16 in the GEMM epilogue); any layer's gradient GEMMs in training
    z.ensure(training ? z_max : (size_t)pixels(0) * layers.back().cout_s);
    if (training) {
      colT.ensure(col_max);
      dcol.ensure(col_max);
      dz.ensure(z_max);
      dzT.ensure(z_max);
    }
    const long P0 = pixels(0);
    in_f.ensure((size_t)P0 * in_ch);
    out_f.ensure(P0);
    tgt_f.ensure(P0);
    last_f.ensure((size_t)P0 * t.back().Cs);
  }

  void gemm(const uint16_t *A, const uint16_t *B, float *C, long M, int N, long K, long lda,
            long ldb, int ldc, float beta, int splits = 1) {
    if (M > INT32_MAX || K > INT32_MAX || lda > INT32_MAX || ldb > INT32_MAX)
      throw NnError("GEMM too large");
    if (splits > 1) split_ws.ensure((size_t)splits * M * ldc);  // deterministic split K
    NCK(tc_gemm(A, B, C, (int)M, N, (int)K, (int)lda, (int)ldb, ldc, 1.f, beta, err.get(), s,
                splits, ConvGeom{nullptr, 0, 0, 0, 0, 0}, BiasActOut{nullptr, nullptr, 0, 0, 0},
                split_ws.get(), split_ws.n));
  }

  void conv_forward(const Layer &L, bool keep_f32) {
    const Tensor &X = t[L.in];
    Tensor &Y = t[L.out];
    const long P = pixels(X.level);
    const int H = cur_h >> X.level, Wd = cur_w >> X.level;
    if (P > INT32_MAX) throw NnError("GEMM too large");
    // all but the last layer: bias, activation and the BF16 store in the
    // GEMM epilogue (the last one keeps its FP32 output for the residual)
    const BiasActOut act = keep_f32 ? BiasActOut{nullptr, nullptr, 0, 0, 0}
                                    : BiasActOut{Y.v.get(), w.get() + L.b_off, L.cout,
                                                 L.cout_s, L.relu};
    const uint16_t *A = nullptr;
    ConvGeom geom{X.v.get(), cur_n, H, Wd, L.cin, X.Cs};  // implicit GEMM
    if (L.in == 0 && L.cin == in_ch && in_ch <= kFirstMaxIn && !keep_f32 && L.cout_s <= 64) {
      // the first layer, from the FP32 input images
      conv_first<<<grid_of(P), kNnThreads, 0, s>>>(in_f.get(), in_ch, cur_n, H, Wd,
                                                   w.get() + L.w_off, w.get() + L.b_off, L.cout,
                                                   L.cout_s, L.relu,
                                                   reinterpret_cast<uint4 *>(Y.v.get()));
      NCK(cudaGetLastError());
      return;
    }
    if (L.cin % 8 != 0) {
      im2col3x3<<<grid_of(P * L.kp), kNnThreads, 0, s>>>(X.v.get(), cur_n, H, Wd, L.cin, X.Cs,
                                                         L.kp, col.get());
      NCK(cudaGetLastError());
      A = col.get();
      geom.x = nullptr;
    }
    const HaloPlan hp = A == nullptr ? halo_plan(geom, L.cout_s, L.kp) : HaloPlan{};
    if (hp.bn > 0) {
      NCK(tc_conv(wp[&L - layers.data()].get(), z.get(), P, L.cout_s, L.cout_s, geom, hp, act,
                  err.get(), s));
    } else {
      NCK(tc_gemm(A, wp[&L - layers.data()].get(), z.get(), (int)P, L.cout_s, L.kp, L.kp, L.kp,
                  L.cout_s, 1.f, 0.f, err.get(), s, 1, geom, act));
    }
    if (keep_f32) {
      bias_act<<<grid_of(P * L.cout_s), kNnThreads, 0, s>>>(
          z.get(), w.get() + L.b_off, P, L.cout, L.cout_s, L.relu, Y.v.get(), last_f.get());
      NCK(cudaGetLastError());
    }
  }

  // n images (device fp32 [n][h][w][in_ch]; in_f itself or copied there) ->
  // out_f = channel 0 + network correction
  void forward(const float *in_dev) {
    const long P0 = pixels(0);
    if (in_dev != in_f.get())
      NCK(cudaMemcpyAsync(in_f.get(), in_dev, (size_t)P0 * in_ch * sizeof(float),
                          cudaMemcpyDeviceToDevice, s));
    if (t[0].Cs == 8) {
      load_input_v<<<grid_of(P0), kNnThreads, 0, s>>>(in_f.get(), in_ch, P0,
                                                      reinterpret_cast<uint4 *>(t[0].v.get()));
    } else {
      load_input<<<grid_of(P0 * t[0].Cs), kNnThreads, 0, s>>>(in_f.get(), in_ch, P0, t[0].Cs,
                                                               t[0].v.get());
    }
    NCK(cudaGetLastError());
    // row-wise 16-byte kernels where the channel stride is 8 times a power of two
    auto c8_shift = [](int cs) {
      int sh = 0;
      while ((8 << sh) < cs) ++sh;
      return (8 << sh) == cs ? sh : -1;
    };
    auto row_grid = [](long rows) {
      return (unsigned)std::max<long>(1, std::min<long>(rows, 148L * 8));
    };
    for (const Op &op : ops) {
      if (op.kind == kConv) {
        conv_forward(layers[op.a], op.a + 1 == (int)layers.size());
      } else if (op.kind == kPool) {
        const Tensor &X = t[op.a];
        const int sh = c8_shift(X.Cs), H = cur_h >> X.level, Wd = cur_w >> X.level;
        if (sh >= 0) {
          avgpool2_v<<<row_grid((long)cur_n * (H / 2)), kNnThreads, 0, s>>>(
              reinterpret_cast<const uint4 *>(X.v.get()), cur_n, H, Wd, sh,
              reinterpret_cast<uint4 *>(t[op.out].v.get()));
        } else {
          avgpool2<<<grid_of(pixels(X.level + 1) * X.Cs), kNnThreads, 0, s>>>(
              X.v.get(), cur_n, H, Wd, X.Cs, t[op.out].v.get());
        }
        NCK(cudaGetLastError());
      } else {
        const Tensor &S = t[op.b];
        const int sh = c8_shift(S.Cs), H = cur_h >> S.level, Wd = cur_w >> S.level;
        if (sh >= 0) {
          upsample2_add_v<<<row_grid((long)cur_n * H), kNnThreads, 0, s>>>(
              reinterpret_cast<const uint4 *>(t[op.a].v.get()),
              reinterpret_cast<const uint4 *>(S.v.get()), cur_n, H, Wd, sh,
              reinterpret_cast<uint4 *>(t[op.out].v.get()));
        } else {
          upsample2_add<<<grid_of(pixels(S.level) * S.Cs), kNnThreads, 0, s>>>(
              t[op.a].v.get(), S.v.get(), cur_n, H, Wd, S.Cs, t[op.out].v.get());
        }
        NCK(cudaGetLastError());
      }
    }
    residual_out<<<grid_of(P0), kNnThreads, 0, s>>>(in_f.get(), in_ch, last_f.get(), P0,
                                                     t.back().Cs, out_f.get());
    NCK(cudaGetLastError());
  }

  // gradients of the MSE loss against tgt_f (device, [n][h][w]) after
  // forward(): grad (zeroed here) and loss_d
  void backward() {
    const long P0 = pixels(0);
    NCK(cudaMemsetAsync(grad.get(), 0, n_params * sizeof(float), s));
    for (Tensor &x : t) NCK(cudaMemsetAsync(x.g.get(), 0, x.g.n * sizeof(float), s));
    NCK(cudaMemsetAsync(loss_d.get(), 0, sizeof(double), s));
    mse_grad<<<grid_of(P0), kNnThreads, 0, s>>>(out_f.get(), tgt_f.get(), P0, t.back().Cs,
                                                 t.back().g.get(), loss_d.get());
    NCK(cudaGetLastError());
    for (int oi = (int)ops.size() - 1; oi >= 0; --oi) {
      const Op &op = ops[oi];
      if (op.kind == kConv) {
        conv_backward(layers[op.a], op.a > 0);
      } else if (op.kind == kPool) {
        const Tensor &X = t[op.a];
        avgpool2_backward<<<grid_of(pixels(X.level) * X.Cs), kNnThreads, 0, s>>>(
            t[op.out].g.get(), cur_n, cur_h >> X.level, cur_w >> X.level, X.Cs, t[op.a].g.get());
        NCK(cudaGetLastError());
      } else {
        const Tensor &S = t[op.b];
        upsample2_backward<<<grid_of(pixels(S.level + 1) * S.Cs), kNnThreads, 0, s>>>(
            t[op.out].g.get(), cur_n, cur_h >> S.level, cur_w >> S.level, S.Cs,
            t[op.a].g.get());
        NCK(cudaGetLastError());
        const long n = pixels(S.level) * S.Cs;
        axpy1<<<grid_of(n), kNnThreads, 0, s>>>(t[op.out].g.get(), n, t[op.b].g.get());
        NCK(cudaGetLastError());
      }
    }
  }

  void conv_backward(const Layer &L, bool need_dx) {
    const size_t li = &L - layers.data();
    const Tensor &X = t[L.in];
    const Tensor &Y = t[L.out];
    const long P = pixels(X.level);
    const int H = cur_h >> X.level, Wd = cur_w >> X.level;
    act_backward<<<grid_of(P * L.cout_s), kNnThreads, 0, s>>>(Y.g.get(), Y.v.get(), P, L.cout,
                                                               L.cout_s, L.relu, dz.get());
    NCK(cudaGetLastError());
    bias_grad<<<L.cout, kNnThreads, 0, s>>>(dz.get(), P, L.cout, L.cout_s,
                                            grad.get() + L.b_off);
    NCK(cudaGetLastError());
    // dW = dZ^T col: both transposed so that the pixels are the K dimension
    im2col3x3<<<grid_of(P * L.kp), kNnThreads, 0, s>>>(X.v.get(), cur_n, H, Wd, L.cin, X.Cs,
                                                       L.kp, col.get());
    NCK(cudaGetLastError());
    const dim3 tb(32, 8);
    transpose_bf16<<<dim3((unsigned)((P + 31) / 32), (unsigned)((L.kp + 31) / 32)), tb, 0, s>>>(
        col.get(), P, L.kp, L.kp, colT.get(), P);
    NCK(cudaGetLastError());
    transpose_bf16<<<dim3((unsigned)((P + 31) / 32), (unsigned)((L.cout_s + 31) / 32)), tb, 0,
                     s>>>(dz.get(), P, L.cout_s, L.cout_s, dzT.get(), P);
    NCK(cudaGetLastError());
    NCK(cudaMemsetAsync(dwp.get(), 0, (size_t)L.cout_s * L.kp * sizeof(float), s));
    const long tiles = ((L.cout_s + 127) / 128) * ((L.kp + (L.kp <= 64 ? 63 : 127)) /
                                                   (L.kp <= 64 ? 64 : 128));
    const int splits = (int)std::max<long>(1, std::min<long>(592 / std::max<long>(tiles, 1),
                                                             (P + 63) / 64));
    gemm(dzT.get(), colT.get(), dwp.get(), L.cout_s, L.kp, P, P, P, L.kp, 0.f, splits);
    unpack_grad<<<grid_of((long)L.cout * 9 * L.cin), kNnThreads, 0, s>>>(
        dwp.get(), L.cout, 9 * L.cin, L.kp, grad.get() + L.w_off);
    NCK(cudaGetLastError());
    if (!need_dx) return;
    // dX = col2im(dZ W)
    gemm(dz.get(), wpt[li].get(), dcol.get(), P, L.kp, L.cout_s, L.cout_s, L.cout_s, L.kp, 0.f);
    col2im3x3<<<grid_of(P * L.cin), kNnThreads, 0, s>>>(dcol.get(), cur_n, H, Wd, L.cin, L.kp,
                                                        t[L.in].g.get(), X.Cs, 1);
    NCK(cudaGetLastError());
  }

  void adam(float lr) {
    ++adam_t;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)adam_t), c2 = 1.f - std::pow(b2, (float)adam_t);
    adam_step<<<grid_of(n_params), kNnThreads, 0, s>>>(w.get(), grad.get(), m.get(), v.get(),
                                                        n_params, lr, b1, b2, 1e-8f, c1, c2,
                                                        nullptr);
    NCK(cudaGetLastError());
    pack_weights();
  }

  void check_errors() {
    int h = 0;
    NCK(cudaMemcpyAsync(&h, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    NCK(cudaStreamSynchronize(s));
    if (h) throw NnError("a tensor-core GEMM gave up waiting for its MMAs");
  }

  double read_loss() {
    double l = 0;
    NCK(cudaMemcpyAsync(&l, loss_d.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
    NCK(cudaStreamSynchronize(s));
    return l;
  }
};

}  // namespace nn
}  // namespace agd

struct agd_nn {
  std::unique_ptr<agd::nn::Net> net;
};

namespace agd {
namespace nn {

int input_channels(const agd_nn *handle) { return handle->net->in_ch; }

void estimate_images(agd_nn *handle, const float *src, float *dst,
                     const std::vector<ImageGroup> &groups, cudaStream_t stream) {
  nvtxRangePushA("agd network estimate");
  Net &nt = *handle->net;
  // the network's stream follows the caller's and the caller's the network's
  cudaEvent_t ev = nullptr;
  NCK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  NCK(cudaEventRecord(ev, stream));
  NCK(cudaStreamWaitEvent(nt.s, ev, 0));
  const long max_pixels = 1L << 23;  // images per network pass
  Buf<float> &rms = nt.rms_buf;
  Buf<long> &bases = nt.base_buf, &nbrs = nt.nbr_buf;
  const int k = nt.in_ch;
  for (const ImageGroup &g : groups) {
    if (g.base.empty()) continue;
    if (k > 1 && g.nbr.size() != g.base.size() * (k - 1))
      throw NnError("image group without the neighbour lines of every input channel");
    const int hp = pad8(g.rows), wp = pad8(g.cols);
    const long per = (long)hp * wp;
    const int chunk = (int)std::max<long>(1, std::min<long>((long)g.base.size(),
                                                            max_pixels / per));
    rms.ensure(chunk);
    bases.ensure(g.base.size());
    NCK(cudaMemcpyAsync(bases.get(), g.base.data(), g.base.size() * sizeof(long),
                        cudaMemcpyHostToDevice, nt.s));
    if (k > 1) {
      nbrs.ensure(g.nbr.size());
      NCK(cudaMemcpyAsync(nbrs.get(), g.nbr.data(), g.nbr.size() * sizeof(long),
                          cudaMemcpyHostToDevice, nt.s));
    }
    for (size_t i0 = 0; i0 < g.base.size(); i0 += chunk) {
      const int n = (int)std::min<size_t>(chunk, g.base.size() - i0);
      nt.shape(n, hp, wp, false);  // the images go straight into the network's input
      gather_images<<<n, kNnThreads, 0, nt.s>>>(src, bases.get() + i0,
                                                 k > 1 ? nbrs.get() + i0 * (k - 1) : nullptr, k,
                                                 g.rows, g.cols, g.row_stride, hp, wp,
                                                 nt.in_f.get(), rms.get());
      NCK(cudaGetLastError());
      nt.forward(nt.in_f.get());
      scatter_images<<<n, kNnThreads, 0, nt.s>>>(nt.out_f.get(), bases.get() + i0, g.rows,
                                                  g.cols, g.row_stride, hp, wp, rms.get(), dst);
      NCK(cudaGetLastError());
    }
  }
  NCK(cudaEventRecord(ev, nt.s));
  NCK(cudaStreamWaitEvent(stream, ev, 0));
  nt.check_errors();  // synchronises the network's stream
  cudaEventDestroy(ev);
  nvtxRangePop();
}

}  // namespace nn
}  // namespace agd

namespace {

template <typename F>
int nn_guarded(const char *name, F &&f) {
  try {
    return f();
  } catch (const std::exception &e) {
    std::fprintf(stderr, "ERROR: %s\nERROR in %s\n", e.what(), name);
    return 1;
  }
}

}  // namespace

extern "C" {

int agd_nn_create_channels(int base_channels, int in_channels, unsigned seed, agd_nn **net) {
  if (net == nullptr || base_channels < 1 || base_channels > 256 || in_channels < 1 ||
      in_channels > 8)
    return 1;
  *net = nullptr;
  return nn_guarded("agd_nn_create", [&] {
    auto h = std::make_unique<agd_nn>();
    h->net = std::make_unique<agd::nn::Net>(base_channels, seed, in_channels);
    *net = h.release();
    return 0;
  });
}

int agd_nn_create(int base_channels, unsigned seed, agd_nn **net) {
  return agd_nn_create_channels(base_channels, 1, seed, net);
}

int agd_nn_input_channels(const agd_nn *net) { return net ? net->net->in_ch : -1; }

void agd_nn_destroy(agd_nn *net) { delete net; }

long agd_nn_param_count(const agd_nn *net) { return net ? net->net->n_params : -1; }

int agd_nn_get_params(const agd_nn *net, float *params) {
  if (net == nullptr || params == nullptr) return 1;
  return nn_guarded("agd_nn_get_params", [&] {
    agd::nn::Net &n = *net->net;
    agd::nn::NCK(cudaMemcpyAsync(params, n.w.get(), n.n_params * sizeof(float),
                                 cudaMemcpyDeviceToHost, n.s));
    agd::nn::NCK(cudaStreamSynchronize(n.s));
    return 0;
  });
}

int agd_nn_set_params(agd_nn *net, const float *params) {
  if (net == nullptr || params == nullptr) return 1;
  return nn_guarded("agd_nn_set_params", [&] {
    agd::nn::Net &n = *net->net;
    agd::nn::NCK(cudaMemcpyAsync(n.w.get(), params, n.n_params * sizeof(float),
                                 cudaMemcpyHostToDevice, n.s));
    n.pack_weights();
    agd::nn::NCK(cudaStreamSynchronize(n.s));
    return 0;
  });
}

int agd_nn_forward(agd_nn *net, const float *input, int n, int h, int w, float *output) {
  if (net == nullptr || input == nullptr || output == nullptr) return 1;
  return nn_guarded("agd_nn_forward", [&] {
    agd::nn::Net &nt = *net->net;
    nt.shape(n, h, w, false);
    const long P0 = (long)n * h * w;
    agd::nn::NCK(cudaMemcpyAsync(nt.in_f.get(), input, (size_t)P0 * nt.in_ch * sizeof(float),
                                 cudaMemcpyHostToDevice, nt.s));
    nt.forward(nt.in_f.get());
    agd::nn::NCK(cudaMemcpyAsync(output, nt.out_f.get(), P0 * sizeof(float),
                                 cudaMemcpyDeviceToHost, nt.s));
    nt.check_errors();
    return 0;
  });
}

int agd_nn_loss_grad(agd_nn *net, const float *input, const float *target, int n, int h, int w,
                     double *loss, float *grad) {
  if (net == nullptr || input == nullptr || target == nullptr) return 1;
  return nn_guarded("agd_nn_loss_grad", [&] {
    agd::nn::Net &nt = *net->net;
    nt.shape(n, h, w);
    const long P0 = (long)n * h * w;
    agd::nn::NCK(cudaMemcpyAsync(nt.in_f.get(), input, (size_t)P0 * nt.in_ch * sizeof(float),
                                 cudaMemcpyHostToDevice, nt.s));
    nt.forward(nt.in_f.get());
    agd::nn::NCK(cudaMemcpyAsync(nt.tgt_f.get(), target, P0 * sizeof(float),
                                 cudaMemcpyHostToDevice, nt.s));
    nt.backward();
    if (loss) *loss = nt.read_loss();
    if (grad)
      agd::nn::NCK(cudaMemcpyAsync(grad, nt.grad.get(), nt.n_params * sizeof(float),
                                   cudaMemcpyDeviceToHost, nt.s));
    nt.check_errors();
    return 0;
  });
}

int agd_nn_train(agd_nn *net, const float *inputs, const float *targets, long n_samples, int h,
                 int w, int batch, int epochs, float lr, unsigned seed, double *epoch_loss) {
  if (net == nullptr || inputs == nullptr || targets == nullptr || n_samples < batch ||
      batch <= 0 || epochs <= 0)
    return 1;
  return nn_guarded("agd_nn_train", [&] {
    agd::nn::Net &nt = *net->net;
    nt.shape(batch, h, w);
    const long hw = (long)h * w, hwc = hw * nt.in_ch;  // values per target, per input
    agd::nn::Buf<float> din, dtg;
    agd::nn::Buf<int> didx;
    din.ensure((size_t)n_samples * hwc);
    dtg.ensure((size_t)n_samples * hw);
    didx.ensure(batch);
    agd::nn::NCK(cudaMemcpyAsync(din.get(), inputs, n_samples * hwc * sizeof(float),
                                 cudaMemcpyHostToDevice, nt.s));
    agd::nn::NCK(cudaMemcpyAsync(dtg.get(), targets, n_samples * hw * sizeof(float),
                                 cudaMemcpyHostToDevice, nt.s));
    std::mt19937 rng(seed);
    std::vector<int> perm(n_samples);
    for (long i = 0; i < n_samples; ++i) perm[i] = (int)i;
    const long steps = n_samples / batch;
    for (int ep = 0; ep < epochs; ++ep) {
      std::shuffle(perm.begin(), perm.end(), rng);
      double sum = 0;
      for (long st = 0; st < steps; ++st) {
        agd::nn::NCK(cudaMemcpyAsync(didx.get(), perm.data() + st * batch, batch * sizeof(int),
                                     cudaMemcpyHostToDevice, nt.s));
        agd::nn::gather_samples<<<agd::nn::grid_of(batch * hwc), agd::nn::kNnThreads, 0,
                                       nt.s>>>(din.get(), didx.get(), batch, hwc,
                                               nt.in_f.get());
        nt.forward(nt.in_f.get());
        agd::nn::gather_samples<<<agd::nn::grid_of(batch * hw), agd::nn::kNnThreads, 0,
                                       nt.s>>>(dtg.get(), didx.get(), batch, hw,
                                               nt.tgt_f.get());
        nt.backward();
        nt.adam(lr);
        sum += nt.read_loss();  // also keeps the host in step with the device
      }
      if (epoch_loss) epoch_loss[ep] = sum / (double)steps;
    }
    nt.check_errors();
    return 0;
  });
}

}  // extern "C"
