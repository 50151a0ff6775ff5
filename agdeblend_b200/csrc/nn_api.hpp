// Interface between the solver (engine.cu) and the warm-start network
// (nn.cu): the network's estimate of deblended data held on the device.
#pragma once

#include <cuda_runtime.h>

#include <vector>

struct agd_nn;

namespace agd {
namespace nn {

// 2-D images cut from patch data in device memory: image i is the rows
// (traces along one space axis) x cols (time samples) block starting at
// base[i], rows row_stride apart.  Images of one group share their shape.
struct ImageGroup {
  std::vector<long> base;
  int rows = 0, cols = 0;
  long row_stride = 0;
};

// Replaces every image of `data` (device, float) by the network's estimate
// of it: each image normalised by its RMS, padded to multiples of 8, run
// through the network, scaled back.  Runs on `stream`; throws on failure.
void estimate_images(agd_nn *net, float *data, const std::vector<ImageGroup> &groups,
                     cudaStream_t stream);

}  // namespace nn
}  // namespace agd
