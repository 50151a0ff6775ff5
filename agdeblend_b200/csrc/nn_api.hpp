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
// For a network with k > 1 input channels, nbr holds k - 1 further starts
// per image (image i's at nbr[i (k - 1) ..]): the blocks fed as channels
// 1 .. k - 1 (neighbouring lines along another space axis).
struct ImageGroup {
  std::vector<long> base, nbr;
  int rows = 0, cols = 0;
  long row_stride = 0;
};

// Input channels of the network (1 unless created with more).
int input_channels(const agd_nn *net);

// Writes the network's estimate of every image of `src` (device, float)
// into the same place in `dst` (src itself is allowed when the network has
// one input channel): each image with its neighbour channels normalised by
// the image's RMS, padded to multiples of 8, run through the network,
// scaled back.  Runs on `stream`; throws on failure.
void estimate_images(agd_nn *net, const float *src, float *dst,
                     const std::vector<ImageGroup> &groups, cudaStream_t stream);

}  // namespace nn
}  // namespace agd
