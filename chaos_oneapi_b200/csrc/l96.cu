// Warp-per-point sweep for the 40-dimensional Lorenz-96 model.
#include "kernels.h"

namespace chaos {

int launch_l96_warp(int, int, const AdaptiveArgs &, int, cudaStream_t) { return kErrUnsupported; }

}  // namespace chaos
