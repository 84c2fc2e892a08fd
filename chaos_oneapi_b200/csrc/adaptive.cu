// Adaptive sweep kernels for the 3-4-dimensional flows (see adaptive.cuh for
// the numerics).  One thread per point.  Two launch forms share one kernel:
//  * direct: thread i integrates point i;
//  * persistent work queue: a grid sized to the machine (a multiple of the
//    SM count) whose threads pull point indices from a device counter, so a
//    thread whose point needed fewer adaptive steps (or a shorter averaging
//    time) starts the next point at once instead of idling until the
//    slowest lane of its warp is done.
#include <algorithm>

#include "adaptive.cuh"

namespace chaos {
namespace adaptive {

// The queue hands out points in the order q -> (q * stride) mod P (stride
// coprime to P, so a permutation): neighbouring grid points cost alike, and
// spreading them over the run keeps a cluster of expensive points (a chaotic
// band, escaping orbits) from forming the tail of the launch.
__device__ __forceinline__ int64_t next_point(const AdaptiveArgs &a) {
  const unsigned long long q = atomicAdd(a.queue, 1ULL);
  if (q >= (unsigned long long)a.P) return a.P;
  return (int64_t)((q * (unsigned long long)a.queue_stride) % (unsigned long long)a.P);
}

template <class M, int K, class R, int INTEG>
__global__ void __launch_bounds__(128) sweep_kernel(const AdaptiveArgs a) {
  int64_t pt = a.queue ? next_point(a) : (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  while (pt < a.P) {
    run_point<M, K, R, INTEG>(a, pt);
    if (!a.queue) break;
    pt = next_point(a);
  }
}

template <class M, class R, int INTEG>
int launch_mri(const AdaptiveArgs &a, int block, int persistent_blocks, cudaStream_t s) {
  if (a.k != M::N) return kErrUnsupported;
  auto kern = sweep_kernel<M, M::N, R, INTEG>;
  unsigned grid;
  if (a.queue) {
    if (persistent_blocks <= 0) {
      // one full wave: resident blocks per SM x SM count
      int dev = 0, sms = 0, per_sm = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, 0);
      persistent_blocks = std::max(1, per_sm) * std::max(1, sms);
    }
    const int64_t need = (a.P + block - 1) / block;  // never more blocks than points need
    grid = (unsigned)std::min<int64_t>(persistent_blocks, need);
  } else {
    grid = (unsigned)((a.P + block - 1) / block);
  }
  kern<<<grid, block, 0, s>>>(a);
  return (int)cudaGetLastError();
}

template <class M>
int launch_m(int integ, int prec, const AdaptiveArgs &a, int block, int pblocks, cudaStream_t s) {
  if (integ == kDverk65) {
    if (prec == kFP64) return launch_mri<M, double, kDverk65>(a, block, pblocks, s);
    if (prec == kFP32) return launch_mri<M, float, kDverk65>(a, block, pblocks, s);
  } else if (integ == kDopri5) {
    if (prec == kFP64) return launch_mri<M, double, kDopri5>(a, block, pblocks, s);
    if (prec == kFP32) return launch_mri<M, float, kDopri5>(a, block, pblocks, s);
  }
  return kErrUnsupported;
}

}  // namespace adaptive

int launch_adaptive(int model, int integ, int prec, const AdaptiveArgs &a, int block,
                    int persistent_blocks, cudaStream_t s) {
  using namespace adaptive;
  if (a.P <= 0) return 0;
  if (block <= 0 || block > 128) block = 128;
  switch (model) {
    case kShimizu: return launch_m<Shimizu>(integ, prec, a, block, persistent_blocks, s);
    case kLorenz: return launch_m<Lorenz>(integ, prec, a, block, persistent_blocks, s);
    case kRossler: return launch_m<Rossler>(integ, prec, a, block, persistent_blocks, s);
    case kChua: return launch_m<Chua>(integ, prec, a, block, persistent_blocks, s);
    case kHyperRossler: return launch_m<HyperRossler>(integ, prec, a, block, persistent_blocks, s);
    default: return kErrUnsupported;
  }
}

}  // namespace chaos
