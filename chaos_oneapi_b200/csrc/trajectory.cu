// Trajectory kernel (trajectory.cuh): one thread per point, the state alone.
#include "trajectory.cuh"

namespace chaos {
namespace adaptive {

template <class M, class R, int INTEG>
__global__ void __launch_bounds__(128) trajectory_kernel(const TrajectoryArgs ta) {
  const int64_t pt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (pt < ta.a.P) run_trajectory<M, R, INTEG>(ta, pt);
}

template <class M>
int launch_traj_m(int integ, int prec, const TrajectoryArgs &ta, cudaStream_t s) {
  const unsigned grid = (unsigned)((ta.a.P + 127) / 128);
  if (integ == kDopri5 && prec == kFP64) trajectory_kernel<M, double, kDopri5><<<grid, 128, 0, s>>>(ta);
  else if (integ == kDopri5 && prec == kFP32) trajectory_kernel<M, float, kDopri5><<<grid, 128, 0, s>>>(ta);
  else if (integ == kDverk65 && prec == kFP64) trajectory_kernel<M, double, kDverk65><<<grid, 128, 0, s>>>(ta);
  else if (integ == kDverk65 && prec == kFP32) trajectory_kernel<M, float, kDverk65><<<grid, 128, 0, s>>>(ta);
  else return kErrUnsupported;
  return (int)cudaGetLastError();
}

}  // namespace adaptive

int launch_trajectory(int model, int integ, int prec, const adaptive::TrajectoryArgs &ta,
                      cudaStream_t s) {
  using namespace adaptive;
  if (ta.a.P <= 0 || ta.nsteps <= 0) return 0;
  switch (model) {
    case kShimizu: return launch_traj_m<Shimizu>(integ, prec, ta, s);
    case kLorenz: return launch_traj_m<Lorenz>(integ, prec, ta, s);
    case kRossler: return launch_traj_m<Rossler>(integ, prec, ta, s);
    case kChua: return launch_traj_m<Chua>(integ, prec, ta, s);
    case kHyperRossler: return launch_traj_m<HyperRossler>(integ, prec, ta, s);
    default: return kErrUnsupported;
  }
}

}  // namespace chaos
