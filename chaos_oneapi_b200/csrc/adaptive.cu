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
// With an explicit order (longest averaging time first, order.cu) the queue
// hands out order[q] instead.
__device__ __forceinline__ int64_t next_point(const AdaptiveArgs &a) {
  const unsigned long long q = atomicAdd(a.queue, 1ULL);
  if (q >= (unsigned long long)a.P) return a.P;
  if (a.order) return (int64_t)a.order[q];
  return (int64_t)((q * (unsigned long long)a.queue_stride) % (unsigned long long)a.P);
}

// Each lane owns one point at a time and runs it as a state machine (one
// step attempt per loop iteration), so a lane never waits for another lane's
// phase or renormalisation interval to end: when its point is done it takes
// the next one from the queue (persistent form) and carries on.  Gram-Schmidt
// is voted per warp: when any lane is due, every lane past its transient
// renormalises in the same pass.
// MINB: resident 128-thread blocks per SM the kernel is compiled for (a
// register cap: 4 -> 128 registers, 5 -> 96 with a few spills); the
// autotuner picks the variant.
template <class M, int K, class R, int INTEG, int MINB>
__global__ void __launch_bounds__(128, MINB) sweep_kernel(const AdaptiveArgs a) {
  const Ctl &c = a.ctl;
  Lane<M, K, R, INTEG> L;
  int64_t pt = a.queue ? next_point(a) : (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool active = pt < a.P;
  if (active) lane_start(L, a, pt);
  while (__any_sync(0xffffffffu, active)) {
    if (active && lane_step(L, a, c) == kFinished) {
      pt = a.queue ? next_point(a) : a.P;
      active = pt < a.P;
      if (active) lane_start(L, a, pt);
    }
    const bool due = active && L.phase != kTransient && L.t_gs >= L.L;
    if (__any_sync(0xffffffffu, due)) {
      if (active && L.phase != kTransient && L.t_gs > 0.f && !lane_gram_schmidt(L, a, c)) {
        lane_finish(L, a, 1);
        pt = a.queue ? next_point(a) : a.P;
        active = pt < a.P;
        if (active) lane_start(L, a, pt);
      }
    }
  }
}

template <class M, class R, int INTEG>
int launch_mri(const AdaptiveArgs &a, int block, int persistent_blocks, int variant,
               cudaStream_t s) {
  if (a.k != M::N) return kErrUnsupported;
  auto kern = sweep_kernel<M, M::N, R, INTEG, 1>;
  if (sizeof(R) == 4) kern = variant == 1 ? sweep_kernel<M, M::N, R, INTEG, 5>
                                          : sweep_kernel<M, M::N, R, INTEG, 4>;
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
  AdaptiveArgs ka = a;
  ka.ctl = make_ctl<R>(a);
  kern<<<grid, block, 0, s>>>(ka);
  return (int)cudaGetLastError();
}

template <class M>
int launch_m(int integ, int prec, const AdaptiveArgs &a, int block, int pblocks, int variant,
             cudaStream_t s) {
  if (integ == kDverk65) {
    if (prec == kFP64) return launch_mri<M, double, kDverk65>(a, block, pblocks, variant, s);
    if (prec == kFP32) return launch_mri<M, float, kDverk65>(a, block, pblocks, variant, s);
  } else if (integ == kDopri5) {
    if (prec == kFP64) return launch_mri<M, double, kDopri5>(a, block, pblocks, variant, s);
    if (prec == kFP32) return launch_mri<M, float, kDopri5>(a, block, pblocks, variant, s);
  }
  return kErrUnsupported;
}

// ----------------------------------------------------------- mixed batch
// One persistent launch over segments of different models (3- and
// 4-dimensional) and per-point averaging times.  Every warp works on one
// segment at a time (warps start on segments round robin); while it does, it
// runs that segment's model-specific loop -- the sweep kernel's loop with the
// segment's queue -- so the step code is specialised to the model, with no
// per-step dispatch, and a lane that finishes a point takes the next point of
// the segment: lanes refill independently, so uneven point lengths do not
// strand warps, and all lanes of a warp run one model's instruction stream.
// When all lanes of the warp are idle (the segment's queue is empty) the warp
// moves on to the next segment with points left.  (Letting lanes move on
// individually mixes models inside warps, which runs every model's step code
// for the warp and measured slower than three separate launches.)

// Next point of segment `seg` for this lane, if any is left.
__device__ __forceinline__ bool batch_take(const BatchArgs &b, int seg, int64_t &pt) {
  const int64_t P = b.seg[seg].P;
  const unsigned long long q = atomicAdd(&b.queues[seg], 1ULL);
  if (q >= (unsigned long long)P) return false;
  pt = b.seg[seg].order
           ? (int64_t)b.seg[seg].order[q]
           : (int64_t)((q * (unsigned long long)b.seg[seg].queue_stride) % (unsigned long long)P);
  return true;
}

template <class M, class R, int INTEG>
__device__ __noinline__ void lane_segment(const BatchArgs &b, int seg, bool active, int64_t pt) {
  const AdaptiveArgs &a = b.seg[seg];
  const Ctl &c = a.ctl;
  Lane<M, M::N, R, INTEG> L;
  if (active) lane_start(L, a, pt);
  while (__any_sync(0xffffffffu, active)) {
    if (active && lane_step(L, a, c) == kFinished) {
      active = batch_take(b, seg, pt);
      if (active) lane_start(L, a, pt);
    }
    const bool due = active && L.phase != kTransient && L.t_gs >= L.L;
    if (__any_sync(0xffffffffu, due)) {
      if (active && L.phase != kTransient && L.t_gs > 0.f && !lane_gram_schmidt(L, a, c)) {
        lane_finish(L, a, 1);
        active = batch_take(b, seg, pt);
        if (active) lane_start(L, a, pt);
      }
    }
  }
}

template <class R, int INTEG>
__global__ void __launch_bounds__(128, sizeof(R) == 4 ? 3 : 1)
    batch_kernel(const __grid_constant__ BatchArgs b) {
  const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  int wseg = warp % b.nseg;
  for (int tried = 0; tried < b.nseg; wseg = (wseg + 1) % b.nseg) {
    int64_t pt = 0;
    const bool active = batch_take(b, wseg, pt);
    if (!__any_sync(0xffffffffu, active)) {  // nothing left here for this warp
      ++tried;
      continue;
    }
    tried = 0;
    switch (b.model[wseg]) {
      case kShimizu: lane_segment<Shimizu, R, INTEG>(b, wseg, active, pt); break;
      case kLorenz: lane_segment<Lorenz, R, INTEG>(b, wseg, active, pt); break;
      case kRossler: lane_segment<Rossler, R, INTEG>(b, wseg, active, pt); break;
      case kChua: lane_segment<Chua, R, INTEG>(b, wseg, active, pt); break;
      default: lane_segment<HyperRossler, R, INTEG>(b, wseg, active, pt); break;
    }
  }
}

}  // namespace adaptive

int launch_batch(int integ, int prec, const BatchArgs &b, int block, cudaStream_t s,
                 double share, bool high_priority) {
  using namespace adaptive;
  if (b.nseg <= 0 || b.nseg > kMaxSegments) return kErrUnsupported;
  int64_t total = 0;
  for (int i = 0; i < b.nseg; i++) {
    if (b.model[i] < 0 || b.model[i] >= kLorenz96) return kErrUnsupported;
    const int dim = b.model[i] == kHyperRossler ? 4 : 3;
    if (b.seg[i].k != dim) return kErrUnsupported;
    total += b.seg[i].P;
  }
  if (total <= 0) return 0;
  if (block <= 0 || block > 128 || block % 32) block = 128;
  void (*kern)(BatchArgs) = nullptr;
  if (integ == kDopri5 && prec == kFP32) kern = batch_kernel<float, kDopri5>;
  else if (integ == kDopri5 && prec == kFP64) kern = batch_kernel<double, kDopri5>;
  else if (integ == kDverk65 && prec == kFP32) kern = batch_kernel<float, kDverk65>;
  else if (integ == kDverk65 && prec == kFP64) kern = batch_kernel<double, kDverk65>;
  else return kErrUnsupported;
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, 0);
  const int64_t full = (int64_t)std::max(1, per_sm) * sms;
  const int64_t cap = std::max<int64_t>(1, (int64_t)(full * std::min(1.0, std::max(share, 0.0))));
  const int64_t grid = std::min<int64_t>(cap, (total + block - 1) / block);
  return (int)launch_with_priority(kern, (unsigned)grid, (unsigned)block, s, high_priority,
                                  with_ctl(b, prec));
}

int launch_adaptive(int model, int integ, int prec, const AdaptiveArgs &a, int block,
                    int persistent_blocks, int variant, cudaStream_t s) {
  using namespace adaptive;
  if (a.P <= 0) return 0;
  if (block <= 0 || block > 128 || block % 32) block = 128;
  const int pb = persistent_blocks, v = variant;
  switch (model) {
    case kShimizu: return launch_m<Shimizu>(integ, prec, a, block, pb, v, s);
    case kLorenz: return launch_m<Lorenz>(integ, prec, a, block, pb, v, s);
    case kRossler: return launch_m<Rossler>(integ, prec, a, block, pb, v, s);
    case kChua: return launch_m<Chua>(integ, prec, a, block, pb, v, s);
    case kHyperRossler: return launch_m<HyperRossler>(integ, prec, a, block, pb, v, s);
    default: return kErrUnsupported;
  }
}

}  // namespace chaos
