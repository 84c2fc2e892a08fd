// Kernels of the split form (split.cuh): a sweep over one model and a mixed
// batch, both with one parameter point per group of four lanes.
#include <algorithm>
#include <type_traits>

#include "split.cuh"

namespace chaos {
namespace adaptive {

// Next point for the group: its first lane takes it from the queue (in the
// queue's order) and hands it to the other three.
__device__ __forceinline__ int64_t group_next_point(const AdaptiveArgs &a, const Group &g) {
  int64_t pt = 0;
  if (g.r == 0) {
    const unsigned long long q = atomicAdd(a.queue, 1ULL);
    if (q >= (unsigned long long)a.P) pt = a.P;
    else if (a.order) pt = (int64_t)a.order[q];
    else pt = (int64_t)((q * (unsigned long long)a.queue_stride) % (unsigned long long)a.P);
  }
  return __shfl_sync(g.mask, pt, g.base);
}

// Direct form: group i integrates point i.  Persistent form: groups pull
// points from the queue until it is empty.  Gram-Schmidt is voted per warp,
// as in the one-lane form.
template <class M, class R, int INTEG, bool XCH>
__global__ void __launch_bounds__(128) split_kernel(const AdaptiveArgs a) {
  const Group g = group_of();
  const Ctl &c = a.ctl;
  SplitLane<M, R, INTEG, XCH> L;
  int64_t pt = a.queue ? group_next_point(a, g)
                       : ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kSplitLanes;
  bool active = pt < a.P;
  if (active) split_start(L, a, pt, g);
  while (__any_sync(0xffffffffu, active)) {
    if (active && split_step(L, a, c, g) == kFinished) {
      pt = a.queue ? group_next_point(a, g) : a.P;
      active = pt < a.P;
      if (active) split_start(L, a, pt, g);
    }
    const bool due = active && L.phase != kTransient && L.t_gs >= L.L;
    if (__any_sync(0xffffffffu, due)) {
      if (active && L.phase != kTransient && L.t_gs > 0.f && !split_gram_schmidt(L, a, c, g)) {
        split_finish(L, a, g, 1);
        pt = a.queue ? group_next_point(a, g) : a.P;
        active = pt < a.P;
        if (active) split_start(L, a, pt, g);
      }
    }
  }
}

// variant 1: the exchange layout (split.cuh: XCH), FP64 and 3-dimensional
// models only; otherwise the default layout.
template <class M, class R, int INTEG>
int launch_split_mri(const AdaptiveArgs &a, int block, int variant, cudaStream_t s) {
  if (a.k != M::N) return kErrUnsupported;
  constexpr bool xch_ok = std::is_same<R, double>::value && M::N == 3;
  void (*kern)(AdaptiveArgs) = split_kernel<M, R, INTEG, false>;
  if constexpr (xch_ok) {
    if (variant == 1) kern = split_kernel<M, R, INTEG, true>;
  }
  unsigned grid;
  const int64_t groups_per_block = block / kSplitLanes;
  const int64_t need = (a.P + groups_per_block - 1) / groups_per_block;
  if (a.queue) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, 0);
    grid = (unsigned)std::min<int64_t>((int64_t)std::max(1, per_sm) * sms, need);
  } else {
    grid = (unsigned)need;
  }
  AdaptiveArgs ka = a;
  ka.ctl = make_ctl<R>(a);
  kern<<<grid, block, 0, s>>>(ka);
  return (int)cudaGetLastError();
}

template <class M>
int launch_split_m(int integ, int prec, const AdaptiveArgs &a, int block, int variant,
                   cudaStream_t s) {
  if (integ == kDverk65) {
    if (prec == kFP64) return launch_split_mri<M, double, kDverk65>(a, block, variant, s);
    if (prec == kFP32) return launch_split_mri<M, float, kDverk65>(a, block, variant, s);
  } else if (integ == kDopri5) {
    if (prec == kFP64) return launch_split_mri<M, double, kDopri5>(a, block, variant, s);
    if (prec == kFP32) return launch_split_mri<M, float, kDopri5>(a, block, variant, s);
  }
  return kErrUnsupported;
}

// ----------------------------------------------------------- mixed batch
// The batch kernel of adaptive.cu in the split form: each warp works on one
// segment at a time (warps start on segments round robin); while it does, it
// runs that segment's model-specific loop -- the sweep kernel's loop with the
// segment's queue -- so the step code is specialised to the model, with no
// per-step dispatch.  When all groups of the warp are idle (the segment's
// queue is empty) the warp moves on to the next segment with points left.
__device__ __forceinline__ bool group_take(const BatchArgs &b, int seg, const Group &g,
                                           int64_t &pt) {
  int64_t v = -1;
  if (g.r == 0) {
    const int64_t P = b.seg[seg].P;
    const unsigned long long q = atomicAdd(&b.queues[seg], 1ULL);
    if (q < (unsigned long long)P)
      v = b.seg[seg].order ? (int64_t)b.seg[seg].order[q]
                           : (int64_t)((q * (unsigned long long)b.seg[seg].queue_stride) %
                                       (unsigned long long)P);
  }
  v = __shfl_sync(g.mask, v, g.base);
  pt = v;
  return v >= 0;
}

template <class M, class R, int INTEG>
__device__ __noinline__ void split_segment(const BatchArgs &b, int seg, const Group &g, bool active,
                              int64_t pt) {
  const AdaptiveArgs &a = b.seg[seg];
  const Ctl &c = a.ctl;
  SplitLane<M, R, INTEG> L;
  if (active) split_start(L, a, pt, g);
  while (__any_sync(0xffffffffu, active)) {
    if (active && split_step(L, a, c, g) == kFinished) {
      active = group_take(b, seg, g, pt);
      if (active) split_start(L, a, pt, g);
    }
    const bool due = active && L.phase != kTransient && L.t_gs >= L.L;
    if (__any_sync(0xffffffffu, due)) {
      if (active && L.phase != kTransient && L.t_gs > 0.f && !split_gram_schmidt(L, a, c, g)) {
        split_finish(L, a, g, 1);
        active = group_take(b, seg, g, pt);
        if (active) split_start(L, a, pt, g);
      }
    }
  }
}

template <class R, int INTEG>
__global__ void __launch_bounds__(128, sizeof(R) == 4 ? 4 : 2)
    batch_split_kernel(const __grid_constant__ BatchArgs b) {
  const Group g = group_of();
  const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  int wseg = warp % b.nseg;
  for (int tried = 0; tried < b.nseg; wseg = (wseg + 1) % b.nseg) {
    int64_t pt = 0;
    const bool active = group_take(b, wseg, g, pt);
    if (!__any_sync(0xffffffffu, active)) {  // nothing left here for this warp
      ++tried;
      continue;
    }
    tried = 0;
    switch (b.model[wseg]) {
      case kShimizu: split_segment<Shimizu, R, INTEG>(b, wseg, g, active, pt); break;
      case kLorenz: split_segment<Lorenz, R, INTEG>(b, wseg, g, active, pt); break;
      case kRossler: split_segment<Rossler, R, INTEG>(b, wseg, g, active, pt); break;
      case kChua: split_segment<Chua, R, INTEG>(b, wseg, g, active, pt); break;
      default: split_segment<HyperRossler, R, INTEG>(b, wseg, g, active, pt); break;
    }
  }
}

}  // namespace adaptive

int launch_split(int model, int integ, int prec, const AdaptiveArgs &a, int block, int variant,
                 cudaStream_t s) {
  using namespace adaptive;
  if (a.P <= 0) return 0;
  if (block <= 0 || block > kMaxLaneBlock || block % 32) block = 64;
  switch (model) {
    case kShimizu: return launch_split_m<Shimizu>(integ, prec, a, block, variant, s);
    case kLorenz: return launch_split_m<Lorenz>(integ, prec, a, block, variant, s);
    case kRossler: return launch_split_m<Rossler>(integ, prec, a, block, variant, s);
    case kChua: return launch_split_m<Chua>(integ, prec, a, block, variant, s);
    case kHyperRossler: return launch_split_m<HyperRossler>(integ, prec, a, block, variant, s);
    default: return kErrUnsupported;
  }
}

int launch_batch_split(int integ, int prec, const BatchArgs &b, int block, cudaStream_t s,
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
  if (block <= 0 || block > kMaxLaneBlock || block % 32) block = 64;
  void (*kern)(BatchArgs) = nullptr;
  if (integ == kDopri5 && prec == kFP32) kern = batch_split_kernel<float, kDopri5>;
  else if (integ == kDopri5 && prec == kFP64) kern = batch_split_kernel<double, kDopri5>;
  else if (integ == kDverk65 && prec == kFP32) kern = batch_split_kernel<float, kDverk65>;
  else if (integ == kDverk65 && prec == kFP64) kern = batch_split_kernel<double, kDverk65>;
  else return kErrUnsupported;
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, 0);
  const int64_t groups = block / kSplitLanes;
  const int64_t full = (int64_t)std::max(1, per_sm) * sms;
  const int64_t cap = std::max<int64_t>(1, (int64_t)(full * std::min(1.0, std::max(share, 0.0))));
  const int64_t grid = std::min<int64_t>(cap, (total + groups - 1) / groups);
  return (int)launch_with_priority(kern, (unsigned)grid, (unsigned)block, s, high_priority,
                                  with_ctl(b, prec));
}

}  // namespace chaos
