// Launch-side declarations shared by the kernel translation units and the
// C-ABI layer.  Plain structs of pointers and scalars; no torch types.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace chaos {

// Strided view of a P x C array of doubles: element (point, comp) lives at
// base[point * ps + comp * cs].  Point-major (the reference's layout,
// tasklyapunov.cpp:47-71) is ps = C, cs = 1; component-major (SoA) is ps = 1,
// cs = P.
struct View {
  double *base;
  int64_t ps, cs;
};
struct CView {
  const double *base;
  int64_t ps, cs;
};

// Reference-exact fixed-step FP64 sweep: cuda/lyapunov.dp.cpp:5-259 (FD, VAR,
// QR) with the DVERK step of cuda/tools/dverk.dp.cpp:7-81.
struct CompatArgs {
  int64_t P;
  int32_t k, method;  // method: 0 FD, 1 VAR, 2 QR
  double eps, step, t_skip, t_skip_clp, calc_time, add_skip;
  CView params;
  View inits;             // advanced in place to the end states
  double *close;          // nullable: P*k*n, the final perturbation / tangent vectors
  View lyap;              // P x k
  int32_t accumulate;     // 1: start each sum from the value already in lyap
  int32_t *status;        // nullable: 0 ok, 1 non-finite spectrum
};

// Tolerances and limits of the adaptive forms in the forms the kernels use
// them (adaptive.cuh: make_ctl).  The launchers fill AdaptiveArgs::ctl, so
// that these loop-invariant values sit in the kernel's parameter space and
// take no registers.
struct Ctl {
  float rtol, atol, tau;  // tau: renormalisation cancellation target
  double rtol64, atol64;  // the tolerances for the FP64 form's error norm
  double hmax, hmin;
  // The step limits as floats, rounded so that a float step compares with
  // them exactly as with the double limits: h >= hmin32 iff h >= hmin
  // (rounded up), h > hmax32 iff h > hmax (rounded down).  The FP32 forms
  // test their steps against these and convert nothing per step.
  float hmin32, hmax32;
  int64_t max_steps;
  double escape;
};

// Adaptive forms (DVERK 6(5) or Dopri5; FP64 or FP32 state and tangent; FP64
// Gram-Schmidt and compensated log-norm sums).
struct AdaptiveArgs {
  int64_t P;
  int32_t k, gs;          // gs: 0 classical, 1 modified Gram-Schmidt
  double rtol, atol, h0, hmax, hmin;
  double t_transient, t_align, t_avg, dt_renorm;
  int64_t max_steps;
  double escape;          // a state component beyond this magnitude ends the point
  CView params;
  CView inits;
  const double *t_avg_per_point;  // nullable: per-point averaging time
  View spectrum;          // P x k
  int32_t *status;        // nullable
  int64_t *steps;         // nullable: attempted steps per point
  // persistent work-queue form
  unsigned long long *queue;  // nullable unless the launch is persistent
  uint64_t queue_stride;      // coprime to P: hand-out order q -> q * stride mod P
  const int32_t *order;       // nullable: hand-out order q -> order[q] (overrides the stride)
  Ctl ctl;                    // set by the launchers from the fields above
};

// Longest-first hand-out order (order.cu): order = a permutation of [0, P)
// by decreasing t_avg (bucketed); scratch holds kOrderScratchBytes.
constexpr int kOrderBuckets = 1024;
constexpr size_t kOrderScratchBytes = 2 * sizeof(unsigned long long) + kOrderBuckets * sizeof(unsigned int);
int launch_order_longest_first(const double *t_avg, int64_t P, int32_t *order, void *scratch,
                               cudaStream_t s);

// A stride for the persistent queue's permutation: a prime that does not
// divide P (so q -> q * stride mod P is a bijection on [0, P)).
inline uint64_t queue_stride_for(int64_t P) {
  if (P <= 1) return 1;
  const uint64_t primes[] = {1000003ULL, 1000033ULL, 1000037ULL, 1000039ULL};
  for (uint64_t s : primes)
    if ((uint64_t)P % s != 0) return s;  // s prime and s does not divide P: gcd = 1
  return 1;
}

enum Integrator : int32_t { kDverkFixed = 0, kDverk65 = 1, kDopri5 = 2 };
enum Precision : int32_t { kCompatFP64 = 0, kFP64 = 1, kFP32 = 2 };

// Returns cudaSuccess or the launch error; kErrUnsupported for a combination
// that has no instantiation.
constexpr int kErrUnsupported = -1;

int launch_compat(int model, const CompatArgs &a, int block, cudaStream_t s);
// variant: 0 = 128-register build, 1 = 96-register build (FP32 only)
int launch_adaptive(int model, int integrator, int precision, const AdaptiveArgs &a, int block,
                    int persistent_blocks, int variant, cudaStream_t s);
int launch_l96_warp(int integrator, int precision, const AdaptiveArgs &a, int warps_per_block,
                    cudaStream_t s);

}  // namespace chaos

namespace chaos {

// Mixed batch: up to kMaxSegments segments (each one model's points, with its
// own arrays and phase times) swept by one persistent launch.  All segments
// share the integrator and precision.
constexpr int kMaxSegments = 8;
struct BatchArgs {
  int32_t nseg;
  int32_t model[kMaxSegments];
  AdaptiveArgs seg[kMaxSegments];  // seg[i].queue is not used; queue_stride is
  unsigned long long *queues;      // nseg point counters, zeroed before the launch
};

// share: fraction (0, 1] of a full machine's resident blocks the persistent
// grid may take; high_priority: launch at the device's greatest stream
// priority (the block scheduler dispatches its pending blocks first when
// another batch kernel runs beside it).
int launch_batch(int integrator, int precision, const BatchArgs &b, int block, cudaStream_t s,
                 double share = 1.0, bool high_priority = false);

// Kernel launch with an optional priority launch attribute (kept by stream
// capture as the graph node's priority).
template <class... Args>
inline cudaError_t launch_with_priority(void (*kern)(Args...), unsigned grid, unsigned block,
                                        cudaStream_t s, bool high_priority, Args... args) {
  if (!high_priority) {
    kern<<<grid, block, 0, s>>>(args...);
    return cudaGetLastError();
  }
  int least = 0, greatest = 0;
  cudaDeviceGetStreamPriorityRange(&least, &greatest);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributePriority;
  attr[0].val.priority = greatest;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, args...);
}

// Split form (split.cu): one point per group of four lanes; variant 1 is the
// exchange layout of the FP64 form for 3-dimensional models.
int launch_split(int model, int integrator, int precision, const AdaptiveArgs &a, int block,
                 int variant, cudaStream_t s);
int launch_batch_split(int integrator, int precision, const BatchArgs &b, int block,
                       cudaStream_t s, double share = 1.0, bool high_priority = false);

}  // namespace chaos

namespace chaos {
// Registry lookup shared by the C ABI translation units: model id, dimension
// and parameter count of a registered name; -1 when unknown.
int model_id_of(const char *name, int *dim, int *nparams);
}  // namespace chaos
