// State trajectories through the adaptive integrators: the reference's
// Dormand-Prince tool dopriStep (cuda/tools/dopri.dp.cpp:7-139) as one lane
// per point.  A caller of that tool starts at time 0 (the first call sets
// facOld = 1e-4 and evaluates k1), and each call makes one accepted step --
// rejected attempts are retried inside the call -- leaving the next step's
// proposal and the FSAL derivative for the following call.  Here one lane
// makes `nsteps` such calls for its point and records, after each, the time,
// the proposal and the state.  The step pass is the sweep kernels' own
// (adaptive.cuh: attempt) and so is the controller, with its arithmetic in
// FP64 for FP64 states (control<..., EXACT>; the sweeps evaluate it in
// FP32), and with the stage combinations in the reference's order y + h
// (sum a k), as in the one-lane sweeps (the four-lane FP64 forms fold h into
// the coefficients instead).  DVERK 6(5) runs the same way with its own
// tableau and exponent.
#pragma once
#include "adaptive.cuh"

namespace chaos {
namespace adaptive {

struct TrajectoryArgs {
  AdaptiveArgs a;   // P, tolerances, h0, hmax, hmin, max_steps, escape, params, inits
  int32_t nsteps;   // accepted steps to record per point
  double *t_out;    // P x nsteps: time after each accepted step
  double *h_out;    // P x nsteps: the step proposal after it
  double *x_out;    // P x nsteps x dim: the state after it
  int32_t *status;  // nullable: P statuses (CHAOS_POINT_* codes)
};

template <class M, class R, int INTEG>
CL_HD void run_trajectory(const TrajectoryArgs &ta, int64_t pt) {
  using C = typename CtlReal<R>::type;
  constexpr int N = M::N, K = M::N;
  const AdaptiveArgs &a = ta.a;
  const Ctl c = make_ctl<R>(a);
  Lane<M, K, R, INTEG> L;
#pragma unroll
  for (int i = 0; i < M::NP; i++) L.p[i] = (R)a.params.base[pt * a.params.ps + i * a.params.cs];
#pragma unroll
  for (int j = 0; j < N; j++) L.x[j] = (R)a.inits.base[pt * a.inits.ps + j * a.inits.cs];
#pragma unroll
  for (int i = 0; i < K; i++)
#pragma unroll
    for (int j = 0; j < N; j++) L.V[i][j] = L.kv[i][j] = R(0);  // not integrated here
  L.h = (R)a.h0;
  L.lfac_old = log2_fac_min<C>();
  L.reject = false;
  L.steps = 0;
  if (INTEG == kDopri5) M::f(L.x, L.kx, L.p);
  double t = 0.0;
  int status = 0, rec = 0;
  const int64_t base = pt * (int64_t)ta.nsteps;
  while (rec < ta.nsteps) {
    if (L.steps >= c.max_steps) {
      status = 3;
      break;
    }
    if (!((double)L.h >= c.hmin)) {
      status = 2;
      break;
    }
    const R h = L.h;
    R x1[N], V1[K][N], kx1[N], kv1[K][N];
    L.steps++;
    // the reference's combination order (HF false): this step sequence is
    // compared with the reference's dopriStep
    const C err2 = attempt<M, K, R, INTEG, false>(L, h, false, ctl_rtol<R>(c), ctl_atol<R>(c),
                                                  x1, V1, kx1, kv1);
    if (!(err2 <= err2_limit<C>())) {  // the sweeps' rule (point_finite)
      if (!point_finite(L.p, L.x)) {
        status = 1;
        break;
      }
      L.h = h / (R)kNonfiniteDiv;
      L.reject = true;
      continue;
    }
    R hnew;
    const bool accepted = control<R, INTEG, true>(err2, h, L.lfac_old, L.reject, c, hnew);
    L.h = hnew;
    if (!accepted) continue;
    bool inside = true;
#pragma unroll
    for (int j = 0; j < N; j++) {
      L.x[j] = x1[j];
      if (INTEG == kDopri5) L.kx[j] = kx1[j];
      inside = inside && (fabs(L.x[j]) <= (R)c.escape);
    }
    t += (double)h;
    ta.t_out[base + rec] = t;
    ta.h_out[base + rec] = (double)hnew;
#pragma unroll
    for (int j = 0; j < N; j++) ta.x_out[(base + rec) * N + j] = (double)L.x[j];
    rec++;
    if (!inside) {
      status = 4;
      break;
    }
  }
  for (int i = rec; i < ta.nsteps; i++) {  // records the point did not reach
    ta.t_out[base + i] = quiet_nan();
    ta.h_out[base + i] = quiet_nan();
#pragma unroll
    for (int j = 0; j < N; j++) ta.x_out[(base + i) * N + j] = quiet_nan();
  }
  if (ta.status) ta.status[pt] = status;
}

}  // namespace adaptive

int launch_trajectory(int model, int integrator, int precision,
                      const adaptive::TrajectoryArgs &ta, cudaStream_t s);

}  // namespace chaos
