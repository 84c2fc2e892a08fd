// Split form of the adaptive integrator: one parameter point per group of
// kSplitLanes = 4 consecutive lanes of a warp.  Lane r of a group carries the
// state and tangent vector v_r (rows r >= k carry none).
//
// Why: with one lane per point a step is a serial chain of passes over the
// state and all k vectors, so a point's time is its step count times that
// chain.  That bounds a sweep whose points are few (a 64 x 64 map fills a
// tenth of the GPU) or whose run is set by its longest point (a batch with
// per-point averaging times: one stiff point with 10^7 steps).  Split over a
// group, each lane advances only the state and one vector per step (in FP32
// one packed pair pass), so a step's chain is about half as long, at the
// price of computing the state in every lane of the group.
//
// Consistency: every lane of a group computes the state with the same
// operations on the same inputs, so the state, the step size, every accept /
// reject decision and every phase change agree bit for bit across the
// group.  The two quantities that combine the lanes -- the error norm (a sum)
// and the Gram-Schmidt cancellation estimate (a max) -- are butterfly
// reductions (__shfl_xor_sync 1, 2), whose result is the same in all four
// lanes because IEEE addition and max are commutative.  Gram-Schmidt runs in
// k rounds: lane q normalises its vector (all projections on earlier vectors
// already subtracted) and broadcasts it; lanes r > q subtract their
// projection on it, with the coefficient taken against the original vector
// (classical, cuda/tools/linalg.dp.cpp:36-51) or the updated one (modified):
// the same FP64 operations in the same order as the one-lane form.
#pragma once
#include "adaptive.cuh"

namespace chaos {
namespace adaptive {

constexpr int kSplitLanes = 4;

struct Group {
  int r;          // this lane's row (tangent vector index)
  int base;       // lane index of the group's first lane
  unsigned mask;  // the group's four lanes
};
__device__ __forceinline__ Group group_of() {
  const int lane = (int)(threadIdx.x & 31);
  return Group{lane & 3, lane & ~3, 0xFu << (lane & ~3)};
}

template <class T> __device__ __forceinline__ T group_sum(T e, unsigned mask) {
  e += __shfl_xor_sync(mask, e, 1);
  e += __shfl_xor_sync(mask, e, 2);
  return e;
}
__device__ __forceinline__ float group_max(float e, unsigned mask) {
  e = fmaxf(e, __shfl_xor_sync(mask, e, 1));
  e = fmaxf(e, __shfl_xor_sync(mask, e, 2));
  return e;
}

// Exchange layout (XCH, FP64 and 3-dimensional models): lane 0 of the group
// advances the state alone and lane 1 + q tangent vector q; at every stage
// the vector lanes take the state's stage point from lane 0 (three FP64
// shuffles) for their Jacobian.  Each lane then combines 3 rows per stage
// instead of 6: on B200 an FP64 instruction holds its pipe for two cycles, so
// the redundant state rows of the default layout are the longer part of a
// step, while the default layout suits FP32, whose packed FFMA2 advances
// state and vector rows in one instruction.  The state is broadcast to the
// vector lanes after every accepted step (they need it for the Jacobian at
// the start of a tangent phase and after Gram-Schmidt, and for the escape
// and finiteness checks that every lane makes alike).
template <bool XCH> __device__ __forceinline__ int vec_of(const Group &g) {
  return XCH ? g.r - 1 : g.r;  // the tangent vector this lane carries (< 0: none)
}

template <class M>
struct ExchangeStages {
  const double *p;
  unsigned mask;
  int base;
  bool state_lane;
  CL_HD void operator()(int, const double *arg, double *out) const {
    constexpr int N = M::N;
    double X[N];
#pragma unroll
    for (int j = 0; j < N; j++) {
#ifdef __CUDA_ARCH__
      X[j] = __shfl_sync(mask, arg[j], base);
#else
      X[j] = arg[j];
#endif
    }
    if (state_lane) M::f(X, out, p);
    else M::jv(arg, out, p, X);
  }
};

template <class M, class R, int INTEG, bool XCH = false>
struct SplitLane {
  static constexpr int N = M::N;
  R p[M::NP];
  R x[N];         // the state (the same in all lanes of the group)
  R v[N];         // this lane's tangent vector (zero for rows >= k)
  R kx[N], kv[N]; // Dopri5 FSAL derivatives
  R h;
  typename CtlReal<R>::type lfac_old;
  int32_t phase;
  bool reject;
  double t_left;  // time left in the current phase
  R t_left_r;     // the same in the step precision, rounded toward zero
  float t_gs, L, rate_max;
  double prod;    // product of this vector's norms since the last log
  int64_t steps;
};

template <class M, class R, int INTEG, bool XCH>
__device__ __forceinline__ void split_flush(SplitLane<M, R, INTEG, XCH> &L) {
  Cold &c = cold_slot();
  const double y = log(L.prod) - c.comp[0];
  const double s = c.sum[0] + y;
  c.comp[0] = (s - c.sum[0]) - y;
  c.sum[0] = s;
  L.prod = 1.0;
}

template <class M, class R, int INTEG, bool XCH>
__device__ void split_finish(SplitLane<M, R, INTEG, XCH> &L, const AdaptiveArgs &a, const Group &g,
                             int status) {
  const Cold &c = cold_slot();
  const int vi = vec_of<XCH>(g);
  if (vi >= 0 && vi < M::N) {
    split_flush(L);
    const double lam = status ? quiet_nan() : c.sum[0] / c.t_avg;
    a.spectrum.base[c.pt * a.spectrum.ps + vi * a.spectrum.cs] = lam;
  }
  if (g.r == 0) {
    if (a.status) a.status[c.pt] = status;
    if (a.steps) a.steps[c.pt] = L.steps;
  }
}

template <class M, class R, int INTEG, bool XCH>
__device__ __forceinline__ void split_set_phase_time(SplitLane<M, R, INTEG, XCH> &L, double len) {
  L.t_left = len;
  L.t_left_r = time_left_as<R>(len);
}

template <class M, class R, int INTEG, bool XCH>
__device__ void split_start_tangent(SplitLane<M, R, INTEG, XCH> &L, const AdaptiveArgs &a,
                                    const Group &g) {
  constexpr int N = M::N;
#pragma unroll
  for (int j = 0; j < N; j++) {  // rows of no vector stay zero
    const int vi = vec_of<XCH>(g);
    L.v[j] = (vi >= 0 && vi < M::N) ? tangent_init<R>(vi, j) : R(0);
  }
  if (INTEG == kDopri5) M::jv(L.v, L.kv, L.p, L.x);
  L.lfac_old = log2_fac_min<typename CtlReal<R>::type>();
  L.t_gs = 0.f;
  if (a.t_align > 0) {
    L.phase = kAlign;
    split_set_phase_time(L, a.t_align);
  } else {
    L.phase = kAverage;
    split_set_phase_time(L, cold_slot().t_avg);
  }
}

template <class M, class R, int INTEG, bool XCH>
__device__ void split_start(SplitLane<M, R, INTEG, XCH> &L, const AdaptiveArgs &a, int64_t pt,
                            const Group &g) {
  constexpr int N = M::N;
  Cold &cs = cold_slot();
  cs.pt = pt;
  cs.t_avg = a.t_avg_per_point ? a.t_avg_per_point[pt] : a.t_avg;
  cs.sum[0] = cs.comp[0] = 0.0;
#pragma unroll
  for (int i = 0; i < M::NP; i++) L.p[i] = (R)a.params.base[pt * a.params.ps + i * a.params.cs];
#pragma unroll
  for (int i = 0; i < N; i++) L.x[i] = (R)a.inits.base[pt * a.inits.ps + i * a.inits.cs];
#pragma unroll
  for (int j = 0; j < N; j++) L.v[j] = L.kv[j] = R(0);
  L.h = (R)a.h0;
  L.lfac_old = log2_fac_min<typename CtlReal<R>::type>();
  L.reject = false;
  L.steps = 0;
  L.L = (float)a.dt_renorm / kRenormSplitInit;
  L.rate_max = initial_renorm_rate(renorm_spread_limit<R>((float)a.rtol), (float)a.dt_renorm);
  L.prod = 1.0;
  if (INTEG == kDopri5) M::f(L.x, L.kx, L.p);
  if (a.t_transient > 0) {
    L.phase = kTransient;
    split_set_phase_time(L, a.t_transient);
    L.t_gs = 0.f;
  } else {
    split_start_tangent(L, a, g);
  }
}

// One step attempt: the state and this lane's vector; returns the group's
// mean square weighted error (the same in all four lanes).
template <class M, class R, int INTEG, bool XCH>
__device__ typename CtlReal<R>::type split_attempt(const SplitLane<M, R, INTEG, XCH> &st, R h,
                                                   bool joint, bool has_vec, const Group &g,
                                                   typename CtlReal<R>::type rtol,
                                                   typename CtlReal<R>::type atol,
                                                   R (&x1)[M::N], R (&v1)[M::N],
                                                   R (&kx1)[M::N], R (&kv1)[M::N]) {
  using C = typename CtlReal<R>::type;
  constexpr int N = M::N;
  constexpr int S = (INTEG == kDverk65) ? 8 : 7;
  C es = C(0), ev = C(0);
  if constexpr (XCH) {  // this lane's rows: the state (lane 0) or its vector
    static_assert(std::is_same<R, double>::value, "the exchange layout is the FP64 form's");
    const bool state_lane = g.r == 0;
    double yr[N], kr[N], y1r[N], k1r[N];
#pragma unroll
    for (int j = 0; j < N; j++) {
      yr[j] = state_lane ? st.x[j] : st.v[j];
      kr[j] = state_lane ? st.kx[j] : st.kv[j];
    }
    double er = 0.0;
    const ExchangeStages<M> fa{st.p, g.mask, g.base, state_lane};
    // step-scaled combinations (FoldH): the exchange rows are latency-bound
    using FA = decltype(fa);
    if (INTEG == kDverk65) dverk_pass<N, double, FA, true>(yr, h, fa, y1r, er, rtol, atol);
    else dopri_pass<N, double, FA, true>(yr, kr, h, fa, y1r, k1r, er, rtol, atol);
#pragma unroll
    for (int j = 0; j < N; j++) {
      x1[j] = __shfl_sync(g.mask, y1r[j], g.base);
      v1[j] = state_lane ? 0.0 : y1r[j];
      if (INTEG == kDopri5) {
        kx1[j] = state_lane ? k1r[j] : 0.0;
        kv1[j] = state_lane ? 0.0 : k1r[j];
      }
    }
    es = state_lane ? er : C(0);
    ev = state_lane ? C(0) : er;
  } else if constexpr (std::is_same<R, float>::value) {  // (state, v_r) as one packed pass
    float X[S][N];
    float2 ya[N], ka[N], ya1[N], ka1[N];
#pragma unroll
    for (int j = 0; j < N; j++) {
      ya[j] = make_float2(st.x[j], st.v[j]);
      ka[j] = make_float2(st.kx[j], st.kv[j]);
    }
    float2 ea = make_float2(0.f, 0.f);
    PairStateStages<M> fa{st.p, X};
    if (INTEG == kDverk65) dverk_pass<N, float2>(ya, h, fa, ya1, ea, rtol, atol);
    else dopri_pass<N, float2>(ya, ka, h, fa, ya1, ka1, ea, rtol, atol);
#pragma unroll
    for (int j = 0; j < N; j++) {
      x1[j] = ya1[j].x;
      v1[j] = ya1[j].y;
      if (INTEG == kDopri5) {
        kx1[j] = ka1[j].x;
        kv1[j] = ka1[j].y;
      }
    }
    es = ea.x;
    ev = ea.y;
  } else {  // (state, v_r) as one pass over FP64 pairs: the two chains interleave
    double X[S][N];
    double2 ya[N], ka[N], ya1[N], ka1[N];
#pragma unroll
    for (int j = 0; j < N; j++) {
      ya[j] = make_double2(st.x[j], st.v[j]);
      ka[j] = make_double2(st.kx[j], st.kv[j]);
    }
    double2 ea = make_double2(0.0, 0.0);
    PairStateStages64<M> fa{st.p, X};
    if (INTEG == kDverk65) dverk_pass<N, double2>(ya, h, fa, ya1, ea, rtol, atol);
    else dopri_pass<N, double2>(ya, ka, h, fa, ya1, ka1, ea, rtol, atol);
#pragma unroll
    for (int j = 0; j < N; j++) {
      x1[j] = ya1[j].x;
      v1[j] = ya1[j].y;
      if (INTEG == kDopri5) {
        kx1[j] = ka1[j].x;
        kv1[j] = ka1[j].y;
      }
    }
    es = ea.x;
    ev = ea.y;
  }
  // the state's error once (lane 0), each vector's in its own lane; summed
  // over the group in FP32 (it only steers the controller, whose arithmetic
  // is FP32 in the sweeps)
  float e = (float)((g.r == 0 ? es : C(0)) + ((joint && has_vec) ? ev : C(0)));
  e = group_sum(e, g.mask);
  const float inv_nc = joint ? 1.0f / float(N * (1 + M::N)) : 1.0f / float(N);
  return (C)(e * inv_nc);
}

// Gram-Schmidt over the group in FP64 (see the header); false on a
// degenerate basis (the same answer in all four lanes).
template <class M, class R, int INTEG, bool XCH>
__device__ bool split_gram_schmidt(SplitLane<M, R, INTEG, XCH> &L, const AdaptiveArgs &a,
                                   const Ctl &c, const Group &g) {
  constexpr int N = M::N;
  constexpr int k = M::N;  // launches take k == dim
  const int vi = vec_of<XCH>(g);
  const bool has_vec = vi >= 0 && vi < k;
  double vo[N], w[N];
  R before = 0;
#pragma unroll
  for (int j = 0; j < N; j++) {
    vo[j] = (double)L.v[j];
    w[j] = vo[j];
    before = vfma(L.v[j], L.v[j], before);
  }
  double rr = 1.0;
  float cancel = 1.0f;
#pragma unroll
  for (int q = 0; q < k; q++) {
    if (vi == q) {
      double s = 0;
#pragma unroll
      for (int j = 0; j < N; j++) s = fma(w[j], w[j], s);
      const double inv = rsqrt_for<R>(s);
      rr = s * inv;
      const float fi = (float)inv;
      cancel = fmaxf(cancel, (float)before * (fi * fi));
#pragma unroll
      for (int j = 0; j < N; j++) w[j] *= inv;
    }
    double qv[N];
#pragma unroll
    for (int j = 0; j < N; j++) qv[j] = __shfl_sync(g.mask, w[j], g.base + q + (XCH ? 1 : 0));
    if (vi > q) {
      double cq = 0;
      if (a.gs == 1) {  // modified: against the updated vector
#pragma unroll
        for (int j = 0; j < N; j++) cq = fma(qv[j], w[j], cq);
      } else {  // classical: against the original vector
#pragma unroll
        for (int j = 0; j < N; j++) cq = fma(qv[j], vo[j], cq);
      }
#pragma unroll
      for (int j = 0; j < N; j++) w[j] = fma(-cq, qv[j], w[j]);
    }
  }
  const bool ok_own = !has_vec || ((rr > 0.0) && (rr < 1e300));
  if (!__all_sync(g.mask, ok_own)) return false;
#pragma unroll
  for (int j = 0; j < N; j++) L.v[j] = has_vec ? (R)w[j] : R(0);
  cancel = group_max(cancel, g.mask);
  float rmin = has_vec ? (float)fmin(rr, 1.0) : 1.0f;  // steers the interval only
  rmin = fminf(rmin, __shfl_xor_sync(g.mask, rmin, 1));
  rmin = fminf(rmin, __shfl_xor_sync(g.mask, rmin, 2));
  if (L.phase == kAverage && has_vec) {
    L.prod *= rr;
    if (!(L.prod < 1e150 && L.prod > 1e-150)) split_flush(L);
  }
  if (L.t_gs > 0.f)  // the interval rule of the one-lane form, on the group's extremes
    next_renorm_interval(L.L, L.rate_max, cancel, rmin, L.t_gs, c.tau, (float)a.dt_renorm);
  L.t_gs = 0.f;
  if (INTEG == kDopri5) M::jv(L.v, L.kv, L.p, L.x);
  return true;
}

// One step attempt of the group, phase bookkeeping included (the one-lane
// form's lane_step, with the group's error norm and Gram-Schmidt).
template <class M, class R, int INTEG, bool XCH>
__device__ int split_step(SplitLane<M, R, INTEG, XCH> &L, const AdaptiveArgs &a, const Ctl &c,
                          const Group &g) {
  using C = typename CtlReal<R>::type;
  constexpr int N = M::N;
  if (L.steps == 0 && !state_inside(L.x, c.escape)) {
    split_finish(L, a, g, 4);
    return kFinished;
  }
  if (L.steps >= c.max_steps) {
    split_finish(L, a, g, 3);
    return kFinished;
  }
  if (!step_at_least_hmin(L.h, c)) {
    split_finish(L, a, g, 2);
    return kFinished;
  }
  const bool clamped = L.h >= L.t_left_r;  // as the one-lane form
  const R h = clamped ? L.t_left_r : L.h;
  const bool joint = L.phase != kTransient;
  const int vi = vec_of<XCH>(g);
  const bool has_vec = vi >= 0 && vi < M::N;  // launches take k == dim
  R x1[N], v1[N], kx1[N], kv1[N];
  L.steps++;
  const C err2 = split_attempt<M, R, INTEG>(L, h, joint, has_vec, g, ctl_rtol<R>(c),
                                            ctl_atol<R>(c), x1, v1, kx1, kv1);
  if (!(err2 <= err2_limit<C>())) {  // the one-lane form's rule (point_finite)
    if (!point_finite(L.p, L.x)) {
      split_finish(L, a, g, 1);
      return kFinished;
    }
    L.h = h / (R)kNonfiniteDiv;
    L.reject = true;
    return kRunning;
  }
  R hnew;
  if (control<R, INTEG>(err2, h, L.lfac_old, L.reject, c, hnew)) {
#pragma unroll
    for (int j = 0; j < N; j++) {
      L.x[j] = x1[j];
      if (INTEG == kDopri5) L.kx[j] = kx1[j];
    }
    if (joint) {
#pragma unroll
      for (int j = 0; j < N; j++) {
        L.v[j] = v1[j];
        if (INTEG == kDopri5) L.kv[j] = kv1[j];
      }
    }
    if (!clamped || hnew < h) L.h = hnew;
    if (!clamped) {
      L.t_left -= (double)h;
      L.t_left_r = time_left_as<R>(L.t_left);
    }
    L.t_gs += (float)h;
    if (!state_inside(L.x, c.escape)) {
      split_finish(L, a, g, 4);
      return kFinished;
    }
    if (clamped) {
      if (L.phase == kTransient) {
        split_start_tangent(L, a, g);
      } else if (L.phase == kAlign) {
        if (!split_gram_schmidt(L, a, c, g)) {
          split_finish(L, a, g, 1);
          return kFinished;
        }
        L.phase = kAverage;
        split_set_phase_time(L, cold_slot().t_avg);
      } else {
        const bool ok = split_gram_schmidt(L, a, c, g);
        split_finish(L, a, g, ok ? 0 : 1);
        return kFinished;
      }
    }
  } else {
    L.h = hnew;
  }
  return kRunning;
}

}  // namespace adaptive
}  // namespace chaos
