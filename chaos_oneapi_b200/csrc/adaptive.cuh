// Adaptive per-point integrator for 3-4-dimensional flows: the state and its
// k tangent vectors under DVERK 6(5) or Dormand-Prince 5(4), one thread per
// parameter point, everything in registers.
//
//  * Tableaux: DVERK a-rows and 6th-order weights of cuda/tools/dverk.dp.cpp
//    :13-41 with the 5th-order weights of Verner's DVERK 6(5) pair for the
//    error estimate; Dopri5 of cuda/tools/dopri.dp.cpp:14-44 (FSAL).
//  * Step-size control: cuda/tools/dopri.dp.cpp:9-12,46-138 (safety 0.9,
//    fac1 0.2, fac2 10, beta 0.04, exponent 1/q - 0.75 beta, error = RMS of
//    e / (atol + rtol max(|y0|,|y1|)), reject / retry), evaluated in FP32
//    (it only steers the step length).
//  * Variational equations are integrated jointly with the state: within one
//    step the state is advanced first and its stage points X_s are kept, then
//    each tangent vector runs the same stages with J(X_s).  This is the same
//    arithmetic as one RK step of the joint (n + k n)-dimensional system, with
//    a register footprint of one vector's stages instead of all of them.
//  * Renormalisation at every multiple of dt_renorm (steps are clamped to
//    land on it), each interval split per point into as many equal parts as
//    the spread of the tangent directions needs (see run_point): Gram-Schmidt
//    (classical as cuda/tools/linalg.dp.cpp:36-51, or modified) in FP64
//    whatever the state precision, log-norms summed in FP64 with Kahan
//    compensation.
#pragma once
#include "kernels.h"
#include "models.cuh"

namespace chaos {
namespace adaptive {

// ---------------------------------------------------------------- tableaux
struct DV {  // DVERK (Verner 6(5)); c = {0, 1/6, 4/15, 2/3, 5/6, 1, 1/15, 1}
  static constexpr double a21 = 1. / 6.;
  static constexpr double a31 = 4. / 75., a32 = 16. / 75.;
  static constexpr double a41 = 5. / 6., a42 = -8. / 3., a43 = 5. / 2.;
  static constexpr double a51 = -165. / 64., a52 = 55. / 6., a53 = -425. / 64., a54 = 85. / 96.;
  static constexpr double a61 = 12. / 5., a62 = -8., a63 = 4015. / 612., a64 = -11. / 36., a65 = 88. / 255.;
  static constexpr double a71 = -8263. / 15000., a72 = 124. / 75., a73 = -643. / 680., a74 = -81. / 250.,
                          a75 = 2484. / 10625.;
  static constexpr double a81 = 3501. / 1720., a82 = -300. / 43., a83 = 297275. / 52632.,
                          a84 = -319. / 2322., a85 = 24068. / 84065., a87 = 3850. / 26703.;
  static constexpr double b1 = 3. / 40., b3 = 875. / 2244., b4 = 23. / 72., b5 = 264. / 1955.,
                          b7 = 125. / 11592., b8 = 43. / 616.;
  // d = b(6th) - b(5th), b(5th) = {13/160, 0, 2375/5984, 5/16, 12/85, 3/44, 0, 0}
  static constexpr double d1 = 3. / 40. - 13. / 160., d3 = 875. / 2244. - 2375. / 5984.,
                          d4 = 23. / 72. - 5. / 16., d5 = 264. / 1955. - 12. / 85., d6 = -3. / 44.,
                          d7 = 125. / 11592., d8 = 43. / 616.;
};

struct DP {  // Dormand-Prince 5(4), FSAL
  static constexpr double a21 = 0.2;
  static constexpr double a31 = 3. / 40., a32 = 9. / 40.;
  static constexpr double a41 = 44. / 45., a42 = -56. / 15., a43 = 32. / 9.;
  static constexpr double a51 = 19372. / 6561., a52 = -25360. / 2187., a53 = 64448. / 6561.,
                          a54 = -212. / 729.;
  static constexpr double a61 = 9017. / 3168., a62 = -355. / 33., a63 = 46732. / 5247.,
                          a64 = 49. / 176., a65 = -5103. / 18656.;
  static constexpr double a71 = 35. / 384., a73 = 500. / 1113., a74 = 125. / 192.,
                          a75 = -2187. / 6784., a76 = 11. / 84.;
  static constexpr double e1 = 71. / 57600., e3 = -71. / 16695., e4 = 71. / 1920.,
                          e5 = -17253. / 339200., e6 = 22. / 525., e7 = -1. / 40.;
};

template <class R> CL_HD R C(double v) { return R(v); }

CL_HD float fast_log2f(float x) {
#ifdef __CUDA_ARCH__
  return __log2f(x);
#else
  return log2f(x);
#endif
}
CL_HD double quiet_nan() {
#ifdef __CUDA_ARCH__
  return __longlong_as_double(0x7ff8000000000000ULL);
#else
  return __builtin_nan("");
#endif
}

// Error weight contribution of one component (the error norm only steers the
// step length, so an approximate reciprocal is enough).
CL_HD float fast_div(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fdividef(a, b);
#else
  return a / b;
#endif
}
template <class R>
CL_HD float err_term(R y0, R y1, R e, float rtol, float atol) {
  const float m = fmaxf(fabsf((float)y0), fabsf((float)y1));
  const float r = fast_div((float)e, fmaf(rtol, m, atol));
  return r * r;
}

// One DVERK 6(5) pass over an N-vector y: y1 = 6th-order solution, err2 +=
// sum of squared weighted error components.  fn(s, arg, out) evaluates the
// derivative of stage s (0-based) at arg.
template <int N, class R, class F>
CL_HD void dverk_pass(const R *y, R h, const F &fn, R *y1, float &err2,
                                           float rtol, float atol) {
  R k1[N], k2[N], k3[N], k4[N], k5[N], k7[N], arg[N], acc[N], e[N];
  using T = DV;
  fn(0, y, k1);
#pragma unroll
  for (int j = 0; j < N; j++) arg[j] = y[j] + h * (C<R>(T::a21) * k1[j]);
  fn(1, arg, k2);
#pragma unroll
  for (int j = 0; j < N; j++) arg[j] = y[j] + h * (C<R>(T::a31) * k1[j] + C<R>(T::a32) * k2[j]);
  fn(2, arg, k3);
#pragma unroll
  for (int j = 0; j < N; j++)
    arg[j] = y[j] + h * (C<R>(T::a41) * k1[j] + C<R>(T::a42) * k2[j] + C<R>(T::a43) * k3[j]);
  fn(3, arg, k4);
#pragma unroll
  for (int j = 0; j < N; j++)
    arg[j] = y[j] + h * (C<R>(T::a51) * k1[j] + C<R>(T::a52) * k2[j] + C<R>(T::a53) * k3[j] +
                         C<R>(T::a54) * k4[j]);
  fn(4, arg, k5);
#pragma unroll
  for (int j = 0; j < N; j++) {
    arg[j] = y[j] + h * (C<R>(T::a61) * k1[j] + C<R>(T::a62) * k2[j] + C<R>(T::a63) * k3[j] +
                         C<R>(T::a64) * k4[j] + C<R>(T::a65) * k5[j]);
    acc[j] = C<R>(T::b1) * k1[j] + C<R>(T::b3) * k3[j] + C<R>(T::b4) * k4[j] + C<R>(T::b5) * k5[j];
    e[j] = C<R>(T::d1) * k1[j] + C<R>(T::d3) * k3[j] + C<R>(T::d4) * k4[j] + C<R>(T::d5) * k5[j];
  }
  {
    R k6[N];
    fn(5, arg, k6);
#pragma unroll
    for (int j = 0; j < N; j++) e[j] += C<R>(T::d6) * k6[j];
  }
#pragma unroll
  for (int j = 0; j < N; j++)
    arg[j] = y[j] + h * (C<R>(T::a71) * k1[j] + C<R>(T::a72) * k2[j] + C<R>(T::a73) * k3[j] +
                         C<R>(T::a74) * k4[j] + C<R>(T::a75) * k5[j]);
  fn(6, arg, k7);
#pragma unroll
  for (int j = 0; j < N; j++) {
    arg[j] = y[j] + h * (C<R>(T::a81) * k1[j] + C<R>(T::a82) * k2[j] + C<R>(T::a83) * k3[j] +
                         C<R>(T::a84) * k4[j] + C<R>(T::a85) * k5[j] + C<R>(T::a87) * k7[j]);
    acc[j] += C<R>(T::b7) * k7[j];
    e[j] += C<R>(T::d7) * k7[j];
  }
  {
    R k8[N];
    fn(7, arg, k8);
#pragma unroll
    for (int j = 0; j < N; j++) {
      acc[j] += C<R>(T::b8) * k8[j];
      e[j] += C<R>(T::d8) * k8[j];
      y1[j] = y[j] + h * acc[j];
      err2 += err_term<R>(y[j], y1[j], h * e[j], rtol, atol);
    }
  }
}

// One Dopri5 pass: k1 = derivative at y (FSAL, given), y1 = 5th-order
// solution, k7 = derivative at y1 (the next step's k1).
template <int N, class R, class F>
CL_HD void dopri_pass(const R *y, const R *k1, R h, const F &fn, R *y1, R *k7,
                                           float &err2, float rtol, float atol) {
  R k2[N], k3[N], k4[N], k5[N], arg[N], e[N];
  using T = DP;
#pragma unroll
  for (int j = 0; j < N; j++) arg[j] = y[j] + h * (C<R>(T::a21) * k1[j]);
  fn(1, arg, k2);
#pragma unroll
  for (int j = 0; j < N; j++) arg[j] = y[j] + h * (C<R>(T::a31) * k1[j] + C<R>(T::a32) * k2[j]);
  fn(2, arg, k3);
#pragma unroll
  for (int j = 0; j < N; j++)
    arg[j] = y[j] + h * (C<R>(T::a41) * k1[j] + C<R>(T::a42) * k2[j] + C<R>(T::a43) * k3[j]);
  fn(3, arg, k4);
#pragma unroll
  for (int j = 0; j < N; j++)
    arg[j] = y[j] + h * (C<R>(T::a51) * k1[j] + C<R>(T::a52) * k2[j] + C<R>(T::a53) * k3[j] +
                         C<R>(T::a54) * k4[j]);
  fn(4, arg, k5);
#pragma unroll
  for (int j = 0; j < N; j++) {
    arg[j] = y[j] + h * (C<R>(T::a61) * k1[j] + C<R>(T::a62) * k2[j] + C<R>(T::a63) * k3[j] +
                         C<R>(T::a64) * k4[j] + C<R>(T::a65) * k5[j]);
    e[j] = C<R>(T::e1) * k1[j] + C<R>(T::e3) * k3[j] + C<R>(T::e4) * k4[j] + C<R>(T::e5) * k5[j];
    y1[j] = C<R>(T::a71) * k1[j] + C<R>(T::a73) * k3[j] + C<R>(T::a74) * k4[j] + C<R>(T::a75) * k5[j];
  }
  {
    R k6[N];
    fn(5, arg, k6);
#pragma unroll
    for (int j = 0; j < N; j++) {
      y1[j] = y[j] + h * (y1[j] + C<R>(T::a76) * k6[j]);
      e[j] += C<R>(T::e6) * k6[j];
    }
  }
  fn(6, y1, k7);
#pragma unroll
  for (int j = 0; j < N; j++) {
    e[j] += C<R>(T::e7) * k7[j];
    err2 += err_term<R>(y[j], y1[j], h * e[j], rtol, atol);
  }
}

// Per-point integrator state.
template <class M, int K, class R, int INTEG>
struct PointState {
  static constexpr int N = M::N;
  static constexpr int S = (INTEG == kDverk65) ? 8 : 7;
  R p[M::NP];
  R x[N];
  R V[K][N];
  R kx[N];      // Dopri5 FSAL: derivative of the state
  R kv[K][N];   // Dopri5 FSAL: derivatives of the tangent vectors
  R h;
  float fac_old;
  int64_t steps;
};

// Stage evaluators for the state pass (records stage points) and the tangent
// passes (J at the recorded stage points).
template <class M, class R, int S>
struct StateStages {
  const R *p;
  R (*X)[M::N];  // X[s] for s >= 1; stage 0 is the current state
  CL_HD void operator()(int s, const R *arg, R *out) const {
    if (s > 0) {
#pragma unroll
      for (int j = 0; j < M::N; j++) X[s][j] = arg[j];
    }
    M::f(arg, out, p);
  }
};
template <class M, class R, int S>
struct TangentStages {
  const R *p;
  const R *x0;
  const R (*X)[M::N];
  CL_HD void operator()(int s, const R *arg, R *out) const {
    M::jv(arg, out, p, s == 0 ? x0 : X[s]);
  }
};

// Attempt one step of length h.  JOINT: also advance the tangent vectors.
// On return x1/V1 (and, for Dopri5, kx1/kv1) hold the candidate; err is the
// RMS weighted error over all integrated components.
template <class M, int K, class R, int INTEG, bool JOINT>
CL_HD float attempt(PointState<M, K, R, INTEG> &st, R h, float rtol, float atol,
                                         R (&x1)[M::N], R (&V1)[K][M::N], R (&kx1)[M::N],
                                         R (&kv1)[K][M::N]) {
  constexpr int N = M::N;
  constexpr int S = PointState<M, K, R, INTEG>::S;
  R X[S][N];
  float err2 = 0.f;
  StateStages<M, R, S> fs{st.p, X};
  if (INTEG == kDverk65) {
    dverk_pass<N, R>(st.x, h, fs, x1, err2, rtol, atol);
  } else {
    dopri_pass<N, R>(st.x, st.kx, h, fs, x1, kx1, err2, rtol, atol);
  }
  if (JOINT) {
    if (INTEG == kDopri5) {
#pragma unroll
      for (int j = 0; j < N; j++) X[6][j] = x1[j];
    }
    TangentStages<M, R, S> ft{st.p, st.x, X};
#pragma unroll
    for (int i = 0; i < K; i++) {
      if (INTEG == kDverk65) dverk_pass<N, R>(st.V[i], h, ft, V1[i], err2, rtol, atol);
      else dopri_pass<N, R>(st.V[i], st.kv[i], h, ft, V1[i], kv1[i], err2, rtol, atol);
    }
  }
  constexpr int NC = JOINT ? N * (1 + K) : N;
  return sqrtf(err2 * (1.0f / NC));  // err2 >= 0
}

struct Ctl {
  float rtol, atol;
  double hmax, hmin;
  int64_t max_steps;
  double escape;
};

// Integrates exactly `len` time units.  Returns 0 or a status code
// (1 non-finite, 2 step underflow, 3 step budget exhausted, 4 escaped: a
// state component left the ball of radius c.escape).
template <class M, int K, class R, int INTEG, bool JOINT>
CL_HD int integrate(PointState<M, K, R, INTEG> &st, double len, const Ctl &c) {
  constexpr int N = M::N;
  constexpr float safe = 0.9f, beta = 0.04f, facc1 = 5.0f, facc2 = 0.1f;
  constexpr float expo1 = (INTEG == kDverk65 ? 1.0f / 6.0f : 0.2f) - beta * 0.75f;
  double t = 0.0;
  bool reject = false;
  if (INTEG == kDopri5) {
    M::f(st.x, st.kx, st.p);
    if (JOINT) {
#pragma unroll
      for (int i = 0; i < K; i++) M::jv(st.V[i], st.kv[i], st.p, st.x);
    }
  }
  while (t < len) {
    if (st.steps >= c.max_steps) return 3;
    if (!((double)st.h >= c.hmin)) return 2;  // also catches h == 0 and NaN
    const double remaining = len - t;
    const bool clamped = (double)st.h >= remaining;
    const R h = clamped ? (R)remaining : st.h;
    R x1[N], V1[K][N], kx1[N], kv1[K][N];
    st.steps++;
    const float err = attempt<M, K, R, INTEG, JOINT>(st, h, c.rtol, c.atol, x1, V1, kx1, kv1);
    if (!(err == err) || err > 3.0e38f) return 1;
    const float fac11 = exp2f(expo1 * fast_log2f(fmaxf(err, 1e-30f)));
    float fac = fac11 * exp2f(-beta * fast_log2f(st.fac_old));
    fac = fmaxf(facc2, fminf(facc1, fac * (1.0f / safe)));
    R hnew = h * (R)fast_div(1.0f, fac);
    if (err <= 1.0f) {
      st.fac_old = fmaxf(err, 1e-4f);
#pragma unroll
      for (int j = 0; j < N; j++) {
        st.x[j] = x1[j];
        if (INTEG == kDopri5) st.kx[j] = kx1[j];
      }
      if (JOINT) {
#pragma unroll
        for (int i = 0; i < K; i++)
#pragma unroll
          for (int j = 0; j < N; j++) {
            st.V[i][j] = V1[i][j];
            if (INTEG == kDopri5) st.kv[i][j] = kv1[i][j];
          }
      }
      if ((double)hnew > c.hmax) hnew = (R)c.hmax;
      if (reject && hnew > h) hnew = h;
      reject = false;
      t = clamped ? len : t + (double)h;
      if (!clamped || hnew < h) st.h = hnew;
      bool inside = true;
#pragma unroll
      for (int j = 0; j < N; j++) inside = inside && (fabs(st.x[j]) <= (R)c.escape);
      if (!inside) return 4;
    } else {
      st.h = h * (R)fast_div(1.0f, fminf(facc1, fac11 * (1.0f / safe)));
      reject = true;
    }
  }
  return 0;
}

// Gram-Schmidt in FP64 on the k tangent vectors; r[i] = norms before scaling.
template <int N, int K, class R>
CL_HD void renormalise(R (&V)[K][N], double (&r)[K], int gs) {
  double v[K][N];
#pragma unroll
  for (int i = 0; i < K; i++)
#pragma unroll
    for (int j = 0; j < N; j++) v[i][j] = (double)V[i][j];
#pragma unroll
  for (int i = 0; i < K; i++) {
    if (gs == 1) {  // modified
#pragma unroll
      for (int q = 0; q < i; q++) {
        double c = 0;
#pragma unroll
        for (int j = 0; j < N; j++) c = fma(v[q][j], v[i][j], c);
#pragma unroll
        for (int j = 0; j < N; j++) v[i][j] = fma(-c, v[q][j], v[i][j]);
      }
    } else {  // classical: all projections against the original v_i
      double cq[K];
#pragma unroll
      for (int q = 0; q < i; q++) {
        double c = 0;
#pragma unroll
        for (int j = 0; j < N; j++) c = fma(v[q][j], v[i][j], c);
        cq[q] = c;
      }
#pragma unroll
      for (int q = 0; q < i; q++)
#pragma unroll
        for (int j = 0; j < N; j++) v[i][j] = fma(-cq[q], v[q][j], v[i][j]);
    }
    double s = 0;
#pragma unroll
    for (int j = 0; j < N; j++) s = fma(v[i][j], v[i][j], s);
    r[i] = sqrt(s);
    const double inv = 1.0 / r[i];
#pragma unroll
    for (int j = 0; j < N; j++) v[i][j] *= inv;
  }
#pragma unroll
  for (int i = 0; i < K; i++)
#pragma unroll
    for (int j = 0; j < N; j++) V[i][j] = (R)v[i][j];
}

constexpr int kRenormSubInit = 16, kRenormSubMax = 64;

// Largest log-norm spread allowed within one renormalisation sub-interval:
// 0.3 ln(1 / max(rtol, unit roundoff of R)).
template <class R> CL_HD float renorm_spread_limit(float rtol) {
  const float ulp = sizeof(R) == 4 ? 5.96e-8f : 1.2e-16f;
  return 0.3f * logf(1.0f / fmaxf(rtol, ulp));
}

// Whole per-point computation.  Returns the status code.
template <class M, int K, class R, int INTEG>
CL_HD int run_point(const AdaptiveArgs &a, int64_t pt) {
  constexpr int N = M::N;
  PointState<M, K, R, INTEG> st;
#pragma unroll
  for (int i = 0; i < M::NP; i++) st.p[i] = (R)a.params.base[pt * a.params.ps + i * a.params.cs];
#pragma unroll
  for (int i = 0; i < N; i++) st.x[i] = (R)a.inits.base[pt * a.inits.ps + i * a.inits.cs];
  st.h = (R)a.h0;
  st.fac_old = 1e-4f;
  st.steps = 0;
  // A step below 1e-12 (model time units) is never meaningful here; it also
  // stops a point whose controller collapsed the step to zero.
  const Ctl c{(float)a.rtol, (float)a.atol, a.hmax > 0 ? a.hmax : 1e300, fmax(a.hmin, 1e-12),
              a.max_steps, a.escape > 0 ? a.escape : 1e4};
  const double t_avg = a.t_avg_per_point ? a.t_avg_per_point[pt] : a.t_avg;

  int status = 0;
  if (a.t_transient > 0) status = integrate<M, K, R, INTEG, false>(st, a.t_transient, c);
#pragma unroll
  for (int i = 0; i < K; i++)
#pragma unroll
    for (int j = 0; j < N; j++) st.V[i][j] = (i == j) ? R(1) : R(0);
  st.fac_old = 1e-4f;

  double sum[K], comp[K];
#pragma unroll
  for (int i = 0; i < K; i++) sum[i] = comp[i] = 0.0;
  const double total = a.t_align + t_avg;
  const double eps_t = 1e-12 * total;
  // Renormalisation sub-intervals.  The exponent estimate is the same for any
  // renormalisation schedule (the R factors of successive Gram-Schmidt steps
  // multiply to the R factor of the whole interval), but the weakest tangent
  // direction is only resolved while its share of each tangent vector stays
  // above the integration error.  So each dt_renorm interval is split into m
  // equal parts, and m adapts per point to the spread of log-norms seen in one
  // part: doubled when it exceeds tau, halved when below tau / 4.
  const float tau = renorm_spread_limit<R>(c.rtol);
  int m = kRenormSubInit;
  double t = 0.0;
  while (status == 0 && t < total) {
    double len = a.dt_renorm;
    if (t + len > total) len = total - t;
    const double sub = len / m;
    float max_spread = 0.f;
    for (int j = 0; j < m; j++) {
      const double l = (j == m - 1) ? len - sub * (m - 1) : sub;
      status = integrate<M, K, R, INTEG, true>(st, l, c);
      if (status) break;
      double r[K];
      renormalise<N, K, R>(st.V, r, a.gs);
      bool ok = true;
#pragma unroll
      for (int i = 0; i < K; i++) ok = ok && (r[i] > 0.0) && (r[i] < 1e300);
      if (!ok) {
        status = 1;
        break;
      }
      double lg[K];
      double lmax = -1e300, lmin = 1e300;
#pragma unroll
      for (int i = 0; i < K; i++) {
        lg[i] = log(r[i]);
        lmax = fmax(lmax, lg[i]);
        lmin = fmin(lmin, lg[i]);
      }
      max_spread = fmaxf(max_spread, (float)(lmax - lmin));
      if (t + sub * (j + 1) > a.t_align + eps_t) {
#pragma unroll
        for (int i = 0; i < K; i++) {  // Kahan-compensated sum of log-norms
          const double y = lg[i] - comp[i];
          const double s2 = sum[i] + y;
          comp[i] = (s2 - sum[i]) - y;
          sum[i] = s2;
        }
      }
    }
    t += len;
    if (max_spread > tau && m < kRenormSubMax) m *= 2;
    else if (max_spread < 0.25f * tau && m > 1) m /= 2;
  }
#pragma unroll
  for (int i = 0; i < K; i++) {
    const double lam = status ? quiet_nan() : sum[i] / t_avg;
    a.spectrum.base[pt * a.spectrum.ps + i * a.spectrum.cs] = lam;
  }
  if (a.status) a.status[pt] = status;
  if (a.steps) a.steps[pt] = st.steps;
  return status;
}

}  // namespace adaptive
}  // namespace chaos
