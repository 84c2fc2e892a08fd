// Test infrastructure only: one Runge-Kutta pass of the adaptive kernels
// (chaos_oneapi_b200/csrc/adaptive.cuh: dverk_pass / dopri_pass) with the
// stage combinations in the reference's order y + h (sum a k) (HF false) and
// step-scaled, y + sum (h a) k (HF true), on the same inputs: single FP64
// rows, FP64 pairs (state, tangent vector) and packed FP32 pairs.  Both
// orders are the same method, so the new state and the error norm must agree
// to rounding; a coefficient mapped to the wrong stage in one of the two
// forms shows up as a difference of the size of the step's increment.
// Built by tests/test_host_lane.py with nvcc; never linked into the library.
//
//   fold_driver SEED N
// Prints per case: integrator element model dy derr errnorm
//   dy: largest |y1(HF) - y1(ref)| / max |y1(ref)|
//   derr: |sqrt(err2(HF)) - sqrt(err2(ref))| / sqrt(err2(ref))
//   errnorm: sqrt(err2(ref))
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>

#include "../../chaos_oneapi_b200/csrc/adaptive.cuh"

using namespace chaos;
using namespace chaos::adaptive;

static double comp(double v, int) { return v; }
static double comp(double2 v, int i) { return i ? v.y : v.x; }
static double comp(float2 v, int i) { return i ? v.y : v.x; }
static double sum_err(double e) { return e; }
static double sum_err(double2 e) { return e.x + e.y; }
static double sum_err(float2 e) { return (double)e.x + (double)e.y; }
template <class E> static E make(double a, double b);
template <> double make<double>(double a, double) { return a; }
template <> double2 make<double2>(double a, double b) { return make_double2(a, b); }
template <> float2 make<float2>(double a, double b) { return make_float2((float)a, (float)b); }
template <class E> static int width() { return 2; }  // pairs
template <> int width<double>() { return 1; }

// stage evaluator per element type: the state alone, or (state, vector)
template <class M, class E> struct Stages;
template <class M> struct Stages<M, double> {
  using type = StateStages<M, double>;
  static type make_fn(const double *p, double (*X)[M::N]) { return type{p, X}; }
};
template <class M> struct Stages<M, double2> {
  using type = PairStateStages64<M>;
  static type make_fn(const double *p, double (*X)[M::N]) { return type{p, X}; }
};
template <class M> struct Stages<M, float2> {
  using type = PairStateStages<M>;
  static type make_fn(const float *p, float (*X)[M::N]) { return type{p, X}; }
};

template <class M, class E, bool DVERK>
static void one(std::mt19937_64 &rng, const double *pd, const char *integ, const char *elem,
                const char *model, double h_in) {
  using S = typename ScalarOf<E>::type;
  using C = typename CtlReal<S>::type;
  constexpr int N = M::N;
  std::normal_distribution<double> g(0.0, 1.0);
  S p[M::NP];
  for (int i = 0; i < M::NP; i++) p[i] = (S)pd[i];
  E y[N], k1[N];
  double xs[N], vs[N];
  for (int j = 0; j < N; j++) {
    xs[j] = 5.0 * g(rng);
    vs[j] = g(rng);
    y[j] = make<E>(xs[j], vs[j]);
  }
  S X[8][N];
  auto fn = Stages<M, E>::make_fn(p, X);
  fn(0, y, k1);
  const S h = (S)h_in;
  const C rtol = (C)1e-6, atol = (C)1e-6;
  E y1a[N], y1b[N], k7a[N], k7b[N];
  typename ErrAcc<E>::type ea{}, eb{};
  if (DVERK) {
    dverk_pass<N, E, decltype(fn), false>(y, h, fn, y1a, ea, rtol, atol);
    dverk_pass<N, E, decltype(fn), true>(y, h, fn, y1b, eb, rtol, atol);
  } else {
    dopri_pass<N, E, decltype(fn), false>(y, k1, h, fn, y1a, k7a, ea, rtol, atol);
    dopri_pass<N, E, decltype(fn), true>(y, k1, h, fn, y1b, k7b, eb, rtol, atol);
  }
  double dy = 0.0, ymax = 0.0;
  for (int j = 0; j < N; j++)
    for (int w = 0; w < width<E>(); w++) {
      dy = std::max(dy, std::fabs(comp(y1b[j], w) - comp(y1a[j], w)));
      ymax = std::max(ymax, std::fabs(comp(y1a[j], w)));
    }
  const double na = std::sqrt(sum_err(ea)), nb = std::sqrt(sum_err(eb));
  printf("%s %s %s %.3e %.3e %.3e\n", integ, elem, model, dy / ymax, std::fabs(nb - na) / na, na);
}

template <class M, class E>
static void both(std::mt19937_64 &rng, const double *p, const char *elem, const char *model,
                 double h) {
  one<M, E, true>(rng, p, "dverk65", elem, model, h);
  one<M, E, false>(rng, p, "dopri5", elem, model, h);
}

int main(int argc, char **argv) {
  const unsigned seed = argc > 1 ? (unsigned)atoi(argv[1]) : 1u;
  const int n = argc > 2 ? atoi(argv[2]) : 20;
  std::mt19937_64 rng(seed);
  const double lorenz[3] = {10.0, 28.0, 8.0 / 3.0}, rossler[3] = {0.2, 0.2, 5.7};
  for (int i = 0; i < n; i++) {
    // steps whose error estimate is of order one, so that its rounding is
    // small against it in either precision
    const double hl = 0.02 + 0.03 * (i % 3), hr = 0.2 + 0.2 * (i % 3);
    both<Lorenz, double>(rng, lorenz, "fp64", "lorenz", hl);
    both<Lorenz, double2>(rng, lorenz, "fp64pair", "lorenz", hl);
    both<Lorenz, float2>(rng, lorenz, "fp32pair", "lorenz", hl);
    both<Rossler, double>(rng, rossler, "fp64", "rossler", hr);
    both<Rossler, double2>(rng, rossler, "fp64pair", "rossler", hr);
    both<Rossler, float2>(rng, rossler, "fp32pair", "rossler", hr);
  }
  return 0;
}
