// Adaptive per-point integrator for 3-4-dimensional flows: the state and its
// k tangent vectors under DVERK 6(5) or Dormand-Prince 5(4), one thread per
// parameter point, everything in registers.
//
//  * Tableaux: DVERK a-rows and 6th-order weights of cuda/tools/dverk.dp.cpp
//    :13-41 with the 5th-order weights of Verner's DVERK 6(5) pair for the
//    error estimate; Dopri5 of cuda/tools/dopri.dp.cpp:14-44 (FSAL).
//  * Step-size control: cuda/tools/dopri.dp.cpp:9-12,46-138 (safety 0.9,
//    fac1 0.2, fac2 10, beta 0.04, exponent 1/q - 0.75 beta, error = RMS of
//    e / (atol + rtol max(|y0|,|y1|)), reject / retry).  The FP64 form
//    evaluates the error norm and the controller in FP64, so that its step
//    sequence follows the reference's dopriStep to rounding; the FP32 form in
//    FP32 with fast reciprocals (there it only steers the step length).
//  * Variational equations are integrated jointly with the state: within one
//    step the state is advanced first and its stage points X_s are kept, then
//    each tangent vector runs the same stages with J(X_s).  This is the same
//    arithmetic as one RK step of the joint (n + k n)-dimensional system, with
//    a register footprint of one vector's stages instead of all of them.
//  * Renormalisation (see Lane): Gram-Schmidt (classical as
//    cuda/tools/linalg.dp.cpp:36-51, or modified) in FP64 whatever the state
//    precision, at intervals of at most dt_renorm and exactly at the phase
//    ends; norms multiplied and log-norms summed in FP64 with Kahan
//    compensation.
#pragma once
#include <type_traits>

#include "kernels.h"
#include "models.cuh"
#include "renorm.cuh"

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

CL_HD double quiet_nan() {
#ifdef __CUDA_ARCH__
  return __longlong_as_double(0x7ff8000000000000ULL);
#else
  return __builtin_nan("");
#endif
}

// ------------------------------------------------- element arithmetic
// The RK passes below are written over an element type E: float or double
// (one row of the joint system per pass), or float2 (two rows side by side,
// advanced by the packed FP32 instructions of sm_100: one FFMA2 performs the
// multiply-add of both rows).  Coefficients and h are scalars of type S.
// Every stage combination is an explicit chain mul, fma, fma, ... so the
// scalar and packed forms do the same operations in the same order.
// double2 pairs two FP64 rows the same way (two scalar FMAs per coefficient:
// FP64 has no packed form, but the two rows' dependency chains interleave in
// one pass, which halves the latency a lane waits on per stage).
template <class E> struct ScalarOf { using type = E; };
template <> struct ScalarOf<float2> { using type = float; };
template <> struct ScalarOf<double2> { using type = double; };

CL_HD float vmul(float a, float b) { return a * b; }
CL_HD double vmul(double a, double b) { return a * b; }
CL_HD float vfma(float a, float b, float c) { return fmaf(a, b, c); }
CL_HD double vfma(double a, double b, double c) { return fma(a, b, c); }
CL_HD float2 vmul(float a, float2 b) {
#ifdef __CUDA_ARCH__
  return __fmul2_rn(make_float2(a, a), b);
#else
  return make_float2(a * b.x, a * b.y);
#endif
}
CL_HD float2 vfma(float a, float2 b, float2 c) {
#ifdef __CUDA_ARCH__
  return __ffma2_rn(make_float2(a, a), b, c);
#else
  return make_float2(fmaf(a, b.x, c.x), fmaf(a, b.y, c.y));
#endif
}
CL_HD float2 vmul2(float2 a, float2 b) {
#ifdef __CUDA_ARCH__
  return __fmul2_rn(a, b);
#else
  return make_float2(a.x * b.x, a.y * b.y);
#endif
}
CL_HD float2 vfma2(float2 a, float2 b, float2 c) {
#ifdef __CUDA_ARCH__
  return __ffma2_rn(a, b, c);
#else
  return make_float2(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y));
#endif
}

CL_HD double2 vmul(double a, double2 b) { return make_double2(a * b.x, a * b.y); }
CL_HD double2 vfma(double a, double2 b, double2 c) {
  return make_double2(fma(a, b.x, c.x), fma(a, b.y, c.y));
}

// lin(c1, k1, c2, k2, ...) = c1 k1 + c2 k2 + ... (left to right)
template <class S, class E> CL_HD E lin_acc(E acc) { return acc; }
// (arguments by value: the coefficients are constexpr members, which device
// code may read but not bind to a reference)
template <class S, class E, class... Rest>
CL_HD E lin_acc(E acc, double c, E k, Rest... rest) {
  return lin_acc<S, E>(vfma(S(c), k, acc), rest...);
}
// FP64 pairs serve the latency-bound forms (a few points, each a long serial
// chain of steps): their combinations run as two interleaved chains -- the
// odd and the even terms -- added at the end, one instruction more for about
// half the dependency depth.
CL_HD double2 lin2_acc(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
template <class... Rest>
CL_HD double2 lin2_acc(double2 a, double2 b, double c, double2 k, Rest... rest) {
  return lin2_acc(b, vfma(c, k, a), rest...);  // alternate the two chains
}
template <class... Rest>
CL_HD double2 lin2_pair(double c1, double2 k1, double c2, double2 k2, Rest... rest) {
  return lin2_acc(vmul(c2, k2), vmul(c1, k1), rest...);
}
template <class S, class E, class... Rest>
CL_HD E lin(double c, E k, Rest... rest) {
  if constexpr (std::is_same<E, double2>::value && sizeof...(Rest) >= 2) {
    return lin2_pair(c, k, rest...);
  } else {
    return lin_acc<S, E>(vmul(S(c), k), rest...);
  }
}

// Step-scaled combinations: acc + (h c1) k1 + (h c2) k2 + ... (left to
// right), one multiply-add per term.  The products h c are formed once per
// pass (scalars, shared by every row), so a stage argument y + h sum a k
// costs one instruction per term instead of one more for the final h, and
// its last term -- the derivative just computed -- is one dependent
// multiply-add away from the argument instead of two.
template <class S, class E> CL_HD E linh(S, E acc) { return acc; }
template <class S, class E, class... Rest>
CL_HD E linh(S h, E acc, double c, E k, Rest... rest) {
  return linh<S, E>(h, vfma(h * S(c), k, acc), rest...);
}
// The same without a starting value: (h c1) k1 + (h c2) k2 + ...
template <class S, class E, class... Rest>
CL_HD E linh0(S h, double c, E k, Rest... rest) {
  return linh<S, E>(h, vmul(h * S(c), k), rest...);
}
// Which element types combine their stages step-scaled (FoldH) rather than
// as y + h (sum a k), the reference's order (cuda/tools/dopri.dp.cpp:54-63).
// Only the FP64 pairs of the four-lane form (and its exchange rows, which
// ask for it explicitly) fold: they are latency-bound, and each stage of
// their serial chain loses one dependent FP64 operation (7 % on the 64^2
// map).  Single FP64 rows -- the one-lane FP64 sweep, bound by FP64
// throughput, which would form the products once per row pass -- measured
// 2.6 % slower folded.  FP32 rows keep the reference's order as well: folded
// they were 1 % faster, but the product h a rounded to FP32 at every step
// moved one of the sensitive Rossler cells held at the full horizon from
// within twice the FP64 method's error to 5x it.  The trajectory kernel,
// whose step sequence is compared with the reference's, never folds.
template <class E> struct FoldH { static constexpr bool value = false; };
template <> struct FoldH<double2> { static constexpr bool value = true; };

// Arithmetic of the error norm and the step-size controller: FP32 for the
// FP32 form, FP64 for the FP64 form.
template <class R> struct CtlReal { using type = float; };
template <> struct CtlReal<double> { using type = double; };

// Squared weighted error e / (atol + rtol max(|y0|, |y1|)) accumulated per
// row: a float accumulator for a scalar FP32 row, a float2 for a packed pair,
// a double for an FP64 row.
template <class E> struct ErrAcc { using type = float; };
template <> struct ErrAcc<float2> { using type = float2; };
template <> struct ErrAcc<double> { using type = double; };
template <> struct ErrAcc<double2> { using type = double2; };

CL_HD void err_acc(float y0, float y1, float e, float rtol, float atol, float &acc) {
  const float m = fmaxf(fabsf(y0), fabsf(y1));
  const float r = fast_div(e, fmaf(rtol, m, atol));
  acc = fmaf(r, r, acc);
}
// The pair shares one reciprocal: 1 / (s_x s_y) scaled by the other weight.
CL_HD void err_acc(float2 y0, float2 y1, float2 e, float rtol, float atol, float2 &acc) {
  const float sx = fmaf(rtol, fmaxf(fabsf(y0.x), fabsf(y1.x)), atol);
  const float sy = fmaf(rtol, fmaxf(fabsf(y0.y), fabsf(y1.y)), atol);
  const float inv = fast_div(1.0f, sx * sy);
  const float2 r = vmul2(e, make_float2(sy * inv, sx * inv));
  acc = vfma2(r, r, acc);
}
CL_HD double recip(double x) {
#ifdef __CUDA_ARCH__
  return __drcp_rn(x);
#else
  return 1.0 / x;
#endif
}
// Error terms of one row of N components; he = h e, the scaled error vector.
// FP64 rows take their components in pairs sharing one correctly rounded
// reciprocal of the product of their weights (a few ulp from the e / s of the
// reference's division).
template <int N, class E, class T, class A>
CL_HD void err_row(const E *y0, const E *y1, const E *he, T rtol, T atol, A &acc) {
  if constexpr (std::is_same<E, double>::value) {
#pragma unroll
    for (int j = 0; j + 1 < N; j += 2) {
      const double sx = fma(rtol, fmax(fabs(y0[j]), fabs(y1[j])), atol);
      const double sy = fma(rtol, fmax(fabs(y0[j + 1]), fabs(y1[j + 1])), atol);
      const double inv = recip(sx * sy);
      const double rx = he[j] * (sy * inv), ry = he[j + 1] * (sx * inv);
      acc = fma(rx, rx, acc);
      acc = fma(ry, ry, acc);
    }
    if (N % 2) {
      const double sk = fma(rtol, fmax(fabs(y0[N - 1]), fabs(y1[N - 1])), atol);
      const double r = he[N - 1] * recip(sk);
      acc = fma(r, r, acc);
    }
  } else if constexpr (std::is_same<E, double2>::value) {
    // a pair of FP64 rows: component j of both rows shares the reciprocal
#pragma unroll
    for (int j = 0; j < N; j++) {
      const double sx = fma(rtol, fmax(fabs(y0[j].x), fabs(y1[j].x)), atol);
      const double sy = fma(rtol, fmax(fabs(y0[j].y), fabs(y1[j].y)), atol);
      const double inv = recip(sx * sy);
      const double rx = he[j].x * (sy * inv), ry = he[j].y * (sx * inv);
      acc.x = fma(rx, rx, acc.x);
      acc.y = fma(ry, ry, acc.y);
    }
  } else {
#pragma unroll
    for (int j = 0; j < N; j++) err_acc(y0[j], y1[j], he[j], rtol, atol, acc);
  }
}

// One DVERK 6(5) pass over an N-vector y of elements E: y1 = 6th-order
// solution, err2 += squared weighted error components.  fn(s, arg, out)
// evaluates the derivative of stage s (0-based) at arg.
template <int N, class E, class F, bool HF = FoldH<E>::value>
CL_HD void dverk_pass(const E *y, typename ScalarOf<E>::type h, const F &fn, E *y1,
                      typename ErrAcc<E>::type &err2,
                      typename CtlReal<typename ScalarOf<E>::type>::type rtol,
                      typename CtlReal<typename ScalarOf<E>::type>::type atol) {
  using S = typename ScalarOf<E>::type;
  using T = DV;
  if constexpr (HF) {
    E k1[N], k2[N], k3[N], k4[N], k5[N], k7[N], arg[N], acc[N], e[N];
    fn(0, y, k1);
#pragma unroll
    for (int j = 0; j < N; j++) arg[j] = linh<S>(h, y[j], T::a21, k1[j]);
    fn(1, arg, k2);
#pragma unroll
    for (int j = 0; j < N; j++) arg[j] = linh<S>(h, y[j], T::a31, k1[j], T::a32, k2[j]);
    fn(2, arg, k3);
#pragma unroll
    for (int j = 0; j < N; j++)
      arg[j] = linh<S>(h, y[j], T::a41, k1[j], T::a42, k2[j], T::a43, k3[j]);
    fn(3, arg, k4);
#pragma unroll
    for (int j = 0; j < N; j++)
      arg[j] = linh<S>(h, y[j], T::a51, k1[j], T::a52, k2[j], T::a53, k3[j], T::a54, k4[j]);
    fn(4, arg, k5);
#pragma unroll
    for (int j = 0; j < N; j++) {
      arg[j] = linh<S>(h, y[j], T::a61, k1[j], T::a62, k2[j], T::a63, k3[j], T::a64, k4[j],
                       T::a65, k5[j]);
      acc[j] = linh<S>(h, y[j], T::b1, k1[j], T::b3, k3[j], T::b4, k4[j], T::b5, k5[j]);
      e[j] = linh0<S>(h, T::d1, k1[j], T::d3, k3[j], T::d4, k4[j], T::d5, k5[j]);
    }
    {
      E k6[N];
      fn(5, arg, k6);
#pragma unroll
      for (int j = 0; j < N; j++) e[j] = linh<S>(h, e[j], T::d6, k6[j]);
    }
#pragma unroll
    for (int j = 0; j < N; j++)
      arg[j] = linh<S>(h, y[j], T::a71, k1[j], T::a72, k2[j], T::a73, k3[j], T::a74, k4[j],
                       T::a75, k5[j]);
    fn(6, arg, k7);
#pragma unroll
    for (int j = 0; j < N; j++) {
      arg[j] = linh<S>(h, y[j], T::a81, k1[j], T::a82, k2[j], T::a83, k3[j], T::a84, k4[j],
                       T::a85, k5[j], T::a87, k7[j]);
      acc[j] = linh<S>(h, acc[j], T::b7, k7[j]);
      e[j] = linh<S>(h, e[j], T::d7, k7[j]);
    }
    {
      E k8[N];
      fn(7, arg, k8);
#pragma unroll
      for (int j = 0; j < N; j++) {
        y1[j] = linh<S>(h, acc[j], T::b8, k8[j]);
        e[j] = linh<S>(h, e[j], T::d8, k8[j]);
      }
    }
    err_row<N>(y, y1, e, rtol, atol, err2);
  } else {
    E k1[N], k2[N], k3[N], k4[N], k5[N], k7[N], arg[N], acc[N], e[N];
    fn(0, y, k1);
#pragma unroll
    for (int j = 0; j < N; j++) arg[j] = vfma(h, lin<S>(T::a21, k1[j]), y[j]);
    fn(1, arg, k2);
#pragma unroll
    for (int j = 0; j < N; j++) arg[j] = vfma(h, lin<S>(T::a31, k1[j], T::a32, k2[j]), y[j]);
    fn(2, arg, k3);
#pragma unroll
    for (int j = 0; j < N; j++)
      arg[j] = vfma(h, lin<S>(T::a41, k1[j], T::a42, k2[j], T::a43, k3[j]), y[j]);
    fn(3, arg, k4);
#pragma unroll
    for (int j = 0; j < N; j++)
      arg[j] = vfma(h, lin<S>(T::a51, k1[j], T::a52, k2[j], T::a53, k3[j], T::a54, k4[j]), y[j]);
    fn(4, arg, k5);
#pragma unroll
    for (int j = 0; j < N; j++) {
      arg[j] = vfma(h, lin<S>(T::a61, k1[j], T::a62, k2[j], T::a63, k3[j], T::a64, k4[j],
                              T::a65, k5[j]), y[j]);
      acc[j] = lin<S>(T::b1, k1[j], T::b3, k3[j], T::b4, k4[j], T::b5, k5[j]);
      e[j] = lin<S>(T::d1, k1[j], T::d3, k3[j], T::d4, k4[j], T::d5, k5[j]);
    }
    {
      E k6[N];
      fn(5, arg, k6);
#pragma unroll
      for (int j = 0; j < N; j++) e[j] = vfma(S(T::d6), k6[j], e[j]);
    }
#pragma unroll
    for (int j = 0; j < N; j++)
      arg[j] = vfma(h, lin<S>(T::a71, k1[j], T::a72, k2[j], T::a73, k3[j], T::a74, k4[j],
                              T::a75, k5[j]), y[j]);
    fn(6, arg, k7);
#pragma unroll
    for (int j = 0; j < N; j++) {
      arg[j] = vfma(h, lin<S>(T::a81, k1[j], T::a82, k2[j], T::a83, k3[j], T::a84, k4[j],
                              T::a85, k5[j], T::a87, k7[j]), y[j]);
      acc[j] = vfma(S(T::b7), k7[j], acc[j]);
      e[j] = vfma(S(T::d7), k7[j], e[j]);
    }
    {
      E k8[N];
      fn(7, arg, k8);
#pragma unroll
      for (int j = 0; j < N; j++) {
        acc[j] = vfma(S(T::b8), k8[j], acc[j]);
        e[j] = vmul(h, vfma(S(T::d8), k8[j], e[j]));
        y1[j] = vfma(h, acc[j], y[j]);
      }
    }
    err_row<N>(y, y1, e, rtol, atol, err2);
  }
}

// One Dopri5 pass: k1 = derivative at y (FSAL, given), y1 = 5th-order
// solution, k7 = derivative at y1 (the next step's k1).
template <int N, class E, class F, bool HF = FoldH<E>::value>
CL_HD void dopri_pass(const E *y, const E *k1, typename ScalarOf<E>::type h, const F &fn,
                      E *y1, E *k7, typename ErrAcc<E>::type &err2,
                      typename CtlReal<typename ScalarOf<E>::type>::type rtol,
                      typename CtlReal<typename ScalarOf<E>::type>::type atol) {
  using S = typename ScalarOf<E>::type;
  using T = DP;
  if constexpr (HF) {
    E k2[N], k3[N], k4[N], k5[N], arg[N], e[N];
#pragma unroll
    for (int j = 0; j < N; j++) arg[j] = linh<S>(h, y[j], T::a21, k1[j]);
    fn(1, arg, k2);
#pragma unroll
    for (int j = 0; j < N; j++) arg[j] = linh<S>(h, y[j], T::a31, k1[j], T::a32, k2[j]);
    fn(2, arg, k3);
#pragma unroll
    for (int j = 0; j < N; j++)
      arg[j] = linh<S>(h, y[j], T::a41, k1[j], T::a42, k2[j], T::a43, k3[j]);
    fn(3, arg, k4);
#pragma unroll
    for (int j = 0; j < N; j++)
      arg[j] = linh<S>(h, y[j], T::a51, k1[j], T::a52, k2[j], T::a53, k3[j], T::a54, k4[j]);
    fn(4, arg, k5);
#pragma unroll
    for (int j = 0; j < N; j++) {
      arg[j] = linh<S>(h, y[j], T::a61, k1[j], T::a62, k2[j], T::a63, k3[j], T::a64, k4[j],
                       T::a65, k5[j]);
      e[j] = linh0<S>(h, T::e1, k1[j], T::e3, k3[j], T::e4, k4[j], T::e5, k5[j]);
      y1[j] = linh<S>(h, y[j], T::a71, k1[j], T::a73, k3[j], T::a74, k4[j], T::a75, k5[j]);
    }
    {
      E k6[N];
      fn(5, arg, k6);
#pragma unroll
      for (int j = 0; j < N; j++) {
        y1[j] = linh<S>(h, y1[j], T::a76, k6[j]);
        e[j] = linh<S>(h, e[j], T::e6, k6[j]);
      }
    }
    fn(6, y1, k7);
#pragma unroll
    for (int j = 0; j < N; j++) e[j] = linh<S>(h, e[j], T::e7, k7[j]);
    err_row<N>(y, y1, e, rtol, atol, err2);
  } else {
    E k2[N], k3[N], k4[N], k5[N], arg[N], e[N];
#pragma unroll
    for (int j = 0; j < N; j++) arg[j] = vfma(h, lin<S>(T::a21, k1[j]), y[j]);
    fn(1, arg, k2);
#pragma unroll
    for (int j = 0; j < N; j++) arg[j] = vfma(h, lin<S>(T::a31, k1[j], T::a32, k2[j]), y[j]);
    fn(2, arg, k3);
#pragma unroll
    for (int j = 0; j < N; j++)
      arg[j] = vfma(h, lin<S>(T::a41, k1[j], T::a42, k2[j], T::a43, k3[j]), y[j]);
    fn(3, arg, k4);
#pragma unroll
    for (int j = 0; j < N; j++)
      arg[j] = vfma(h, lin<S>(T::a51, k1[j], T::a52, k2[j], T::a53, k3[j], T::a54, k4[j]), y[j]);
    fn(4, arg, k5);
#pragma unroll
    for (int j = 0; j < N; j++) {
      arg[j] = vfma(h, lin<S>(T::a61, k1[j], T::a62, k2[j], T::a63, k3[j], T::a64, k4[j],
                              T::a65, k5[j]), y[j]);
      e[j] = lin<S>(T::e1, k1[j], T::e3, k3[j], T::e4, k4[j], T::e5, k5[j]);
      y1[j] = lin<S>(T::a71, k1[j], T::a73, k3[j], T::a74, k4[j], T::a75, k5[j]);
    }
    {
      E k6[N];
      fn(5, arg, k6);
#pragma unroll
      for (int j = 0; j < N; j++) {
        y1[j] = vfma(h, vfma(S(T::a76), k6[j], y1[j]), y[j]);
        e[j] = vfma(S(T::e6), k6[j], e[j]);
      }
    }
    fn(6, y1, k7);
#pragma unroll
    for (int j = 0; j < N; j++) e[j] = vmul(h, vfma(S(T::e7), k7[j], e[j]));
    err_row<N>(y, y1, e, rtol, atol, err2);
  }
}

// Stage evaluators for the state pass (records stage points) and the tangent
// passes (J at the recorded stage points).
template <class M, class R>
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
template <class M, class R>
struct TangentStages {
  const R *p;
  const R *x0;
  const R (*X)[M::N];
  CL_HD void operator()(int s, const R *arg, R *out) const {
    M::jv(arg, out, p, s == 0 ? x0 : X[s]);
  }
};

enum Phase : int32_t { kTransient = 0, kAlign = 1, kAverage = 2 };
enum LaneResult : int32_t { kRunning = 0, kFinished = 1 };


// log2 of the floor of the previous step's error (dopri.dp.cpp:65-68: 1e-4),
// the controller's state at the start of an integration.
template <class C> CL_HD C log2_fac_min() { return C(-13.287712379549449); }

// Largest log of the Gram-Schmidt cancellation factor (|v_i| / r_i) allowed
// between two renormalisations: 0.3 ln(1 / max(rtol, unit roundoff of R)).
template <class R> CL_HD float renorm_spread_limit(float rtol) {
  const float ulp = sizeof(R) == 4 ? 5.96e-8f : 1.2e-16f;
  return 0.3f * logf(1.0f / fmaxf(rtol, ulp));
}

template <class R> CL_HD typename CtlReal<R>::type ctl_rtol(const Ctl &c) { return c.rtol; }
template <> CL_HD double ctl_rtol<double>(const Ctl &c) { return c.rtol64; }
template <class R> CL_HD typename CtlReal<R>::type ctl_atol(const Ctl &c) { return c.atol; }
template <> CL_HD double ctl_atol<double>(const Ctl &c) { return c.atol64; }

// Float nearest to x in the direction of +inf / -inf / zero.
CL_HD float float_ru(double x) {
#ifdef __CUDA_ARCH__
  return __double2float_ru(x);
#else
  float f = (float)x;
  return (double)f < x ? nextafterf(f, INFINITY) : f;
#endif
}
CL_HD float float_rd(double x) {
#ifdef __CUDA_ARCH__
  return __double2float_rd(x);
#else
  float f = (float)x;
  return (double)f > x ? nextafterf(f, -INFINITY) : f;
#endif
}
CL_HD float float_rz(double x) { return x >= 0.0 ? float_rd(x) : float_ru(x); }

// h >= hmin and h > hmax for a step of either precision.
CL_HD bool step_at_least_hmin(float h, const Ctl &c) { return h >= c.hmin32; }
CL_HD bool step_at_least_hmin(double h, const Ctl &c) { return h >= c.hmin; }
CL_HD bool step_above_hmax(float h, const Ctl &c) { return h > c.hmax32; }
CL_HD bool step_above_hmax(double h, const Ctl &c) { return h > c.hmax; }

// Time left in a phase as the step precision, never above the exact time
// left (rounded toward zero), so that a step no longer than it never
// passes the phase end.
template <class R> CL_HD R time_left_as(double t) { return (R)t; }
template <> CL_HD float time_left_as<float>(double t) { return float_rz(t); }

// Controller arithmetic of either precision: base-2 logarithm and power.
CL_HD float ctl_log2(float x) { return fast_log2f(x); }
CL_HD double ctl_log2(double x) { return log2(x); }
CL_HD float ctl_exp2(float x) { return exp2f(x); }
CL_HD double ctl_exp2(double x) { return exp2(x); }
CL_HD float ctl_fma(float a, float b, float c) { return fmaf(a, b, c); }
CL_HD double ctl_fma(double a, double b, double c) { return fma(a, b, c); }

// Largest error mean square that counts as finite.
template <class C> CL_HD C err2_limit() { return sizeof(C) == 4 ? C(3.4e38f) : C(1e300); }

// An attempt whose error estimate is not finite.  From a finite point this
// is an overflow: a step far beyond the stability bound, which the
// controller proposes after a run of steps whose error vanished (a state
// resting on a stable equilibrium, where FP32 rounds the derivative to
// zero, lets the proposal grow by 5x per step).  The reference's controller
// meets an infinite error with its largest reduction,
// newStep = step / min(facc1, fac11 / safeFac) = step / 5
// (cuda/tools/dopri.dp.cpp:134), and so does this one, for NaN as well: the
// attempt is rejected with h / 5.  A point whose parameters or state are not
// finite is not an overflow and ends with status 1.
constexpr int kNonfiniteDiv = 5;

// Every state component within the escape radius (status 4 otherwise: after
// an accepted step, and for the initial state before the first attempt).
template <class R, int N> CL_HD bool state_inside(const R (&x)[N], double escape) {
  bool inside = true;
#pragma unroll
  for (int j = 0; j < N; j++) inside = inside && (fabs(x[j]) <= (R)escape);
  return inside;
}
template <class R, int NP, int N>
CL_HD bool point_finite(const R (&p)[NP], const R (&x)[N]) {
  bool ok = true;  // v - v is 0 for finite v, NaN for Inf and NaN
#pragma unroll
  for (int i = 0; i < NP; i++) ok = ok && (p[i] - p[i] == R(0));
#pragma unroll
  for (int j = 0; j < N; j++) ok = ok && (x[j] - x[j] == R(0));
  return ok;
}

// The step-size controller of dopri.dp.cpp:46-138 after an attempted step of
// length h with error mean square err2, in the log2 domain: with
// l = log2 err, the reference's fac = err^expo1 facOld^-beta / safe clamped
// to [facc2, facc1] = [0.1, 5] is lf = expo1 l - beta l_old - log2 safe
// clamped to [log2 0.1, log2 5], and h_new = h 2^-lf.  Accepted (err <= 1):
// returns true, hnew = the next proposal (at most hmax; after a rejection no
// longer than h), lfac_old = max(l, log2 1e-4).  Rejected: returns false,
// hnew = h / min(facc1, err^expo1 / safe).  R the state precision.
// EXACT: the arithmetic in the error norm's precision (FP64 for FP64
// states), so that a state trajectory's step sequence follows the
// reference's dopriStep to rounding (trajectory.cuh).  Otherwise -- the
// sweeps -- in FP32 with the hardware log2 / exp2: the controller only
// picks the next step's length, and on B200 the FP64 form's log2 / exp2
// chain was a fifth of a step's latency where a step is latency-bound.
template <class R, int INTEG, bool EXACT = false>
CL_HD bool control(typename CtlReal<R>::type err2_in, R h, typename CtlReal<R>::type &lfac_old,
                   bool &reject, const Ctl &c, R &hnew) {
  using C = typename CtlReal<R>::type;
  using T = typename std::conditional<EXACT, C, float>::type;
  constexpr T beta = T(0.04);
  constexpr T expo1 = (INTEG == kDverk65 ? T(1.0 / 6.0) : T(0.2)) - beta * T(0.75);
  constexpr T log2_safe = T(-0.15200309344504995);   // log2 0.9
  constexpr T log2_facc1 = T(2.321928094887362);     // log2 5
  constexpr T log2_facc2 = T(-3.321928094887362);    // log2 0.1
  const T err2 = (T)err2_in;  // beyond FP32's range: +inf, rejected with h / 5 below
  const T lerr = T(0.5) * ctl_log2(err2 > T(1e-38f) ? err2 : T(1e-38f));
  if (err2 <= T(1)) {
    T lf = ctl_fma(expo1, lerr, ctl_fma(-beta, (T)lfac_old, -log2_safe));
    lf = lf < log2_facc2 ? log2_facc2 : lf;
    lf = lf < log2_facc1 ? lf : log2_facc1;
    R hn = h * (R)ctl_exp2(-lf);
    lfac_old = (C)(lerr > log2_fac_min<T>() ? lerr : log2_fac_min<T>());
    if (step_above_hmax(hn, c)) hn = (R)c.hmax;
    if (reject && hn > h) hn = h;
    reject = false;
    hnew = hn;
    return true;
  }
  T lr = ctl_fma(expo1, lerr, -log2_safe);
  lr = lr < log2_facc1 ? lr : log2_facc1;
  hnew = h * (R)ctl_exp2(-lr);
  reject = true;
  return false;
}

// The whole integration state of one parameter point, owned by one lane.
//
// Phases: transient (state only) over t_transient; alignment (state +
// tangent, renormalised, not accumulated) over t_align; averaging over t_avg.
// Steps are clamped to land exactly on each phase end.  Between phase ends,
// Gram-Schmidt runs whenever the time since the last one reaches the point's
// interval L (<= dt_renorm), and -- in the device kernel -- whenever any lane
// of the warp runs it, so that the whole warp renormalises in one pass
// instead of one lane at a time.  The exponent estimate does not depend on
// when renormalisations happen (the R factors of successive Gram-Schmidt steps
// multiply to the R factor over the whole window); L only keeps the weakest
// tangent direction above the integration error: errors in a tangent vector
// are relative to its length, and Gram-Schmidt keeps only the part of it not
// along the earlier vectors, so they grow by the cancellation factor
// |v_i| / r_i.  L adapts so that the log of that factor over one interval, at
// the largest recent rate, stays near tau / 4, and the norms shrink by at
// most e^2 over one interval (renorm.cuh).
template <class M, int K, class R, int INTEG>
struct Lane {
  static constexpr int N = M::N;
  R p[M::NP];
  R x[N];
  R V[K][N];
  R kx[N];      // Dopri5 FSAL: derivative of the state
  R kv[K][N];   // Dopri5 FSAL: derivatives of the tangent vectors
  R h;
  typename CtlReal<R>::type lfac_old;  // log2 of the previous accepted step's error (>= log2 1e-4)
  int32_t phase;
  bool reject;
  double t_left;  // time left in the current phase
  R t_left_r;     // the same in the step precision, rounded toward zero
  float t_gs, L;  // time since the last Gram-Schmidt, its target
  float rate_max; // largest recent log-cancellation per unit time
  int64_t steps;
};

// The part of a lane's state that a step does not touch -- the products of
// the norms (touched at renormalisations), the compensated log-norm sums
// (read at the rare flushes of those products), the averaging time and the
// point index (read at phase ends) -- lives in a per-thread slot of shared
// memory instead of registers, which leaves the registers to the step
// itself.  Blocks have at most kMaxLaneBlock threads.
constexpr int kMaxLaneBlock = 128;
struct Cold {
  double prod[4];          // product of the norms since the last log (k <= 4)
  double sum[4], comp[4];  // Kahan-compensated sums of log-norms
  double t_avg;
  int64_t pt;
};
#ifdef __CUDA_ARCH__
static __shared__ Cold g_cold[kMaxLaneBlock];
#endif
CL_HD Cold &cold_slot() {
#ifdef __CUDA_ARCH__
  return g_cold[threadIdx.x];
#else
  static thread_local Cold c;  // host form: one lane per thread
  return c;
#endif
}

// Packed FP32 form: the rows of the joint system -- the state and the k
// tangent vectors -- advance two at a time as float2 pairs.  Odd k:
// (state, v_{k-1}) in one pass, which also records the stage points, then
// (v_0, v_1), (v_2, v_3), ... at those stage points.  Even k: the state alone
// (recording the stage points), then the same vector pairs.  Each stage
// combination of two rows is then one packed multiply-add per coefficient
// instead of two.
template <class M, int K, class R>
struct Packed {
  static constexpr bool value = std::is_same<R, float>::value && K >= 2;
  static constexpr bool state_paired = (K % 2 == 1);
};

// (state, one tangent vector) as FP64 pairs: the state's stage point is
// recorded and the vector's derivative taken at it, in the same pass.
template <class M>
struct PairStateStages64 {
  const double *p;
  double (*X)[M::N];
  CL_HD void operator()(int s, const double2 *arg, double2 *out) const {
    constexpr int N = M::N;
    double ax[N], av[N], ox[N], ov[N];
#pragma unroll
    for (int j = 0; j < N; j++) {
      ax[j] = arg[j].x;
      av[j] = arg[j].y;
    }
    if (s > 0) {
#pragma unroll
      for (int j = 0; j < N; j++) X[s][j] = ax[j];
    }
    M::f(ax, ox, p);
    M::jv(av, ov, p, ax);
#pragma unroll
    for (int j = 0; j < N; j++) out[j] = make_double2(ox[j], ov[j]);
  }
};

template <class M>
struct PairStateStages {  // (state, last tangent vector)
  const float *p;
  float (*X)[M::N];
  CL_HD void operator()(int s, const float2 *arg, float2 *out) const {
    constexpr int N = M::N;
    float ax[N], av[N], ox[N], ov[N];
#pragma unroll
    for (int j = 0; j < N; j++) {
      ax[j] = arg[j].x;
      av[j] = arg[j].y;
    }
    if (s > 0) {
#pragma unroll
      for (int j = 0; j < N; j++) X[s][j] = ax[j];
    }
    M::f(ax, ox, p);
    M::jv(av, ov, p, ax);
#pragma unroll
    for (int j = 0; j < N; j++) out[j] = make_float2(ox[j], ov[j]);
  }
};
template <class M>
struct PairTangentStages {  // two tangent vectors at the recorded stage points
  const float *p;
  const float *x0;
  const float (*X)[M::N];
  CL_HD void operator()(int s, const float2 *arg, float2 *out) const {
    constexpr int N = M::N;
    const float *xs = s == 0 ? x0 : X[s];
    float a0[N], a1[N], o0[N], o1[N];
#pragma unroll
    for (int j = 0; j < N; j++) {
      a0[j] = arg[j].x;
      a1[j] = arg[j].y;
    }
    M::jv(a0, o0, p, xs);
    M::jv(a1, o1, p, xs);
#pragma unroll
    for (int j = 0; j < N; j++) out[j] = make_float2(o0[j], o1[j]);
  }
};

// Attempt one step of length h; the tangent vectors only when `joint`.
// Returns the mean square of the weighted error components (err^2).
template <class M, int K, class R, int INTEG, bool HF = FoldH<R>::value>
CL_HD typename CtlReal<R>::type attempt(const Lane<M, K, R, INTEG> &st, R h, bool joint,
                                        typename CtlReal<R>::type rtol,
                                        typename CtlReal<R>::type atol, R (&x1)[M::N],
                                        R (&V1)[K][M::N], R (&kx1)[M::N], R (&kv1)[K][M::N]) {
  using C = typename CtlReal<R>::type;
  constexpr int N = M::N;
  constexpr int S = (INTEG == kDverk65) ? 8 : 7;
  const C inv_nc = joint ? C(1) / C(N * (1 + K)) : C(1) / C(N);
  R X[S][N];
  if constexpr (Packed<M, K, R>::value) {
    constexpr bool SP = Packed<M, K, R>::state_paired;
    constexpr int KV = SP ? K - 1 : K;  // vectors advanced in pairs (v_0 .. v_{KV-1})
    float2 ea = make_float2(0.f, 0.f);
    if constexpr (SP) {
      float2 ya[N], ka[N], ya1[N], ka1[N];
#pragma unroll
      for (int j = 0; j < N; j++) {
        ya[j] = make_float2(st.x[j], st.V[K - 1][j]);
        ka[j] = make_float2(st.kx[j], st.kv[K - 1][j]);
      }
      PairStateStages<M> fa{st.p, X};
      if (INTEG == kDverk65) dverk_pass<N, float2, decltype(fa), HF>(ya, h, fa, ya1, ea, rtol, atol);
      else dopri_pass<N, float2, decltype(fa), HF>(ya, ka, h, fa, ya1, ka1, ea, rtol, atol);
#pragma unroll
      for (int j = 0; j < N; j++) {
        x1[j] = ya1[j].x;
        V1[K - 1][j] = ya1[j].y;
        if (INTEG == kDopri5) {
          kx1[j] = ka1[j].x;
          kv1[K - 1][j] = ka1[j].y;
        }
      }
    } else {
      StateStages<M, R> fs{st.p, X};
      if (INTEG == kDverk65) dverk_pass<N, R, decltype(fs), HF>(st.x, h, fs, x1, ea.x, rtol, atol);
      else dopri_pass<N, R, decltype(fs), HF>(st.x, st.kx, h, fs, x1, kx1, ea.x, rtol, atol);
    }
    float err2 = ea.x;
    if (joint) {
      float2 eb = make_float2(0.f, 0.f);
      PairTangentStages<M> fb{st.p, st.x, X};
#pragma unroll
      for (int m = 0; m + 1 < KV; m += 2) {
        float2 yb[N], kb[N], yb1[N], kb1[N];
#pragma unroll
        for (int j = 0; j < N; j++) {
          yb[j] = make_float2(st.V[m][j], st.V[m + 1][j]);
          kb[j] = make_float2(st.kv[m][j], st.kv[m + 1][j]);
        }
        if (INTEG == kDverk65) dverk_pass<N, float2, decltype(fb), HF>(yb, h, fb, yb1, eb, rtol, atol);
        else dopri_pass<N, float2, decltype(fb), HF>(yb, kb, h, fb, yb1, kb1, eb, rtol, atol);
#pragma unroll
        for (int j = 0; j < N; j++) {
          V1[m][j] = yb1[j].x;
          V1[m + 1][j] = yb1[j].y;
          if (INTEG == kDopri5) {
            kv1[m][j] = kb1[j].x;
            kv1[m + 1][j] = kb1[j].y;
          }
        }
      }
      err2 += ea.y + (eb.x + eb.y);
    }
    return err2 * inv_nc;
  } else {
    C err2 = C(0);
    StateStages<M, R> fs{st.p, X};
    if (INTEG == kDverk65) dverk_pass<N, R, decltype(fs), HF>(st.x, h, fs, x1, err2, rtol, atol);
    else dopri_pass<N, R, decltype(fs), HF>(st.x, st.kx, h, fs, x1, kx1, err2, rtol, atol);
    if (joint) {
      TangentStages<M, R> ft{st.p, st.x, X};
#pragma unroll
      for (int i = 0; i < K; i++) {
        if (INTEG == kDverk65) dverk_pass<N, R, decltype(ft), HF>(st.V[i], h, ft, V1[i], err2, rtol, atol);
        else dopri_pass<N, R, decltype(ft), HF>(st.V[i], st.kv[i], h, ft, V1[i], kv1[i], err2, rtol, atol);
      }
    }
    return err2 * inv_nc;
  }
}

// Gram-Schmidt in FP64 on the k tangent vectors (whatever their precision R);
// r[i] = norms after the projections (the R diagonal).  Returns
// max_i |v_i|^2 / r_i^2: how much of each vector cancelled, i.e. the factor
// by which errors in the vectors grew relative to what is left of them (an
// estimate that only steers the renormalisation interval, so |v_i|^2 before
// the projections is taken in the vectors' own precision).
//
template <class R> CL_HD double rsqrt_for(double s) {
#ifdef __CUDA_ARCH__
  return rsqrt(s);
#else
  return 1.0 / sqrt(s);
#endif
}

template <int N, int K, class R>
CL_HD float renormalise(R (&V)[K][N], double (&r)[K], int gs) {
  double v[K][N];
  float cancel = 1.0f;
#pragma unroll
  for (int i = 0; i < K; i++)
#pragma unroll
    for (int j = 0; j < N; j++) v[i][j] = (double)V[i][j];
#pragma unroll
  for (int i = 0; i < K; i++) {
    R before = 0;
#pragma unroll
    for (int j = 0; j < N; j++) before = vfma(V[i][j], V[i][j], before);
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
    const double inv = rsqrt_for<R>(s);
    r[i] = s * inv;
    const float fi = (float)inv;
    cancel = fmaxf(cancel, (float)before * (fi * fi));
#pragma unroll
    for (int j = 0; j < N; j++) v[i][j] *= inv;
  }
#pragma unroll
  for (int i = 0; i < K; i++)
#pragma unroll
    for (int j = 0; j < N; j++) V[i][j] = (R)v[i][j];
  return cancel;
}

template <class M, int K, class R, int INTEG>
CL_HD void refresh_tangent_derivs(Lane<M, K, R, INTEG> &L) {
  if (INTEG == kDopri5) {
#pragma unroll
    for (int i = 0; i < K; i++) M::jv(L.V[i], L.kv[i], L.p, L.x);
  }
}

// Moves the running norm products into the compensated log sums.
template <class M, int K, class R, int INTEG>
CL_HD void lane_flush_logs(Lane<M, K, R, INTEG> &) {
  Cold &c = cold_slot();
#pragma unroll
  for (int i = 0; i < K; i++) {  // Kahan-compensated sum of log-norms
    const double y = log(c.prod[i]) - c.comp[i];
    const double s = c.sum[i] + y;
    c.comp[i] = (s - c.sum[i]) - y;
    c.sum[i] = s;
    c.prod[i] = 1.0;
  }
}

template <class M, int K, class R, int INTEG>
CL_HD void lane_finish(Lane<M, K, R, INTEG> &L, const AdaptiveArgs &a, int status) {
  lane_flush_logs(L);
  const Cold &c = cold_slot();
#pragma unroll
  for (int i = 0; i < K; i++) {
    const double lam = status ? quiet_nan() : c.sum[i] / c.t_avg;
    a.spectrum.base[c.pt * a.spectrum.ps + i * a.spectrum.cs] = lam;
  }
  if (a.status) a.status[c.pt] = status;
  if (a.steps) a.steps[c.pt] = L.steps;
}

// Tangent basis = identity, start of the alignment / averaging phases.
// Component j of tangent vector i at the start of the tangent phase: the
// identity basis (cuda/lyapunov.dp.cpp:133-226 starts from I), tilted in the
// FP32 forms by 1e-6 along every other axis.  Why: a stable equilibrium at
// the origin (Lorenz at rho < 1) decays below FP32's smallest denormal during
// the transient, the state becomes exactly zero, and the variational
// equations split exactly into invariant subspaces (for Lorenz, the x-y
// block and z); an axis-aligned vector then never acquires the component
// along the slower direction and Gram-Schmidt reports the exponents out of
// order.  In FP64 the state stays nonzero and rounding supplies that
// component.  The tilt changes an exponent by about 1e-6 / t_avg.
template <class R> CL_HD R tangent_init(int i, int j) {
  return i == j ? R(1) : (sizeof(R) == 4 ? R(1e-6f) : R(0));
}

template <class M, int K, class R, int INTEG>
CL_HD void lane_set_phase_time(Lane<M, K, R, INTEG> &L, double len) {
  L.t_left = len;
  L.t_left_r = time_left_as<R>(len);
}

template <class M, int K, class R, int INTEG>
CL_HD void lane_start_tangent(Lane<M, K, R, INTEG> &L, const AdaptiveArgs &a) {
  constexpr int N = M::N;
#pragma unroll
  for (int i = 0; i < K; i++)
#pragma unroll
    for (int j = 0; j < N; j++) L.V[i][j] = tangent_init<R>(i, j);
  refresh_tangent_derivs(L);
  L.lfac_old = log2_fac_min<typename CtlReal<R>::type>();
  L.t_gs = 0.f;
  if (a.t_align > 0) {
    L.phase = kAlign;
    lane_set_phase_time(L, a.t_align);
  } else {
    L.phase = kAverage;
    lane_set_phase_time(L, cold_slot().t_avg);
  }
}

template <class M, int K, class R, int INTEG>
CL_HD void lane_start(Lane<M, K, R, INTEG> &L, const AdaptiveArgs &a, int64_t pt) {
  constexpr int N = M::N;
  Cold &cs = cold_slot();
  cs.pt = pt;
#pragma unroll
  for (int i = 0; i < M::NP; i++) L.p[i] = (R)a.params.base[pt * a.params.ps + i * a.params.cs];
#pragma unroll
  for (int i = 0; i < N; i++) L.x[i] = (R)a.inits.base[pt * a.inits.ps + i * a.inits.cs];
  L.h = (R)a.h0;
  L.lfac_old = log2_fac_min<typename CtlReal<R>::type>();
  L.reject = false;
  L.steps = 0;
  cs.t_avg = a.t_avg_per_point ? a.t_avg_per_point[pt] : a.t_avg;
  L.L = (float)a.dt_renorm / kRenormSplitInit;
  L.rate_max = initial_renorm_rate(renorm_spread_limit<R>((float)a.rtol), (float)a.dt_renorm);
#pragma unroll
  for (int i = 0; i < K; i++) {
    cs.sum[i] = cs.comp[i] = 0.0;
    cs.prod[i] = 1.0;
  }
  // The tangent rows ride along in the packed transient pass; start them
  // from zero so that they stay finite until the alignment phase sets them.
#pragma unroll
  for (int i = 0; i < K; i++)
#pragma unroll
    for (int j = 0; j < N; j++) L.V[i][j] = L.kv[i][j] = R(0);
  if (INTEG == kDopri5) M::f(L.x, L.kx, L.p);
  if (a.t_transient > 0) {
    L.phase = kTransient;
    lane_set_phase_time(L, a.t_transient);
    L.t_gs = 0.f;
  } else {
    lane_start_tangent(L, a);
  }
}

// Gram-Schmidt step of one lane: log-norms accumulated in the averaging
// phase, interval target adapted.  Returns false on a degenerate basis.
template <class M, int K, class R, int INTEG>
CL_HD bool lane_gram_schmidt(Lane<M, K, R, INTEG> &L, const AdaptiveArgs &a, const Ctl &c) {
  double r[K];
  const float cancel = renormalise<M::N, K, R>(L.V, r, a.gs);
  bool ok = true;
#pragma unroll
  for (int i = 0; i < K; i++) ok = ok && (r[i] > 0.0) && (r[i] < 1e300);
  if (!ok) return false;
  if (L.phase == kAverage) {
    // Norms multiply into a running FP64 product; its log joins the
    // compensated sum only when it nears the edge of the double range (and
    // at the end), so most renormalisations take no logarithm at all.
    Cold &cs = cold_slot();
    bool flush = false;
#pragma unroll
    for (int i = 0; i < K; i++) {
      cs.prod[i] *= r[i];
      flush = flush || !(cs.prod[i] < 1e150 && cs.prod[i] > 1e-150);
    }
    if (flush) lane_flush_logs(L);
  }
  if (L.t_gs > 0.f) {  // strain per unit time -> next interval
    double rmin = r[0];
#pragma unroll
    for (int i = 1; i < K; i++) rmin = fmin(rmin, r[i]);
    next_renorm_interval(L.L, L.rate_max, cancel, rmin, L.t_gs, c.tau, (float)a.dt_renorm);
  }
  L.t_gs = 0.f;
  refresh_tangent_derivs(L);
  return true;
}

// One step attempt of one lane, phase bookkeeping included.  Returns
// kFinished once the point's outputs are written.
template <class M, int K, class R, int INTEG>
CL_HD int lane_step(Lane<M, K, R, INTEG> &L, const AdaptiveArgs &a, const Ctl &c) {
  using C = typename CtlReal<R>::type;
  constexpr int N = M::N;
  if (L.steps == 0 && !state_inside(L.x, c.escape)) {
    lane_finish(L, a, 4);
    return kFinished;
  }
  if (L.steps >= c.max_steps) {
    lane_finish(L, a, 3);
    return kFinished;
  }
  if (!step_at_least_hmin(L.h, c)) {  // also catches h == 0 and NaN
    lane_finish(L, a, 2);
    return kFinished;
  }
  // A proposal that reaches the phase end lands on it (t_left_r is the time
  // left rounded toward zero, so a step that is not clamped never passes it)
  const bool clamped = L.h >= L.t_left_r;
  const R h = clamped ? L.t_left_r : L.h;
  const bool joint = L.phase != kTransient;
  R x1[N], V1[K][N], kx1[N], kv1[K][N];
  L.steps++;
  const C err2 = attempt<M, K, R, INTEG>(L, h, joint, ctl_rtol<R>(c), ctl_atol<R>(c), x1, V1,
                                         kx1, kv1);
  if (!(err2 <= err2_limit<C>())) {  // NaN or an overflowed error norm
    if (!point_finite(L.p, L.x)) {
      lane_finish(L, a, 1);
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
      for (int i = 0; i < K; i++)
#pragma unroll
        for (int j = 0; j < N; j++) {
          L.V[i][j] = V1[i][j];
          if (INTEG == kDopri5) L.kv[i][j] = kv1[i][j];
        }
    }
    if (!clamped || hnew < h) L.h = hnew;  // else keep the unclamped proposal
    if (!clamped) {
      L.t_left -= (double)h;
      L.t_left_r = time_left_as<R>(L.t_left);
    }
    L.t_gs += (float)h;
    if (!state_inside(L.x, c.escape)) {
      lane_finish(L, a, 4);
      return kFinished;
    }
    if (clamped) {  // landed on a phase end
      if (L.phase == kTransient) {
        lane_start_tangent(L, a);
      } else if (L.phase == kAlign) {
        if (!lane_gram_schmidt(L, a, c)) {
          lane_finish(L, a, 1);
          return kFinished;
        }
        L.phase = kAverage;
        lane_set_phase_time(L, cold_slot().t_avg);
      } else {
        const bool ok = lane_gram_schmidt(L, a, c);
        lane_finish(L, a, ok ? 0 : 1);
        return kFinished;
      }
    }
  } else {
    L.h = hnew;
  }
  return kRunning;
}

template <class R>
CL_HD Ctl make_ctl(const AdaptiveArgs &a) {
  // A step below 1e-12 (model time units) is never meaningful here; it also
  // stops a point whose controller collapsed the step to zero.
  const double hmax = a.hmax > 0 ? a.hmax : 1e300, hmin = fmax(a.hmin, 1e-12);
  return Ctl{(float)a.rtol, (float)a.atol, renorm_spread_limit<R>((float)a.rtol), a.rtol, a.atol,
             hmax, hmin, float_ru(hmin), float_rd(hmax), a.max_steps,
             a.escape > 0 ? a.escape : 1e4};
}

// A batch's arguments with every segment's limits filled in for the
// batch's precision (host side, before the launch).
inline BatchArgs with_ctl(const BatchArgs &b, int prec) {
  BatchArgs out = b;
  for (int i = 0; i < b.nseg; i++)
    out.seg[i].ctl = prec == kFP32 ? make_ctl<float>(b.seg[i]) : make_ctl<double>(b.seg[i]);
  return out;
}

// One point start to finish on one thread (the host form of the kernel
// loop, used by tests that run the integrator on the CPU).
template <class M, int K, class R, int INTEG>
CL_HD void run_point(const AdaptiveArgs &a, int64_t pt) {
  const Ctl c = make_ctl<R>(a);
  Lane<M, K, R, INTEG> L;
  lane_start(L, a, pt);
  for (;;) {
    if (lane_step(L, a, c) == kFinished) return;
    if (L.phase != kTransient && L.t_gs >= L.L && !lane_gram_schmidt(L, a, c)) {
      lane_finish(L, a, 1);
      return;
    }
  }
}

}  // namespace adaptive
}  // namespace chaos
