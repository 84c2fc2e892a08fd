// Pieces shared by every adaptive form (one lane per point, four lanes per
// point, warp per point): fast single-precision helpers and the policy that
// sets the interval between two Gram-Schmidt renormalisations.
#pragma once
#include <cmath>

#include "models.cuh"

namespace chaos {
namespace adaptive {

CL_HD float fast_log2f(float x) {
#ifdef __CUDA_ARCH__
  return __log2f(x);
#else
  return log2f(x);
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

// Initial renormalisation interval dt_renorm / kRenormSplitInit; the
// interval never falls below dt_renorm / kRenormSplitMax.
constexpr int kRenormSplitInit = 16, kRenormSplitMax = 64;

// Renormalisation interval, shared by every form.  Two things degrade the
// tangent vectors between two Gram-Schmidt passes, and the interval L keeps
// both bounded:
//  * cancellation: errors in a vector are relative to its length, and
//    Gram-Schmidt keeps only its part not along the earlier vectors, so they
//    grow by |v_i| / r_i -- allowed up to exp(kCancelFrac tau) = exp(tau / 4);
//  * shrinking: a vector in a contracting direction loses length, and once
//    its components fall below atol / rtol the error control on it is
//    absolute, not relative -- the norms may shrink by at most
//    exp(kShrinkMax) (measured: letting them shrink to 1e-10 between passes
//    biased the most negative exponent of regular Rossler cells by 1e-3 at
//    rtol 1e-6; bounded at e^-2 the bias falls to the level of the FP64
//    method at the same tolerance).
// Both are measured at each pass as a "strain" per unit time; the interval
// follows the largest recent rate (forgotten by 0.5 % per pass, so a calm
// part of an orbit does not open an interval that a contraction burst later
// crosses), grows at most 2x per pass, and lies in [dt / 64, dt].  The rate
// starts at the value that gives L = dt / 16 (initial_renorm_rate).
// kCancelFrac: tau / 8 and tau / 4 give the same FP32 spectra on 512 Rossler
// and 256 Lorenz cells of the 1024^2 maps against the FP64 oracle (regular
// cells within 1e-3: 95.6 % and 91.2 % both; median errors within 10 %;
// Lorenz trace identity, median 1.28e-5 -> 1.41e-5), with half the
// Gram-Schmidt passes -- a third of a step's latency in the four-lane form.
constexpr float kShrinkMax = 2.0f;
constexpr float kCancelFrac = 0.25f;
CL_HD float initial_renorm_rate(float tau, float dt) {
  return kCancelFrac * tau * kRenormSplitInit / dt;
}
template <class T>
CL_HD void next_renorm_interval(T &L, T &rate_max, float cancel, double rmin, T t_gs, float tau,
                                T dt) {
  constexpr float ln2 = 0.6931471805599453f;
  const float cancel_strain = 0.5f * ln2 * fast_log2f(cancel);
  const float shrink_strain =
      (kCancelFrac * tau / kShrinkMax) * (-ln2) * fast_log2f(fminf((float)rmin, 1.0f));
  const float strain = fmaxf(cancel_strain, shrink_strain);
  const T rate = sizeof(T) == 4 ? (T)fast_div(strain, (float)t_gs) : (T)strain / t_gs;
  rate_max = rate > T(0.995) * rate_max ? rate : T(0.995) * rate_max;
  const T rm = rate_max > T(1e-30) ? rate_max : T(1e-30);
  const T target = sizeof(T) == 4 ? (T)fast_div(kCancelFrac * tau, (float)rm)
                                   : T(kCancelFrac) * tau / rm;
  const T lo = dt * T(1.0 / kRenormSplitMax);
  T next = target > lo ? target : lo;
  next = next < T(2) * L ? next : T(2) * L;
  L = next < dt ? next : dt;
}

}  // namespace adaptive
}  // namespace chaos
