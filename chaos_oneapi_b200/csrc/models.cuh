// Flow models as compile-time types: the device right-hand sides that the
// reference reaches through device function pointers (types.h:17-24,
// cuda/models/flows/shimizu.dp.cpp:63-68) become template parameters here, so
// every kernel instantiation inlines its model.
//
// Each model provides, for any arithmetic type T:
//   f(x, dx, p)          dx = F(x)                    (types.h:18 diffSysFunc)
//   jv(v, dv, p, x)      dv = J(x) v                  (types.h:21 diffSysFuncVar)
//   jq_col(v, dv, p, x)  dv = column of J(x) Q        (the f_Q plug-in)
// The expression order is the one the reference's Shimizu-Morioka model uses
// (shimizu.dp.cpp:15-52), and for the other models the one of the oracle's
// reference-format model files; under -fmad=false the fixed-step kernels
// therefore reproduce the reference's arithmetic bit for bit.
#pragma once
#include <cmath>
#include <cstdint>

#define CL_HD __host__ __device__ __forceinline__

namespace chaos {

enum ModelId : int32_t {
  kShimizu = 0,
  kLorenz = 1,
  kRossler = 2,
  kChua = 3,
  kHyperRossler = 4,
  kLorenz96 = 5,
  kHenon = 6,
  kNumModels = 7
};

// Model type (model_factory.h ModelType): flows are integrated, maps
// iterated (cuda/tools/mapstep.dp.cpp:6-19: the new state is f(state), the
// new tangent vector J(state) v).  Flows are the default.
template <class M> struct IsMap { static constexpr bool value = false; };

// Shimizu-Morioka: x' = y, y' = -a y - x z + x, z' = -l z + x^2 ; p = (alpha, lamda)
struct Shimizu {
  static constexpr int N = 3, NP = 2, ID = kShimizu;
  template <class T> CL_HD static void f(const T *x, T *dx, const T *p) {
    dx[0] = x[1];
    dx[1] = -p[0] * x[1] - x[0] * x[2] + x[0];
    dx[2] = -p[1] * x[2] + x[0] * x[0];
  }
  template <class T> CL_HD static void jv(const T *v, T *dv, const T *p, const T *x) {
    dv[0] = v[1] * T(1);
    dv[1] = v[0] * (T(1) - x[2]) + v[1] * (-p[0]) + v[2] * (-x[0]);
    dv[2] = v[0] * (T(2.0) * x[0]) + v[2] * (-p[1]);
  }
  // shimizu.dp.cpp:39-52 keeps explicit zero terms; they are kept here too.
  template <class T> CL_HD static void jq_col(const T *q, T *dq, const T *p, const T *x) {
    dq[0] = T(0) * q[0] + T(1) * q[1] + T(0) * q[2];
    dq[1] = (T(1) - x[2]) * q[0] + (-p[0]) * q[1] + (-x[0]) * q[2];
    dq[2] = (T(2.0) * x[0]) * q[0] + T(0) * q[1] + (-p[1]) * q[2];
  }
  static constexpr int kFlopsF = 7, kFlopsJv = 9;
};

// Lorenz: x' = s (y - x), y' = x (r - z) - y, z' = x y - b z ; p = (sigma, rho, beta)
struct Lorenz {
  static constexpr int N = 3, NP = 3, ID = kLorenz;
  template <class T> CL_HD static void f(const T *x, T *dx, const T *p) {
    dx[0] = p[0] * (x[1] - x[0]);
    dx[1] = x[0] * (p[1] - x[2]) - x[1];
    dx[2] = x[0] * x[1] - p[2] * x[2];
  }
  template <class T> CL_HD static void jv(const T *v, T *dv, const T *p, const T *x) {
    dv[0] = p[0] * (v[1] - v[0]);
    dv[1] = (p[1] - x[2]) * v[0] - v[1] - x[0] * v[2];
    dv[2] = x[1] * v[0] + x[0] * v[1] - p[2] * v[2];
  }
  template <class T> CL_HD static void jq_col(const T *q, T *dq, const T *p, const T *x) { jv(q, dq, p, x); }
  static constexpr int kFlopsF = 9, kFlopsJv = 12;
};

// Rossler: x' = -y - z, y' = x + a y, z' = b + z (x - c) ; p = (a, b, c)
struct Rossler {
  static constexpr int N = 3, NP = 3, ID = kRossler;
  template <class T> CL_HD static void f(const T *x, T *dx, const T *p) {
    dx[0] = -x[1] - x[2];
    dx[1] = x[0] + p[0] * x[1];
    dx[2] = p[1] + x[2] * (x[0] - p[2]);
  }
  template <class T> CL_HD static void jv(const T *v, T *dv, const T *p, const T *x) {
    dv[0] = -v[1] - v[2];
    dv[1] = v[0] + p[0] * v[1];
    dv[2] = x[2] * v[0] + (x[0] - p[2]) * v[2];
  }
  template <class T> CL_HD static void jq_col(const T *q, T *dq, const T *p, const T *x) { jv(q, dq, p, x); }
  static constexpr int kFlopsF = 7, kFlopsJv = 8;
};

// Chua double scroll: x' = al (y - x - f(x)), y' = x - y + z, z' = -be y,
// f(x) = m1 x + (m0 - m1)(|x + 1| - |x - 1|) / 2 ; p = (alpha, beta, m0, m1)
struct Chua {
  static constexpr int N = 3, NP = 4, ID = kChua;
  template <class T> CL_HD static void f(const T *x, T *dx, const T *p) {
    const T fx = p[3] * x[0] + T(0.5) * (p[2] - p[3]) * (fabs(x[0] + T(1.0)) - fabs(x[0] - T(1.0)));
    dx[0] = p[0] * (x[1] - x[0] - fx);
    dx[1] = x[0] - x[1] + x[2];
    dx[2] = -p[1] * x[1];
  }
  template <class T> CL_HD static void jv(const T *v, T *dv, const T *p, const T *x) {
    const T fp = (fabs(x[0]) < T(1.0)) ? p[2] : p[3];
    dv[0] = p[0] * (v[1] - v[0] - fp * v[0]);
    dv[1] = v[0] - v[1] + v[2];
    dv[2] = -p[1] * v[1];
  }
  template <class T> CL_HD static void jq_col(const T *q, T *dq, const T *p, const T *x) { jv(q, dq, p, x); }
  static constexpr int kFlopsF = 14, kFlopsJv = 9;
};

// Hyperchaotic Rossler 4-D: x' = -y - z, y' = x + 0.25 y + w, z' = 3 + x z,
// w' = -c z + d w ; p = (c, d)
struct HyperRossler {
  static constexpr int N = 4, NP = 2, ID = kHyperRossler;
  template <class T> CL_HD static void f(const T *x, T *dx, const T *p) {
    dx[0] = -x[1] - x[2];
    dx[1] = x[0] + T(0.25) * x[1] + x[3];
    dx[2] = T(3.0) + x[0] * x[2];
    dx[3] = -p[0] * x[2] + p[1] * x[3];
  }
  template <class T> CL_HD static void jv(const T *v, T *dv, const T *p, const T *x) {
    dv[0] = -v[1] - v[2];
    dv[1] = v[0] + T(0.25) * v[1] + v[3];
    dv[2] = x[2] * v[0] + x[0] * v[2];
    dv[3] = -p[0] * v[2] + p[1] * v[3];
  }
  template <class T> CL_HD static void jq_col(const T *q, T *dq, const T *p, const T *x) { jv(q, dq, p, x); }
  static constexpr int kFlopsF = 10, kFlopsJv = 11;
};

// Lorenz-96, N = 40, cyclic: x_i' = (x_{i+1} - x_{i-2}) x_{i-1} - g x_i + F ; p = (F, gamma)
struct Lorenz96 {
  static constexpr int N = 40, NP = 2, ID = kLorenz96;
  CL_HD static int w(int i) { return (i + N) % N; }
  template <class T> CL_HD static void f(const T *x, T *dx, const T *p) {
    for (int i = 0; i < N; ++i) dx[i] = (x[w(i + 1)] - x[w(i - 2)]) * x[w(i - 1)] - p[1] * x[i] + p[0];
  }
  template <class T> CL_HD static void jv(const T *v, T *dv, const T *p, const T *x) {
    for (int i = 0; i < N; ++i)
      dv[i] = (v[w(i + 1)] - v[w(i - 2)]) * x[w(i - 1)] + (x[w(i + 1)] - x[w(i - 2)]) * v[w(i - 1)] - p[1] * v[i];
  }
  template <class T> CL_HD static void jq_col(const T *q, T *dq, const T *p, const T *x) { jv(q, dq, p, x); }
  static constexpr int kFlopsF = 5 * N, kFlopsJv = 8 * N;
};

// Henon map: x -> 1 - a x^2 + y, y -> b x ; p = (a, b).  A map-type model
// (the reference registers none; its configuration lists map entries and its
// method code has map branches, cuda/lyapunov.dp.cpp:70-125,182-222).
// lambda_1 + lambda_2 = ln |b| (det J = -b).
struct Henon {
  static constexpr int N = 2, NP = 2, ID = kHenon;
  template <class T> CL_HD static void f(const T *x, T *dx, const T *p) {
    dx[0] = T(1.0) - p[0] * x[0] * x[0] + x[1];
    dx[1] = p[1] * x[0];
  }
  template <class T> CL_HD static void jv(const T *v, T *dv, const T *p, const T *x) {
    dv[0] = T(-2.0) * p[0] * x[0] * v[0] + v[1];
    dv[1] = p[1] * v[0];
  }
  template <class T> CL_HD static void jq_col(const T *q, T *dq, const T *p, const T *x) { jv(q, dq, p, x); }
  static constexpr int kFlopsF = 6, kFlopsJv = 6;
};
template <> struct IsMap<Henon> { static constexpr bool value = true; };

}  // namespace chaos
