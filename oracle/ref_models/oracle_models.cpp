// Test infrastructure only (oracle build): extra models written in the
// reference's own model-plugin format so that the reference's Lyapunov path
// (cuda/lyapunov.dp.cpp) can be run on them as the parity oracle.  The
// reference ships only Shimizu-Morioka (cuda/models/flows/shimizu.dp.cpp);
// these files follow its interface:
//   f    (const double* x, double* dx, const double* p)                 types.h:18
//   f_var(const double* v, double* dv, const double* p, const double* x)  types.h:21
//   f_Q  (const double* Q, double* JQ, const double* p, const double* x)  J*Q, row-major n*n
// and register through ModelFactoryRegistry::RegisterModel
// (model_factory.h:36-39) the way shimizu.dp.cpp:70-211 does.
//
// The expression order of every right-hand side below is the one the CUDA
// models and the C restatement use, so that fixed-step runs agree bit for bit.
#include <CL/sycl.hpp>
#include <dpct/dpct.hpp>
#include <cmath>
#include "model_factory.h"

namespace {

// ---------------------------------------------------------------- Lorenz
// dx = s(y-x), dy = x(r-z) - y, dz = xy - b z ; p = (sigma, rho, beta)
void lorenz(const double *x, double *dx, const double *p) {
  dx[0] = p[0] * (x[1] - x[0]);
  dx[1] = x[0] * (p[1] - x[2]) - x[1];
  dx[2] = x[0] * x[1] - p[2] * x[2];
}
void lorenz_var(const double *v, double *dv, const double *p, const double *x) {
  dv[0] = p[0] * (v[1] - v[0]);
  dv[1] = (p[1] - x[2]) * v[0] - v[1] - x[0] * v[2];
  dv[2] = x[1] * v[0] + x[0] * v[1] - p[2] * v[2];
}

// --------------------------------------------------------------- Rossler
// dx = -y - z, dy = x + a y, dz = b + z (x - c) ; p = (a, b, c)
void rossler(const double *x, double *dx, const double *p) {
  dx[0] = -x[1] - x[2];
  dx[1] = x[0] + p[0] * x[1];
  dx[2] = p[1] + x[2] * (x[0] - p[2]);
}
void rossler_var(const double *v, double *dv, const double *p, const double *x) {
  dv[0] = -v[1] - v[2];
  dv[1] = v[0] + p[0] * v[1];
  dv[2] = x[2] * v[0] + (x[0] - p[2]) * v[2];
}

// ------------------------------------------------------------------ Chua
// x' = al (y - x - f(x)), y' = x - y + z, z' = -be y,
// f(x) = m1 x + 0.5 (m0 - m1)(|x+1| - |x-1|) ; p = (alpha, beta, m0, m1)
void chua(const double *x, double *dx, const double *p) {
  const double fx = p[3] * x[0] + 0.5 * (p[2] - p[3]) * (std::fabs(x[0] + 1.0) - std::fabs(x[0] - 1.0));
  dx[0] = p[0] * (x[1] - x[0] - fx);
  dx[1] = x[0] - x[1] + x[2];
  dx[2] = -p[1] * x[1];
}
void chua_var(const double *v, double *dv, const double *p, const double *x) {
  const double fp = (std::fabs(x[0]) < 1.0) ? p[2] : p[3];
  dv[0] = p[0] * (v[1] - v[0] - fp * v[0]);
  dv[1] = v[0] - v[1] + v[2];
  dv[2] = -p[1] * v[1];
}

// ------------------------------------------------- hyperchaotic Rossler 4-D
// x' = -y - z, y' = x + 0.25 y + w, z' = 3 + x z, w' = -c z + d w ; p = (c, d)
void hyper_rossler(const double *x, double *dx, const double *p) {
  dx[0] = -x[1] - x[2];
  dx[1] = x[0] + 0.25 * x[1] + x[3];
  dx[2] = 3.0 + x[0] * x[2];
  dx[3] = -p[0] * x[2] + p[1] * x[3];
}
void hyper_rossler_var(const double *v, double *dv, const double *p, const double *x) {
  dv[0] = -v[1] - v[2];
  dv[1] = v[0] + 0.25 * v[1] + v[3];
  dv[2] = x[2] * v[0] + x[0] * v[2];
  dv[3] = -p[0] * v[2] + p[1] * v[3];
}

// ----------------------------------------------------- Lorenz-96, N = 40
// dx_i = (x_{i+1} - x_{i-2}) x_{i-1} - g x_i + F (cyclic) ; p = (F, gamma)
constexpr int L96_N = 40;
inline int wrap(int i) { return (i + L96_N) % L96_N; }
void lorenz96(const double *x, double *dx, const double *p) {
  for (int i = 0; i < L96_N; ++i)
    dx[i] = (x[wrap(i + 1)] - x[wrap(i - 2)]) * x[wrap(i - 1)] - p[1] * x[i] + p[0];
}
void lorenz96_var(const double *v, double *dv, const double *p, const double *x) {
  for (int i = 0; i < L96_N; ++i)
    dv[i] = (v[wrap(i + 1)] - v[wrap(i - 2)]) * x[wrap(i - 1)] +
            (x[wrap(i + 1)] - x[wrap(i - 2)]) * v[wrap(i - 1)] - p[1] * v[i];
}

// ------------------------------------------------------------ Henon map
// x -> 1 - a x^2 + y, y -> b x ; p = (a, b).  A map-type model: f writes the
// next state (cuda/tools/mapstep.dp.cpp:6-11), f_var the tangent image J(x) v.
void henon(const double *x, double *dx, const double *p) {
  dx[0] = 1.0 - p[0] * x[0] * x[0] + x[1];
  dx[1] = p[1] * x[0];
}
void henon_var(const double *v, double *dv, const double *p, const double *x) {
  dv[0] = -2.0 * p[0] * x[0] * v[0] + v[1];
  dv[1] = p[1] * v[0];
}

// J*Q for a row-major n*n Q: column c of the result is J applied to column c
// of Q, evaluated with the model's own tangent expression.
template <int N, void (*VAR)(const double *, double *, const double *, const double *)>
void linear_q(const double *Q, double *res, const double *p, const double *x) {
  double col[N], out[N];
  for (int c = 0; c < N; ++c) {
    for (int r = 0; r < N; ++r) col[r] = Q[r * N + c];
    VAR(col, out, p, x);
    for (int r = 0; r < N; ++r) res[r * N + c] = out[r];
  }
}

template <diffSysFunc F, diffSysFuncVar V, diffSysFuncVar Q, ModelType TYPE = ModelType::flow>
struct Registrar : public ModelFactoryRegistry {
  Registrar(const char *name, int dim, int np, const char *pnames, const char *phase, const char *eq) {
    auto f = [](diffSysFunc *out) { *out = F; };
    auto fv = [](diffSysFuncVar *out) { *out = V; };
    auto fq = [](diffSysFuncVar *out) { *out = Q; };
    RegisterModel(name, dim, np, TYPE, f, fv, nullptr, nullptr, fq, pnames, phase, eq);
  }
};

Registrar<lorenz, lorenz_var, linear_q<3, lorenz_var>> reg_lorenz(
    "lorenz", 3, 3, "sigma, rho, beta", "x, y, z",
    "x' = sigma * (y - x);y' = x * (rho - z) - y;z' = x * y - beta * z");
Registrar<rossler, rossler_var, linear_q<3, rossler_var>> reg_rossler(
    "rossler", 3, 3, "a, b, c", "x, y, z", "x' = - y - z;y' = x + a * y;z' = b + z * (x - c)");
Registrar<chua, chua_var, linear_q<3, chua_var>> reg_chua(
    "chua", 3, 4, "alpha, beta, m0, m1", "x, y, z",
    "x' = alpha * (y - x - f(x));y' = x - y + z;z' = - beta * y;"
    "f(x) = m1 * x + 0.5 * (m0 - m1) * (|x + 1| - |x - 1|)");
Registrar<hyper_rossler, hyper_rossler_var, linear_q<4, hyper_rossler_var>> reg_hyper_rossler(
    "hyper_rossler", 4, 2, "c, d", "x, y, z, w",
    "x' = - y - z;y' = x + 0.25 * y + w;z' = 3 + x * z;w' = - c * z + d * w");
Registrar<henon, henon_var, linear_q<2, henon_var>, ModelType::map> reg_henon(
    "henon", 2, 2, "a, b", "x, y", "x -> 1 - a * x^2 + y;y -> b * x");
Registrar<lorenz96, lorenz96_var, linear_q<L96_N, lorenz96_var>> reg_lorenz96(
    "lorenz96", L96_N, 2, "F, gamma", "x0..x39",
    "x_i' = (x_{i+1} - x_{i-2}) * x_{i-1} - gamma * x_i + F (cyclic, N = 40)");

}  // namespace
