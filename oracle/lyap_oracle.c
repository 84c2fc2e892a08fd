/* Test infrastructure only: the oracle (see lyap_oracle.h).  A CPU restatement
 * of the reference's Lyapunov-spectrum path, used by tests, the smoke check and
 * the bench's CPU-baseline leg to compare against.  The product never links it.
 *
 * Fixed-step part: reproduces cuda/lyapunov.dp.cpp:5-259 with the tableau and
 * operation order of cuda/tools/dverk.dp.cpp:7-81 and the Gram-Schmidt of
 * cuda/tools/linalg.dp.cpp:5-127, so that it agrees bit for bit with the
 * reference compiled on the host (strict IEEE double, no FMA contraction:
 * build with -ffp-contract=off).
 *
 * Adaptive part: DVERK 6(5) (Verner's pair; 6th-order weights from
 * cuda/tools/dverk.dp.cpp:41, 5th-order weights from Verner's published
 * DVERK pair) and Dormand-Prince 5(4) (cuda/tools/dopri.dp.cpp:14-44), with
 * the step-size controller of cuda/tools/dopri.dp.cpp:9-12,46-138, applied to
 * the state and its variational equations integrated jointly.
 */
#include "lyap_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ models */
/* Expression order matches oracle/ref_models/oracle_models.cpp and, for
 * Shimizu-Morioka, cuda/models/flows/shimizu.dp.cpp:15-52. */

#define L96_N 40
static int l96w(int i) { return (i + L96_N) % L96_N; }

int orc_model_dim(int model) {
  static const int d[ORC_NMODELS] = {3, 3, 3, 3, 4, L96_N, 2};
  return (model >= 0 && model < ORC_NMODELS) ? d[model] : -1;
}
int orc_model_nparams(int model) {
  static const int m[ORC_NMODELS] = {2, 3, 3, 4, 2, 2, 2};
  return (model >= 0 && model < ORC_NMODELS) ? m[model] : -1;
}
int orc_model_is_map(int model) { return model == ORC_HENON; }

static void model_f(int model, const double *x, double *dx, const double *p) {
  switch (model) {
    case ORC_SHIMIZU:  /* shimizu.dp.cpp:15-19 */
      dx[0] = x[1];
      dx[1] = -p[0] * x[1] - x[0] * x[2] + x[0];
      dx[2] = -p[1] * x[2] + x[0] * x[0];
      break;
    case ORC_LORENZ:
      dx[0] = p[0] * (x[1] - x[0]);
      dx[1] = x[0] * (p[1] - x[2]) - x[1];
      dx[2] = x[0] * x[1] - p[2] * x[2];
      break;
    case ORC_ROSSLER:
      dx[0] = -x[1] - x[2];
      dx[1] = x[0] + p[0] * x[1];
      dx[2] = p[1] + x[2] * (x[0] - p[2]);
      break;
    case ORC_CHUA: {
      const double fx = p[3] * x[0] + 0.5 * (p[2] - p[3]) * (fabs(x[0] + 1.0) - fabs(x[0] - 1.0));
      dx[0] = p[0] * (x[1] - x[0] - fx);
      dx[1] = x[0] - x[1] + x[2];
      dx[2] = -p[1] * x[1];
    } break;
    case ORC_HYPER_ROSSLER:
      dx[0] = -x[1] - x[2];
      dx[1] = x[0] + 0.25 * x[1] + x[3];
      dx[2] = 3.0 + x[0] * x[2];
      dx[3] = -p[0] * x[2] + p[1] * x[3];
      break;
    case ORC_LORENZ96:
      for (int i = 0; i < L96_N; ++i)
        dx[i] = (x[l96w(i + 1)] - x[l96w(i - 2)]) * x[l96w(i - 1)] - p[1] * x[i] + p[0];
      break;
    case ORC_HENON: /* map: dx is the next state */
      dx[0] = 1.0 - p[0] * x[0] * x[0] + x[1];
      dx[1] = p[1] * x[0];
      break;
  }
}

/* Tangent right-hand side dv = J(x) v. */
static void model_var(int model, const double *v, double *dv, const double *p, const double *x) {
  switch (model) {
    case ORC_SHIMIZU:  /* shimizu.dp.cpp:22-27; pow(x, 1.0) == x exactly */
      dv[0] = v[1] * 1;
      dv[1] = v[0] * (1 - x[2]) + v[1] * (-p[0]) + v[2] * (-x[0]);
      dv[2] = v[0] * (2.0 * pow(x[0], 1.0)) + v[2] * (-p[1]);
      break;
    case ORC_LORENZ:
      dv[0] = p[0] * (v[1] - v[0]);
      dv[1] = (p[1] - x[2]) * v[0] - v[1] - x[0] * v[2];
      dv[2] = x[1] * v[0] + x[0] * v[1] - p[2] * v[2];
      break;
    case ORC_ROSSLER:
      dv[0] = -v[1] - v[2];
      dv[1] = v[0] + p[0] * v[1];
      dv[2] = x[2] * v[0] + (x[0] - p[2]) * v[2];
      break;
    case ORC_CHUA: {
      const double fp = (fabs(x[0]) < 1.0) ? p[2] : p[3];
      dv[0] = p[0] * (v[1] - v[0] - fp * v[0]);
      dv[1] = v[0] - v[1] + v[2];
      dv[2] = -p[1] * v[1];
    } break;
    case ORC_HYPER_ROSSLER:
      dv[0] = -v[1] - v[2];
      dv[1] = v[0] + 0.25 * v[1] + v[3];
      dv[2] = x[2] * v[0] + x[0] * v[2];
      dv[3] = -p[0] * v[2] + p[1] * v[3];
      break;
    case ORC_LORENZ96:
      for (int i = 0; i < L96_N; ++i)
        dv[i] = (v[l96w(i + 1)] - v[l96w(i - 2)]) * x[l96w(i - 1)] +
                (x[l96w(i + 1)] - x[l96w(i - 2)]) * v[l96w(i - 1)] - p[1] * v[i];
      break;
    case ORC_HENON:
      dv[0] = -2.0 * p[0] * x[0] * v[0] + v[1];
      dv[1] = p[1] * v[0];
      break;
  }
}

/* J(x) Q for a row-major n*n Q (the reference's f_Q plug-in).  Shimizu keeps
 * the reference's own expression (shimizu.dp.cpp:39-52); the other models
 * apply their tangent expression column by column. */
static void model_q(int model, const double *Q, double *res, const double *p, const double *x) {
  const int n = orc_model_dim(model);
  if (model == ORC_SHIMIZU) {
    for (int c = 0; c < 3; ++c) {
      res[c] = 0 * Q[c] + (1) * Q[3 + c] + 0 * Q[6 + c];
      res[3 + c] = (1 - x[2]) * Q[c] + (-p[0]) * Q[3 + c] + (-x[0]) * Q[6 + c];
      res[6 + c] = (2.0 * pow(x[0], 1.0)) * Q[c] + 0 * Q[3 + c] + (-p[1]) * Q[6 + c];
    }
    return;
  }
  double col[L96_N], out[L96_N];
  for (int c = 0; c < n; ++c) {
    for (int r = 0; r < n; ++r) col[r] = Q[r * n + c];
    model_var(model, col, out, p, x);
    for (int r = 0; r < n; ++r) res[r * n + c] = out[r];
  }
}

/* ------------------------------------------------- fixed-step DVERK (ref) */
typedef struct {
  int model, kind; /* kind 0: f(y); 1: J(xf) y; 2: J(xf) Q */
  const double *p, *xf;
} deriv_ctx;

static void deriv(const deriv_ctx *c, const double *y, double *dy) {
  if (c->kind == 0) model_f(c->model, y, dy, c->p);
  else if (c->kind == 1) model_var(c->model, y, dy, c->p, c->xf);
  else model_q(c->model, y, dy, c->p, c->xf);
}

/* cuda/tools/dverk.dp.cpp:7-43 (and :45-81, identical with the tangent
 * right-hand side): same stage order, same coefficient grouping. */
static void dverk_fixed(double *val, int dim, const deriv_ctx *c, double step, double *w) {
  double *arg = w, *k1 = w + dim, *k2 = w + 2 * dim, *k3 = w + 3 * dim, *k4 = w + 4 * dim,
         *k5 = w + 5 * dim, *k6 = w + 6 * dim, *k7 = w + 7 * dim, *k8 = w + 8 * dim;
  int j;
  deriv(c, val, k1);
  for (j = 0; j < dim; j++) arg[j] = val[j] + step / 6. * k1[j];
  deriv(c, arg, k2);
  for (j = 0; j < dim; j++) arg[j] = val[j] + step * (4. / 75. * k1[j] + 16. / 75. * k2[j]);
  deriv(c, arg, k3);
  for (j = 0; j < dim; j++)
    arg[j] = val[j] + step * (5. / 6. * k1[j] - 8. / 3. * k2[j] + 5. / 2. * k3[j]);
  deriv(c, arg, k4);
  for (j = 0; j < dim; j++)
    arg[j] = val[j] + step * (-165. / 64. * k1[j] + 55. / 6. * k2[j] - 425. / 64. * k3[j] +
                              85. / 96. * k4[j]);
  deriv(c, arg, k5);
  for (j = 0; j < dim; j++)
    arg[j] = val[j] + step * (12. / 5. * k1[j] - 8. * k2[j] + 4015. / 612. * k3[j] -
                              11. / 36. * k4[j] + 88. / 255. * k5[j]);
  deriv(c, arg, k6);
  for (j = 0; j < dim; j++)
    arg[j] = val[j] + step * (-8263. / 15000. * k1[j] + 124. / 75. * k2[j] - 643. / 680. * k3[j] -
                              81. / 250. * k4[j] + 2484. / 10625. * k5[j]);
  deriv(c, arg, k7);
  for (j = 0; j < dim; j++)
    arg[j] = val[j] + step * (3501. / 1720. * k1[j] - 300. / 43. * k2[j] +
                              297275. / 52632. * k3[j] - 319. / 2322. * k4[j] +
                              24068. / 84065. * k5[j] + 3850. / 26703. * k7[j]);
  deriv(c, arg, k8);
  for (j = 0; j < dim; j++)
    val[j] = val[j] + step * (3. / 40. * k1[j] + 875. / 2244. * k3[j] + 23. / 72. * k4[j] +
                              264. / 1955. * k5[j] + 125. / 11592. * k7[j] + 43. / 616. * k8[j]);
}

void orc_dverk_step(int model, double *x, const double *p, double h) {
  double w[9 * L96_N];
  deriv_ctx c = {model, 0, p, 0};
  dverk_fixed(x, orc_model_dim(model), &c, h, w);
}

/* ------------------------------------------ Gram-Schmidt (linalg.dp.cpp) */
static double dot_seq(const double *a, const double *b, int n) {
  double r = 0;
  for (int i = 0; i < n; i++) r += a[i] * b[i];
  return r;
}
static double norm_seq(const double *v, int n) { return sqrt(dot_seq(v, v, n)); }

/* Classical GS with an accumulated projection sum (linalg.dp.cpp:36-51). */
static void ort_vecs(double *v, int n, int k, double *proj) {
  for (int i = 1; i < k; i++) {
    for (int j = 0; j < i; j++) {
      double c = dot_seq(&v[j * n], &v[i * n], n) / dot_seq(&v[j * n], &v[j * n], n);
      for (int q = 0; q < n; q++) proj[q] += c * v[j * n + q];
    }
    for (int q = 0; q < n; q++) {
      v[i * n + q] -= proj[q];
      proj[q] = 0;
    }
  }
}
/* linalg.dp.cpp:20-28 */
static void normalize_vecs(double *v, int n, int k, double eps) {
  for (int i = 0; i < k; i++) {
    double nr = norm_seq(&v[i * n], n);
    for (int q = 0; q < n; q++) v[i * n + q] = (v[i * n + q] / nr) * eps;
  }
}

/* qrDecomposition (linalg.dp.cpp:120-127) for a square rows == cols matrix:
 * CGS on the columns of the row-major matrix, unit columns, R = Q^T A. */
static void qr_decomp(double *R, double *Q, const double *A, int n, double *proj) {
  memcpy(Q, A, sizeof(double) * n * n);
  for (int i = 1; i < n; i++) {
    for (int j = 0; j < i; j++) {
      double num = 0, den = 0;
      for (int r = 0; r < n; r++) num += Q[j + r * n] * Q[i + r * n];
      for (int r = 0; r < n; r++) den += Q[j + r * n] * Q[j + r * n];
      double c = num / den;
      for (int r = 0; r < n; r++) proj[r] += c * Q[j + r * n];
    }
    for (int r = 0; r < n; r++) {
      Q[i + r * n] -= proj[r];
      proj[r] = 0;
    }
  }
  for (int i = 0; i < n; i++) {
    double s = 0;
    for (int r = 0; r < n; r++) s += Q[i + r * n] * Q[i + r * n];
    double nr = sqrt(s);
    for (int r = 0; r < n; r++) Q[i + r * n] = (Q[i + r * n] / nr) * 1;
  }
  /* R[i][j] = sum_q Q^T[i][q] A[q][j] = sum_q Q[q][i] A[q][j], summed from 0 */
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      double s = 0;
      for (int q = 0; q < n; q++) s += Q[q * n + i] * A[q * n + j];
      R[i * n + j] = s;
    }
}

/* -------------------------------------------- fixed-step methods (ref) */
typedef struct {
  int model, method, k;
  double eps, h, t_skip, t_skip_clp, calc_time, add_skip;
} fixed_cfg;

static void point_var(const fixed_cfg *c, const double *p, double *x, double *lyap) {
  const int n = orc_model_dim(c->model), k = c->k;
  double V[L96_N * L96_N], proj[L96_N], w[9 * L96_N];
  deriv_ctx fs = {c->model, 0, p, 0}, fv = {c->model, 1, p, x};
  int32_t skip = 0;
  double t;
  memset(proj, 0, sizeof proj);
  for (t = 0; t < c->t_skip; t += c->h) dverk_fixed(x, n, &fs, c->h, w);
  memset(V, 0, sizeof(double) * k * n);
  for (int i = 0; i < k; i++) V[i * n + i] += c->eps;
  for (t = 0; t < c->t_skip_clp; t += c->h) {
    for (int i = 0; i < k; i++) dverk_fixed(&V[i * n], n, &fv, c->h, w);
    dverk_fixed(x, n, &fs, c->h, w);
    ort_vecs(V, n, k, proj);
    normalize_vecs(V, n, k, c->eps);
  }
  for (t = 0; t < c->calc_time; t += c->h) {
    skip++;
    for (int i = 0; i < k; i++) dverk_fixed(&V[i * n], n, &fv, c->h, w);
    dverk_fixed(x, n, &fs, c->h, w);
    if (skip == c->add_skip) {
      ort_vecs(V, n, k, proj);
      for (int i = 0; i < k; i++) lyap[i] += log(norm_seq(&V[i * n], n) / c->eps);
      normalize_vecs(V, n, k, c->eps);
      skip = 0;
    }
  }
  for (int i = 0; i < k; i++) lyap[i] = lyap[i] / c->calc_time;
}

static void point_fd(const fixed_cfg *c, const double *p, double *x, double *lyap) {
  const int n = orc_model_dim(c->model), k = c->k;
  double S[L96_N * L96_N], proj[L96_N], w[9 * L96_N];
  deriv_ctx fs = {c->model, 0, p, 0};
  int32_t skip = 0;
  double t;
  memset(proj, 0, sizeof proj);
  for (t = 0; t < c->t_skip; t += c->h) dverk_fixed(x, n, &fs, c->h, w);
  for (int i = 0; i < k; i++) {
    memcpy(&S[i * n], x, sizeof(double) * n);
    S[i * n + i] += c->eps;
  }
  for (t = 0; t < c->t_skip_clp; t += c->h) {
    dverk_fixed(x, n, &fs, c->h, w);
    for (int i = 0; i < k; i++) {
      dverk_fixed(&S[i * n], n, &fs, c->h, w);
      for (int j = 0; j < n; j++) S[i * n + j] -= x[j];
    }
    ort_vecs(S, n, k, proj);
    normalize_vecs(S, n, k, c->eps);
    for (int i = 0; i < k; i++)
      for (int j = 0; j < n; j++) S[i * n + j] += x[j];
  }
  for (t = 0; t < c->calc_time; t += c->h) {
    skip++;
    dverk_fixed(x, n, &fs, c->h, w);
    for (int i = 0; i < k; i++) dverk_fixed(&S[i * n], n, &fs, c->h, w);
    if (skip == c->add_skip) {
      for (int i = 0; i < k; i++)
        for (int j = 0; j < n; j++) S[i * n + j] -= x[j];
      ort_vecs(S, n, k, proj);
      for (int i = 0; i < k; i++) lyap[i] += log(norm_seq(&S[i * n], n) / c->eps);
      normalize_vecs(S, n, k, c->eps);
      for (int i = 0; i < k; i++)
        for (int j = 0; j < n; j++) S[i * n + j] += x[j];
      skip = 0;
    }
  }
  for (int i = 0; i < k; i++) lyap[i] = lyap[i] / c->calc_time;
}

/* One map iteration through a scratch copy: cuda/tools/mapstep.dp.cpp:6-11
 * (StepMAP, ctx kind 0) and :13-19 (StepMAPVAR, kind 1). */
static void map_step(double *val, int n, const deriv_ctx *c) {
  double arg[L96_N];
  deriv(c, val, arg);
  for (int j = 0; j < n; j++) val[j] = arg[j];
}

/* cuda/lyapunov.dp.cpp:182-225: VAR map branch (double counters stepped by
 * 1, Gram-Schmidt and log-norms every iteration). */
static void point_var_map(const fixed_cfg *c, const double *p, double *x, double *lyap) {
  const int n = orc_model_dim(c->model), k = c->k;
  double V[L96_N * L96_N], proj[L96_N];
  deriv_ctx fs = {c->model, 0, p, 0}, fv = {c->model, 1, p, x};
  double t;
  memset(proj, 0, sizeof proj);
  for (t = 0; t < c->t_skip; t += 1) map_step(x, n, &fs);
  memset(V, 0, sizeof(double) * k * n);
  for (int i = 0; i < k; i++) V[i * n + i] += c->eps;
  for (t = 0; t < c->t_skip_clp; t += 1) {
    for (int i = 0; i < k; i++) map_step(&V[i * n], n, &fv);
    map_step(x, n, &fs);
    ort_vecs(V, n, k, proj);
    normalize_vecs(V, n, k, c->eps);
  }
  for (t = 0; t < c->calc_time; t += 1) {
    for (int i = 0; i < k; i++) map_step(&V[i * n], n, &fv);
    map_step(x, n, &fs);
    ort_vecs(V, n, k, proj);
    for (int i = 0; i < k; i++) lyap[i] += log(norm_seq(&V[i * n], n) / c->eps);
    normalize_vecs(V, n, k, c->eps);
  }
  for (int i = 0; i < k; i++) lyap[i] = lyap[i] / c->calc_time;
}

/* cuda/lyapunov.dp.cpp:70-128: FD map branch (int32_t counters compared
 * with the double times, renormalisation every iteration). */
static void point_fd_map(const fixed_cfg *c, const double *p, double *x, double *lyap) {
  const int n = orc_model_dim(c->model), k = c->k;
  double S[L96_N * L96_N], proj[L96_N];
  deriv_ctx fs = {c->model, 0, p, 0};
  memset(proj, 0, sizeof proj);
  for (int32_t t = 0; t < c->t_skip; t++) map_step(x, n, &fs);
  for (int i = 0; i < k; i++) {
    memcpy(&S[i * n], x, sizeof(double) * n);
    S[i * n + i] += c->eps;
  }
  for (int32_t t = 0; t < c->t_skip_clp; t++) {
    map_step(x, n, &fs);
    for (int i = 0; i < k; i++) {
      map_step(&S[i * n], n, &fs);
      for (int j = 0; j < n; j++) S[i * n + j] -= x[j];
    }
    ort_vecs(S, n, k, proj);
    normalize_vecs(S, n, k, c->eps);
    for (int i = 0; i < k; i++)
      for (int j = 0; j < n; j++) S[i * n + j] += x[j];
  }
  for (int32_t t = 0; t < c->calc_time; t++) {
    map_step(x, n, &fs);
    for (int i = 0; i < k; i++) map_step(&S[i * n], n, &fs);
    for (int i = 0; i < k; i++)
      for (int j = 0; j < n; j++) S[i * n + j] -= x[j];
    ort_vecs(S, n, k, proj);
    for (int i = 0; i < k; i++) lyap[i] += log(norm_seq(&S[i * n], n) / c->eps);
    normalize_vecs(S, n, k, c->eps);
    for (int i = 0; i < k; i++)
      for (int j = 0; j < n; j++) S[i * n + j] += x[j];
  }
  for (int i = 0; i < k; i++) lyap[i] = lyap[i] / c->calc_time;
}

static void point_qr(const fixed_cfg *c, const double *p, double *x, double *lyap) {
  const int n = orc_model_dim(c->model), nn = n * n;
  double *Q = malloc(sizeof(double) * nn * 12 + sizeof(double) * n);
  double *U = Q + nn, *R = U + nn, *w = R + nn, *proj = w + 9 * nn;
  deriv_ctx fs = {c->model, 0, p, 0}, fq = {c->model, 2, p, x};
  double t;
  double wx[9 * L96_N];
  memset(proj, 0, sizeof(double) * n);
  for (t = 0; t < c->t_skip; t += c->h) dverk_fixed(x, n, &fs, c->h, wx);
  memset(Q, 0, sizeof(double) * nn);
  for (int i = 0; i < n; i++) Q[i * n + i] = 1;
  for (t = c->t_skip; t < c->t_skip + c->calc_time; t += c->h) {
    dverk_fixed(x, n, &fs, c->h, wx);
    dverk_fixed(Q, nn, &fq, c->h, w);
    memcpy(U, Q, sizeof(double) * nn);
    qr_decomp(R, Q, U, n, proj);
    for (int i = 0; i < n; i++) lyap[i] += log(fabs(R[i * n + i]));
  }
  for (int i = 0; i < n; i++) lyap[i] = lyap[i] / c->calc_time;
  free(Q);
}

/* --------------------------------------------------------- thread pool */
typedef struct {
  atomic_llong next;
  int64_t P;
  void (*fn)(void *, int64_t);
  void *arg;
} pool_t;

static void *pool_worker(void *a) {
  pool_t *pl = (pool_t *)a;
  for (;;) {
    int64_t i = atomic_fetch_add(&pl->next, 1);
    if (i >= pl->P) break;
    pl->fn(pl->arg, i);
  }
  return 0;
}

static void run_parallel(int64_t P, int threads, void (*fn)(void *, int64_t), void *arg) {
  pool_t pl;
  atomic_init(&pl.next, 0);
  pl.P = P;
  pl.fn = fn;
  pl.arg = arg;
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  pthread_t th[256];
  pthread_attr_t attr;
  pthread_attr_init(&attr);
  pthread_attr_setstacksize(&attr, 16u << 20);
  int started = 0;
  for (int t = 1; t < threads; ++t)
    if (pthread_create(&th[started], &attr, pool_worker, &pl) == 0) started++;
  pool_worker(&pl);
  for (int t = 0; t < started; ++t) pthread_join(th[t], 0);
  pthread_attr_destroy(&attr);
}

typedef struct {
  fixed_cfg c;
  int m, n;
  const double *params;
  double *inits, *out;
} fixed_job;

static void fixed_point(void *a, int64_t i) {
  fixed_job *j = (fixed_job *)a;
  const double *p = j->params + i * j->m;
  double *x = j->inits + i * j->n, *o = j->out + i * j->c.k;
  for (int q = 0; q < j->c.k; q++) o[q] = 0;
  if (orc_model_is_map(j->c.model)) {
    if (j->c.method == ORC_VAR) point_var_map(&j->c, p, x, o);
    else point_fd_map(&j->c, p, x, o);
  } else if (j->c.method == ORC_VAR) point_var(&j->c, p, x, o);
  else if (j->c.method == ORC_FD) point_fd(&j->c, p, x, o);
  else point_qr(&j->c, p, x, o);
}

int orc_lyap_fixed(int model, int method, int64_t P, const double *params, double *inits,
                   double eps, double h, int k, double t_skip, double t_skip_clp,
                   double calc_time, double add_skip_steps, double *out, int threads) {
  const int n = orc_model_dim(model);
  if (n < 0 || P < 0 || k < 1 || k > n || !(h > 0)) return -1;
  if (method == ORC_QR && (k != n || orc_model_is_map(model))) return -1;
  if (method < ORC_FD || method > ORC_QR) return -1;
  fixed_job j = {{model, method, k, eps, h, t_skip, t_skip_clp, calc_time, add_skip_steps},
                 orc_model_nparams(model), n, params, inits, out};
  run_parallel(P, threads, fixed_point, &j);
  return 0;
}

/* ------------------------------------------------------ adaptive forms */
/* Joint system y = [x (n) | v_0 (n) | ... | v_{k-1} (n)], dv_i = J(x) v_i. */
static void joint_rhs(int model, int n, int k, const double *p, const double *y, double *dy) {
  model_f(model, y, dy, p);
  for (int i = 0; i < k; i++) model_var(model, y + n + i * n, dy + n + i * n, p, y);
}

/* DVERK: c and a-rows of cuda/tools/dverk.dp.cpp:13-39, 6th-order weights
 * :41, 5th-order weights of Verner's DVERK 6(5) pair. */
static const double DV_A[8][7] = {
    {0},
    {1. / 6.},
    {4. / 75., 16. / 75.},
    {5. / 6., -8. / 3., 5. / 2.},
    {-165. / 64., 55. / 6., -425. / 64., 85. / 96.},
    {12. / 5., -8., 4015. / 612., -11. / 36., 88. / 255.},
    {-8263. / 15000., 124. / 75., -643. / 680., -81. / 250., 2484. / 10625., 0.},
    {3501. / 1720., -300. / 43., 297275. / 52632., -319. / 2322., 24068. / 84065., 0.,
     3850. / 26703.}};
static const double DV_B6[8] = {3. / 40., 0., 875. / 2244., 23. / 72., 264. / 1955., 0.,
                                125. / 11592., 43. / 616.};
static const double DV_B5[8] = {13. / 160., 0., 2375. / 5984., 5. / 16., 12. / 85., 3. / 44., 0., 0.};

/* Dormand-Prince 5(4), cuda/tools/dopri.dp.cpp:14-44. */
static const double DP_A[7][6] = {
    {0},
    {0.2},
    {3. / 40., 9. / 40.},
    {44. / 45., -56. / 15., 32. / 9.},
    {19372. / 6561., -25360. / 2187., 64448. / 6561., -212. / 729.},
    {9017. / 3168., -355. / 33., 46732. / 5247., 49. / 176., -5103. / 18656.},
    {35. / 384., 0., 500. / 1113., 125. / 192., -2187. / 6784., 11. / 84.}};
static const double DP_E[7] = {71. / 57600., 0., -71. / 16695., 71. / 1920., -17253. / 339200.,
                               22. / 525., -1. / 40.};

typedef struct {
  const orc_adaptive_cfg *cfg;
  int n, k, N; /* N: components integrated (n or n(1+k)) */
  const double *p;
  double h, fac_old;
  int first, have_k1;
  int64_t steps;
  double *K; /* 8*N stage storage */
  double *y1, *tmp;
} integ_t;

/* One attempted step of length h from y; on success y <- y1 and returns 1. */
static int try_step(integ_t *s, double *y, double h, double *err_out) {
  const int N = s->N, n = s->n, k = (N == s->n) ? 0 : s->k;
  const int model = s->cfg->model;
  double *K = s->K, *arg = s->tmp, *y1 = s->y1;
  double err = 0;
  if (s->cfg->integrator == ORC_DVERK65) {
    joint_rhs(model, n, k, s->p, y, K);
    for (int st = 1; st < 8; st++) {
      for (int c = 0; c < N; c++) {
        double acc = 0;
        for (int q = 0; q < st; q++) acc += DV_A[st][q] * K[q * N + c];
        arg[c] = y[c] + h * acc;
      }
      joint_rhs(model, n, k, s->p, arg, K + st * N);
    }
    for (int c = 0; c < N; c++) {
      double a6 = 0, e = 0;
      for (int q = 0; q < 8; q++) {
        a6 += DV_B6[q] * K[q * N + c];
        e += (DV_B6[q] - DV_B5[q]) * K[q * N + c];
      }
      y1[c] = y[c] + h * a6;
      double sk = s->cfg->atol + s->cfg->rtol * fmax(fabs(y[c]), fabs(y1[c]));
      double r = h * e / sk;
      err += r * r;
    }
  } else {
    if (!s->have_k1) {
      joint_rhs(model, n, k, s->p, y, K);
      s->have_k1 = 1;
    }
    for (int st = 1; st < 7; st++) {
      for (int c = 0; c < N; c++) {
        if (st == 1) { /* dopri.dp.cpp:71: val + step * a21 * k1, no parentheses */
          arg[c] = y[c] + h * DP_A[1][0] * K[c];
          continue;
        }
        double acc = 0;
        for (int q = 0; q < st; q++) acc += DP_A[st][q] * K[q * N + c];
        arg[c] = y[c] + h * acc;
      }
      if (st == 6) memcpy(y1, arg, sizeof(double) * N);
      joint_rhs(model, n, k, s->p, arg, K + st * N);
    }
    for (int c = 0; c < N; c++) {
      double e = 0;
      for (int q = 0; q < 7; q++) e += DP_E[q] * K[q * N + c];
      double sk = s->cfg->atol + s->cfg->rtol * fmax(fabs(y[c]), fabs(y1[c]));
      double r = h * e / sk;
      err += r * r;
    }
  }
  err = sqrt(err / N);
  *err_out = err;
  return err <= 1.0;
}

/* The step-size controller of cuda/tools/dopri.dp.cpp:46-138 after an
 * attempted step of length h whose error norm is err: safety 0.9, the step
 * shrinks by at most 1 / fac1 = 5 and grows by at most 1 / fac2 = 10, PI
 * exponent expo1 = 1/q - 0.75 beta with beta = 0.04 (q = 5 for Dopri5, 6 for
 * DVERK 6(5)), previous error floored at 1e-4, the step after a rejection no
 * longer than the rejected one.  Returns 1 when the step is accepted (*hnext =
 * the next proposal), 0 when it is rejected (*hnext = the retry length). */
static int control(integ_t *s, double err, double h, double hmax, int *reject, double *hnext) {
  const double safe = 0.9, fac1 = 0.2, fac2 = 10., beta = 0.04;
  const double expo1 = (s->cfg->integrator == ORC_DVERK65 ? 1. / 6. : 0.2) - beta * 0.75;
  const double facc1 = 1. / fac1, facc2 = 1. / fac2;
  double fac11 = pow(err, expo1);
  double fac = fac11 / pow(s->fac_old, beta);
  fac = fmax(facc2, fmin(facc1, fac / safe));
  double hnew = h / fac;
  if (err <= 1.0) {
    s->fac_old = fmax(err, 1e-4);
    if (hnew > hmax) hnew = hmax;
    if (*reject) hnew = fmin(hnew, h);
    *reject = 0;
    *hnext = hnew;
    return 1;
  }
  *reject = 1;
  *hnext = h / fmin(facc1, fac11 / safe);
  return 0;
}

/* An attempt whose error norm is not finite.  From a finite point it is an
 * overflow (a step far beyond the stability bound, proposed after steps whose
 * error vanished); the reference's controller meets an infinite error with
 * its largest reduction, newStep = step / min(facc1, fac11 / safeFac) =
 * step / 5 (cuda/tools/dopri.dp.cpp:134), and so does this one, for NaN as
 * well.  A point whose parameters or state are not finite ends: returns 1
 * then, else 0 with the retry length in *hnext. */
static int nonfinite_error(const integ_t *s, const double *y, double h, int *reject,
                           double *hnext) {
  for (int i = 0; i < orc_model_nparams(s->cfg->model); i++)
    if (!isfinite(s->p[i])) return 1;
  for (int c = 0; c < s->n; c++)
    if (!isfinite(y[c])) return 1;
  *reject = 1;
  *hnext = h / 5.0;
  return 0;
}

/* Takes the attempted step: y <- y1 (and, for Dopri5, the FSAL derivative). */
static void take_step(integ_t *s, double *y) {
  memcpy(y, s->y1, sizeof(double) * s->N);
  if (s->cfg->integrator == ORC_DOPRI5) memcpy(s->K, s->K + 6 * s->N, sizeof(double) * s->N);
}

/* Integrates y over exactly `len` time units with the controller above.  A
 * step clamped to land on the end point does not shrink the proposal carried
 * on.  Returns 0, or the status code of the failure. */
static int integrate(integ_t *s, double *y, double len) {
  const double hmax = s->cfg->hmax > 0 ? s->cfg->hmax : 1e300;
  double t = 0;
  int reject = 0;
  if (s->steps == 0 && s->cfg->escape > 0) /* an initial state outside the escape radius */
    for (int c = 0; c < s->n; c++)
      if (!(fabs(y[c]) <= s->cfg->escape)) return 4;
  while (t < len) {
    if (s->steps >= s->cfg->max_steps) return 3;
    if (s->h < s->cfg->hmin) return 2;
    double remaining = len - t;
    int clamped = s->h >= remaining;
    double h = clamped ? remaining : s->h;
    double err, hnew;
    s->steps++;
    try_step(s, y, h, &err);
    if (!isfinite(err)) {
      if (nonfinite_error(s, y, h, &reject, &s->h)) return 1;
      continue;
    }
    if (control(s, err, h, hmax, &reject, &hnew)) {
      take_step(s, y);
      t = clamped ? len : t + h;
      if (!clamped || hnew < h) s->h = hnew; /* else keep the unclamped proposal */
      if (s->cfg->escape > 0)
        for (int c = 0; c < s->n; c++)
          if (!(fabs(y[c]) <= s->cfg->escape)) return 4;
    } else {
      s->h = hnew;
    }
  }
  return 0;
}

int orc_dopri_trajectory(int model, const double *p, const double *x0, double h0, double hmax,
                         double atol, double rtol, int nsteps, double *t_out, double *h_out,
                         double *x_out) {
  const int n = orc_model_dim(model);
  if (n < 0 || orc_model_is_map(model) || nsteps < 0 || !(h0 > 0)) return -1;
  orc_adaptive_cfg cfg = {model, 0, ORC_DOPRI5, ORC_CGS, rtol, atol, h0, hmax, 0.0,
                          0.0, 0.0, 1.0, 1.0, INT64_MAX, 0.0};
  double buf[12 * L96_N];
  double *y = buf, *K = y + n, *y1 = K + 8 * n, *tmp = y1 + n;
  integ_t s = {&cfg, n, 0, n, p, h0, 1e-4, 1, 0, 0, K, y1, tmp};
  double t = 0;
  memcpy(y, x0, sizeof(double) * n);
  for (int i = 0; i < nsteps; i++) {
    int reject = 0, ok = 0;
    while (!ok) { /* one accepted step, rejected attempts retried */
      const double h = s.h;
      double err, hnew;
      s.steps++;
      try_step(&s, y, h, &err);
      if (!isfinite(err)) {
        if (nonfinite_error(&s, y, h, &reject, &s.h)) return 1;
        continue;
      }
      ok = control(&s, err, h, hmax, &reject, &hnew);
      if (ok) {
        take_step(&s, y);
        t += h;
      }
      s.h = hnew;
    }
    t_out[i] = t;
    h_out[i] = s.h;
    memcpy(x_out + (size_t)i * n, y, sizeof(double) * n);
  }
  return 0;
}

typedef struct {
  const orc_adaptive_cfg *cfg;
  int m, n;
  const double *params, *inits;
  double *out;
  int32_t *status;
  int64_t *steps;
} adapt_job;

static void adaptive_point(void *a, int64_t i) {
  adapt_job *j = (adapt_job *)a;
  const orc_adaptive_cfg *cfg = j->cfg;
  const int n = j->n, k = cfg->k, Nj = n * (1 + k);
  double *buf = malloc(sizeof(double) * (size_t)Nj * 12);
  double *y = buf, *K = y + Nj, *y1 = K + 8 * Nj, *tmp = y1 + Nj;
  long double sums[L96_N];
  double r[L96_N];
  integ_t s = {cfg, n, k, n, j->params + i * j->m, cfg->h0 > 0 ? cfg->h0 : 1e-3, 1e-4, 1, 0, 0,
               K, y1, tmp};
  int st = 0;
  double *o = j->out + i * k;
  memcpy(y, j->inits + i * n, sizeof(double) * n);
  for (int q = 0; q < k; q++) sums[q] = 0;

  if (cfg->t_transient > 0) st = integrate(&s, y, cfg->t_transient);
  /* tangent basis = first k columns of the identity */
  memset(y + n, 0, sizeof(double) * n * k);
  for (int q = 0; q < k; q++) y[n + q * n + q] = 1.0;
  s.N = Nj;
  s.fac_old = 1e-4;
  const double total = cfg->t_align + cfg->t_avg;
  /* Renormalisation sub-intervals, the same per-point policy as the device
   * kernels: each dt_renorm interval is split into m equal parts, m doubled
   * when one part's log-norm spread exceeds tau = 0.3 ln(1/max(rtol, u)),
   * halved when below tau / 4 (m in 1..64, starting at 16). */
  const float tau = 0.3f * logf(1.0f / fmaxf((float)cfg->rtol, 1.2e-16f));
  int m = 16;
  double t = 0;
  while (!st && t < total) {
    double len = cfg->dt_renorm;
    if (t + len > total) len = total - t;
    const double sub = len / m;
    float max_spread = 0.f;
    for (int jj = 0; jj < m; jj++) {
      const double l = (jj == m - 1) ? len - sub * (m - 1) : sub;
      s.have_k1 = 0;
      st = integrate(&s, y, l);
      if (st) break;
      /* Gram-Schmidt on the tangent vectors (CGS as linalg.dp.cpp:36-51, or MGS) */
      double *V = y + n;
      for (int q = 0; q < k; q++) {
        double *vq = V + q * n;
        if (cfg->gs == ORC_MGS) {
          for (int pq = 0; pq < q; pq++) {
            double c = dot_seq(V + pq * n, vq, n);
            for (int c2 = 0; c2 < n; c2++) vq[c2] -= c * V[pq * n + c2];
          }
        } else {
          double proj[L96_N];
          for (int c2 = 0; c2 < n; c2++) proj[c2] = 0;
          for (int pq = 0; pq < q; pq++) {
            double c = dot_seq(V + pq * n, vq, n);
            for (int c2 = 0; c2 < n; c2++) proj[c2] += c * V[pq * n + c2];
          }
          for (int c2 = 0; c2 < n; c2++) vq[c2] -= proj[c2];
        }
        r[q] = norm_seq(vq, n);
        for (int c2 = 0; c2 < n; c2++) vq[c2] /= r[q];
      }
      for (int q = 0; q < k; q++)
        if (!isfinite(r[q]) || r[q] <= 0) st = 1;
      if (st) break;
      double lmax = -1e300, lmin = 1e300;
      for (int q = 0; q < k; q++) {
        double lg = log(r[q]);
        lmax = fmax(lmax, lg);
        lmin = fmin(lmin, lg);
      }
      if ((float)(lmax - lmin) > max_spread) max_spread = (float)(lmax - lmin);
      if (t + sub * (jj + 1) > cfg->t_align + 1e-12 * total)
        for (int q = 0; q < k; q++) sums[q] += logl((long double)r[q]);
    }
    t += len;
    if (max_spread > tau && m < 64) m *= 2;
    else if (max_spread < 0.25f * tau && m > 1) m /= 2;
  }
  for (int q = 0; q < k; q++) o[q] = st ? NAN : (double)(sums[q] / (long double)cfg->t_avg);
  if (j->status) j->status[i] = st;
  if (j->steps) j->steps[i] = s.steps;
  free(buf);
}

int orc_lyap_adaptive(const orc_adaptive_cfg *cfg, int64_t P, const double *params,
                      const double *inits, double *out, int32_t *status, int64_t *steps,
                      int threads) {
  const int n = orc_model_dim(cfg->model);
  if (n < 0 || P < 0 || cfg->k < 1 || cfg->k > n || !(cfg->dt_renorm > 0) || !(cfg->t_avg > 0))
    return -1;
  if (orc_model_is_map(cfg->model)) return -1; /* maps are iterated, not integrated */
  adapt_job j = {cfg, orc_model_nparams(cfg->model), n, params, inits, out, status, steps};
  run_parallel(P, threads, adaptive_point, &j);
  return 0;
}

/* ------------------------------------------------------ inputs (grid, RNG) */
static uint64_t mulhilo64(uint64_t a, uint64_t b, uint64_t *hi) {
  unsigned __int128 p = (unsigned __int128)a * b;
  *hi = (uint64_t)(p >> 64);
  return (uint64_t)p;
}

void orc_philox4x64(const uint64_t ctr[4], const uint64_t key[2], uint64_t out[4]) {
  uint64_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    uint64_t hi0, hi1;
    uint64_t lo0 = mulhilo64(0xD2E7470EE14C6C93ULL, c0, &hi0);
    uint64_t lo1 = mulhilo64(0xCA5A826395121157ULL, c2, &hi1);
    uint64_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B97F4A7C15ULL;
    k1 += 0xBB67AE8584CAA73BULL;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

int64_t orc_make_grid(int m, const double *base, const double s1[4], const double s2[4],
                      double *out) {
  const int n1 = (int)s1[3], n2 = (int)s2[3];
  const double d1 = fabs(s1[2] - s1[1]) / (s1[3] - 1), d2 = fabs(s2[2] - s2[1]) / (s2[3] - 1);
  int64_t c = 0;
  for (int a = 0; a < n1; a++)
    for (int b = 0; b < n2; b++) {
      double v1 = s1[1] + a * d1, v2 = s2[1] + b * d2;
      for (int i = 0; i < m; i++) {
        double v = base[i];
        if (i == (int)s1[0]) v = v1;
        else if (i == (int)s2[0]) v = v2;
        out[c * m + i] = v;
      }
      c++;
    }
  return c;
}

/* 53-bit uniform in [0,1) from a 64-bit word */
static double u53(uint64_t w) { return (double)(w >> 11) * (1.0 / 9007199254740992.0); }

void orc_make_inits(int n, int64_t P, const double *base, double amp, int dist, uint64_t seed,
                    double *out) {
  const uint64_t key[2] = {seed, 0x6368616F735F6C79ULL};
  for (int64_t p = 0; p < P; p++) {
    for (int blk = 0; blk * 4 < n; blk++) {
      uint64_t ctr[4] = {(uint64_t)p, (uint64_t)blk, 0, 0}, r[4];
      orc_philox4x64(ctr, key, r);
      for (int q = 0; q < 4 && blk * 4 + q < n; q++) {
        int c = blk * 4 + q;
        double d;
        if (dist == 0) {
          d = (2.0 * u53(r[q]) - 1.0) * amp;
        } else {
          /* Box-Muller on the pair (r[q & ~1], r[q | 1]) */
          double u1 = 1.0 - u53(r[q & ~1]), u2 = u53(r[q | 1]);
          double rad = sqrt(-2.0 * log(u1));
          d = amp * ((q & 1) ? rad * sin(6.283185307179586 * u2) : rad * cos(6.283185307179586 * u2));
        }
        out[p * n + c] = base[c] + d;
      }
    }
  }
}
