/* Test infrastructure only: the oracle.  A CPU restatement, in plain C, of the
 * reference's Lyapunov-spectrum path (cuda/lyapunov.dp.cpp,
 * cuda/tools/dverk.dp.cpp, cuda/tools/dopri.dp.cpp, cuda/tools/linalg.dp.cpp)
 * plus the adaptive forms built on it.  Only tests, the smoke check and the
 * bench's CPU-baseline leg use it, to compare against; the product never links it.
 *
 * Pinned: the fixed-step methods are checked bit for bit against the
 * reference's own sources compiled on the host (oracle/_ref, recipe in
 * oracle/Makefile) and against fixtures generated from them
 * (tests/golden/make_golden.py).
 */
#ifndef LYAP_ORACLE_H
#define LYAP_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_SHIMIZU = 0, ORC_LORENZ = 1, ORC_ROSSLER = 2, ORC_CHUA = 3, ORC_HYPER_ROSSLER = 4,
       ORC_LORENZ96 = 5, ORC_HENON = 6, ORC_NMODELS = 7 };
enum { ORC_FD = 0, ORC_VAR = 1, ORC_QR = 2 };
enum { ORC_DVERK65 = 0, ORC_DOPRI5 = 1 };
enum { ORC_CGS = 0, ORC_MGS = 1 };

int orc_model_dim(int model);
int orc_model_nparams(int model);
/* 1 for map-type models (iterated: cuda/tools/mapstep.dp.cpp:6-19). */
int orc_model_is_map(int model);

/* One fixed DVERK step of the state, in the reference's operation order
 * (cuda/tools/dverk.dp.cpp:7-43). */
void orc_dverk_step(int model, double *x, const double *p, double h);

/* Fixed-step reference methods (cuda/lyapunov.dp.cpp:5-259); map models take
 * the FD / VAR map branches (:70-125, :182-222; no QR).
 * params P*m and inits P*n are point-major; inits are advanced in place to the
 * end states; out is P*k.  Returns 0, or -1 on bad arguments. */
int orc_lyap_fixed(int model, int method, int64_t P, const double *params, double *inits,
                   double eps, double h, int k, double t_skip, double t_skip_clp,
                   double calc_time, double add_skip_steps, double *out, int threads);

/* Adaptive forms: transient (state only), then the state and its k tangent
 * vectors integrated jointly (variational equations at the stage states),
 * renormalised by Gram-Schmidt at every multiple of dt_renorm; the first
 * t_align time units renormalise without accumulating; log-norms summed in
 * long double over t_avg.  status: 0 ok, 1 non-finite, 2 step underflow,
 * 3 step budget exhausted, 4 escaped.  steps (optional) receives accepted+rejected. */
typedef struct {
  int model, k, integrator, gs;
  double rtol, atol, h0, hmax, hmin;
  double t_transient, t_align, t_avg, dt_renorm;
  int64_t max_steps;
  double escape; /* status 4 once a state component exceeds it (<= 0: never) */
} orc_adaptive_cfg;

int orc_lyap_adaptive(const orc_adaptive_cfg *cfg, int64_t P, const double *params,
                      const double *inits, double *out, int32_t *status, int64_t *steps,
                      int threads);

/* The state alone under Dormand-Prince 5(4) with the controller of the
 * adaptive forms (cuda/tools/dopri.dp.cpp:46-138), stepped the way the
 * reference's dopriStep is called: time from 0, one accepted step per entry
 * (rejections retried), no end point to land on.  After step i: t_out[i] =
 * time, h_out[i] = the next step's proposal, x_out[i*n..] = the state.
 * Returns 0, 1 on a non-finite error norm, or -1 on bad arguments. */
int orc_dopri_trajectory(int model, const double *p, const double *x0, double h0, double hmax,
                         double atol, double rtol, int nsteps, double *t_out, double *h_out,
                         double *x_out);

/* Philox4x64-10 (Salmon et al., SC'11): out[4] = philox(ctr[4], key[2]). */
void orc_philox4x64(const uint64_t ctr[4], const uint64_t key[2], uint64_t out[4]);

/* Sweep grid in the reference's order (tasklyapunov.cpp:45-63): p1 outer,
 * p2 inner, delta = |end-start|/(count-1).  sweep = {index, start, end, count}.
 * params_out P*m point-major.  Returns P. */
int64_t orc_make_grid(int m, const double *base_params, const double sweep1[4],
                      const double sweep2[4], double *params_out);

/* Seeded per-point initial states, point-major P*n: base + U(-amp, amp) when
 * dist == 0, base + N(0, amp^2) when dist == 1. */
void orc_make_inits(int n, int64_t P, const double *base, double amp, int dist, uint64_t seed,
                    double *inits_out);

#ifdef __cplusplus
}
#endif
#endif
