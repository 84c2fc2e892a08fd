/* chaos_lyap host surface: the reference program's flow (main.cpp:11-80:
 * config.json -> LyapunovParameters -> TaskLyapunov -> Data/Lyapunov <model>.json)
 * as C entry points over libchaos_lyap.so.  The C++ classes behind them mirror
 * the reference's (ModelFactoryRegistry, LyapunovParameters, ConfigFactory,
 * TaskLyapunov, saveCalculatedData) and are declared in
 * chaos_oneapi_b200/host/*.h. */
#ifndef CHAOS_LYAP_HOST_H
#define CHAOS_LYAP_HOST_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The whole run of the reference's main() (main.cpp:11-80) for one model:
 * reads the config, sweeps on config's num_GPUs devices, writes
 * <out_dir>/Lyapunov <model>.json (+ .npy with full precision).  verbose:
 * print the parameters and the time report like the reference.  Returns 0,
 * or -1 with a message on stderr. */
int chaos_host_run_config(const char *config_path, const char *model, const char *out_dir,
                          int verbose);

/* TaskLyapunov::allocate's host half (tasklyapunov.cpp:45-71) without a
 * device: the parameter grid (P x nparams) and initial states (P x dim),
 * point-major.  *P_out receives the point count; the arrays may be NULL to
 * query it. */
int chaos_host_plan(const char *config_path, const char *model, double *params_out,
                    double *inits_out, int64_t *P_out);

/* The output writer (filehandler.cpp:35-89) for a spectrum computed
 * elsewhere (P x k, point-major), rows built as TaskLyapunov::execute does. */
int chaos_host_save(const char *config_path, const char *model, const double *spectrum,
                    const char *out_dir);

#ifdef __cplusplus
}
#endif
#endif
