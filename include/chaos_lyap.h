/* chaos_lyap: C ABI of the B200 Lyapunov-spectrum sweep.
 *
 * Plain C types only (pointers, sizes, doubles); every function returns an
 * int status (CHAOS_LYAP_OK == 0) and never throws.  A human-readable message
 * for the last failure on the calling thread is available from
 * chaos_lyap_last_error().
 *
 * The reference's only boundary on this path is the C++ launcher
 *   void cudaLyapunov(int bn, int bs, size_t taskNum, bool isQr, bool isVar,
 *                     ModelType, double* inits, double* closePoints, int32_t dim,
 *                     diffSysFunc, diffSysFuncVar, diffSysFuncVar, double* params,
 *                     int32_t paramsDim, double eps, double step, double* lyapExps,
 *                     int32_t expsNum, double timeSkip, double timeSkipClP,
 *                     double calcTime, double addSkipSteps, <28 scratch pointers>)
 * (reference cuda/lyapunov.dp.hpp:10-17, cuda/lyapunov.dp.cpp:321-367), called
 * only by TaskLyapunov::execute (tasklyapunov.cpp:204-208), plus the model
 * registry lookups TaskLyapunov::init / execute make
 * (tasklyapunov.cpp:15-16,195-203; model_factory.h:22-68).
 */
#ifndef CHAOS_LYAP_H
#define CHAOS_LYAP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CHAOS_LYAP_ABI_VERSION 1

/* ------------------------------------------------------------- statuses */
enum {
  CHAOS_LYAP_OK = 0,
  CHAOS_LYAP_EINVAL = 1,       /* bad argument (null pointer, size, option) */
  CHAOS_LYAP_ENOMODEL = 2,     /* unknown model name */
  CHAOS_LYAP_EUNSUPPORTED = 3, /* valid but not provided combination */
  CHAOS_LYAP_ECUDA = 4,        /* CUDA runtime error (message has details) */
  CHAOS_LYAP_ENOMEM = 5        /* device allocation failed */
};

/* Per-point status written by the sweeps (status_out arrays). */
enum {
  CHAOS_POINT_OK = 0,
  CHAOS_POINT_NONFINITE = 1,      /* NaN / Inf in the state or a log-norm */
  CHAOS_POINT_STEP_UNDERFLOW = 2, /* adaptive step fell below h_min */
  CHAOS_POINT_MAX_STEPS = 3,      /* per-point step budget exhausted */
  CHAOS_POINT_ESCAPED = 4         /* a state component outside |x| <= escape (after a
                                     step, or the initial state) */
};

/* Methods: reference cuda/lyapunov.dp.cpp:5-129 (FD, slave trajectories),
 * :133-226 (VAR, variational equations), :229-259 (QR on J*Q). */
enum { CHAOS_METHOD_FD = 0, CHAOS_METHOD_VAR = 1, CHAOS_METHOD_QR = 2 };

/* Integrators: the reference's fixed-step DVERK (cuda/tools/dverk.dp.cpp),
 * adaptive DVERK 6(5), adaptive Dormand-Prince 5(4) (cuda/tools/dopri.dp.cpp). */
enum { CHAOS_INTEG_DVERK_FIXED = 0, CHAOS_INTEG_DVERK65 = 1, CHAOS_INTEG_DOPRI5 = 2 };

/* Precision forms.
 *  COMPAT_FP64: the reference's arithmetic operation by operation (fixed-step
 *               DVERK only); bit-identical trajectories to the reference.
 *  FP64:        state and tangent in FP64 (adaptive integrators).
 *  FP32:        state and tangent in FP32; Gram-Schmidt and the compensated
 *               log-norm sums in FP64. */
enum { CHAOS_PREC_COMPAT_FP64 = 0, CHAOS_PREC_FP64 = 1, CHAOS_PREC_FP32 = 2 };

enum { CHAOS_GS_CLASSICAL = 0, CHAOS_GS_MODIFIED = 1 };

/* Memory layout of the params / inits / spectrum arrays.
 *  POINT_MAJOR: element (point, c) at a[point * C + c]   (the reference's)
 *  COMP_MAJOR:  element (point, c) at a[c * P + point]   (SoA) */
enum { CHAOS_LAYOUT_POINT_MAJOR = 0, CHAOS_LAYOUT_COMP_MAJOR = 1 };

/* Launch schedule for the adaptive forms of the 3-4-dimensional models.
 *  DIRECT / PERSISTENT: one lane per point; thread i takes point i, or
 *    threads pull points from a device work queue.
 *  SPLIT_DIRECT / SPLIT_PERSISTENT: one point per group of four lanes (each
 *    lane the state and one tangent vector): about half the work per lane and
 *    step, for sweeps of few points or runs bounded by their longest point.
 *    A batch runs each segment in the form of its handle's schedule; with
 *    both forms present the two batch kernels run side by side, the split
 *    one first and at the greatest stream priority.
 *  AUTO: persistent until chaos_lyap_autotune picks one. */
enum {
  CHAOS_SCHED_AUTO = 0,
  CHAOS_SCHED_DIRECT = 1,
  CHAOS_SCHED_PERSISTENT = 2,
  CHAOS_SCHED_SPLIT_DIRECT = 3,
  CHAOS_SCHED_SPLIT_PERSISTENT = 4
};

/* Sweep description.  Times are in model time units.  Fields mirror the
 * reference's LyapunovParameters (tool_params.h:23-44): eps = epsilon,
 * h = integration_step, t_transient = skip_time_attractor, t_align =
 * skip_time_slave_trajectory, dt_renorm = skip_time_normalization, t_avg =
 * total_time, k = lyapunov_exponent_num, method = using_qr / using_var.
 * Map models (type 1) take compat precision and FD or VAR; their times are
 * iteration counts and they renormalise every iteration, as the reference's
 * map branches do (cuda/lyapunov.dp.cpp:70-125,182-222). */
typedef struct chaos_lyap_desc {
  int32_t struct_size;      /* sizeof(chaos_lyap_desc) */
  char model[32];           /* registered model name, e.g. "lorenz" */
  int32_t method;           /* CHAOS_METHOD_* */
  int32_t integrator;       /* CHAOS_INTEG_* */
  int32_t precision;        /* CHAOS_PREC_* */
  int32_t gs;               /* CHAOS_GS_* (adaptive forms) */
  int32_t k;                /* number of exponents (1..dim) */
  int32_t layout;           /* CHAOS_LAYOUT_* */
  double eps;               /* compat: perturbation / tangent length */
  double h;                 /* compat: fixed step; adaptive: initial step */
  double rtol, atol;        /* adaptive tolerances */
  double h_max, h_min;      /* adaptive step bounds (0: unbounded / 0) */
  double t_transient, t_align, t_avg, dt_renorm;
  int64_t max_steps;        /* adaptive: per-point budget of attempted steps */
  int32_t device;           /* CUDA device ordinal */
  int32_t schedule;         /* CHAOS_SCHED_* */
  int32_t block;            /* threads per block, 0 = tuned default */
  int32_t variant;          /* 0 = default.  1 = FP32 one-lane kernels: the 96-register
                               build (more resident warps, a few spills); FP64 split
                               kernels of 3-dimensional models: the exchange layout
                               (the state in one lane of the group, the vectors in the
                               others); autotuned */
  double escape;            /* adaptive: escape radius of the state (0: 1e4) */
  int32_t reserved[4];
} chaos_lyap_desc;

typedef struct chaos_lyap_handle chaos_lyap_handle;

/* Library ABI version (CHAOS_LYAP_ABI_VERSION). */
int chaos_lyap_abi_version(void);

/* Message of the last failing call on this thread ("" if none). */
const char *chaos_lyap_last_error(void);

/* Fills desc with defaults: VAR, DVERK 6(5), FP64, classical GS, k = 0
 * (= model dimension at create), point-major, eps 1e-7, h 1e-3, rtol = atol
 * = 1e-10, max_steps 1e8, escape radius 1e4. */
int chaos_lyap_desc_init(chaos_lyap_desc *desc);

/* Model registry (replaces the registry lookups of tasklyapunov.cpp:15-16 and
 * the function-pointer fetches of tasklyapunov.cpp:195-203; the reference's
 * registry is model_factory.h:22-68).  type: 0 flow, 1 map. */
int chaos_lyap_model_count(void);
int chaos_lyap_model_name(int index, char *buf, int buflen);
int chaos_lyap_query_model(const char *name, int32_t *dim, int32_t *nparams, int32_t *type);
/* Description strings the output writer stores (filehandler.cpp:70-76):
 * which: 0 parameter names, 1 phase variable names, 2 equations. */
int chaos_lyap_model_text(const char *name, int which, char *buf, int buflen);

/* Creates a sweep handle for one device (what TaskLyapunov::allocate does
 * for one GPU, tasklyapunov.cpp:104-176, without the per-work-item scratch:
 * the kernels keep their working state on chip). */
int chaos_lyap_create(const chaos_lyap_desc *desc, chaos_lyap_handle **out);
int chaos_lyap_destroy(chaos_lyap_handle *h);

/* Stream-ordered sweep over P points, DEVICE pointers (replaces
 * cudaLyapunov's launch, cuda/lyapunov.dp.cpp:339-366).
 *   params   P x nparams (layout per desc)
 *   inits    P x dim; compat precision advances them in place to the end
 *            states (as the reference does); adaptive forms only read them
 *   spectrum P x k output
 *   status   optional P int32 (CHAOS_POINT_*)
 *   steps    optional P int64 attempted steps (adaptive forms)
 *   t_avg_per_point optional P doubles (adaptive forms): per-point averaging
 *            time overriding desc.t_avg
 *   stream   cudaStream_t (NULL = legacy default stream)
 * Returns after enqueueing; chaos_lyap_sync() waits. */
int chaos_lyap_run(chaos_lyap_handle *h, int64_t P, const double *params, double *inits,
                   double *spectrum, int32_t *status, int64_t *steps,
                   const double *t_avg_per_point, void *stream);

/* Same sweep with HOST buffers: copies in, runs, copies out and waits.
 * Device staging buffers are owned by the handle and reused across calls. */
int chaos_lyap_run_host(chaos_lyap_handle *h, int64_t P, const double *params, double *inits,
                        double *spectrum, int32_t *status, int64_t *steps,
                        const double *t_avg_per_point);

/* Waits for the handle's last stream and reports a CUDA error, if any. */
int chaos_lyap_sync(chaos_lyap_handle *h);

/* Picks the launch shape (block size, direct vs persistent work queue, grid
 * of the persistent form, one lane or four lanes per point, kernel variant)
 * by timing short runs on `sample` points of the given device inputs: every
 * shape over 20 renormalisation intervals, then the shapes within 15 % of
 * the fastest over a horizon four times longer.  Stores the choice in the
 * handle.  Returns the chosen block size in *block_out and schedule in
 * *schedule_out when non-null. */
int chaos_lyap_autotune(chaos_lyap_handle *h, int64_t sample, const double *params,
                        const double *inits, int32_t *block_out, int32_t *schedule_out);

/* The same over a whole map of P points: the sample is every (P / sample)-th
 * point, spread over the map instead of its first rows (a map's cost varies
 * across it: chaotic bands, escaping corners). */
int chaos_lyap_autotune_map(chaos_lyap_handle *h, int64_t P, int64_t sample,
                            const double *params, const double *inits, int32_t *block_out,
                            int32_t *schedule_out);

/* ---------------------------------------------------------- mixed batches
 * Several sweeps (segments: different 3- or 4-dimensional models, each with
 * its own handle, arrays and phase times; per-point averaging times allowed)
 * in ONE persistent launch whose lanes take points segment after segment, so
 * points of uneven dimension and length share warps without idling them.
 * All handles must use the same integrator and precision; nseg <= 8; every
 * segment has its own handle (a handle in two segments is rejected).  The
 * point counters live in the first segment's handle: do not run that handle
 * on another stream while a batch on it is in flight.  No reference
 * counterpart (the reference launches one model per run, tasklyapunov.cpp:204). */
typedef struct chaos_lyap_segment {
  chaos_lyap_handle *handle;
  int64_t P;
  const double *params;
  const double *inits;
  double *spectrum;
  int32_t *status;               /* optional */
  int64_t *steps;                /* optional */
  const double *t_avg_per_point; /* optional */
} chaos_lyap_segment;

int chaos_lyap_run_batch(const chaos_lyap_segment *segs, int nseg, void *stream);

/* The same batch captured once into a CUDA graph (counter reset + launch)
 * and replayed by chaos_lyap_graph_launch on any stream; the segments'
 * arrays are baked in: refill them and replay.  The graph owns the buffers
 * of its longest-first orderings, so later runs of its handles do not
 * disturb it. */
typedef struct chaos_lyap_graph chaos_lyap_graph;
int chaos_lyap_batch_graph_create(const chaos_lyap_segment *segs, int nseg, chaos_lyap_graph **out);
int chaos_lyap_graph_launch(chaos_lyap_graph *g, void *stream);
int chaos_lyap_graph_destroy(chaos_lyap_graph *g);

/* The mixed batch above for callers that cannot allocate device memory while
 * they run: their device memory belongs to their own allocator, or an
 * allocation (and the synchronisation a free implies) would stall a real-time
 * loop, or their plugin host forbids device allocations.  No counterpart in
 * the reference.  Takes one descriptor per segment instead of handles
 * (segs[i].handle is ignored) and allocates nothing: the batch kernel's point
 * counters live in a fixed 8-entry device array inside the library, which
 * every GPU that loads it holds until the process exits, so nseg > 8 is
 * rejected.  All calls share those counters: calls that overlap on the GPU
 * race, so serialise them.  Each call zeroes the counters it uses on `stream`
 * before launching.  The first call on a device looks up the array's device
 * address; make it before any stream capture begins.  That address is kept
 * for the life of the process: the entry point does not survive a device
 * reset (cudaDeviceReset).  Descriptors are checked as chaos_lyap_create
 * checks them.  On failure the message is in chaos_lyap_static_last_error(). */
int chaos_lyap_run_batch_static(const chaos_lyap_desc *descs, const chaos_lyap_segment *segs,
                                int nseg, void *stream);
const char *chaos_lyap_static_last_error(void);

/* State trajectories through the adaptive integrators: the reference's
 * Dormand-Prince tool dopriStep (cuda/tools/dopri.dp.cpp:7-139, declared in
 * cuda/tools/dopri.dp.hpp:7-8) as a batched call, one lane per point.  A
 * caller of dopriStep starts at time 0 and makes one accepted step per call
 * (rejections retried inside), keeping the step proposal and the FSAL
 * derivative between calls; here every point makes `nsteps` such steps of
 * the STATE alone with the handle's integrator (DOPRI5 as the reference,
 * or DVERK65), precision (FP64: error norm and controller in FP64, the
 * reference's arithmetic to rounding; FP32), rtol / atol (the reference's
 * tolGlobErr / tolLocErr), h (initial step), h_max (maxStep; 0 = unbounded),
 * h_min, max_steps (attempted steps) and escape radius.  DEVICE pointers:
 *   params  P x nparams, inits P x dim (layout per desc)
 *   t_out   P x nsteps time after each accepted step
 *   h_out   P x nsteps the step proposal after it
 *   x_out   P x nsteps x dim the state after it (point-major)
 *   status  optional P int32 (CHAOS_POINT_*); records a point did not reach
 *           are NaN.
 * Flows of dimension <= 4.  Stream-ordered; returns after enqueueing. */
int chaos_lyap_trajectory(chaos_lyap_handle *h, int64_t P, const double *params,
                          const double *inits, int32_t nsteps, double *t_out, double *h_out,
                          double *x_out, int32_t *status, void *stream);

/* The kernel variant in use (desc.variant, or the autotuner's choice). */
int chaos_lyap_get_variant(chaos_lyap_handle *h, int32_t *variant);

/* Drop-in for the reference launcher cudaLyapunov (cuda/lyapunov.dp.hpp:10-17)
 * with the same argument meaning, DEVICE pointers, point-major layout:
 *   - the model is named instead of passed as three device function
 *     pointers (diffFunc / diffFuncVar / diffFuncVarQ);
 *   - the 28 scratch pointers are gone (state stays on chip);
 *   - bn / bs are accepted and ignored (the reference also overrides them,
 *     cuda/lyapunov.dp.cpp:331-332);
 *   - lyapExps is accumulated into, exactly like the reference
 *     (cuda/lyapunov.dp.cpp:169,253): zero it for a plain result;
 *   - inits and closePoints are written like the reference writes them;
 *   - modelType (0 flow, 1 map) must be the named model's type; maps run the
 *     reference's FD / VAR map branches (cuda/lyapunov.dp.cpp:70-125,
 *     182-222), and QR on a map is rejected (the reference has no QR map
 *     branch).
 * Arithmetic is the compat FP64 form (bit-identical trajectories).
 * Enqueued on `stream`; returns after the launch. */
int chaos_lyap_cudaLyapunov(int bn, int bs, size_t taskNum, int isQr, int isVar, int modelType,
                            double *inits, double *closePoints, int32_t dimension,
                            const char *model, double *params, int32_t paramsDim, double eps,
                            double integrationStep, double *lyapExps, int32_t expsNum,
                            double timeSkip, double timeSkipClP, double calcTime,
                            double addSkipSteps, void *stream);

/* Host-side inputs in the reference's conventions (TaskLyapunov::allocate,
 * tasklyapunov.cpp:45-71): the sweep grid, p1 outer / p2 inner, delta =
 * |end - start| / (count - 1); sweep = {param_index, start, end, count}.
 * Writes P x nparams point-major into out (may be NULL to query P). */
int64_t chaos_lyap_make_grid(int32_t nparams, const double *base_params, const double sweep1[4],
                             const double sweep2[4], double *out);

/* Seeded per-point initial states, point-major P x dim: base + U(-amp, amp)
 * (dist 0) or base + N(0, amp^2) (dist 1), counter-based (Philox4x64-10 on
 * (point, block) with key (seed, constant)), so any subset of points can be
 * regenerated independently. */
int chaos_lyap_make_inits(int32_t dim, int64_t P, const double *base, double amp, int32_t dist,
                          uint64_t seed, double *out);

/* Measures the FP32 (precision = CHAOS_PREC_FP32) or FP64 (CHAOS_PREC_FP64)
 * fused-multiply-add throughput of `device` with a kernel of independent FMA
 * chains running for about `seconds` (FP32: the faster of scalar FFMA and
 * packed FFMA2 chains); the roofline denominator of the sweep kernels, which
 * are bound by the FMA pipe.  No reference counterpart (the
 * reference reports whole-run wall time only, raiitimer.h). */
int chaos_lyap_fma_peak(int device, int precision, double seconds, double *tflops);

/* The same initial states for an arbitrary list of point indices: out[i] is
 * what chaos_lyap_make_inits writes for point index[i] (used to integrate a
 * scattered subset of a large grid, e.g. the cells a surrogate flags). */
int chaos_lyap_make_inits_at(int32_t dim, int64_t count, const int64_t *index, const double *base,
                             double amp, int32_t dist, uint64_t seed, double *out);

#ifdef __cplusplus
}
#endif
#endif /* CHAOS_LYAP_H */
