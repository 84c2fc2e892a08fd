// C ABI of the sweep (include/chaos_lyap.h): model registry, handles,
// argument checking, launch dispatch, host-buffer path, autotuner and the
// drop-in for the reference launcher cudaLyapunov.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/chaos_lyap.h"
#include "kernels.h"
#include "models.cuh"
#include "trajectory.cuh"

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  return fail(CHAOS_LYAP_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

struct ModelInfo {
  const char *name;
  int id, dim, nparams, type;
  const char *pnames, *phase, *eq;
};

// The registry the reference fills at static-initialisation time
// (model_factory.h:36-39, shimizu.dp.cpp:203-204); here the device code is
// compiled in (models.cuh) and the table only carries the descriptions.
const ModelInfo kModels[] = {
    {"chua", chaos::kChua, 3, 4, 0, "alpha, beta, m0, m1", "x, y, z",
     "x' = alpha * (y - x - f(x));y' = x - y + z;z' = - beta * y;"
     "f(x) = m1 * x + 0.5 * (m0 - m1) * (|x + 1| - |x - 1|)"},
    {"henon", chaos::kHenon, 2, 2, 1, "a, b", "x, y", "x -> 1 - a * x^2 + y;y -> b * x"},
    {"hyper_rossler", chaos::kHyperRossler, 4, 2, 0, "c, d", "x, y, z, w",
     "x' = - y - z;y' = x + 0.25 * y + w;z' = 3 + x * z;w' = - c * z + d * w"},
    {"lorenz", chaos::kLorenz, 3, 3, 0, "sigma, rho, beta", "x, y, z",
     "x' = sigma * (y - x);y' = x * (rho - z) - y;z' = x * y - beta * z"},
    {"lorenz96", chaos::kLorenz96, 40, 2, 0, "F, gamma", "x0..x39",
     "x_i' = (x_{i+1} - x_{i-2}) * x_{i-1} - gamma * x_i + F (cyclic, N = 40)"},
    {"rossler", chaos::kRossler, 3, 3, 0, "a, b, c", "x, y, z",
     "x' = - y - z;y' = x + a * y;z' = b + z * (x - c)"},
    {"shimizu", chaos::kShimizu, 3, 2, 0, "alpha, lamda", "x, y, z",
     "x' = y;y' = - alpha * y - x * z + x;z' = - lamda * z + x ** 2.0"},
};
constexpr int kModelCount = sizeof(kModels) / sizeof(kModels[0]);

const ModelInfo *find_model(const char *name) {
  if (!name) return nullptr;
  for (const auto &m : kModels)
    if (std::strcmp(m.name, name) == 0) return &m;
  return nullptr;
}

// Keeps the caller's current device across a call.
struct DeviceGuard {
  int prev = -1;
  bool ok = false;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    ok = (prev == dev) || cudaSetDevice(dev) == cudaSuccess;
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

chaos::View view(double *p, int64_t P, int C, int layout) {
  return layout == CHAOS_LAYOUT_COMP_MAJOR ? chaos::View{p, 1, P} : chaos::View{p, C, 1};
}
chaos::CView cview(const double *p, int64_t P, int C, int layout) {
  return layout == CHAOS_LAYOUT_COMP_MAJOR ? chaos::CView{p, 1, P} : chaos::CView{p, C, 1};
}

}  // namespace

namespace chaos {
int model_id_of(const char *name, int *dim, int *nparams) {
  const ModelInfo *m = find_model(name);
  if (!m) return -1;
  if (dim) *dim = m->dim;
  if (nparams) *nparams = m->nparams;
  return m->id;
}
}  // namespace chaos

struct chaos_lyap_handle {
  chaos_lyap_desc d;
  const ModelInfo *model;
  int sm_count = 0;
  int block = 0;
  int schedule = CHAOS_SCHED_PERSISTENT;
  int variant = 0;  // kernel variant (chaos_lyap_desc.variant; autotuned)
  cudaStream_t own_stream = nullptr;
  cudaStream_t last_stream = nullptr;
  unsigned long long *queue = nullptr;  // point counters: persistent sweep / batch segments
  // longest-first hand-out order of points with their own averaging times
  int32_t *order = nullptr;
  void *order_scratch = nullptr;
  int64_t order_cap = 0;
  // second stream and fork / join events of a batch with both kernel forms
  cudaStream_t aux_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // host-path staging
  double *s_params = nullptr, *s_inits = nullptr, *s_spec = nullptr, *s_tavg = nullptr;
  int32_t *s_status = nullptr;
  int64_t *s_steps = nullptr;
  int64_t s_cap = 0;
};

extern "C" {

int chaos_lyap_abi_version(void) { return CHAOS_LYAP_ABI_VERSION; }

const char *chaos_lyap_last_error(void) { return g_err.c_str(); }

int chaos_lyap_desc_init(chaos_lyap_desc *d) {
  if (!d) return fail(CHAOS_LYAP_EINVAL, "desc is null");
  std::memset(d, 0, sizeof *d);
  d->struct_size = (int32_t)sizeof *d;
  std::strcpy(d->model, "lorenz");
  d->method = CHAOS_METHOD_VAR;
  d->integrator = CHAOS_INTEG_DVERK65;
  d->precision = CHAOS_PREC_FP64;
  d->gs = CHAOS_GS_CLASSICAL;
  d->layout = CHAOS_LAYOUT_POINT_MAJOR;
  d->eps = 1e-7;
  d->h = 1e-3;
  d->rtol = d->atol = 1e-10;
  d->max_steps = 100000000LL;
  d->escape = 1e4;
  d->schedule = CHAOS_SCHED_AUTO;
  return CHAOS_LYAP_OK;
}

int chaos_lyap_model_count(void) { return kModelCount; }

int chaos_lyap_model_name(int index, char *buf, int buflen) {
  if (index < 0 || index >= kModelCount || !buf || buflen <= 0)
    return fail(CHAOS_LYAP_EINVAL, "model index %d out of range", index);
  std::snprintf(buf, (size_t)buflen, "%s", kModels[index].name);
  return CHAOS_LYAP_OK;
}

int chaos_lyap_query_model(const char *name, int32_t *dim, int32_t *nparams, int32_t *type) {
  const ModelInfo *m = find_model(name);
  if (!m) return fail(CHAOS_LYAP_ENOMODEL, "unknown model '%s'", name ? name : "(null)");
  if (dim) *dim = m->dim;
  if (nparams) *nparams = m->nparams;
  if (type) *type = m->type;
  return CHAOS_LYAP_OK;
}

int chaos_lyap_model_text(const char *name, int which, char *buf, int buflen) {
  const ModelInfo *m = find_model(name);
  if (!m) return fail(CHAOS_LYAP_ENOMODEL, "unknown model '%s'", name ? name : "(null)");
  if (!buf || buflen <= 0 || which < 0 || which > 2) return fail(CHAOS_LYAP_EINVAL, "bad buffer");
  const char *s = which == 0 ? m->pnames : which == 1 ? m->phase : m->eq;
  std::snprintf(buf, (size_t)buflen, "%s", s);
  return (int)std::strlen(s) < buflen ? CHAOS_LYAP_OK
                                      : fail(CHAOS_LYAP_EINVAL, "buffer too small");
}

}  // extern "C"

namespace chaos {
static int msg_fail(char *msg, size_t len, int code, const char *fmt, ...)
    __attribute__((format(printf, 4, 5)));
static int msg_fail(char *msg, size_t len, int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, len, fmt, ap);
  va_end(ap);
  return code;
}

// Descriptor validation shared by the handle path (chaos_lyap_create) and
// the no-allocation batch entry: CHAOS_LYAP_OK, or an error code with the
// reason in msg.  k must already be resolved (k == 0 means "dim" only at
// create time).
int validate_desc(const chaos_lyap_desc *d, char *msg, size_t len) {
  if (!d) return msg_fail(msg, len, CHAOS_LYAP_EINVAL, "desc is null");
  if (d->struct_size != (int32_t)sizeof(chaos_lyap_desc))
    return msg_fail(msg, len, CHAOS_LYAP_EINVAL, "desc.struct_size %d != %d", d->struct_size,
                (int)sizeof(chaos_lyap_desc));
  char name[33];
  std::memcpy(name, d->model, 32);
  name[32] = 0;
  const ModelInfo *m = find_model(name);
  if (!m) return msg_fail(msg, len, CHAOS_LYAP_ENOMODEL, "unknown model '%s'", name);
  if (d->k < 1 || d->k > m->dim)
    return msg_fail(msg, len, CHAOS_LYAP_EINVAL,
        "k = %d outside 1..%d for model %s", d->k, m->dim, m->name);
  if (d->layout != CHAOS_LAYOUT_POINT_MAJOR && d->layout != CHAOS_LAYOUT_COMP_MAJOR)
    return msg_fail(msg, len, CHAOS_LYAP_EINVAL, "bad layout %d", d->layout);
  if (d->method < CHAOS_METHOD_FD || d->method > CHAOS_METHOD_QR)
    return msg_fail(msg, len, CHAOS_LYAP_EINVAL, "bad method %d", d->method);
  if (!(d->h > 0) || !std::isfinite(d->h)) return msg_fail(msg, len, CHAOS_LYAP_EINVAL,
      "h must be > 0");
  if (d->precision == CHAOS_PREC_COMPAT_FP64) {
    if (d->integrator != CHAOS_INTEG_DVERK_FIXED)
      return msg_fail(msg, len, CHAOS_LYAP_EINVAL,
          "compat precision needs the fixed-step DVERK integrator");
    if (d->method == CHAOS_METHOD_QR && d->k != m->dim)
      return msg_fail(msg, len, CHAOS_LYAP_EUNSUPPORTED,
                  "QR method needs k == dim (the reference's QR assumes a square matrix)");
    if (!(d->t_avg > 0)) return msg_fail(msg, len, CHAOS_LYAP_EINVAL, "t_avg must be > 0");
  } else if (d->precision == CHAOS_PREC_FP64 || d->precision == CHAOS_PREC_FP32) {
    if (d->integrator != CHAOS_INTEG_DVERK65 && d->integrator != CHAOS_INTEG_DOPRI5)
      return msg_fail(msg, len, CHAOS_LYAP_EINVAL,
          "adaptive precision forms need DVERK65 or DOPRI5");
    if (d->method != CHAOS_METHOD_VAR)
      return msg_fail(msg, len, CHAOS_LYAP_EUNSUPPORTED,
          "adaptive forms integrate the variational equations (VAR)");
    if (d->k != m->dim && m->dim <= 4)
      return msg_fail(msg, len, CHAOS_LYAP_EUNSUPPORTED,
          "adaptive forms compute the full spectrum (k == dim)");
    if (!(d->rtol > 0) || !(d->atol > 0)) return msg_fail(msg, len, CHAOS_LYAP_EINVAL,
        "rtol/atol must be > 0");
    if (!(d->dt_renorm > 0) || !(d->t_avg > 0) || d->t_transient < 0 || d->t_align < 0)
      return msg_fail(msg, len, CHAOS_LYAP_EINVAL,
          "times: dt_renorm, t_avg > 0; t_transient, t_align >= 0");
    if (d->max_steps <= 0) return msg_fail(msg, len, CHAOS_LYAP_EINVAL, "max_steps must be > 0");
    if (d->gs != CHAOS_GS_CLASSICAL && d->gs != CHAOS_GS_MODIFIED)
      return msg_fail(msg, len, CHAOS_LYAP_EINVAL, "bad gs %d", d->gs);
  } else {
    return msg_fail(msg, len, CHAOS_LYAP_EINVAL, "bad precision %d", d->precision);
  }
  if (m->type != 0) {  // maps: the reference's FD / VAR map branches, in compat precision
    if (d->precision != CHAOS_PREC_COMPAT_FP64)
      return msg_fail(msg, len, CHAOS_LYAP_EUNSUPPORTED,
                  "map model %s: maps are iterated, not integrated; use compat precision", m->name);
    if (d->method == CHAOS_METHOD_QR)
      return msg_fail(msg, len, CHAOS_LYAP_EUNSUPPORTED,
          "map model %s: the QR method has no map branch",
                  m->name);
  }
  return CHAOS_LYAP_OK;
}
}  // namespace chaos

static int check_desc(const chaos_lyap_desc *d, const ModelInfo **mout) {
  char msg[512];
  const int rc = chaos::validate_desc(d, msg, sizeof msg);
  if (rc) return fail(rc, "%s", msg);
  char name[33];
  std::memcpy(name, d->model, 32);
  name[32] = 0;
  *mout = find_model(name);
  return CHAOS_LYAP_OK;
}

extern "C" {

int chaos_lyap_create(const chaos_lyap_desc *desc, chaos_lyap_handle **out) {
  if (!out) return fail(CHAOS_LYAP_EINVAL, "out is null");
  *out = nullptr;
  chaos_lyap_desc d;
  if (!desc) return fail(CHAOS_LYAP_EINVAL, "desc is null");
  d = *desc;
  const ModelInfo *m0 = find_model(d.model);
  if (d.k == 0 && m0) d.k = m0->dim;
  const ModelInfo *m = nullptr;
  int rc = check_desc(&d, &m);
  if (rc) return rc;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
  if (d.device < 0 || d.device >= ndev)
    return fail(CHAOS_LYAP_EINVAL, "device %d not present (%d devices)", d.device, ndev);
  DeviceGuard g(d.device);
  if (!g.ok) return fail(CHAOS_LYAP_ECUDA, "cannot select device %d", d.device);
  auto *h = new chaos_lyap_handle();
  h->d = d;
  h->model = m;
  cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, d.device);
  h->block = d.block > 0 ? d.block : (d.precision == CHAOS_PREC_COMPAT_FP64 ? 64 : 128);
  h->schedule = (d.schedule >= CHAOS_SCHED_DIRECT && d.schedule <= CHAOS_SCHED_SPLIT_PERSISTENT)
                    ? d.schedule
                    : CHAOS_SCHED_PERSISTENT;
  h->variant = d.variant == 1 ? 1 : 0;
  if ((e = cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking)) != cudaSuccess) {
    delete h;
    return cuda_fail(e, "cudaStreamCreate");
  }
  if ((e = cudaMalloc(&h->queue, sizeof(unsigned long long) * chaos::kMaxSegments)) != cudaSuccess) {
    cudaStreamDestroy(h->own_stream);
    delete h;
    return fail(CHAOS_LYAP_ENOMEM, "cudaMalloc(queue): %s", cudaGetErrorString(e));
  }
  *out = h;
  return CHAOS_LYAP_OK;
}

static void free_staging(chaos_lyap_handle *h) {
  cudaFree(h->s_params);
  cudaFree(h->s_inits);
  cudaFree(h->s_spec);
  cudaFree(h->s_tavg);
  cudaFree(h->s_status);
  cudaFree(h->s_steps);
  h->s_params = h->s_inits = h->s_spec = h->s_tavg = nullptr;
  h->s_status = nullptr;
  h->s_steps = nullptr;
  h->s_cap = 0;
}

int chaos_lyap_destroy(chaos_lyap_handle *h) {
  if (!h) return CHAOS_LYAP_OK;
  DeviceGuard g(h->d.device);
  cudaStreamSynchronize(h->own_stream);
  free_staging(h);
  cudaFree(h->queue);
  cudaFree(h->order);
  cudaFree(h->order_scratch);
  if (h->aux_stream) {
    cudaStreamSynchronize(h->aux_stream);
    cudaStreamDestroy(h->aux_stream);
  }
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  cudaStreamDestroy(h->own_stream);
  delete h;
  return CHAOS_LYAP_OK;
}

// Device buffers for the longest-first order of P points (grown on demand;
// allocated outside any stream capture: before a run or a graph capture).
static int ensure_order(chaos_lyap_handle *h, int64_t P) {
  if (P <= h->order_cap) return CHAOS_LYAP_OK;
  DeviceGuard g(h->d.device);
  cudaFree(h->order);
  h->order = nullptr;
  h->order_cap = 0;
  cudaError_t e = cudaMalloc(&h->order, sizeof(int32_t) * P);
  if (e == cudaSuccess && !h->order_scratch) e = cudaMalloc(&h->order_scratch, chaos::kOrderScratchBytes);
  if (e != cudaSuccess) {
    cudaFree(h->order);
    h->order = nullptr;
    return fail(CHAOS_LYAP_ENOMEM, "cudaMalloc(order): %s", cudaGetErrorString(e));
  }
  h->order_cap = P;
  return CHAOS_LYAP_OK;
}

// P points of params / inits are read at every `stride`-th point of arrays
// that hold P_full points (stride 1, P_full = 0: the arrays themselves); the
// spectrum, status and steps arrays hold P points.
static int enqueue(chaos_lyap_handle *h, int64_t P, const double *params, double *inits,
                   double *spectrum, int32_t *status, int64_t *steps, const double *tavg,
                   cudaStream_t s, int block, int schedule, int variant, double t_avg_override,
                   double t_transient_override, int64_t P_full = 0, int64_t stride = 1) {
  const chaos_lyap_desc &d = h->d;
  const ModelInfo *m = h->model;
  int rc;
  if (d.precision == CHAOS_PREC_COMPAT_FP64) {
    chaos::CompatArgs a{};
    a.P = P;
    a.k = d.k;
    a.method = d.method;
    a.eps = d.eps;
    a.step = d.h;
    a.t_skip = d.t_transient;
    a.t_skip_clp = d.t_align;
    a.calc_time = d.t_avg;
    a.add_skip = d.dt_renorm / d.h;  // tasklyapunov.cpp:65
    a.params = cview(params, P, m->nparams, d.layout);
    a.inits = view(inits, P, m->dim, d.layout);
    a.close = nullptr;
    a.lyap = view(spectrum, P, d.k, d.layout);
    a.accumulate = 0;
    a.status = status;
    rc = chaos::launch_compat(m->id, a, block, s);
  } else {
    chaos::AdaptiveArgs a{};
    a.P = P;
    a.k = d.k;
    a.gs = d.gs;
    a.rtol = d.rtol;
    a.atol = d.atol;
    a.h0 = d.h;
    a.hmax = d.h_max;
    a.hmin = d.h_min;
    a.t_transient = t_transient_override >= 0 ? t_transient_override : d.t_transient;
    a.t_align = d.t_align;
    a.t_avg = t_avg_override > 0 ? t_avg_override : d.t_avg;
    a.dt_renorm = d.dt_renorm;
    a.max_steps = d.max_steps;
    a.escape = d.escape > 0 ? d.escape : 1e4;
    a.params = cview(params, P_full > 0 ? P_full : P, m->nparams, d.layout);
    a.inits = cview(inits, P_full > 0 ? P_full : P, m->dim, d.layout);
    a.params.ps *= stride;
    a.inits.ps *= stride;
    a.t_avg_per_point = t_avg_override > 0 ? nullptr : tavg;
    a.spectrum = view(spectrum, P, d.k, d.layout);
    a.status = status;
    a.steps = steps;
    const int integ = d.integrator == CHAOS_INTEG_DOPRI5 ? chaos::kDopri5 : chaos::kDverk65;
    const int prec = d.precision == CHAOS_PREC_FP32 ? chaos::kFP32 : chaos::kFP64;
    const bool split = schedule == CHAOS_SCHED_SPLIT_DIRECT || schedule == CHAOS_SCHED_SPLIT_PERSISTENT;
    if (schedule == CHAOS_SCHED_PERSISTENT || schedule == CHAOS_SCHED_SPLIT_PERSISTENT) {
      cudaError_t e = cudaMemsetAsync(h->queue, 0, sizeof(unsigned long long), s);
      if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(queue)");
      a.queue = h->queue;
      a.queue_stride = chaos::queue_stride_for(P);
      if (a.t_avg_per_point && m->dim <= 4) {  // longest averaging time first
        if ((rc = ensure_order(h, P))) return rc;
        rc = chaos::launch_order_longest_first(a.t_avg_per_point, P, h->order, h->order_scratch, s);
        if (rc) return cuda_fail((cudaError_t)rc, "order launch");
        a.order = h->order;
      }
    }
    if (m->dim > 4) rc = chaos::launch_l96_warp(integ, prec, a, 0, s);
    else if (split) rc = chaos::launch_split(m->id, integ, prec, a, block, variant, s);
    else rc = chaos::launch_adaptive(m->id, integ, prec, a, block, 0, variant, s);
  }
  if (rc == chaos::kErrUnsupported)
    return fail(CHAOS_LYAP_EUNSUPPORTED, "no kernel for model %s with this integrator/precision/k",
                m->name);
  if (rc != 0) return cuda_fail((cudaError_t)rc, "kernel launch");
  h->last_stream = s;
  return CHAOS_LYAP_OK;
}

int chaos_lyap_run(chaos_lyap_handle *h, int64_t P, const double *params, double *inits,
                   double *spectrum, int32_t *status, int64_t *steps, const double *tavg,
                   void *stream) {
  if (!h) return fail(CHAOS_LYAP_EINVAL, "handle is null");
  if (P < 0) return fail(CHAOS_LYAP_EINVAL, "P < 0");
  if (P == 0) return CHAOS_LYAP_OK;
  if (!params || !inits || !spectrum) return fail(CHAOS_LYAP_EINVAL, "null array");
  DeviceGuard g(h->d.device);
  if (!g.ok) return fail(CHAOS_LYAP_ECUDA, "cannot select device %d", h->d.device);
  return enqueue(h, P, params, inits, spectrum, status, steps, tavg, (cudaStream_t)stream, h->block,
                 h->schedule, h->variant, -1.0, -1.0);
}

int chaos_lyap_sync(chaos_lyap_handle *h) {
  if (!h) return fail(CHAOS_LYAP_EINVAL, "handle is null");
  DeviceGuard g(h->d.device);
  cudaError_t e = h->last_stream ? cudaStreamSynchronize(h->last_stream) : cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_fail(e, "synchronize");
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "sweep");
  return CHAOS_LYAP_OK;
}

int chaos_lyap_run_host(chaos_lyap_handle *h, int64_t P, const double *params, double *inits,
                        double *spectrum, int32_t *status, int64_t *steps, const double *tavg) {
  if (!h) return fail(CHAOS_LYAP_EINVAL, "handle is null");
  if (P < 0) return fail(CHAOS_LYAP_EINVAL, "P < 0");
  if (P == 0) return CHAOS_LYAP_OK;
  if (!params || !inits || !spectrum) return fail(CHAOS_LYAP_EINVAL, "null array");
  DeviceGuard g(h->d.device);
  if (!g.ok) return fail(CHAOS_LYAP_ECUDA, "cannot select device %d", h->d.device);
  const ModelInfo *m = h->model;
  const int k = h->d.k;
  cudaError_t e;
  if (P > h->s_cap) {
    free_staging(h);
    if ((e = cudaMalloc(&h->s_params, sizeof(double) * P * m->nparams)) != cudaSuccess ||
        (e = cudaMalloc(&h->s_inits, sizeof(double) * P * m->dim)) != cudaSuccess ||
        (e = cudaMalloc(&h->s_spec, sizeof(double) * P * k)) != cudaSuccess ||
        (e = cudaMalloc(&h->s_tavg, sizeof(double) * P)) != cudaSuccess ||
        (e = cudaMalloc(&h->s_status, sizeof(int32_t) * P)) != cudaSuccess ||
        (e = cudaMalloc(&h->s_steps, sizeof(int64_t) * P)) != cudaSuccess) {
      free_staging(h);
      return fail(CHAOS_LYAP_ENOMEM, "staging for %lld points: %s", (long long)P,
                  cudaGetErrorString(e));
    }
    h->s_cap = P;
  }
  cudaStream_t s = h->own_stream;
  const size_t bp = sizeof(double) * P * m->nparams, bx = sizeof(double) * P * m->dim,
               bs = sizeof(double) * P * k;
  if ((e = cudaMemcpyAsync(h->s_params, params, bp, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(h->s_inits, inits, bx, cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return cuda_fail(e, "copy in");
  if (tavg && (e = cudaMemcpyAsync(h->s_tavg, tavg, sizeof(double) * P, cudaMemcpyHostToDevice,
                                   s)) != cudaSuccess)
    return cuda_fail(e, "copy in");
  int rc = enqueue(h, P, h->s_params, h->s_inits, h->s_spec, status ? h->s_status : nullptr,
                   steps ? h->s_steps : nullptr, tavg ? h->s_tavg : nullptr, s, h->block,
                   h->schedule, h->variant, -1.0, -1.0);
  if (rc) return rc;
  if ((e = cudaMemcpyAsync(spectrum, h->s_spec, bs, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return cuda_fail(e, "copy out");
  if (h->d.precision == CHAOS_PREC_COMPAT_FP64 &&
      (e = cudaMemcpyAsync(inits, h->s_inits, bx, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return cuda_fail(e, "copy out");
  if (status && (e = cudaMemcpyAsync(status, h->s_status, sizeof(int32_t) * P,
                                     cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return cuda_fail(e, "copy out");
  if (steps && (e = cudaMemcpyAsync(steps, h->s_steps, sizeof(int64_t) * P,
                                    cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return cuda_fail(e, "copy out");
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "synchronize");
  return CHAOS_LYAP_OK;
}

// Times short runs of `sample` points -- every `stride`-th of the P_full
// points of the arrays -- in every launch shape and keeps the fastest.
static int autotune(chaos_lyap_handle *h, int64_t P_full, int64_t sample, int64_t stride,
                    const double *params, const double *inits, int32_t *block_out,
                    int32_t *schedule_out) {
  if (!h) return fail(CHAOS_LYAP_EINVAL, "handle is null");
  if (sample <= 0 || !params || !inits) return fail(CHAOS_LYAP_EINVAL, "bad sample");
  if (h->d.precision == CHAOS_PREC_COMPAT_FP64 || h->model->dim > 4) {
    if (block_out) *block_out = h->block;
    if (schedule_out) *schedule_out = h->schedule;
    return CHAOS_LYAP_OK;
  }
  DeviceGuard g(h->d.device);
  const int k = h->d.k;
  double *spec = nullptr;
  cudaError_t e;
  if ((e = cudaMalloc(&spec, sizeof(double) * sample * k)) != cudaSuccess)
    return fail(CHAOS_LYAP_ENOMEM, "autotune buffer: %s", cudaGetErrorString(e));
  // Short horizons: the launch-shape ranking does not need the full run.
  // Stage 1 times every shape on a horizon of 20 renormalisation intervals;
  // stage 2 re-times the shapes within 15 % of the fastest on a horizon four
  // times longer, where the few points whose chains set a small map's
  // length weigh as they do in the full run (on a 64^2 map the short
  // horizon alone ranked two split layouts 10 % apart the wrong way round).
  const double t_avg1 = std::min(h->d.t_avg, 20.0 * h->d.dt_renorm);
  const double t_tr1 = std::min(h->d.t_transient, 5.0 * h->d.dt_renorm);
  const double t_avg2 = std::min(h->d.t_avg, 80.0 * h->d.dt_renorm);
  const double t_tr2 = std::min(h->d.t_transient, 20.0 * h->d.dt_renorm);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks[] = {64, 128};
  const int scheds[] = {CHAOS_SCHED_DIRECT, CHAOS_SCHED_PERSISTENT, CHAOS_SCHED_SPLIT_DIRECT,
                        CHAOS_SCHED_SPLIT_PERSISTENT};
  const bool fp32 = h->d.precision == CHAOS_PREC_FP32;
  struct Shape {
    int b, sc, v;
    float ms;
  };
  Shape shapes[16];
  int n = 0, rc = CHAOS_LYAP_OK;
  cudaStream_t s = h->own_stream;
  auto time_shape = [&](Shape &x, double t_avg, double t_tr) {
    for (int rep = 0; rep < 2 && rc == CHAOS_LYAP_OK; ++rep) {
      cudaEventRecord(e0, s);
      rc = enqueue(h, sample, params, const_cast<double *>(inits), spec, nullptr, nullptr,
                   nullptr, s, x.b, x.sc, x.v, t_avg, t_tr, P_full, stride);
      cudaEventRecord(e1, s);
      cudaEventSynchronize(e1);
      cudaEventElapsedTime(&x.ms, e0, e1);  // second repetition is the warm one
    }
  };
  for (int v = 0; v < 2 && rc == CHAOS_LYAP_OK; v++)
    for (int b : blocks)
      for (int sc : scheds) {
        // variant 1: the register cap of the FP32 one-lane forms, the
        // exchange layout of the FP64 split forms of 3-dimensional models
        const bool split = sc == CHAOS_SCHED_SPLIT_DIRECT || sc == CHAOS_SCHED_SPLIT_PERSISTENT;
        if (v > 0 && (split ? (fp32 || h->model->dim != 3) : !fp32)) continue;
        if (rc != CHAOS_LYAP_OK || n >= 16) break;
        shapes[n] = Shape{b, sc, v, 0.f};
        time_shape(shapes[n], t_avg1, t_tr1);
        ++n;
      }
  float best1 = 1e30f;
  for (int i = 0; i < n; i++) best1 = std::min(best1, shapes[i].ms);
  Shape best{h->block, h->schedule, h->variant, 1e30f};
  const bool longer = t_avg2 > t_avg1 || t_tr2 > t_tr1;
  for (int i = 0; i < n && rc == CHAOS_LYAP_OK; i++) {
    Shape x = shapes[i];
    if (x.ms > 1.15f * best1) continue;
    if (longer) time_shape(x, t_avg2, t_tr2);
    if (rc == CHAOS_LYAP_OK && x.ms < best.ms) best = x;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(spec);
  if (rc) return rc;
  const int best_b = best.b, best_s = best.sc, best_v = best.v;
  h->block = best_b;
  h->schedule = best_s;
  h->variant = best_v;
  if (block_out) *block_out = best_b;
  if (schedule_out) *schedule_out = best_s;
  return CHAOS_LYAP_OK;
}

int chaos_lyap_autotune(chaos_lyap_handle *h, int64_t sample, const double *params,
                        const double *inits, int32_t *block_out, int32_t *schedule_out) {
  return autotune(h, sample, sample, 1, params, inits, block_out, schedule_out);
}

int chaos_lyap_autotune_map(chaos_lyap_handle *h, int64_t P, int64_t sample,
                            const double *params, const double *inits, int32_t *block_out,
                            int32_t *schedule_out) {
  if (P <= 0 || sample <= 0) return fail(CHAOS_LYAP_EINVAL, "P and sample must be > 0");
  const int64_t n = std::min(P, sample);
  return autotune(h, P, n, P / n, params, inits, block_out, schedule_out);
}

// A batch runs each segment in the form of its handle's schedule: segments
// with a split schedule in the split batch kernel, the others in the
// one-lane batch kernel.  When both kinds are present the two persistent
// kernels run side by side (forked onto the first handle's second stream,
// joined before the batch ends; captured as two branches of a graph).  The
// split kernel -- the form chosen for segments whose longest points set the
// run's length -- is launched first and at the device's greatest priority
// with a full machine's grid; the one-lane kernel's blocks take the SM slots
// that its blocks free as its queues run dry.
struct BatchPlan {
  chaos::BatchArgs lane, split;
  chaos_lyap_handle *lane_h[chaos::kMaxSegments], *split_h[chaos::kMaxSegments];
  // scratch of the longest-first ordering of each segment with per-point times
  void *lane_scratch[chaos::kMaxSegments], *split_scratch[chaos::kMaxSegments];
  int integ, prec, lane_block, split_block;
};

// Device buffers of one segment's longest-first hand-out order.
struct OrderBuf {
  int32_t *order;
  void *scratch;
};

static bool is_split(const chaos_lyap_handle *h) {
  return h->schedule == CHAOS_SCHED_SPLIT_DIRECT || h->schedule == CHAOS_SCHED_SPLIT_PERSISTENT;
}

// Checks the segments and lays out the launch.  Each segment's longest-first
// order goes into `own[i]` when given (buffers a graph owns, sized for the
// segment), else into the segment handle's own buffers (grown on demand).
// Every segment has its own handle: two segments of one handle would share
// that handle's order buffer.
static int check_segments(const chaos_lyap_segment *segs, int nseg) {
  if (!segs || nseg <= 0 || nseg > chaos::kMaxSegments)
    return fail(CHAOS_LYAP_EINVAL, "nseg must be 1..%d", chaos::kMaxSegments);
  for (int i = 0; i < nseg; i++) {
    if (!segs[i].handle) return fail(CHAOS_LYAP_EINVAL, "segment %d: null handle", i);
    for (int j = 0; j < i; j++)
      if (segs[j].handle == segs[i].handle)
        return fail(CHAOS_LYAP_EINVAL,
                    "segments %d and %d share a handle: every segment needs its own", j, i);
  }
  return CHAOS_LYAP_OK;
}

static int build_batch(const chaos_lyap_segment *segs, int nseg, BatchPlan *plan,
                       const OrderBuf *own) {
  int rc0 = check_segments(segs, nseg);
  if (rc0) return rc0;
  std::memset(plan, 0, sizeof *plan);
  for (int i = 0; i < nseg; i++) {
    const chaos_lyap_segment &sg = segs[i];
    const chaos_lyap_desc &d = sg.handle->d;
    if (d.precision == CHAOS_PREC_COMPAT_FP64 || sg.handle->model->dim > 4)
      return fail(CHAOS_LYAP_EUNSUPPORTED,
                  "segment %d: batches take the adaptive forms of 3-4 dimensional models", i);
    if (i > 0 && (d.precision != segs[0].handle->d.precision ||
                  d.integrator != segs[0].handle->d.integrator ||
                  d.device != segs[0].handle->d.device))
      return fail(CHAOS_LYAP_EINVAL, "segment %d: integrator / precision / device differ", i);
    if (sg.P < 0 || (sg.P > 0 && (!sg.params || !sg.inits || !sg.spectrum)))
      return fail(CHAOS_LYAP_EINVAL, "segment %d: bad arrays", i);
    const bool sp = is_split(sg.handle);
    chaos::BatchArgs &b = sp ? plan->split : plan->lane;
    const int j = b.nseg++;
    (sp ? plan->split_h : plan->lane_h)[j] = sg.handle;
    chaos::AdaptiveArgs &a = b.seg[j];
    a.P = sg.P;
    a.k = d.k;
    a.gs = d.gs;
    a.rtol = d.rtol;
    a.atol = d.atol;
    a.h0 = d.h;
    a.hmax = d.h_max;
    a.hmin = d.h_min;
    a.t_transient = d.t_transient;
    a.t_align = d.t_align;
    a.t_avg = d.t_avg;
    a.dt_renorm = d.dt_renorm;
    a.max_steps = d.max_steps;
    a.escape = d.escape > 0 ? d.escape : 1e4;
    const ModelInfo *m = sg.handle->model;
    a.params = cview(sg.params, sg.P, m->nparams, d.layout);
    a.inits = cview(sg.inits, sg.P, m->dim, d.layout);
    a.t_avg_per_point = sg.t_avg_per_point;
    a.spectrum = view(sg.spectrum, sg.P, d.k, d.layout);
    a.status = sg.status;
    a.steps = sg.steps;
    a.queue_stride = chaos::queue_stride_for(sg.P);
    a.order = nullptr;
    void *scratch = nullptr;
    if (sg.t_avg_per_point && sg.P > 0) {  // longest averaging time first
      if (own) {
        a.order = own[i].order;
        scratch = own[i].scratch;
      } else {
        int rc = ensure_order(sg.handle, sg.P);
        if (rc) return rc;
        a.order = sg.handle->order;
        scratch = sg.handle->order_scratch;
      }
    }
    (sp ? plan->split_scratch : plan->lane_scratch)[j] = scratch;
    b.model[j] = m->id;
  }
  chaos_lyap_handle *h0 = segs[0].handle;
  // the first handle's counters: one-lane segments first, then split ones
  plan->lane.queues = h0->queue;
  plan->split.queues = h0->queue + plan->lane.nseg;
  const chaos_lyap_desc &d0 = h0->d;
  plan->integ = d0.integrator == CHAOS_INTEG_DOPRI5 ? chaos::kDopri5 : chaos::kDverk65;
  plan->prec = d0.precision == CHAOS_PREC_FP32 ? chaos::kFP32 : chaos::kFP64;
  plan->lane_block = plan->lane.nseg ? plan->lane_h[0]->block : 128;
  plan->split_block = plan->split.nseg ? plan->split_h[0]->block : 64;
  if (plan->lane.nseg && plan->split.nseg && !h0->aux_stream) {  // fork / join resources
    DeviceGuard g(d0.device);
    cudaError_t e = cudaStreamCreateWithFlags(&h0->aux_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h0->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h0->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_fail(e, "batch fork stream / events");
  }
  return CHAOS_LYAP_OK;
}

static int launch_orders(const chaos::BatchArgs &b, void *const *scratch, cudaStream_t s) {
  for (int i = 0; i < b.nseg; i++) {
    if (!b.seg[i].order) continue;
    int rc = chaos::launch_order_longest_first(b.seg[i].t_avg_per_point, b.seg[i].P,
                                               const_cast<int32_t *>(b.seg[i].order), scratch[i], s);
    if (rc) return cuda_fail((cudaError_t)rc, "order launch");
  }
  return CHAOS_LYAP_OK;
}

static int batch_rc(int rc) {
  if (rc == chaos::kErrUnsupported) return fail(CHAOS_LYAP_EUNSUPPORTED, "no batch kernel for this mix");
  if (rc) return cuda_fail((cudaError_t)rc, "batch launch");
  return CHAOS_LYAP_OK;
}

static int enqueue_batch(const BatchPlan &p, chaos_lyap_handle *h0, cudaStream_t s) {
  const int nseg = p.lane.nseg + p.split.nseg;
  cudaError_t e = cudaMemsetAsync(h0->queue, 0, sizeof(unsigned long long) * nseg, s);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(queues)");
  int rc = launch_orders(p.lane, p.lane_scratch, s);
  if (!rc) rc = launch_orders(p.split, p.split_scratch, s);
  if (rc) return rc;
  if (p.lane.nseg && p.split.nseg) {
    cudaStream_t aux = h0->aux_stream;
    if ((e = cudaEventRecord(h0->ev_fork, s)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(aux, h0->ev_fork, 0)) != cudaSuccess)
      return cuda_fail(e, "batch fork");
    rc = batch_rc(chaos::launch_batch_split(p.integ, p.prec, p.split, p.split_block, s, 1.0, true));
    const int rc2 = batch_rc(chaos::launch_batch(p.integ, p.prec, p.lane, p.lane_block, aux, 1.0));
    // join even after a failed launch, so that a capture still ends cleanly
    if ((e = cudaEventRecord(h0->ev_join, aux)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(s, h0->ev_join, 0)) != cudaSuccess)
      return cuda_fail(e, "batch join");
    return rc ? rc : rc2;
  }
  if (p.split.nseg)
    return batch_rc(chaos::launch_batch_split(p.integ, p.prec, p.split, p.split_block, s));
  return batch_rc(chaos::launch_batch(p.integ, p.prec, p.lane, p.lane_block, s));
}

int chaos_lyap_run_batch(const chaos_lyap_segment *segs, int nseg, void *stream) {
  BatchPlan plan;
  int rc = build_batch(segs, nseg, &plan, nullptr);
  if (rc) return rc;
  DeviceGuard g(segs[0].handle->d.device);
  rc = enqueue_batch(plan, segs[0].handle, (cudaStream_t)stream);
  if (!rc) segs[0].handle->last_stream = (cudaStream_t)stream;
  return rc;
}

// A captured batch.  The graph owns the longest-first order buffers of its
// segments, so a later run on one of its handles (which may regrow that
// handle's own buffer) cannot leave the graph reading freed memory.
struct chaos_lyap_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int device = 0;
  OrderBuf order[chaos::kMaxSegments] = {};
};

static void free_graph(chaos_lyap_graph *gr) {
  if (gr->exec) cudaGraphExecDestroy(gr->exec);
  if (gr->graph) cudaGraphDestroy(gr->graph);
  for (auto &o : gr->order) {
    cudaFree(o.order);
    cudaFree(o.scratch);
  }
  delete gr;
}

int chaos_lyap_batch_graph_create(const chaos_lyap_segment *segs, int nseg, chaos_lyap_graph **out) {
  if (!out) return fail(CHAOS_LYAP_EINVAL, "out is null");
  *out = nullptr;
  int rc = check_segments(segs, nseg);
  if (rc) return rc;
  DeviceGuard g(segs[0].handle->d.device);
  auto *gr = new chaos_lyap_graph();
  gr->device = segs[0].handle->d.device;
  for (int i = 0; i < nseg; i++) {
    if (!segs[i].t_avg_per_point || segs[i].P <= 0) continue;
    cudaError_t e = cudaMalloc(&gr->order[i].order, sizeof(int32_t) * segs[i].P);
    if (e == cudaSuccess) e = cudaMalloc(&gr->order[i].scratch, chaos::kOrderScratchBytes);
    if (e != cudaSuccess) {
      free_graph(gr);
      return fail(CHAOS_LYAP_ENOMEM, "cudaMalloc(graph order): %s", cudaGetErrorString(e));
    }
  }
  BatchPlan plan;
  rc = build_batch(segs, nseg, &plan, gr->order);
  if (rc) {
    free_graph(gr);
    return rc;
  }
  cudaStream_t cs;
  cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    free_graph(gr);
    return cuda_fail(e, "cudaStreamCreate");
  }
  e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    rc = enqueue_batch(plan, segs[0].handle, cs);
    cudaError_t e2 = cudaStreamEndCapture(cs, &gr->graph);
    if (!rc && e2 != cudaSuccess) rc = cuda_fail(e2, "cudaStreamEndCapture");
  } else {
    rc = cuda_fail(e, "cudaStreamBeginCapture");
  }
  // per-node priorities: the split kernel's blocks are dispatched first
  if (!rc && (e = cudaGraphInstantiate(&gr->exec, gr->graph, cudaGraphInstantiateFlagUseNodePriority)) !=
                 cudaSuccess)
    rc = cuda_fail(e, "cudaGraphInstantiate");
  cudaStreamDestroy(cs);
  if (rc) {
    free_graph(gr);
    return rc;
  }
  *out = gr;
  return CHAOS_LYAP_OK;
}

int chaos_lyap_graph_launch(chaos_lyap_graph *g, void *stream) {
  if (!g) return fail(CHAOS_LYAP_EINVAL, "graph is null");
  DeviceGuard dg(g->device);
  cudaError_t e = cudaGraphLaunch(g->exec, (cudaStream_t)stream);
  return e == cudaSuccess ? CHAOS_LYAP_OK : cuda_fail(e, "cudaGraphLaunch");
}

int chaos_lyap_graph_destroy(chaos_lyap_graph *g) {
  if (!g) return CHAOS_LYAP_OK;
  DeviceGuard dg(g->device);
  free_graph(g);
  return CHAOS_LYAP_OK;
}

int chaos_lyap_trajectory(chaos_lyap_handle *h, int64_t P, const double *params,
                          const double *inits, int32_t nsteps, double *t_out, double *h_out,
                          double *x_out, int32_t *status, void *stream) {
  if (!h) return fail(CHAOS_LYAP_EINVAL, "handle is null");
  const chaos_lyap_desc &d = h->d;
  const ModelInfo *m = h->model;
  if (d.precision == CHAOS_PREC_COMPAT_FP64)
    return fail(CHAOS_LYAP_EUNSUPPORTED, "trajectories take the adaptive forms (FP64 or FP32)");
  if (m->type != 0 || m->dim > 4)
    return fail(CHAOS_LYAP_EUNSUPPORTED, "trajectories of flows of dimension <= 4 (model %s)",
                m->name);
  if (P < 0 || nsteps < 0) return fail(CHAOS_LYAP_EINVAL, "P and nsteps must be >= 0");
  if (P == 0 || nsteps == 0) return CHAOS_LYAP_OK;
  if (!params || !inits || !t_out || !h_out || !x_out) return fail(CHAOS_LYAP_EINVAL, "null array");
  DeviceGuard g(d.device);
  if (!g.ok) return fail(CHAOS_LYAP_ECUDA, "cannot select device %d", d.device);
  chaos::adaptive::TrajectoryArgs ta{};
  chaos::AdaptiveArgs &a = ta.a;
  a.P = P;
  a.k = m->dim;
  a.rtol = d.rtol;
  a.atol = d.atol;
  a.h0 = d.h;
  a.hmax = d.h_max;
  a.hmin = d.h_min;
  a.max_steps = d.max_steps;
  a.escape = d.escape > 0 ? d.escape : 1e4;
  a.params = cview(params, P, m->nparams, d.layout);
  a.inits = cview(inits, P, m->dim, d.layout);
  ta.nsteps = nsteps;
  ta.t_out = t_out;
  ta.h_out = h_out;
  ta.x_out = x_out;
  ta.status = status;
  const int integ = d.integrator == CHAOS_INTEG_DOPRI5 ? chaos::kDopri5 : chaos::kDverk65;
  const int prec = d.precision == CHAOS_PREC_FP32 ? chaos::kFP32 : chaos::kFP64;
  const int rc = chaos::launch_trajectory(m->id, integ, prec, ta, (cudaStream_t)stream);
  if (rc == chaos::kErrUnsupported)
    return fail(CHAOS_LYAP_EUNSUPPORTED, "no trajectory kernel for model %s", m->name);
  if (rc) return cuda_fail((cudaError_t)rc, "trajectory launch");
  h->last_stream = (cudaStream_t)stream;
  return CHAOS_LYAP_OK;
}

int chaos_lyap_get_variant(chaos_lyap_handle *h, int32_t *variant) {
  if (!h || !variant) return fail(CHAOS_LYAP_EINVAL, "null argument");
  *variant = h->variant;
  return CHAOS_LYAP_OK;
}

int chaos_lyap_cudaLyapunov(int bn, int bs, size_t taskNum, int isQr, int isVar, int modelType,
                            double *inits, double *closePoints, int32_t dimension,
                            const char *model, double *params, int32_t paramsDim, double eps,
                            double integrationStep, double *lyapExps, int32_t expsNum,
                            double timeSkip, double timeSkipClP, double calcTime,
                            double addSkipSteps, void *stream) {
  (void)bn;
  (void)bs;
  const ModelInfo *m = find_model(model);
  if (!m) return fail(CHAOS_LYAP_ENOMODEL, "unknown model '%s'", model ? model : "(null)");
  if (modelType != m->type)
    return fail(CHAOS_LYAP_EINVAL, "model %s is a %s, modelType %d", m->name,
                m->type ? "map" : "flow", modelType);
  if (m->type != 0 && isQr)
    return fail(CHAOS_LYAP_EUNSUPPORTED, "map model %s: the QR method has no map branch", m->name);
  if (dimension != m->dim || paramsDim != m->nparams)
    return fail(CHAOS_LYAP_EINVAL, "model %s has dim %d and %d params (got %d, %d)", m->name,
                m->dim, m->nparams, dimension, paramsDim);
  if (expsNum < 1 || expsNum > m->dim) return fail(CHAOS_LYAP_EINVAL, "expsNum out of range");
  if (isQr && expsNum != m->dim)
    return fail(CHAOS_LYAP_EUNSUPPORTED, "QR method needs expsNum == dimension");
  if (!(integrationStep > 0)) return fail(CHAOS_LYAP_EINVAL, "integrationStep must be > 0");
  if (taskNum == 0) return CHAOS_LYAP_OK;
  if (!inits || !params || !lyapExps) return fail(CHAOS_LYAP_EINVAL, "null array");
  chaos::CompatArgs a{};
  a.P = (int64_t)taskNum;
  a.k = expsNum;
  a.method = isQr ? 2 : (isVar ? 1 : 0);
  a.eps = eps;
  a.step = integrationStep;
  a.t_skip = timeSkip;
  a.t_skip_clp = timeSkipClP;
  a.calc_time = calcTime;
  a.add_skip = addSkipSteps;
  a.params = chaos::CView{params, paramsDim, 1};
  a.inits = chaos::View{inits, dimension, 1};
  a.close = closePoints;
  a.lyap = chaos::View{lyapExps, expsNum, 1};
  a.accumulate = 1;
  a.status = nullptr;
  int rc = chaos::launch_compat(m->id, a, 64, (cudaStream_t)stream);
  if (rc == chaos::kErrUnsupported) return fail(CHAOS_LYAP_EUNSUPPORTED, "no kernel for this k");
  if (rc) return cuda_fail((cudaError_t)rc, "cudaLyapunov launch");
  return CHAOS_LYAP_OK;
}

}  // extern "C"
