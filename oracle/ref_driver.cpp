// Test infrastructure only (oracle build).  A C entry point into the
// reference's own Lyapunov launcher, cudaLyapunov (cuda/lyapunov.dp.hpp:10-17,
// cuda/lyapunov.dp.cpp:321-367), compiled from the reference sources on the
// host (see oracle/Makefile).  It does what TaskLyapunov::allocate/execute
// (tasklyapunov.cpp:37-250) do around that call, except that the caller
// supplies the per-point parameters and initial states, so seeded per-point
// inputs can be fed to the reference unchanged:
//   * looks the model up in the reference's registry (model_factory.h:65-68)
//     and fetches its function pointers the way tasklyapunov.cpp:195-203 does;
//   * sizes the work-item scratch for the 32x32 work-items the launcher
//     forces (cuda/lyapunov.dp.cpp:331-332), times n (times n again for QR),
//     like tasklyapunov.cpp:104-176;
//   * zero-initialises lyapExps (the reference accumulates into it with +=).
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "cuda/lyapunov.dp.hpp"
#include "cuda/tools/dopri.dp.hpp"
#include "singleton.h"

namespace {
struct Buf {
  double *p = nullptr;
  explicit Buf(size_t n) { p = static_cast<double *>(std::calloc(n ? n : 1, sizeof(double))); }
  ~Buf() { std::free(p); }
};
}  // namespace

extern "C" {

// Comma-separated names of every registered model. Returns the length needed.
int chaos_ref_model_names(char *buf, int buflen) {
  auto &storage = Singleton<ModelFactoryRegistry::Storage>::Instance();
  std::string s;
  for (auto &kv : storage._data) {
    if (!s.empty()) s += ",";
    s += kv.first;
  }
  if (buf && buflen > 0) {
    std::strncpy(buf, s.c_str(), (size_t)buflen - 1);
    buf[buflen - 1] = 0;
  }
  return (int)s.size() + 1;
}

int chaos_ref_model_info(const char *name, int *dim, int *nparams, int *is_map) {
  auto &storage = Singleton<ModelFactoryRegistry::Storage>::Instance();
  auto it = storage._data.find(name);
  if (it == storage._data.end()) return -1;
  *dim = it->second._dimension;
  *nparams = it->second._param_number;
  *is_map = it->second._type == ModelType::map ? 1 : 0;
  return 0;
}

// params: P*m (AoS, point-major, as tasklyapunov.cpp:47-63 lays them out);
// inits: P*n, advanced in place to the end states (as the reference does);
// lyap_out: P*k.  Returns 0, or -1 for an unknown model / bad arguments.
int chaos_ref_lyapunov(const char *name, int is_qr, int is_var, long long P, const double *params,
                       double *inits, double eps, double step, int k, double t_skip,
                       double t_skip_clp, double calc_time, double add_skip_steps, double *lyap_out) {
  auto &storage = Singleton<ModelFactoryRegistry::Storage>::Instance();
  auto it = storage._data.find(name);
  if (it == storage._data.end() || P <= 0 || k <= 0) return -1;
  ModelFactoryRegistry::ModelData &md = it->second;
  const int n = md._dimension, m = md._param_number;

  diffSysFunc f = nullptr;
  diffSysFuncVar fv = nullptr, fq = nullptr;
  md._model_func(&f);
  if (md._func_var) md._func_var(&fv);
  if (md._func_Q) md._func_Q(&fq);

  const size_t items = 32 * 32;
  const size_t cuda_size = items * (size_t)n;  // doubles per scratch buffer
  Buf prm((size_t)P * m), ini((size_t)P * n), close((size_t)P * k * n), lyap((size_t)P * k);
  std::memcpy(prm.p, params, sizeof(double) * (size_t)P * m);
  std::memcpy(ini.p, inits, sizeof(double) * (size_t)P * n);
  Buf arg(cuda_size), k1(cuda_size), k2(cuda_size), k3(cuda_size), k4(cuda_size), k5(cuda_size),
      k6(cuda_size), k7(cuda_size), k8(cuda_size), proj(cuda_size);
  const size_t qn = is_qr ? cuda_size * n : 1;
  Buf U(qn), R(qn), Q(qn), argQ(qn), k1Q(qn), k2Q(qn), k3Q(qn), k4Q(qn), k5Q(qn), k6Q(qn), k7Q(qn),
      k8Q(qn);

  cudaLyapunov(32, 32, (size_t)P, is_qr != 0, is_var != 0, md._type, ini.p, close.p, n, f, fv, fq,
               prm.p, m, eps, step, lyap.p, k, t_skip, t_skip_clp, calc_time, add_skip_steps, arg.p,
               U.p, R.p, Q.p, k1.p, k2.p, k3.p, k4.p, k5.p, k6.p, k7.p, k8.p, argQ.p, k1Q.p, k2Q.p,
               k3Q.p, k4Q.p, k5Q.p, k6Q.p, k7Q.p, k8Q.p, proj.p);
  dpct::get_current_device().queues_wait_and_throw();

  std::memcpy(lyap_out, lyap.p, sizeof(double) * (size_t)P * k);
  std::memcpy(inits, ini.p, sizeof(double) * (size_t)P * n);
  return 0;
}

// The reference's Dormand-Prince step, dopriStep (cuda/tools/dopri.dp.cpp:7-139),
// driven over one state trajectory the way a caller of that tool drives it:
// time starts at 0 (the first call sets facOld = 1e-4 and evaluates k1,
// :65-68), each call makes one accepted step (rejected attempts are retried
// inside the call, :133-138) and leaves the next step's proposal in `step` and
// the FSAL derivative in k1.  After call i: t_out[i] = time, h_out[i] = step,
// x_out[i*n .. i*n+n-1] = the state.  tolLocErr = atol, tolGlobErr = rtol
// (error weights atol + rtol max(|y0|, |y1|), :98-104).  Returns 0, or -1 for
// an unknown model / bad arguments.
int chaos_ref_dopri_trajectory(const char *name, const double *params, const double *x0,
                               double h0, double hmax, double atol, double rtol, int nsteps,
                               double *t_out, double *h_out, double *x_out) {
  auto &storage = Singleton<ModelFactoryRegistry::Storage>::Instance();
  auto it = storage._data.find(name);
  if (it == storage._data.end() || nsteps < 0 || !(h0 > 0)) return -1;
  ModelFactoryRegistry::ModelData &md = it->second;
  if (md._type != ModelType::flow) return -1;
  const int n = md._dimension, m = md._param_number;
  diffSysFunc f = nullptr;
  md._model_func(&f);
  std::vector<double> prm(params, params + m), x(x0, x0 + n), spare(n), ysti(n), arg(n), k1(n),
      k2(n), k3(n), k4(n), k5(n), k6(n);
  double step = h0, time = 0.0, fac_old = 0.0;
  for (int i = 0; i < nsteps; i++) {
    dopriStep(x.data(), n, f, prm.data(), step, hmax, atol, rtol, spare.data(), ysti.data(),
              arg.data(), k1.data(), k2.data(), k3.data(), k4.data(), k5.data(), k6.data(), time,
              fac_old);
    t_out[i] = time;
    h_out[i] = step;
    std::memcpy(x_out + (size_t)i * n, x.data(), sizeof(double) * n);
  }
  return 0;
}

}  // extern "C"
