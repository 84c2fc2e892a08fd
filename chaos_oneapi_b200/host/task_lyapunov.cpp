// TaskLyapunov over the C ABI (reference tasklyapunov.cpp:13-327).
//  init:     model lookup, node count (tasklyapunov.cpp:13-35)
//  allocate: parameter grid in the reference's order and initial states
//            (:37-71); one sweep handle per GPU instead of 28 scratch buffers
//  execute:  each GPU sweeps a contiguous block of points (remainder spread
//            over the first GPUs; the reference drops it, :19), results as
//            rows [p1, p2, lambda_1..lambda_k] (:230-246)
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <thread>

#include "task.h"

void Task::printTimeReport() const {
  std::printf("\n========TIME REPORT==========\n");
  std::printf(" allocation: %.3f s\n", mClocks.allocate);
  std::printf(" execution:  %.3f s\n", mClocks.execute);
  std::printf(" clear:      %.3f s\n", mClocks.clear);
  std::printf(" Total:      %.3f s\n", mClocks.allocate + mClocks.execute + mClocks.clear);
  std::printf("==============================\n\n");
}

int TaskLyapunov::init(std::shared_ptr<Parameters> paramsBase, const std::string &modelName) {
  mParameters = std::dynamic_pointer_cast<LyapunovParameters>(paramsBase);
  if (!mParameters) return -1;
  auto &storage = Singleton<ModelFactoryRegistry::Storage>::Instance();
  auto it = storage._data.find(modelName);
  if (it == storage._data.end()) {
    mError = "unknown model " + modelName;
    return -1;
  }
  mModel = &it->second;
  mNodes = (int64_t)mParameters->first_sweep_param[3] * (int64_t)mParameters->second_sweep_param[3];
  return 0;
}

static int fill_desc(const LyapunovParameters &p, const std::string &model, int device,
                     chaos_lyap_desc *d) {
  chaos_lyap_desc_init(d);
  std::snprintf(d->model, sizeof d->model, "%s", model.c_str());
  d->k = p.lyapunov_exponent_num;
  d->method = p.is_qr ? CHAOS_METHOD_QR : (p.is_var ? CHAOS_METHOD_VAR : CHAOS_METHOD_FD);
  d->eps = p.epsilon;
  d->h = p.integration_step;
  d->t_transient = p.skip_time_attractor;
  d->t_align = p.skip_time_slave_trajectory;
  d->t_avg = p.total_time;
  d->dt_renorm = p.skip_time_normalization;
  d->rtol = p.rtol;
  d->atol = p.atol;
  d->escape = p.escape;
  d->max_steps = p.max_steps;
  d->device = device;
  d->gs = p.gram_schmidt == "mgs" ? CHAOS_GS_MODIFIED : CHAOS_GS_CLASSICAL;
  if (p.integrator == "dverk65") d->integrator = CHAOS_INTEG_DVERK65;
  else if (p.integrator == "dopri5") d->integrator = CHAOS_INTEG_DOPRI5;
  else d->integrator = CHAOS_INTEG_DVERK_FIXED;
  if (p.precision == "fp32") d->precision = CHAOS_PREC_FP32;
  else if (p.precision == "fp64") d->precision = CHAOS_PREC_FP64;
  else d->precision = CHAOS_PREC_COMPAT_FP64;
  return 0;
}

int TaskLyapunov::prepareInputs() {
  if (!mModel) return -1;
  const LyapunovParameters &p = *mParameters;
  const int m = mModel->_param_number, n = mModel->_dimension;
  if ((int)p.initial_model_params.size() < m || (int)p.initial_state.size() < n) {
    mError = "initial_model_params / initial_state shorter than the model";
    return -1;
  }
  mDelta1 = std::fabs(p.first_sweep_param[2] - p.first_sweep_param[1]) / (p.first_sweep_param[3] - 1);
  mDelta2 = std::fabs(p.second_sweep_param[2] - p.second_sweep_param[1]) / (p.second_sweep_param[3] - 1);
  mParams.assign((size_t)mNodes * m, 0.0);
  chaos_lyap_make_grid(m, p.initial_model_params.data(), p.first_sweep_param.data(),
                       p.second_sweep_param.data(), mParams.data());
  mInits.assign((size_t)mNodes * n, 0.0);
  if (p.init_jitter > 0) {
    chaos_lyap_make_inits(n, mNodes, p.initial_state.data(), p.init_jitter, 0, p.seed, mInits.data());
  } else {
    for (int64_t i = 0; i < mNodes; ++i)
      std::memcpy(&mInits[i * n], p.initial_state.data(), sizeof(double) * n);
  }
  mSpectrum.assign((size_t)mNodes * p.lyapunov_exponent_num, 0.0);
  mStatus.assign((size_t)mNodes, 0);
  mResults.reserve(mNodes);
  return 0;
}

int TaskLyapunov::allocate() {
  ScopeTimer t(&mClocks.allocate);
  if (prepareInputs()) return -1;
  const LyapunovParameters &p = *mParameters;
  for (int g = 0; g < std::max(1, p.num_GPUs); ++g) {
    chaos_lyap_desc d;
    fill_desc(p, mModel->_model_name, g, &d);
    chaos_lyap_handle *h = nullptr;
    if (chaos_lyap_create(&d, &h) != CHAOS_LYAP_OK) {
      mError = chaos_lyap_last_error();
      std::cerr << "error: " << mError << std::endl;
      clear();
      return -1;
    }
    mHandles.push_back(h);
  }
  return 0;
}

int TaskLyapunov::execute() {
  ScopeTimer t(&mClocks.execute);
  mResults.clear();
  mReady = false;
  if (mHandles.empty()) return -1;
  const LyapunovParameters &p = *mParameters;
  const int m = mModel->_param_number, n = mModel->_dimension, k = p.lyapunov_exponent_num;
  const int G = (int)mHandles.size();
  (void)p;
  std::vector<int> rc(G, 0);
  std::vector<std::string> err(G);
  std::vector<std::thread> workers;
  for (int g = 0; g < G; ++g) {
    const int64_t base = mNodes / G, extra = mNodes % G;
    const int64_t s = g * base + std::min<int64_t>(g, extra);
    const int64_t cnt = base + (g < extra ? 1 : 0);
    workers.emplace_back([&, g, s, cnt] {
      if (cnt == 0) return;
      rc[g] = chaos_lyap_run_host(mHandles[g], cnt, &mParams[s * m], &mInits[s * n],
                                  &mSpectrum[s * k], &mStatus[s], nullptr, nullptr);
      if (rc[g]) err[g] = chaos_lyap_last_error();
    });
  }
  for (auto &w : workers) w.join();
  for (int g = 0; g < G; ++g)
    if (rc[g]) {
      mError = err[g];
      std::cerr << "error: GPU " << g << ": " << mError << std::endl;
      return -1;
    }
  buildRows();
  return (int)mNodes;
}

void TaskLyapunov::adoptSpectrum(const double *spectrum) {
  std::memcpy(mSpectrum.data(), spectrum, sizeof(double) * mSpectrum.size());
  buildRows();
}

// Rows [p1, p2, lambda_1..lambda_k] in the reference's order (tasklyapunov.cpp:230-246).
void TaskLyapunov::buildRows() {
  const LyapunovParameters &p = *mParameters;
  const int k = p.lyapunov_exponent_num;
  mResults.clear();
  int64_t row = 0;
  for (int a = 0; a < (int)p.first_sweep_param[3]; ++a)
    for (int b = 0; b < (int)p.second_sweep_param[3]; ++b) {
      std::vector<double> r;
      r.reserve(2 + k);
      r.push_back(p.first_sweep_param[1] + a * mDelta1);
      r.push_back(p.second_sweep_param[1] + b * mDelta2);
      for (int i = 0; i < k; ++i) r.push_back(mSpectrum[row * k + i]);
      mResults.push_back(std::move(r));
      ++row;
    }
  mReady = true;
}

int TaskLyapunov::clear() {
  ScopeTimer t(&mClocks.clear);
  for (auto *h : mHandles) chaos_lyap_destroy(h);
  mHandles.clear();
  return 0;
}
