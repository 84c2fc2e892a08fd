// C entry points of the host surface (include/chaos_lyap_host.h).
#include <iostream>

#include "chaos_lyap_host.h"
#include "task.h"

namespace {
std::shared_ptr<LyapunovParameters> load(const char *config_path, const char *model) {
  try {
    auto p = ConfigFactory::paramsFromConfigFile(ToolID::LYAPUNOV, model, config_path);
    return std::dynamic_pointer_cast<LyapunovParameters>(p);
  } catch (const std::exception &e) {
    std::cerr << "error: " << e.what() << std::endl;
    return nullptr;
  }
}
}  // namespace

extern "C" int chaos_host_run_config(const char *config_path, const char *model, const char *out_dir,
                                     int verbose) {
  auto params = load(config_path, model);
  if (!params) return -1;
  if (verbose) params->Print();
  TaskLyapunov task;
  if (task.init(params, model) || task.allocate() || task.execute() < 0) {
    std::cerr << "error: " << task.lastError() << std::endl;
    return -1;
  }
  int rc = 0;
  if (task.isReady()) rc = saveCalculatedData(ToolID::LYAPUNOV, model, params.get(), &task, out_dir);
  task.clear();
  if (verbose) task.printTimeReport();
  return rc;
}

extern "C" int chaos_host_plan(const char *config_path, const char *model, double *params_out,
                               double *inits_out, int64_t *P_out) {
  auto params = load(config_path, model);
  if (!params) return -1;
  TaskLyapunov task;
  if (task.init(params, model) || task.prepareInputs()) return -1;
  if (P_out) *P_out = task.points();
  if (params_out) std::copy(task.params().begin(), task.params().end(), params_out);
  if (inits_out) std::copy(task.inits().begin(), task.inits().end(), inits_out);
  return 0;
}

extern "C" int chaos_host_save(const char *config_path, const char *model, const double *spectrum,
                               const char *out_dir) {
  auto params = load(config_path, model);
  if (!params || !spectrum) return -1;
  TaskLyapunov task;
  if (task.init(params, model) || task.prepareInputs()) return -1;
  task.adoptSpectrum(spectrum);
  return saveCalculatedData(ToolID::LYAPUNOV, model, params.get(), &task, out_dir);
}
