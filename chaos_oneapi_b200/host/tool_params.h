// Configuration of the Lyapunov tool: the reference's LyapunovParameters
// (tool_params.h:23-44, tool_params.cpp:77-122) with the same config.json keys,
// plus optional keys that select this library's integrators and precision
// forms.  Without the optional keys the sweep is the reference's (fixed-step
// DVERK, reference-exact FP64).
#pragma once
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include <nlohmann/json.hpp>

using json = nlohmann::json;

enum ToolID { UNDEFINED = -1, LYAPUNOV = 0, ANGLE = 2, KNEADING = 1 };

class Parameters {
 public:
  virtual ~Parameters() = default;
  virtual void Print() const {}
  virtual json paramsToJson() const = 0;
};

class LyapunovParameters : public Parameters {
 public:
  LyapunovParameters(const json &jsonConfig, const std::string &modelName);
  void Print() const override;
  json paramsToJson() const override;

  // reference keys (tool_params.cpp:80-104)
  bool is_qr = true;
  bool is_var = true;
  int32_t lyapunov_exponent_num = 0;
  int32_t num_GPUs = 1;
  int32_t samples_num = 1;
  double epsilon = 0;
  double integration_step = 0;
  double skip_time_attractor = 0;
  double skip_time_slave_trajectory = 0;
  double skip_time_normalization = 0;
  double total_time = 0;
  std::vector<double> initial_state;
  std::vector<double> initial_model_params;
  std::vector<double> first_sweep_param;
  std::vector<double> second_sweep_param;

  // optional keys of this library (in the system entry; absent = reference)
  std::string integrator = "dverk";   // dverk | dverk65 | dopri5
  std::string precision = "compat";   // compat | fp64 | fp32
  std::string gram_schmidt = "cgs";   // cgs | mgs
  double rtol = 1e-10, atol = 1e-10;
  double init_jitter = 0.0;           // U(-a, a) added per point to initial_state
  uint64_t seed = 0;
  double escape = 1e4;
  int64_t max_steps = 100000000;
  json extended;                      // the optional keys as given, echoed in the output
};

struct ConfigFactory {
  static std::shared_ptr<Parameters> paramsFromConfigFile(ToolID toolId, const std::string &modelName,
                                                          const std::string &path = "config.json");
  static std::shared_ptr<Parameters> paramsFromJson(ToolID toolId, const std::string &modelName,
                                                    const json &jsonConfig);
};
