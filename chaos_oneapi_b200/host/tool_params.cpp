#include "tool_params.h"

#include <cstdio>
#include <fstream>
#include <iostream>
#include <stdexcept>

namespace {
void print_vec(const char *title, const std::vector<double> &v) {
  std::cout << title;
  int count = 0;
  for (const auto &e : v) std::cout << " [" << count++ << "] = " << e << " ";
  std::cout << std::endl;
}
}  // namespace

void LyapunovParameters::Print() const {
  std::cout << "************************************************************************" << std::endl;
  std::cout << "Lyapunov's parameters: " << std::endl;
  std::cout << "Number of lyapunov's exponent: " << lyapunov_exponent_num << std::endl;
  std::cout << "Epsilon: " << epsilon << std::endl;
  std::cout << "Step of integration: " << integration_step << std::endl;
  std::cout << "Time skip to reach attractor: " << skip_time_attractor << std::endl;
  std::cout << "Time skip for complementary trajectories: " << skip_time_slave_trajectory << std::endl;
  std::cout << "Time skip for Lyapunov's normalization: " << skip_time_normalization << std::endl;
  std::cout << "Total time: " << total_time << std::endl;
  std::cout << "Samples num: " << samples_num << std::endl;
  print_vec("Initial state: ", initial_state);
  print_vec("Initial parameters of model: ", initial_model_params);
  print_vec("First sweep parameter: ", first_sweep_param);
  print_vec("Second sweep parameter: ", second_sweep_param);
  std::cout << "Number of GPUs: " << num_GPUs << std::endl;
  std::cout << "Using QR: " << std::boolalpha << is_qr << std::endl;
  std::cout << "Using VAR: " << std::boolalpha << is_var << std::endl;
  std::cout << "Integrator: " << integrator << ", precision: " << precision << std::endl;
  std::cout << "************************************************************************" << std::endl
            << std::endl;
}

// Same keys as tool_params.cpp:53-75; the optional keys only when given.
json LyapunovParameters::paramsToJson() const {
  json params;
  params["lyapunov_exponent_num"] = lyapunov_exponent_num;
  params["epsilon"] = epsilon;
  params["integration_step"] = integration_step;
  params["skip_time_attractor"] = skip_time_attractor;
  params["skip_time_slave_trajectory"] = skip_time_slave_trajectory;
  params["skip_time_normalization"] = skip_time_normalization;
  params["total_time"] = total_time;
  params["samples_num"] = samples_num;
  params["initial_state"] = initial_state;
  params["initial_model_params"] = initial_model_params;
  params["first_sweep_param"] = first_sweep_param;
  params["second_sweep_param"] = second_sweep_param;
  params["num_GPUs"] = num_GPUs;
  params["using_qr"] = is_qr;
  params["using_var"] = is_var;
  for (auto &kv : extended.items()) params[kv.key()] = kv.value();
  return params;
}

LyapunovParameters::LyapunovParameters(const json &jsonConfig, const std::string &modelName) {
  bool found = false;
  try {
    jsonConfig.at("hardware").at("num_GPUs").get_to(num_GPUs);
    auto conf = jsonConfig.at("tool").at("lyapunov");
    conf.at("samples_num").get_to(samples_num);
    conf.at("using_qr").get_to(is_qr);
    conf.at("using_var").get_to(is_var);
    for (const auto &c : jsonConfig.at("systems").items()) {
      const json &v = c.value();
      if (v.at("model_name") != modelName) continue;
      found = true;
      v.at("lyapunov_exponent_num").get_to(lyapunov_exponent_num);
      v.at("epsilon").get_to(epsilon);
      v.at("integration_step").get_to(integration_step);
      v.at("skip_time_attractor").get_to(skip_time_attractor);
      v.at("skip_time_slave_trajectory").get_to(skip_time_slave_trajectory);
      v.at("skip_time_normalization").get_to(skip_time_normalization);
      v.at("total_time").get_to(total_time);
      v.at("initial_state").get_to(initial_state);
      v.at("initial_model_params").get_to(initial_model_params);
      v.at("first_sweep_param").get_to(first_sweep_param);
      v.at("second_sweep_param").get_to(second_sweep_param);
      const char *opt[] = {"integrator", "precision", "gram_schmidt", "rtol", "atol",
                           "init_jitter", "seed", "escape", "max_steps"};
      for (const char *k : opt)
        if (v.contains(k)) extended[k] = v.at(k);
      if (v.contains("integrator")) v.at("integrator").get_to(integrator);
      if (v.contains("precision")) v.at("precision").get_to(precision);
      if (v.contains("gram_schmidt")) v.at("gram_schmidt").get_to(gram_schmidt);
      if (v.contains("rtol")) v.at("rtol").get_to(rtol);
      if (v.contains("atol")) v.at("atol").get_to(atol);
      if (v.contains("init_jitter")) v.at("init_jitter").get_to(init_jitter);
      if (v.contains("seed")) v.at("seed").get_to(seed);
      if (v.contains("escape")) v.at("escape").get_to(escape);
      if (v.contains("max_steps")) v.at("max_steps").get_to(max_steps);
      break;
    }
  } catch (std::exception &e) {
    std::printf("error: model: %s config exception: %s\n", modelName.c_str(), e.what());
    throw std::runtime_error("config error");
  }
  if (!found) {
    std::printf("error: model: %s config not found\n", modelName.c_str());
    throw std::runtime_error("config error");
  }
  if (first_sweep_param.size() != 4 || second_sweep_param.size() != 4) {
    std::printf("error: model: %s config sweep parameters size error\n", modelName.c_str());
    throw std::runtime_error("config error");
  }
  // The fixed-step integrator is the reference-exact path; the adaptive ones
  // default to FP64 when no precision form is named.
  if (integrator == "dverk") precision = "compat";
  else if (precision == "compat") precision = "fp64";
}

std::shared_ptr<Parameters> ConfigFactory::paramsFromConfigFile(ToolID toolId,
                                                                const std::string &modelName,
                                                                const std::string &path) {
  if (toolId != ToolID::LYAPUNOV && toolId != ToolID::ANGLE) return nullptr;
  std::ifstream config(path);
  if (!config.good()) {
    std::printf("error: config file: %s not found\n", path.c_str());
    return nullptr;
  }
  json jsonConfig;
  try {
    config >> jsonConfig;
  } catch (...) {
    std::printf("error: config file: %s parse failure\n", path.c_str());
    return nullptr;
  }
  return std::make_shared<LyapunovParameters>(jsonConfig, modelName);
}

std::shared_ptr<Parameters> ConfigFactory::paramsFromJson(ToolID toolId, const std::string &modelName,
                                                          const json &jsonConfig) {
  if (toolId != ToolID::LYAPUNOV && toolId != ToolID::ANGLE) return nullptr;
  return std::make_shared<LyapunovParameters>(jsonConfig, modelName);
}
