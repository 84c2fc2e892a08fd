// Command-line program with the reference's flow (main.cpp:11-80): list the
// registered models, read config.json, run the Lyapunov task, write
// Data/Lyapunov <model>.json, print the time report.
//
//   chaos_lyapunov [--model NAME] [--config PATH] [--out DIR]
//
// The reference hard-codes the first registered model (model_id 0,
// main.cpp:12), which with its single registration is Shimizu-Morioka; here
// the model is chosen with --model and defaults to "shimizu".
#include <cstring>
#include <iostream>
#include <string>

#include "chaos_lyap_host.h"
#include "model_factory.h"

int main(int argc, char **argv) {
  std::string model = "shimizu", config = "config.json", out = "Data";
  for (int i = 1; i + 1 < argc; i += 2) {
    if (!std::strcmp(argv[i], "--model")) model = argv[i + 1];
    else if (!std::strcmp(argv[i], "--config")) config = argv[i + 1];
    else if (!std::strcmp(argv[i], "--out")) out = argv[i + 1];
    else {
      std::cerr << "usage: chaos_lyapunov [--model NAME] [--config PATH] [--out DIR]" << std::endl;
      return 2;
    }
  }
  auto &storage = Singleton<ModelFactoryRegistry::Storage>::Instance();
  std::cout << "Available models: " << std::endl;
  int count = 0;
  for (const auto &e : storage._data) {
    std::cout << "Model[" << count++ << "]: \"" << e.first << "\"";
    std::cout << "  Dimension: " << e.second._dimension;
    std::cout << " Number of parameters: " << e.second._param_number << std::endl;
  }
  if (!storage._data.count(model)) {
    std::cout << "Model " << model << " is not registered" << std::endl;
    return 1;
  }
  return chaos_host_run_config(config.c_str(), model.c_str(), out.c_str(), 1) == 0 ? 0 : 1;
}
