// Model registry of the reference's plugin surface (model_factory.h:22-68):
// name -> {dimension, parameter count, type, description strings}.  The
// reference also stores five getters of device function pointers; here the
// device code is compiled into libchaos_lyap.so and selected by name through
// the C ABI, so a registry entry carries the name instead.
#pragma once
#include <cstdint>
#include <map>
#include <string>

enum class ModelType { flow, map };

template <typename T> class Singleton {
 public:
  static T &Instance() {
    static T instance;
    return instance;
  }
};

class ModelFactoryRegistry {
 public:
  struct ModelData {
    int32_t _dimension;
    int32_t _param_number;
    std::string _model_name;
    ModelType _type;
    std::string _model_param;
    std::string _model_phase;
    std::string _model_equat;
  };
  struct Storage {
    std::map<std::string, ModelData> _data;
  };

  // Adds a model (the reference's RegisterModel, model_factory.h:36-39).
  static void RegisterModel(const std::string &name, int32_t dim, int32_t param_num, ModelType type,
                            const std::string &model_param, const std::string &model_phase,
                            const std::string &model_equat);
  // Registers every model the native library provides (idempotent).
  static void RegisterNativeModels();
};
