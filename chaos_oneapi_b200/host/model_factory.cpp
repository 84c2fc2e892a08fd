#include "model_factory.h"

#include "chaos_lyap.h"

void ModelFactoryRegistry::RegisterModel(const std::string &name, int32_t dim, int32_t param_num,
                                         ModelType type, const std::string &model_param,
                                         const std::string &model_phase,
                                         const std::string &model_equat) {
  Storage &storage = Singleton<Storage>::Instance();
  storage._data.insert(std::make_pair(
      name, ModelData{dim, param_num, name, type, model_param, model_phase, model_equat}));
}

void ModelFactoryRegistry::RegisterNativeModels() {
  const int n = chaos_lyap_model_count();
  for (int i = 0; i < n; ++i) {
    char name[64], text[3][512];
    if (chaos_lyap_model_name(i, name, sizeof name) != CHAOS_LYAP_OK) continue;
    int32_t dim = 0, np = 0, type = 0;
    chaos_lyap_query_model(name, &dim, &np, &type);
    for (int w = 0; w < 3; ++w) chaos_lyap_model_text(name, w, text[w], sizeof text[w]);
    RegisterModel(name, dim, np, type == 0 ? ModelType::flow : ModelType::map, text[0], text[1],
                  text[2]);
  }
}

namespace {
// Static registration, like the reference's per-model registrar objects
// (shimizu.dp.cpp:70-211).
struct NativeModels {
  NativeModels() { ModelFactoryRegistry::RegisterNativeModels(); }
} register_native_models;
}  // namespace
