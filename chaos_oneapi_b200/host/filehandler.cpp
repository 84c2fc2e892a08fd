// Output writer of the reference (filehandler.cpp:35-89): Data/<Tool> <model>.json
// with {"Parameters", "ID_Tool", "_Data", "Model"}, _Data one row per point of
// std::to_string values (6 decimals) separated by spaces, rows by '\n'.  Next
// to it a full-precision copy of the same rows (.npy, float64), since six
// decimals hide differences far above double rounding.
#include <cassert>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <iostream>

#include "task.h"

static std::string tool_name_of(int tool_id) {
  switch (tool_id) {
    case 0: return "Lyapunov";
    case 1: return "Kneadings";
    case 2: return "Angle";
    case 3: return "minDistance";
    default: return "Unknown";
  }
}

static bool write_npy(const std::string &path, const std::vector<std::vector<double>> &rows) {
  const size_t R = rows.size(), C = R ? rows[0].size() : 0;
  std::string hdr = "{'descr': '<f8', 'fortran_order': False, 'shape': (" + std::to_string(R) +
                    ", " + std::to_string(C) + "), }";
  const size_t total = 10 + hdr.size() + 1;
  hdr.append((64 - total % 64) % 64, ' ');
  hdr.push_back('\n');
  std::ofstream f(path, std::ios::binary);
  if (!f) return false;
  const char magic[] = {'\x93', 'N', 'U', 'M', 'P', 'Y', 1, 0};
  f.write(magic, 8);
  const uint16_t hl = (uint16_t)hdr.size();
  f.write(reinterpret_cast<const char *>(&hl), 2);
  f.write(hdr.data(), (std::streamsize)hdr.size());
  for (const auto &r : rows) f.write(reinterpret_cast<const char *>(r.data()), sizeof(double) * C);
  return (bool)f;
}

int32_t saveCalculatedData(ToolID tool_id, const std::string &modelName, const Parameters *params,
                           const Task *task, const std::string &dir) {
  if (!params || !task || task->mResults.empty()) return -1;
  if (!task->mResultsStr.empty() && task->mResultsStr.size() != task->mResults.size()) return -1;
  json outputData;
  outputData["Parameters"] = params->paramsToJson();
  const std::string tool_name = tool_name_of(tool_id);
  outputData["ID_Tool"] = tool_name;

  std::string data_str;
  data_str.reserve(task->mResults.size() * task->mResults.at(0).size() * 9);
  size_t row_cnt = 0;
  for (const auto &row : task->mResults) {
    for (const auto &val : row) {
      data_str.append(std::to_string(val));
      data_str.append(" ");
    }
    if (!task->mResultsStr.empty()) {
      data_str.append(task->mResultsStr.at(row_cnt));
      data_str.append(" ");
    }
    data_str.at(data_str.size() - 1) = '\n';
    row_cnt += 1;
  }
  outputData["_Data"] = data_str;

  auto &storage = Singleton<ModelFactoryRegistry::Storage>::Instance();
  auto it = storage._data.find(modelName);
  if (it == storage._data.end()) return -1;
  const auto &model = it->second;
  json modelData;
  modelData["Name"] = model._model_name;
  modelData["Dimension"] = model._dimension;
  modelData["Number of parameters"] = model._param_number;
  modelData["Name of parameters"] = model._model_param;
  modelData["Name of phase"] = model._model_phase;
  modelData["Equations"] = model._model_equat;
  modelData["systemType"] = model._type;
  outputData["Model"] = modelData;

  const std::string base = dir + "/" + tool_name + " " + model._model_name;
  std::ofstream out(base + ".json");
  if (!out) {
    std::cout << "Unable to write the file: " << base << ".json" << std::endl;
    return -1;
  }
  out << std::setw(4) << outputData << std::endl;
  if (!out) return -1;
  return write_npy(base + ".npy", task->mResults) ? 0 : -1;
}
