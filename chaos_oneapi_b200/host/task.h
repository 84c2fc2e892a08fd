// Task surface of the reference (task.h:11-73, tasklyapunov.h:8-59):
// init -> allocate -> execute -> accessResult / save -> clear, with a time
// report.  Timings are kept in seconds as doubles (the reference's RaiiTimer
// truncates to whole seconds, raiitimer.h:21).
#pragma once
#include <chrono>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "chaos_lyap.h"
#include "model_factory.h"
#include "tool_params.h"

class Task;
int32_t saveCalculatedData(ToolID tool_id, const std::string &modelName, const Parameters *params,
                           const Task *task, const std::string &dir = "Data");

class Task {
 public:
  struct Clocks {
    double allocate = 0, execute = 0, clear = 0;
  };
  virtual ~Task() = default;
  virtual int init(std::shared_ptr<Parameters> paramsBase, const std::string &modelName) = 0;
  virtual int allocate() = 0;
  virtual int execute() = 0;
  virtual int clear() = 0;
  bool isReady() const { return mReady; }
  double getAllocationTime() const { return mClocks.allocate; }
  double getExecutionTime() const { return mClocks.execute; }
  virtual std::vector<std::vector<double>> &accessResult() = 0;
  void printTimeReport() const;

 protected:
  Clocks mClocks;
  std::vector<std::string> mResultsStr;
  std::vector<std::vector<double>> mResults;
  bool mReady = false;
  friend int32_t saveCalculatedData(ToolID, const std::string &, const Parameters *, const Task *,
                                    const std::string &);
};

// Wall-clock scope timer writing seconds into a slot.
class ScopeTimer {
 public:
  explicit ScopeTimer(double *slot) : slot_(slot), t0_(std::chrono::steady_clock::now()) {}
  ~ScopeTimer() {
    *slot_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
  }

 private:
  double *slot_;
  std::chrono::steady_clock::time_point t0_;
};

class TaskLyapunov : public Task {
 public:
  ~TaskLyapunov() override { clear(); }
  int init(std::shared_ptr<Parameters> paramsBase, const std::string &modelName) override;
  int allocate() override;
  int execute() override;
  int clear() override;
  std::vector<std::vector<double>> &accessResult() override { return mResults; }

  // The host half of allocate(): parameter grid and initial states, no device.
  int prepareInputs();
  // Takes a spectrum (P x k, point-major) computed elsewhere and builds the
  // result rows as execute() does.
  void adoptSpectrum(const double *spectrum);

  // Inputs and per-point outputs of the last run (point-major).
  const std::vector<double> &params() const { return mParams; }
  const std::vector<double> &inits() const { return mInits; }
  const std::vector<int32_t> &status() const { return mStatus; }
  const std::string &lastError() const { return mError; }
  int64_t points() const { return mNodes; }

 private:
  std::shared_ptr<LyapunovParameters> mParameters;
  const ModelFactoryRegistry::ModelData *mModel = nullptr;
  int64_t mNodes = 0;
  double mDelta1 = 0, mDelta2 = 0;
  std::vector<double> mParams, mInits, mSpectrum;
  std::vector<int32_t> mStatus;
  std::vector<chaos_lyap_handle *> mHandles;  // one per GPU
  std::string mError;
  void buildRows();
};
