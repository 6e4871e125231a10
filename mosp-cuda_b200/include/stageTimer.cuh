#ifndef MOSP_B200_STAGE_TIMER_CUH
#define MOSP_B200_STAGE_TIMER_CUH

// Optional stage instrumentation (wall-clock stage timers, counters, NVTX
// ranges), declared as in the reference (SMShovan/MOSP-CUDA
// headers/stageTimer.cuh:21-66). Disabled unless enabled (mosp --timing);
// the CSV format is "kind,name,value".

#include <chrono>
#include <iosfwd>
#include <string>

void setInstrumentation(bool enabled);
bool instrumentationEnabled();

void setStagePrefix(const std::string &prefix);
const std::string &stagePrefix();

void recordStage(const std::string &name, double milliseconds);
void recordCounter(const std::string &name, double value);
double totalStageTime(const std::string &suffix);
void clearInstrumentation();
void printInstrumentation(std::ostream &out);
bool writeInstrumentationCsv(const std::string &path);
void instrumentationSync();

/// RAII stage timer; with syncDevice the device is synchronized at both
/// ends (only while instrumentation is enabled).
class ScopedStage {
public:
  explicit ScopedStage(const std::string &name, bool syncDevice = false);
  ~ScopedStage() { stop(); }
  ScopedStage(const ScopedStage &) = delete;
  ScopedStage &operator=(const ScopedStage &) = delete;
  void stop();

private:
  std::string name_;
  bool active_;
  bool sync_;
  std::chrono::steady_clock::time_point start_;
};

#endif // MOSP_B200_STAGE_TIMER_CUH
