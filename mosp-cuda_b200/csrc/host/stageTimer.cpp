// stageTimer.cpp - optional stage timers, counters and NVTX ranges
// (interface: include/stageTimer.cuh; CSV format "kind,name,value" as in
// SMShovan/MOSP-CUDA src/stageTimer.cu:87-100).
#include "stageTimer.cuh"

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdio>
#include <map>
#include <ostream>
#include <string>
#include <utility>
#include <vector>

namespace {

struct Records {
  bool enabled = false;
  std::string prefix;
  std::vector<std::pair<std::string, double>> stages;
  std::map<std::string, double> counters;
};

Records &records() {
  static Records r;
  return r;
}

}  // namespace

void setInstrumentation(bool enabled) { records().enabled = enabled; }
bool instrumentationEnabled() { return records().enabled; }
void setStagePrefix(const std::string &prefix) { records().prefix = prefix; }
const std::string &stagePrefix() { return records().prefix; }

void recordStage(const std::string &name, double milliseconds) {
  if (records().enabled) records().stages.emplace_back(records().prefix + name, milliseconds);
}

void recordCounter(const std::string &name, double value) {
  if (records().enabled) records().counters[records().prefix + name] += value;
}

double totalStageTime(const std::string &suffix) {
  double total = 0;
  for (const auto &s : records().stages) {
    const std::string &name = s.first;
    if (name.size() >= suffix.size() &&
        name.compare(name.size() - suffix.size(), suffix.size(), suffix) == 0) {
      total += s.second;
    }
  }
  return total;
}

void clearInstrumentation() {
  records().stages.clear();
  records().counters.clear();
}

void printInstrumentation(std::ostream &out) {
  char line[256];
  for (const auto &s : records().stages) {
    std::snprintf(line, sizeof(line), "STAGE   %-52s %12.3f ms\n", s.first.c_str(), s.second);
    out << line;
  }
  for (const auto &c : records().counters) {
    std::snprintf(line, sizeof(line), "COUNTER %-52s %15.0f\n", c.first.c_str(), c.second);
    out << line;
  }
}

bool writeInstrumentationCsv(const std::string &path) {
  FILE *f = std::fopen(path.c_str(), "w");
  if (f == nullptr) return false;
  std::fprintf(f, "kind,name,value\n");
  for (const auto &s : records().stages) std::fprintf(f, "stage,%s,%.6f\n", s.first.c_str(), s.second);
  for (const auto &c : records().counters) std::fprintf(f, "counter,%s,%.0f\n", c.first.c_str(), c.second);
  return std::fclose(f) == 0;
}

void instrumentationSync() {
  if (records().enabled) cudaDeviceSynchronize();
}

ScopedStage::ScopedStage(const std::string &name, bool syncDevice)
    : name_(records().prefix + name), active_(records().enabled), sync_(syncDevice) {
  if (!active_) return;
  if (sync_) cudaDeviceSynchronize();
  nvtxRangePushA(name_.c_str());
  start_ = std::chrono::steady_clock::now();
}

void ScopedStage::stop() {
  if (!active_) return;
  if (sync_) cudaDeviceSynchronize();
  const double ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - start_).count();
  nvtxRangePop();
  records().stages.emplace_back(name_, ms);
  active_ = false;
}
