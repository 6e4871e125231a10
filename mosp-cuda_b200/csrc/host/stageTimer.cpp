// stageTimer.cpp - optional stage instrumentation (interface:
// include/stageTimer.cuh).
//
// One process-wide ledger, guarded by a mutex so that the worker threads of
// the serving loop and the pipeline's helper threads can record into it at
// once. Stages keep the order in which they finished; counters are summed
// per name and listed by name. The text forms are the contract the
// reference's tools print and scripts read: "STAGE <name> <ms> ms" and
// "COUNTER <name> <value>" lines, and a "kind,name,value" CSV.
#include "stageTimer.cuh"

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <fstream>
#include <iomanip>
#include <map>
#include <mutex>
#include <ostream>
#include <string>
#include <vector>

namespace {

class Ledger {
public:
  bool on() const { return on_; }
  void setOn(bool on) { on_ = on; }

  std::string qualified(const std::string &name) {
    std::lock_guard<std::mutex> hold(mutex_);
    return scope_ + name;
  }
  void setScope(const std::string &scope) {
    std::lock_guard<std::mutex> hold(mutex_);
    scope_ = scope;
  }
  const std::string &scope() const { return scope_; }

  void stage(const std::string &fullName, double ms) {
    std::lock_guard<std::mutex> hold(mutex_);
    stages_.push_back(Stage{fullName, ms});
  }
  void count(const std::string &fullName, double value) {
    std::lock_guard<std::mutex> hold(mutex_);
    counters_[fullName] += value;
  }
  double sumEndingWith(const std::string &suffix) {
    std::lock_guard<std::mutex> hold(mutex_);
    double sum = 0.0;
    for (const Stage &s : stages_) {
      if (endsWith(s.name, suffix)) sum += s.ms;
    }
    return sum;
  }
  void reset() {
    std::lock_guard<std::mutex> hold(mutex_);
    stages_.clear();
    counters_.clear();
  }

  // "STAGE   <name, 52 wide> <ms, 12 wide, 3 decimals> ms" and
  // "COUNTER <name, 52 wide> <value, 15 wide, no decimals>"
  void render(std::ostream &out) {
    std::lock_guard<std::mutex> hold(mutex_);
    const std::ios::fmtflags flags = out.flags();
    const std::streamsize precision = out.precision();
    out << std::fixed;
    for (const Stage &s : stages_) {
      out << "STAGE   " << std::left << std::setw(52) << s.name << ' ' << std::right << std::setw(12)
          << std::setprecision(3) << s.ms << " ms\n";
    }
    for (const auto &kv : counters_) {
      out << "COUNTER " << std::left << std::setw(52) << kv.first << ' ' << std::right << std::setw(15)
          << std::setprecision(0) << kv.second << '\n';
    }
    out.flags(flags);
    out.precision(precision);
  }

  bool saveCsv(const std::string &path) {
    std::ofstream file(path);
    if (!file) return false;
    std::lock_guard<std::mutex> hold(mutex_);
    file << "kind,name,value\n" << std::fixed;
    for (const Stage &s : stages_) file << "stage," << s.name << ',' << std::setprecision(6) << s.ms << '\n';
    for (const auto &kv : counters_) {
      file << "counter," << kv.first << ',' << std::setprecision(0) << kv.second << '\n';
    }
    file.flush();
    return static_cast<bool>(file);
  }

private:
  struct Stage {
    std::string name;
    double ms;
  };
  static bool endsWith(const std::string &s, const std::string &tail) {
    return s.size() >= tail.size() && std::equal(tail.rbegin(), tail.rend(), s.rbegin());
  }

  bool on_ = false;
  std::mutex mutex_;
  std::string scope_;
  std::vector<Stage> stages_;
  std::map<std::string, double> counters_;
};

Ledger &ledger() {
  static Ledger instance;
  return instance;
}

}  // namespace

void setInstrumentation(bool enabled) { ledger().setOn(enabled); }
bool instrumentationEnabled() { return ledger().on(); }
void setStagePrefix(const std::string &prefix) { ledger().setScope(prefix); }
const std::string &stagePrefix() { return ledger().scope(); }

void recordStage(const std::string &name, double milliseconds) {
  if (ledger().on()) ledger().stage(ledger().qualified(name), milliseconds);
}

void recordCounter(const std::string &name, double value) {
  if (ledger().on()) ledger().count(ledger().qualified(name), value);
}

double totalStageTime(const std::string &suffix) { return ledger().sumEndingWith(suffix); }
void clearInstrumentation() { ledger().reset(); }
void printInstrumentation(std::ostream &out) { ledger().render(out); }
bool writeInstrumentationCsv(const std::string &path) { return ledger().saveCsv(path); }

void instrumentationSync() {
  if (ledger().on()) cudaDeviceSynchronize();
}

// A stage that asks for device synchronization measures the GPU work queued
// inside it on any stream: the device is drained when the stage opens (so
// earlier work is not counted) and when it closes.
ScopedStage::ScopedStage(const std::string &name, bool syncDevice)
    : name_(), active_(ledger().on()), sync_(syncDevice) {
  if (!active_) return;
  name_ = ledger().qualified(name);
  if (sync_) cudaDeviceSynchronize();
  nvtxRangePushA(name_.c_str());
  start_ = std::chrono::steady_clock::now();
}

void ScopedStage::stop() {
  if (!active_) return;
  active_ = false;
  if (sync_) cudaDeviceSynchronize();
  const std::chrono::duration<double, std::milli> elapsed = std::chrono::steady_clock::now() - start_;
  nvtxRangePop();
  ledger().stage(name_, elapsed.count());
}
