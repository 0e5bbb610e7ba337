// TimeDurations: named wall-clock phases (the reference's singleton,
// src/time_durations.cuh:7-39), same interface; also thread-safe here.
#pragma once

#include <chrono>
#include <map>
#include <mutex>
#include <string>

class TimeDurations {
 public:
  static TimeDurations* Get() {
    static TimeDurations instance;
    return &instance;
  }
  TimeDurations(const TimeDurations&) = delete;
  void operator=(const TimeDurations&) = delete;

  void Tic(const std::string& key) {
    std::lock_guard<std::mutex> lock(mutex_);
    begin_time_[key] = std::chrono::high_resolution_clock::now();
  }
  void Toc(const std::string& key) {
    std::lock_guard<std::mutex> lock(mutex_);
    durations[key] = std::chrono::high_resolution_clock::now() - begin_time_.at(key);
  }
  // Records a phase measured elsewhere (the engine reports its own phases).
  void Set(const std::string& key, double seconds) {
    std::lock_guard<std::mutex> lock(mutex_);
    durations[key] = std::chrono::duration<double>(seconds);
  }
  std::chrono::duration<double> TotalExecutionTime() {
    std::lock_guard<std::mutex> lock(mutex_);
    std::chrono::duration<double> total(0);
    for (const auto& d : durations) total += d.second;
    return total;
  }

  std::map<std::string, std::chrono::duration<double>> durations;

 private:
  TimeDurations() = default;
  std::mutex mutex_;
  std::map<std::string, std::chrono::time_point<std::chrono::high_resolution_clock>> begin_time_;
};
