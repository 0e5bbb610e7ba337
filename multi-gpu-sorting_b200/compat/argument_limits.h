// ArgumentLimits: validation of the sort_benchmark options
// (src/argument_limits.cuh:15-311): same names, defaults and accepted values.
// Differences: the gpu-count check is the intended power-of-two test (the
// reference's `size & (size - 1) != 0` parses as `size & ((size - 1) != 0)`,
// :200, and accepts e.g. 6 GPUs); num_buffers is checked against {2, 3}; the
// engine's key types uint32/uint64 and workload distributions are accepted in
// addition to the reference's.
#pragma once

#include <omp.h>

#include <algorithm>
#include <cctype>
#include <cstdint>
#include <limits>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "mgs.h"

class ArgumentLimits {
 public:
  ArgumentLimits() = delete;

  static bool IsDigits(const std::string& s) {
    return !s.empty() && std::all_of(s.begin(), s.end(), [](unsigned char c) { return std::isdigit(c); });
  }
  static bool ParseNumElements(const std::string& s, size_t* v) {
    if (!IsDigits(s)) return false;
    *v = std::stoull(s);
    return true;
  }
  static bool ParseAlgorithm(const std::string& s, std::string* v) {
    *v = s;
    return Contains(Algorithms(), s);
  }
  static bool ParseGpus(const std::string& in, std::vector<int>* gpus) {
    std::string t;
    for (char c : in)
      if (!std::isspace(static_cast<unsigned char>(c))) t += c;
    if (!t.empty() && (t.front() == '{' || t.back() == '}')) {
      if ((t.front() == '{') != (t.back() == '}')) return false;
      t = t.substr(1, t.size() - 2);
    }
    if (t.empty() || t.front() == ',' || t.back() == ',' || t.find(",,") != std::string::npos) return false;
    if (!std::all_of(t.begin(), t.end(), [](unsigned char c) { return std::isdigit(c) || c == ','; })) return false;
    gpus->clear();
    std::stringstream ss(t);
    std::string item;
    while (std::getline(ss, item, ',')) gpus->push_back(std::stoi(item));
    const size_t g = gpus->size();
    if (g == 0 || (g & (g - 1)) != 0) return false;
    if (std::set<int>(gpus->begin(), gpus->end()).size() != g) return false;
    const int count = DeviceCount();
    return std::all_of(gpus->begin(), gpus->end(), [&](int x) { return x >= 0 && x < count; });
  }
  static bool ParseDataType(const std::string& s, std::string* v) {
    *v = s;
    return Contains(DataTypes(), s);
  }
  static bool ParseDistributionType(const std::string& s, std::string* v) {
    *v = s;
    return Contains(Distributions(), s);
  }
  static bool ParseDistributionSeed(const std::string& s, uint32_t* v) {
    if (!IsDigits(s) || std::stoull(s) > std::numeric_limits<uint32_t>::max()) return false;
    *v = static_cast<uint32_t>(std::stoull(s));
    return true;
  }
  static bool ParseNumThreads(const std::string& s, int* v) {
    if (!IsDigits(s)) return false;
    *v = std::stoi(s);
    return *v >= 1 && *v <= omp_get_num_procs();
  }
  static bool ParseChunkSize(const std::string& s, size_t* v) { return ParseNumElements(s, v); }
  static bool ParseMergeGroupSize(const std::string& s, size_t* v) { return ParseNumElements(s, v); }
  static bool ParseNumBuffers(const std::string& s, size_t* v) {
    if (!IsDigits(s)) return false;
    *v = std::stoull(s);
    return *v == 2 || *v == 3;
  }

  static size_t GetDefaultNumElements() { return 0; }
  static std::string GetDefaultAlgorithm() { return Algorithms().front(); }
  static std::vector<int> GetDefaultGpus() { return {0}; }
  static std::string GetDefaultDataType() { return DataTypes().front(); }
  static std::string GetDefaultDistributionType() { return Distributions().front(); }
  static uint32_t GetDefaultDistributionSeed() { return 2147483647u; }
  static int GetDefaultNumThreads() { return omp_get_num_procs(); }
  static size_t GetDefaultChunkSize() { return 0; }
  static size_t GetDefaultMergeGroupSize() { return 1; }
  static size_t GetDefaultNumBuffers() { return 2; }

  static const std::vector<std::string>& Algorithms() {
    static const std::vector<std::string> v = {"tanasic", "gowanlock", "thrust", "boost", "gnu_parallel", "std",
                                               "paradis"};
    return v;
  }
  static const std::vector<std::string>& DataTypes() {
    static const std::vector<std::string> v = {"int", "long", "float", "double", "uint32", "uint64"};
    return v;
  }
  static const std::vector<std::string>& Distributions() {
    static const std::vector<std::string> v = {
        "uniform", "normal", "zero", "staggered", "sorted", "reverse-sorted", "nearly-sorted", "bucket-sorted",
        "full-uniform", "normal0", "zipf", "sorted-full", "reverse-sorted-full", "nearly-sorted-swaps", "all-equal",
        "full-uniform-specials", "zipf-specials", "normal0-specials"};
    return v;
  }
  static int DeviceCount() {
    int c = 0;
    if (mgs_device_count(&c) != MGS_OK) return 0;
    return c;
  }
  static std::string Join(const std::vector<std::string>& v) {
    std::string s = "{";
    for (size_t i = 0; i < v.size(); ++i) s += (i ? ", " : "") + v[i];
    return s + "}";
  }

 private:
  static bool Contains(const std::vector<std::string>& v, const std::string& s) {
    return std::find(v.begin(), v.end(), s) != v.end();
  }
};
