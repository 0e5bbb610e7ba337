// DataGenerator (src/data_generator.cuh:12-211): same constructor and
// ComputeDistribution<T>(begin, n, name); generation runs in the engine
// (mgs_generate), value for value equal to the reference's distributions.
#pragma once

#include <cstdint>
#include <string>

#include "mgs_runtime.h"

class DataGenerator {
 public:
  explicit DataGenerator(uint32_t distribution_seed, int num_threads = kNumThreads)
      : distribution_seed_(distribution_seed), num_threads_(num_threads) {}

  template <typename T>
  void ComputeDistribution(T* begin, size_t num_elements, const std::string& distribution_type) {
    mgs_compat::check(mgs_generate(mgs_compat::DType<T>::value, distribution_type.c_str(), distribution_seed_, begin,
                                   num_elements),
                      "DataGenerator::ComputeDistribution");
  }

 private:
  const uint32_t distribution_seed_;
  const int num_threads_;  // the reference fixes 128 generator threads; kept for the signature
  inline static constexpr int kNumThreads = 128;
};
