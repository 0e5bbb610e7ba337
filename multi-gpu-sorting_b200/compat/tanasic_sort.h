// P2P sort entry points (src/tanasic_sort.cuh:206-299) on the engine: the
// partitions of `gpus` become gpus.size() chunks of the first listed GPU.
#pragma once

#include <vector>

#include "host_vector.h"
#include "mgs_runtime.h"
#include "time_durations.h"

inline void SetupTanasicSort(const std::vector<int>& gpus) {
  if (!gpus.empty()) mgs_compat::Contexts::get(gpus.front());
}

template <typename T>
void TanasicSort(HostVector<T>* elements, std::vector<int> gpus) {
  if (elements->empty()) return;  // src/tanasic_sort.cuh:225-227
  mgs_ctx* ctx = mgs_compat::Contexts::get(gpus.front());
  TimeDurations::Get()->Tic("memory_allocation");
  TimeDurations::Get()->Toc("memory_allocation");  // the context arena is reserved on first use
  TimeDurations::Get()->Tic("sort_phase");
  mgs_compat::check(mgs_tanasic_sort(ctx, mgs_compat::DType<T>::value, elements->data(), elements->size(),
                                     static_cast<int>(gpus.size())),
                    "TanasicSort");
  TimeDurations::Get()->Toc("sort_phase");
  TimeDurations::Get()->Tic("memory_deallocation");
  TimeDurations::Get()->Toc("memory_deallocation");
}
