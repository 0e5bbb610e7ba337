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
  mgs_compat::check(mgs_tanasic_sort(ctx, mgs_compat::DType<T>::value, elements->data(), elements->size(),
                                     static_cast<int>(gpus.size())),
                    "TanasicSort");
  // The engine times the call's phases itself: memory_allocation is the growth
  // of the context's device arena (the first call, or a larger input), and
  // sort_phase the copies, sorts and merges; the arena is kept between calls.
  for (const char* phase : {"memory_allocation", "sort_phase", "memory_deallocation"}) {
    double s = 0;
    mgs_ctx_phase_seconds(ctx, phase, &s);
    TimeDurations::Get()->Set(phase, s);
  }
}
