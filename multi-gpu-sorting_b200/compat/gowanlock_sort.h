// HET sort entry points (src/gowanlock_sort.cuh:117-125,395-483) on the engine:
// the out-of-core chunk pipeline of one GPU (the first listed) with the GPU
// k-way merge, or the reference's CPU multiway merge when MGS_HET_CPU_MERGE
// is set in the environment.
#pragma once

#include <omp.h>

#include <cstdlib>
#include <vector>

#include "host_vector.h"
#include "mgs_runtime.h"
#include "time_durations.h"

inline void SetupGowanlockSort(const std::vector<int>& gpus, int num_threads) {
  omp_set_num_threads(num_threads);
  if (!gpus.empty()) mgs_compat::Contexts::get(gpus.front());
}

template <typename T>
void GowanlockSort(HostVector<T>* elements, size_t chunk_size, size_t merge_group_size, size_t num_buffers,
                   const std::vector<int>& gpus) {
  if (elements->empty()) return;  // src/gowanlock_sort.cuh:398-400
  mgs_ctx* ctx = mgs_compat::Contexts::get(gpus.front());
  const int mode = std::getenv("MGS_HET_CPU_MERGE") ? MGS_MERGE_CPU : MGS_MERGE_GPU;
  mgs_compat::check(mgs_gowanlock_sort(ctx, mgs_compat::DType<T>::value, elements->data(), elements->size(),
                                       chunk_size, merge_group_size, num_buffers, mode),
                    "GowanlockSort");
  for (const char* phase : {"memory_allocation", "sort_phase", "memory_deallocation"}) {
    double s = 0;
    mgs_ctx_phase_seconds(ctx, phase, &s);
    TimeDurations::Get()->Set(phase, s);
  }
}
