// Out-of-core chunk pipeline (GowanlockSort on one GPU), see out_of_core.cu.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace mgs {

struct Context;

struct OocPlan {
  size_t chunk;       // keys per chunk
  size_t num_chunks;  // sorted runs produced by phase A
  int num_buffers;    // device chunk buffers in the ring (2 or 3)
  size_t window;      // keys per GPU merge window (phase B)
  size_t phase_a_bytes, phase_b_bytes;  // device memory of each phase
};

struct OocTimes {
  double allocation_s = 0, sort_s = 0, merge_s = 0;
};

// chunk == 0: the whole input if it fits `device_budget` bytes, else the largest
// chunk that does. window == 0: 512 MiB of keys.
OocPlan plan_out_of_core(int dtype, size_t n, size_t chunk, int num_buffers, size_t window, size_t device_budget);

// Sorts h_keys[0..n) (host, pinned for full speed) in place. h_secondary is a
// host buffer of n keys used for the sorted runs when there is more than one
// chunk. merge_on_cpu selects the reference's CPU multiway merge for phase B.
cudaError_t out_of_core_sort(Context& c, int dtype, void* h_keys, size_t n, const OocPlan& p, int merge_on_cpu,
                             void* h_secondary, OocTimes* times);

}  // namespace mgs
