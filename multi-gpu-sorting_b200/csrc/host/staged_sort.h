// Sort of a host buffer through one GPU with the host<->device copies
// overlapped with the device work. The reference's single-GPU TanasicSort runs
// copy-in, sort and copy-out one after another (src/tanasic_sort.cuh:250-253,
// 264-266, 286-289); here:
//   1. the keys go to the device in slabs on the H2D stream, and the compute
//      stream sorts each slab (onesweep radix sort) as soon as its copy landed,
//      while the next slab is in flight;
//   2. the sorted slabs are merged (stable k-way merge) into a second device
//      buffer window by window, and each window goes back to the host on the
//      D2H stream while the next window is merged.
// Stable slab sorts and a merge that takes equal keys from the lower slab first
// give exactly the order of one stable sort of the whole buffer.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "context.h"

namespace mgs {

struct StagedPlan {
  int slabs = 1;            // input slabs (sorted runs); 1 = no staging
  size_t slab_keys = 0;     // keys per slab (the last one may be shorter)
  size_t window_keys = 0;   // output keys per merge window / D2H copy
};

// Staging plan for n keys of w bytes; slabs == 1 when n is too small for the
// overlap to pay (the plain copy-sort-copy path is used then).
StagedPlan plan_staged(size_t n, size_t w);

// Device bytes staged_host_sort needs for (dtype, n) under plan_staged().
size_t staged_sort_device_bytes(int dtype, size_t n);

// Sorts h_keys[0..n) in place (host memory, pinned for the overlap to happen)
// using the context's arena, streams and status word. Synchronous: returns
// after the last D2H copy finished. Device-side status bits are left in
// c.d_status for the caller to read.
cudaError_t staged_host_sort(Context& c, int dtype, void* h_keys, size_t n);

}  // namespace mgs
