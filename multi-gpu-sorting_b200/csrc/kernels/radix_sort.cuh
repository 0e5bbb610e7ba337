// Host-side interface of the onesweep LSD radix sort (replaces thrust::sort /
// CUB DeviceRadixSort, the call at src/tanasic_sort.cuh:264-266 of the
// reference).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "launch.cuh"

namespace mgs {

// Bytes of scratch memory (device) one sort of n keys of the given dtype needs:
// the ping-pong key buffer, the per-sort state block and two look-back arrays.
size_t radix_sort_temp_bytes(int dtype, size_t n);

// Sorts d_keys[0..n) ascending and stably, in place, on `stream`. d_temp must
// hold radix_sort_temp_bytes(dtype, n) bytes. Device-side failures (a bounded
// wait that gave up) are OR-ed into *d_status (a device word) when it is not
// null. Asynchronous.
cudaError_t radix_sort(int dtype, void* d_keys, size_t n, void* d_temp, size_t temp_bytes, cudaStream_t stream,
                       uint32_t* d_status, LaunchRecorder* rec);

// Batched segmented sort: each segment [d_offsets[s], d_offsets[s+1]) of
// d_keys (device, n keys; offsets are num_segments + 1 device uint64 values)
// sorted on its own, stably, in a fixed number of launches that depend on no
// host readback (capturable in a CUDA graph). Segments must lie inside [0, n);
// bad offsets set kStatusBadInput in *d_status and leave the segment unsorted.
size_t segmented_sort_temp_bytes(int dtype, size_t n, size_t num_segments);
cudaError_t segmented_sort(int dtype, void* d_keys, size_t n, const uint64_t* d_offsets, size_t num_segments,
                           void* d_temp, size_t temp_bytes, cudaStream_t stream, uint32_t* d_status,
                           LaunchRecorder* rec);

// Number of kernel launches radix_sort issues for (dtype, n).
int radix_sort_launches(int dtype, size_t n);

}  // namespace mgs
