// Gather / scatter of a coalesced batch of sort requests (the serving loop):
// the requests' keys are copied into one contiguous staging array, sorted
// there by one segmented-sort launch sequence, and copied back.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "launch.cuh"

namespace mgs {

// One request of a batch. `device` is the request's own device buffer, or null
// when its keys are copied to and from the staging array by the host (a host
// request). `offset` is the request's first key in the staging array. With
// `flip`, the top bit of every key is inverted on the way in and back on the
// way out: signed keys then sort as unsigned ones of the same width, so that
// int32 requests share a batch with uint32 ones (and int64 with uint64).
struct BatchEntry {
  void* device;
  uint64_t offset;
  uint64_t n;
  uint32_t flip;
  uint32_t pad;
};

// Stage in: for every entry, staging[offset, offset + n) = its device keys (or,
// for a host entry, the keys already there), top bit inverted when flip is set.
// entries lives in device memory. Asynchronous on `stream`.
cudaError_t batch_stage_in(void* staging, const BatchEntry* entries, uint32_t count, int key_bytes,
                           cudaStream_t stream, LaunchRecorder* rec);
// Stage out: the inverse of batch_stage_in (device entries receive their sorted
// keys; host entries get their top bit restored in place, for the host copy).
cudaError_t batch_stage_out(void* staging, const BatchEntry* entries, uint32_t count, int key_bytes,
                            cudaStream_t stream, LaunchRecorder* rec);

}  // namespace mgs
