// Host-side interface of the merge kernels: the merge-path pivot search of P2P
// sort (SelectPivot/FindPivot, src/tanasic_sort.cuh:15-87 of the reference),
// the two-way merge (thrust::merge, src/tanasic_sort.cuh:163-167) and the k-way
// merge that replaces HET sort's CPU multiway merge
// (__gnu_parallel::multiway_merge, src/gowanlock_sort.cuh:73-74,91-92).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <functional>

#include "launch.cuh"

namespace mgs {

constexpr int kMaxPivotHalf = 64;  // at most 128 chunks in one merge step

// FindPivot over two halves of `half` chunks each (chunk size psize): the
// largest p such that left[N - p] > right[p - 1] (radix order), N = half*psize,
// where left/right index the virtual concatenations of the chunk pointers.
// Writes the pivot (uint64) to d_pivot.
cudaError_t pivot_search(int dtype, const void* const* left, const void* const* right, int half, size_t psize,
                         uint64_t* d_pivot, cudaStream_t stream, LaunchRecorder* rec);

// Scratch bytes of a k-way merge of `total` keys (k runs).
size_t kway_merge_temp_bytes(int dtype, int k, size_t total);

// Stable k-way merge: out = merge of runs[0..k), where runs (host array of
// device pointers) are sorted and hold lens[r] keys each (host array). On equal
// keys the lower run index comes first, so k = 2 gives thrust::merge's order
// (ties take the first range). d_temp must hold kway_merge_temp_bytes(). At
// most kMaxKwayRuns runs.
constexpr int kMaxKwayRuns = 1024;
cudaError_t kway_merge(int dtype, const void* const* runs, const size_t* lens, int k, void* out, void* d_temp,
                       size_t temp_bytes, cudaStream_t stream, LaunchRecorder* rec);

// As kway_merge, with the output merged in windows of about window_keys keys
// (whole merge tiles), in output order: after the launch of each window is
// enqueued on `stream`, on_window(first, count) is called with the window's
// output range, so that the caller can hand it to another stream (a D2H copy
// that overlaps the merge of the next window).
using MergeWindowFn = std::function<cudaError_t(size_t first, size_t count)>;
cudaError_t kway_merge_windowed(int dtype, const void* const* runs, const size_t* lens, int k, void* out,
                                void* d_temp, size_t temp_bytes, size_t window_keys, const MergeWindowFn& on_window,
                                cudaStream_t stream, LaunchRecorder* rec);

}  // namespace mgs
