// Host-side interface of the onesweep LSD radix sort (replaces thrust::sort /
// CUB DeviceRadixSort, the call at src/tanasic_sort.cuh:264-266 of the
// reference).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <vector>

#include "launch.cuh"

namespace mgs {

// Bounds of the radix kernels' device-side waits on the current device (0 =
// the default bound) and the failure-injection hook: the plain sort's tile
// `hold_tile` never publishes its look-back status (0xFFFFFFFF: none), so the
// look-back waits after it run out and the sort reports a timeout. Synchronous;
// applies to sorts launched afterwards.
cudaError_t set_wait_control(uint32_t lookback_spins, uint32_t tma_polls, uint32_t hold_tile);

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

// Key-value sort (thrust::sort_by_key order): d_keys[0..n) sorted as by
// radix_sort, stably, and d_values[0..n) (value_bytes = 4 or 8, opaque) moved
// with their keys. d_temp must hold radix_sort_pairs_temp_bytes() bytes.
size_t radix_sort_pairs_temp_bytes(int dtype, size_t value_bytes, size_t n);
cudaError_t radix_sort_pairs(int dtype, void* d_keys, void* d_values, size_t value_bytes, size_t n, void* d_temp,
                             size_t temp_bytes, cudaStream_t stream, uint32_t* d_status, LaunchRecorder* rec);

// Sort by bits [begin_bit, end_bit) of the ordered key (CUB's begin_bit /
// end_bit), ascending or descending, stable; with value_bytes 4 or 8 the values
// move with their keys (0: keys only, d_values unused). Scratch as for
// radix_sort (keys only) or radix_sort_pairs.
cudaError_t radix_sort_range(int dtype, void* d_keys, void* d_values, size_t value_bytes, size_t n, int begin_bit,
                             int end_bit, int descending, void* d_temp, size_t temp_bytes, cudaStream_t stream,
                             uint32_t* d_status, LaunchRecorder* rec);

// Argsort: d_indices[0..n) (index_bytes = 4 or 8) receives the input position
// of every key in sorted order; the keys are sorted in place on the way.
// Scratch: radix_sort_pairs_temp_bytes(dtype, index_bytes, n).
cudaError_t radix_argsort(int dtype, void* d_keys, void* d_indices, size_t index_bytes, size_t n, void* d_temp,
                          size_t temp_bytes, cudaStream_t stream, uint32_t* d_status, LaunchRecorder* rec);

// K-way merge tiles sorted in shared memory (the merge of many runs of 4-byte
// keys): tile j in [tile0, tile0 + tiles) of the output is out[j*T, (j+1)*T)
// (T = kway_radix_tile_keys(dtype), the last tile shorter), filled from the
// slices splits[j*k + r] .. splits[(j+1)*k + r) of the k device runs (d_runs:
// a device array of k run pointers; splits: a device (tiles+1) x k uint64
// split matrix of a stable k-way merge at spacing T) by range-limited LSD
// passes. kway_radix_tile_keys is 0 for dtypes without this path (8-byte keys).
constexpr int kMaxKwayTileRuns = 1024;
size_t kway_radix_tile_keys(int dtype);
cudaError_t kway_radix_tiles(int dtype, const void* d_runs, int k, const uint64_t* d_splits, void* out,
                             uint64_t total, uint64_t tile0, uint64_t tiles, cudaStream_t stream,
                             LaunchRecorder* rec);

// Number of kernel launches radix_sort issues for (dtype, n).// Number of kernel launches radix_sort issues for (dtype, n).
int radix_sort_launches(int dtype, size_t n);

// Onesweep variant choice. Key widths 4 and 8 bytes each have a table of
// kSizeClasses entries (size_class: n < 2^16, < 2^18, < 2^20, < 2^22, < 2^26,
// larger); each entry names a tile shape (0..6: threads x keys per thread, see
// OnesweepShape) and a ranking mode (2: shared-memory peer masks, 3: ballots
// for half of the items). radix_sort reads the entry of its (width, n).
constexpr int kSizeClasses = 6;
struct SortVariant {
  int shape;
  int mode;
};
int size_class(size_t n);
size_t size_class_sample(int size_class);  // the key count the autotuner times for a class
bool valid_variant(SortVariant v);
bool set_sort_variant(int key_bytes, int size_class, SortVariant v);  // false when out of range
SortVariant sort_variant(int key_bytes, size_t n);  // the table's entry, then the environment overrides
SortVariant table_variant(int key_bytes, int size_class);  // the table's entry alone
// Tuning files (format in tune.cu): load returns the number of entries read,
// -1 when the file cannot be opened, -2 when a line is malformed (valid lines
// before and after it are still applied); save writes the whole table.
int load_tuning_file(const char* path);
bool save_tuning_file(const char* path);
// The default tuning file (the MGS_TUNE_FILE path, else tuning/b200.tune
// beside the library's own directory) is read once, before the table is first
// read or set: ensure_default_tuning runs load_default_tuning on that first use.
// store_sort_variant writes an entry without that step (file reading uses it).
void ensure_default_tuning();
void load_default_tuning();
bool store_sort_variant(int key_bytes, int size_class, SortVariant v);

// Autotuner: for each size class whose sample size is at most max_n, times every
// variant (CUDA events, median of `reps` sorts of uniformly random keys of the
// dtype's width) and stores the fastest in the table. Allocates its own device
// buffers (keys, a pristine copy, scratch) and frees them. Sorts must not be
// issued from other threads meanwhile. Synchronous.
struct TuneSample {
  int key_bytes, size_class;
  size_t n;
  SortVariant variant;
  double ms;
  bool chosen;
};
cudaError_t autotune(int dtype, size_t max_n, int reps, std::vector<TuneSample>* out);

}  // namespace mgs
