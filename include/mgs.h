/*
 * mgs.h — C ABI of the B200 sort engine (libmgs.so).
 *
 * Every entry point returns an int status (MGS_OK on success). A failing call
 * leaves a human-readable message for the calling thread in
 * mgs_last_error_string(). No C++ or torch types cross this boundary: keys are
 * raw bytes described by an mgs_dtype, sizes are counts of keys, streams are
 * cudaStream_t passed as void*.
 *
 * Reference surface replaced (hpides/multi-gpu-sorting, paths inside that
 * project):
 *   TanasicSort<T>(HostVector<T>*, gpus)            src/tanasic_sort.cuh:223-299
 *   SetupTanasicSort(gpus)                          src/tanasic_sort.cuh:206-221
 *   GowanlockSort<T>(HostVector<T>*, chunk, group,  src/gowanlock_sort.cuh:395-483
 *                    buffers, gpus)
 *   SetupGowanlockSort(gpus, threads)               src/gowanlock_sort.cuh:117-125
 *   thrust::sort(par.on(stream), begin, end)        src/tanasic_sort.cuh:264-266
 *   thrust::merge(...)                              src/tanasic_sort.cuh:163-167
 *   SelectPivot / FindPivot                         src/tanasic_sort.cuh:15-87
 *   __gnu_parallel::multiway_merge(...)             src/gowanlock_sort.cuh:73-74,91-92
 *   DataGenerator::ComputeDistribution<T>           src/data_generator.cuh:18-36
 *   HostVector<T> (pinned thrust::host_vector)      src/host_vector.cuh:7
 *
 * The reference's CheckCudaError ignores errors in release builds
 * (src/cuda_error.cuh:5-10); this ABI reports every error as a status.
 */
#ifndef MGS_H_
#define MGS_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define MGS_OK 0
#define MGS_ERR_INVALID 1   /* bad argument (null pointer, unknown dtype, size limit) */
#define MGS_ERR_OOM 2       /* device or pinned host allocation failed */
#define MGS_ERR_CUDA 3      /* a CUDA runtime call failed */
#define MGS_ERR_TIMEOUT 4   /* a bounded device-side wait gave up (status word set by a kernel) */
#define MGS_ERR_NO_DEVICE 5 /* no CUDA device, or the device id is out of range */
#define MGS_ERR_CANCELLED 6 /* a queued request was cancelled before it ran */
#define MGS_ERR_BUSY 7      /* admission refused: not enough free device memory right now */

/* ---- key types ---------------------------------------------------------
 * The reference CLI accepts int, long, float, double (src/sort_benchmark.cu:209-221);
 * the unsigned types are the ones the sort path is benchmarked on. Keys are
 * sorted ascending in the order thrust::sort / CUB DeviceRadixSort 2.8.2 gives:
 * signed by value, IEEE-754 by value with -0.0 equal to +0.0 (input order kept,
 * the sort is stable), NaNs placed by their bit pattern (negative-sign NaNs
 * before -inf, positive-sign NaNs after +inf). */
typedef enum mgs_dtype {
  MGS_U32 = 0,
  MGS_I32 = 1,
  MGS_F32 = 2,
  MGS_U64 = 3,
  MGS_I64 = 4,
  MGS_F64 = 5
} mgs_dtype;

typedef struct mgs_ctx mgs_ctx;

/* ---- library ----------------------------------------------------------- */
int mgs_version(void);                   /* 10000 * major + 100 * minor + patch */
const char* mgs_last_error_string(void); /* thread-local; "" when the last call succeeded */
size_t mgs_dtype_size(int dtype);        /* 4 or 8; 0 for an unknown dtype */
int mgs_device_count(int* count);

/* ---- context: one per device; owns streams and a grow-only device arena ----
 * Replaces DeviceBuffers<T> (src/device_buffers.cuh:15-135) and its bump
 * allocator (src/device_allocator.cuh:10-92): device memory is reserved once
 * per context instead of per call. arena_bytes == 0 reserves lazily.
 * Calls on one context must not run concurrently from several host threads. */
int mgs_ctx_create(int device, size_t arena_bytes, mgs_ctx** out);
int mgs_ctx_destroy(mgs_ctx* ctx);
int mgs_ctx_synchronize(mgs_ctx* ctx); /* waits for the context's streams; reports device status words */
int mgs_ctx_arena_bytes(mgs_ctx* ctx, size_t* bytes);

/* Profiling: when enabled, every kernel launch of the context is bracketed by
 * CUDA events on its stream. mgs_ctx_kernel_times synchronizes and returns, per
 * kernel name, the number of launches and the summed device time; it then
 * clears the record. */
typedef struct mgs_kernel_time {
  char name[48];
  uint64_t launches;
  double total_ms;
} mgs_kernel_time;
int mgs_ctx_set_profiling(mgs_ctx* ctx, int enabled);
int mgs_ctx_kernel_times(mgs_ctx* ctx, mgs_kernel_time* out, int capacity, int* count);
/* Number of kernels the context launched since the counter was last reset. */
int mgs_ctx_launch_count(mgs_ctx* ctx, uint64_t* launches, int reset);

/* ---- pinned host memory (HostVector<T>, src/host_vector.cuh:7) ---------- */
int mgs_host_alloc(size_t bytes, void** out);
int mgs_host_free(void* ptr);

/* ---- device radix sort (thrust::sort on one GPU, src/tanasic_sort.cuh:264) ----
 * Ascending, stable, in place on d_keys. d_temp must hold mgs_sort_temp_bytes()
 * bytes, or be NULL to use the context arena. stream is a cudaStream_t (NULL =
 * the context's compute stream). Asynchronous: device status is reported by
 * mgs_ctx_synchronize. n must be below 2^32. */
int mgs_sort_temp_bytes(int dtype, size_t n, size_t* bytes);
int mgs_sort_device(mgs_ctx* ctx, int dtype, void* d_keys, size_t n, void* d_temp, size_t temp_bytes,
                    void* stream);

/* ---- device radix sort without any allocation ------------------------------
 * No counterpart in the reference. For callers that cannot allocate device
 * memory (code running while a pool or arena owns the device memory,
 * allocators and runtimes that must not re-enter cudaMalloc, servers that
 * forbid allocation after start-up): the same sort as mgs_sort_device, with
 * its scratch in a fixed 32 MiB area that is part of the library's device
 * image (held by every GPU that loads the library until exit). No context,
 * no cudaMalloc/cudaFree. At most 2^22 (4,194,304) keys of 4 bytes or 2^21
 * (2,097,152) keys of 8 bytes; larger n returns MGS_ERR_INVALID. All calls on a GPU share the
 * area: calls that overlap on that GPU race, so order them on one stream. The
 * first call on a device looks up the area's address for that device; make it
 * before any stream capture. After cudaDeviceReset (or any other teardown of
 * the device's context) the area may move: the next call notices the new
 * context and looks the address up again, so it counts as a first call again.
 * Asynchronous on `stream` (a cudaStream_t, NULL = the legacy default
 * stream); device-side timeouts are not reported. */
int mgs_sort_device_noalloc(int dtype, void* d_keys, size_t n, void* stream);

/* ---- TanasicSort with one GPU (src/tanasic_sort.cuh:223-299) ------------
 * h_keys is the caller's host buffer (pinned for full link speed); sorted in
 * place: H2D, device sort, D2H, synchronous. Returns early on n == 0 like the
 * reference (src/tanasic_sort.cuh:225-227). */
int mgs_sort_host(mgs_ctx* ctx, int dtype, void* h_keys, size_t n);

/* ---- TanasicSort with g partitions as chunks of one GPU --------------------
 * (src/tanasic_sort.cuh:223-299 with MergePartitions :176-204). The reference's
 * per-GPU partitions become num_chunks (a power of two, <= 128) chunks of this
 * GPU's HBM; the pivot search (FindPivot :45-87), the exchange of the pivot
 * ranges (SwapPartitions :89-146) and the boundary merges
 * (MergeLocalPartitions :148-174) run between those chunks. n is padded to a
 * multiple of num_chunks with the type's maximum like the reference
 * (:231-238,255-259), including its effect on +inf / NaN keys (the padding
 * sorts before them and the copy-back keeps the padding). num_chunks == 1 is
 * mgs_sort_host. Synchronous. */
int mgs_tanasic_sort(mgs_ctx* ctx, int dtype, void* h_keys, size_t n, int num_chunks);
/* Same on a device buffer (in/out), using the context arena. Synchronous. */
int mgs_tanasic_sort_device(mgs_ctx* ctx, int dtype, void* d_keys, size_t n, int num_chunks);

/* ---- merge-path pivot (SelectPivot/FindPivot, src/tanasic_sort.cuh:15-87) ----
 * d_left/d_right: host arrays of `half` device pointers to sorted chunks of
 * chunk_size keys. Returns the largest p with left[N-p] > right[p-1] over the
 * virtual concatenations (N = half * chunk_size). Synchronous. */
int mgs_find_pivot_device(mgs_ctx* ctx, int dtype, const void* const* d_left, const void* const* d_right, int half,
                          size_t chunk_size, size_t* pivot);

/* ---- merges ---------------------------------------------------------------
 * thrust::merge of two sorted device ranges (src/tanasic_sort.cuh:163-167):
 * stable, on equal keys the first range first. k-way merge of k sorted device
 * runs (HET sort's __gnu_parallel::multiway_merge, src/gowanlock_sort.cuh:73-74,
 * 91-92): stable by run index, k <= 1024. d_runs and lens are host arrays.
 * d_temp may be NULL (context arena). Asynchronous on `stream`. */
int mgs_merge_temp_bytes(int dtype, int k, size_t total, size_t* bytes);
int mgs_merge_device(mgs_ctx* ctx, int dtype, const void* d_a, size_t na, const void* d_b, size_t nb, void* d_out,
                     void* d_temp, size_t temp_bytes, void* stream);
int mgs_kway_merge_device(mgs_ctx* ctx, int dtype, const void* const* d_runs, const size_t* lens, int k, void* d_out,
                          void* d_temp, size_t temp_bytes, void* stream);

/* ---- batched segmented sort (no counterpart in the reference; the batched form
 * of the device sort) --------------------------------------------------------
 * Every segment [d_offsets[s], d_offsets[s+1]) of d_keys (device, n keys) is
 * sorted on its own, ascending and stably, in the same order as
 * mgs_sort_device. d_offsets: num_segments + 1 device uint64 values, each
 * segment inside [0, n). Segments of up to 1024 4-byte / 512 8-byte keys are
 * sorted by one warp, up to one tile (16384 / 8192 keys) by one CTA entirely in
 * shared memory, both classes in one persistent launch; longer segments go
 * through the onesweep passes all at once. The launch sequence does not read
 * anything back to the host (stream-ordered, capturable in a CUDA graph).
 * Invalid offsets (decreasing, or beyond n) leave that segment unsorted and
 * make the next mgs_ctx_synchronize return MGS_ERR_INVALID. Asynchronous. */
int mgs_segmented_sort_temp_bytes(int dtype, size_t n, size_t num_segments, size_t* bytes);
int mgs_segmented_sort_device(mgs_ctx* ctx, int dtype, void* d_keys, size_t n, const uint64_t* d_offsets,
                              size_t num_segments, void* d_temp, size_t temp_bytes, void* stream);

/* ---- key-value sort and argsort ---------------------------------------------
 * Not in the reference, whose sorts carry keys only; this is the
 * thrust::sort_by_key form of the library it sorts with (src/tanasic_sort.cuh:264):
 * d_keys[0..n) sorted exactly as mgs_sort_device sorts them (stable), and
 * d_values[0..n) (value_bytes = 4 or 8 per key; any payload: row ids, pointers,
 * indices) moved with their keys, so values of equal keys keep their input
 * order. mgs_argsort_device writes into d_indices the input position of each
 * key in sorted order (index_bytes = 4 or 8) and sorts the keys in place.
 * Scratch as for mgs_sort_device (NULL: the context's arena). Asynchronous. */
int mgs_sort_pairs_temp_bytes(int dtype, size_t value_bytes, size_t n, size_t* bytes);
int mgs_sort_pairs_device(mgs_ctx* ctx, int dtype, void* d_keys, void* d_values, size_t value_bytes, size_t n,
                          void* d_temp, size_t temp_bytes, void* stream);
int mgs_argsort_device(mgs_ctx* ctx, int dtype, void* d_keys, void* d_indices, size_t index_bytes, size_t n,
                       void* d_temp, size_t temp_bytes, void* stream);

/* ---- bit ranges and descending order -----------------------------------------
 * Not in the reference; the begin_bit / end_bit and descending forms of
 * cub::DeviceRadixSort (SortKeys[Descending], SortPairs[Descending]), the
 * library behind the thrust::sort the reference calls (src/tanasic_sort.cuh:264).
 * Keys are compared by bits [begin_bit, end_bit) of their ordered form (the
 * order of mgs_sort_device: unsigned, two's complement, IEEE with -0.0 equal to
 * +0.0), ascending or descending (descending != 0); the sort is stable, so keys
 * equal on those bits keep their input order. value_bytes 4 or 8 moves d_values
 * with their keys; 0 sorts keys only (d_values unused). 0 <= begin_bit <=
 * end_bit <= key bits. Scratch: mgs_sort_temp_bytes (keys only) or
 * mgs_sort_pairs_temp_bytes; NULL: the context's arena. Asynchronous. */
int mgs_sort_range_device(mgs_ctx* ctx, int dtype, void* d_keys, void* d_values, size_t value_bytes, size_t n,
                          int begin_bit, int end_bit, int descending, void* d_temp, size_t temp_bytes, void* stream);

/* ---- recorded sorts (CUDA graphs) -------------------------------------------
 * No counterpart in the reference (its sorts are host-driven thrust calls). A
 * plan records once, into a CUDA graph, the launches of one device sort or one
 * segmented sort of a FIXED buffer (keys, offsets and scratch pointers are baked
 * in); mgs_plan_launch replays them with a single graph launch on any stream,
 * sorting whatever the buffer holds at that time. For callers that sort the same
 * buffers again and again (a batch loop, a serving slot): one launch instead of
 * seven or more, no host work per sort. d_temp NULL: the plan allocates and owns
 * its scratch (mgs_sort_temp_bytes / mgs_segmented_sort_temp_bytes); otherwise
 * the caller's scratch must outlive the plan. Device status goes to the
 * context's status word (read by mgs_ctx_synchronize), so the context must
 * outlive the plan. Creating a plan runs nothing on the GPU. Replays of one
 * plan, or of two plans sharing scratch, must not overlap on the GPU. */
typedef struct mgs_plan mgs_plan;
int mgs_plan_sort_create(mgs_ctx* ctx, int dtype, void* d_keys, size_t n, void* d_temp, size_t temp_bytes,
                         mgs_plan** out);
int mgs_plan_segmented_create(mgs_ctx* ctx, int dtype, void* d_keys, size_t n, const uint64_t* d_offsets,
                              size_t num_segments, void* d_temp, size_t temp_bytes, mgs_plan** out);
int mgs_plan_launch(mgs_plan* plan, void* stream); /* NULL stream: the context's compute stream; asynchronous */
int mgs_plan_launch_count(mgs_plan* plan, uint64_t* launches); /* kernel launches one replay performs */
int mgs_plan_destroy(mgs_plan* plan); /* waits for the device first (replays may still run) */

/* ---- onesweep variants and the autotuner ------------------------------------
 * No counterpart in the reference (it calls thrust::sort with CUB's own tuning).
 * The radix sort picks, per key width (4 or 8 bytes) and size class of n
 * (0: n < 2^16, 1: < 2^18, 2: < 2^20, 3: < 2^22, 4: < 2^26, 5: larger), a tile
 * shape (0..6: threads x keys per thread) and a ranking mode (2: shared-memory
 * peer masks, 3: ballots for half of the keys). The table is read from a tuning
 * file on first use (MGS_TUNE_FILE, else tuning/b200.tune beside the library's
 * directory; format: lines "key_bytes size_class shape rank_mode"), and the
 * environment variables MGS_ONESWEEP_SHAPE / MGS_RANK_MODE override it.
 * mgs_autotune times every variant on a sample of each size class up to max_n
 * (uniformly random keys of the dtype's width, median of reps sorts), keeps the
 * fastest in the table and reports every timing in out (count = number of
 * samples, also when more than capacity). It allocates and frees its own
 * device buffers; no other sort may be issued meanwhile. Changing the table
 * (set, load, autotune) while sorts are being issued from other threads races. */
typedef struct mgs_tune_sample {
  int key_bytes;
  int size_class;
  size_t n;
  int shape;
  int rank_mode;
  double ms;
  int chosen; /* 1 for the variant the table now holds for this class */
} mgs_tune_sample;
int mgs_tune_get(int dtype, size_t n, int* shape, int* rank_mode); /* the variant a sort of n keys uses */
int mgs_tune_set(int dtype, int size_class, int shape, int rank_mode);
int mgs_tune_load(const char* path);
int mgs_tune_save(const char* path);
int mgs_autotune(mgs_ctx* ctx, int dtype, size_t max_n, int reps, mgs_tune_sample* out, int capacity, int* count);

/* ---- GowanlockSort on one GPU: out-of-core chunk pipeline -------------------
 * (HET sort, src/gowanlock_sort.cuh:127-483). h_keys (host, pinned for full link
 * speed) is sorted in place. Phase 1 streams chunks of chunk_size keys through
 * num_buffers (2 or 3, src/gowanlock_sort.cuh:460-469) device buffers: H2D on
 * one copy engine, radix sort, D2H on the other, overlapped. Phase 2 merges the
 * sorted chunks: MGS_MERGE_GPU streams windows of the runs through the GPU k-way
 * merge; MGS_MERGE_CPU runs the reference's __gnu_parallel::multiway_merge with
 * std::less<T> (src/gowanlock_sort.cuh:73-74,91-92) on the host cores.
 * chunk_size 0 = the whole input if it fits in 80% of free device memory, else
 * the largest chunk that does (the reference's default is n / num_gpus,
 * src/gowanlock_sort.cuh:402-404). merge_group_size is accepted for API parity
 * (the reference merges groups of chunks on a CPU thread while sorting,
 * src/gowanlock_sort.cuh:29-84); here the merge is one k-way pass after all
 * chunks are sorted. At most 1024 chunks with MGS_MERGE_GPU. A pinned host
 * buffer of n keys holds the sorted chunks; it is kept by the context
 * (grow-only). Synchronous. Phase times: mgs_ctx_phase_seconds. */
#define MGS_MERGE_GPU 0
#define MGS_MERGE_CPU 1
int mgs_gowanlock_sort(mgs_ctx* ctx, int dtype, void* h_keys, size_t n, size_t chunk_size, size_t merge_group_size,
                       size_t num_buffers, int merge_mode);
/* Wall-clock seconds of the context's last GowanlockSort call per phase, named
 * like the reference's TimeDurations keys (src/time_durations.cuh): "memory_allocation",
 * "sort_phase" (chunk sorting and merging), "merge_phase", "memory_deallocation". */
int mgs_ctx_phase_seconds(mgs_ctx* ctx, const char* phase, double* seconds);

/* ---- serving loop (no counterpart in the reference) -------------------------
 * Sort requests of mixed sizes and key types, submitted from any thread, are
 * batched onto one GPU by a dispatcher thread (continuous batching).
 *   Memory: one device pool of device_budget_bytes is reserved at creation
 *   (0: half the free device memory, at most 32 GiB). Each batch takes exactly
 *   the bytes it needs (staging keys, offsets, sort scratch) from the pool and
 *   returns them when it finishes: a queued request is admitted when a stream
 *   is free and the pool has room for it (admission by free HBM), in arrival
 *   order. A request that would not fit even in the empty pool, or that has
 *   more than slot_keys keys (0: no such limit), is refused at submission.
 *   In flight: up to num_slots batches (default 4), each on its own stream.
 *   Coalescing: a request of at most coalesce_keys keys (0: no coalescing)
 *   opens a batch that queued small requests of a compatible key type join
 *   (up to max_batch_requests, default 4096): uint32 with int32, uint64 with
 *   int64 (signed keys sort as unsigned ones with the top bit inverted on the
 *   way in and out), float32 and float64 each on their own; the batch is sorted
 *   by one segmented-sort launch sequence. Larger requests run alone.
 *   Requests: mgs_server_submit takes a host buffer (pinned for full speed),
 *   mgs_server_submit_device a buffer in this GPU's memory, which a request
 *   running alone sorts in place without any copy. Either is sorted in place
 *   and must stay valid until mgs_server_wait reports it finished.
 * num_slots = 1 with coalesce_keys = 0 gives the plain one-request-per-launch
 * form. */
typedef struct mgs_server mgs_server;
typedef struct mgs_server_config {
  int device;
  int num_slots;             /* batches in flight (streams) */
  size_t slot_keys;          /* largest request in keys; 0 = limited by the pool only */
  size_t coalesce_keys;      /* requests up to this many keys may share a batch; 0 = none */
  size_t max_batch_requests; /* requests per coalesced batch */
  size_t device_budget_bytes; /* device pool */
} mgs_server_config;
typedef struct mgs_server_stats {
  uint64_t submitted, completed, rejected, cancelled, batches, keys, kernel_launches;
  int num_slots;
  double p50_us, p99_us, mean_us, max_us; /* latency: completion - submission */
  double busy_s;                          /* first submission to last completion */
  uint64_t pool_bytes, pool_free_bytes;   /* the device pool and its free bytes now */
} mgs_server_stats;
int mgs_server_create(const mgs_server_config* config, mgs_server** out);
int mgs_server_destroy(mgs_server* server); /* finishes queued and running requests first */
int mgs_server_submit(mgs_server* server, int dtype, void* h_keys, size_t n, uint64_t* request_id);
int mgs_server_submit_device(mgs_server* server, int dtype, void* d_keys, size_t n, uint64_t* request_id);
/* Waits for a request (timeout_ms < 0: no limit); MGS_ERR_TIMEOUT if it is still
 * running. *request_status: MGS_OK, MGS_ERR_CANCELLED or the failure. A request
 * is forgotten once a wait has reported it finished. */
int mgs_server_wait(mgs_server* server, uint64_t request_id, int timeout_ms, int* request_status);
int mgs_server_cancel(mgs_server* server, uint64_t request_id); /* queued requests only, else MGS_ERR_BUSY */
int mgs_server_stats_get(mgs_server* server, mgs_server_stats* out, int reset);

/* ---- DataGenerator::ComputeDistribution<T> (src/data_generator.cuh:18-36) ----
 * Fills the host buffer out[0..n) exactly as the reference generator does for
 * the reference's distributions: "uniform", "normal", "zero", "staggered",
 * "sorted", "reverse-sorted", "nearly-sorted", "bucket-sorted" (128 OpenMP
 * threads, mt19937 per thread). Additional seeded distributions of the sort
 * engine's workload sweep: "full-uniform", "normal0", "zipf", "sorted-full",
 * "reverse-sorted-full", "nearly-sorted-swaps", "all-equal". For f32/f64 the
 * "-specials" suffix (e.g. "full-uniform-specials") additionally replaces 0.1%
 * of the keys with -0.0 and 0.1% with NaNs of both signs. */
int mgs_generate(int dtype, const char* distribution, uint32_t seed, void* out, size_t n);

/* ---- DataGenerator::ComputeDistribution<T> into device memory
 * (src/data_generator.cuh:18-36, with the buffer on the GPU) ----
 * Fills the device buffer d_out[0..n) with the same bytes mgs_generate writes
 * for the same (dtype, distribution, seed, n), without the host generation and
 * the copy. Every distribution above except "normal", "nearly-sorted" and
 * "normal0": those draw through the host C library's log / cos, which the
 * device does not reproduce bit for bit, and are refused (MGS_ERR_INVALID).
 * Entries the host generator leaves untouched (staggered and bucket-sorted with
 * n < 10) stay untouched. Uses the context's arena and compute stream; returns
 * when the buffer is filled. n must be below 2^32. */
int mgs_generate_device(mgs_ctx* ctx, int dtype, const char* distribution, uint32_t seed, void* d_out, size_t n);

/* ---- failure injection for tests (no counterpart in the reference, whose
 * CheckCudaError ignores errors in release builds, src/cuda_error.cuh:5-10) ----
 * mgs_test_set_waits: bounds of the sort kernels' device-side waits on
 * `device` (polls of a look-back status word, polls of a tile-copy barrier;
 * 0 = the default bound) for sorts launched afterwards, and one tile of the
 * plain device sort whose look-back status is never published (hold_tile;
 * 0xFFFFFFFF = none). With a tile held, the look-back after it waits on a word
 * that nothing sets until its bound runs out; the sort then finishes, its
 * output unspecified (every write stays inside the keys), and reports
 * MGS_ERR_TIMEOUT through mgs_ctx_synchronize. Call with (device, 0, 0,
 * 0xFFFFFFFF) to restore the defaults. Synchronous.
 * mgs_test_fail_device_allocations: the next `count` growths of any context's
 * device arena fail as an out-of-memory cudaMalloc would (MGS_ERR_OOM); 0
 * cancels. */
int mgs_test_set_waits(int device, uint32_t lookback_spins, uint32_t tma_polls, uint32_t hold_tile);
int mgs_test_fail_device_allocations(int count);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* MGS_H_ */
