// C ABI of the sort engine (include/mgs.h). Argument checking, error strings,
// context lifetime and the synchronous host-buffer entry points live here; the
// device work is in csrc/kernels.
#include "mgs.h"

#include <cuda_runtime.h>

#include <chrono>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../kernels/engine_types.h"
#include "../kernels/merge.cuh"
#include "../kernels/radix_sort.cuh"
#include "chunk_sort.h"
#include "staged_sort.h"
#include "context.h"
#include "out_of_core.h"

#include "data_generator.h"
#include "../kernels/generate.cuh"

using mgs::Context;
using mgs::set_last_error;

namespace {

constexpr size_t kMaxDeviceSortKeys = (size_t(1) << 32) - 1;

int cuda_fail(cudaError_t e, const char* what) {
  set_last_error("%s: %s", what, cudaGetErrorString(e));
  cudaGetLastError();  // clear the sticky-free error state
  return e == cudaErrorMemoryAllocation ? MGS_ERR_OOM : MGS_ERR_CUDA;
}

int invalid(const char* msg) {
  set_last_error("%s", msg);
  return MGS_ERR_INVALID;
}

int status_to_code(uint32_t status) {
  if (status == 0) return MGS_OK;
  if (status == mgs::kStatusBadInput) {
    set_last_error("device status 0x%x: invalid input found by a kernel (segment offsets out of order or range)",
                   status);
    return MGS_ERR_INVALID;
  }
  set_last_error("device status 0x%x: a bounded device-side wait gave up (%s%s%s)", status,
                 (status & mgs::kStatusLookbackTimeout) ? "look-back " : "",
                 (status & mgs::kStatusTmaTimeout) ? "tma " : "", (status & mgs::kStatusQueueTimeout) ? "queue " : "");
  return MGS_ERR_TIMEOUT;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

inline size_t align256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace

// A recorded sort: the instantiated CUDA graph of one sort's launches.
struct mgs_plan {
  mgs_ctx* ctx = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  void* owned_temp = nullptr;  // scratch the plan allocated itself
  uint64_t launches = 0;       // kernel launches one replay performs
};

namespace {

// Counts the launches issued while a plan is recorded (no timing events, which
// would become graph nodes).
struct CountingRecorder : mgs::LaunchRecorder {
  uint64_t launches = 0;
  void before(const char*, cudaStream_t) override { ++launches; }
  void after(const char*, cudaStream_t) override {}
};

void plan_release(mgs_plan* p) {
  if (!p) return;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  if (p->owned_temp) cudaFree(p->owned_temp);
  delete p;
}

// Records body(d_temp, temp_bytes, stream, recorder) into a graph on a private
// stream (relaxed capture mode: the one-time per-kernel attribute calls the
// launch path makes are allowed during the capture) and instantiates it.
template <class Body>
int plan_record(mgs_ctx* ctx, const char* what, size_t need, void* d_temp, size_t temp_bytes, Body body,
                mgs_plan** out) {
  Context& c = ctx->impl;
  DeviceGuard g(c.device);
  mgs_plan* p = new (std::nothrow) mgs_plan;
  if (!p) {
    set_last_error("%s: out of host memory", what);
    return MGS_ERR_OOM;
  }
  p->ctx = ctx;
  if (d_temp == nullptr) {
    if (need > 0) {
      const cudaError_t e = cudaMalloc(&p->owned_temp, need);
      if (e != cudaSuccess) {
        plan_release(p);
        return cuda_fail(e, what);
      }
    }
    d_temp = p->owned_temp;
    temp_bytes = need;
  } else if (temp_bytes < need) {
    plan_release(p);
    set_last_error("%s: d_temp holds %zu bytes, %zu needed", what, temp_bytes, need);
    return MGS_ERR_INVALID;
  }
  cudaStream_t s = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed);
  if (e == cudaSuccess) {
    CountingRecorder rec;
    const cudaError_t eb = body(d_temp, temp_bytes, s, &rec);
    cudaGraph_t graph = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(s, &graph);
    p->graph = graph;
    p->launches = rec.launches;
    e = (eb != cudaSuccess) ? eb : ee;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&p->exec, p->graph, 0);
  }
  if (s) cudaStreamDestroy(s);
  if (e != cudaSuccess) {
    plan_release(p);
    return cuda_fail(e, what);
  }
  *out = p;
  mgs::clear_last_error();
  return MGS_OK;
}

}  // namespace

extern "C" {

int mgs_version(void) { return 10000 * 0 + 100 * 1 + 0; }

const char* mgs_last_error_string(void) { return mgs::last_error(); }

size_t mgs_dtype_size(int dtype) { return mgs::dtype_bytes(dtype); }

int mgs_device_count(int* count) {
  if (!count) return invalid("mgs_device_count: count is null");
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (e != cudaSuccess) {
    *count = 0;
    cudaGetLastError();
    set_last_error("cudaGetDeviceCount: %s", cudaGetErrorString(e));
    return MGS_ERR_NO_DEVICE;
  }
  *count = c;
  mgs::clear_last_error();
  return MGS_OK;
}

int mgs_ctx_create(int device, size_t arena_bytes, mgs_ctx** out) {
  if (!out) return invalid("mgs_ctx_create: out is null");
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    set_last_error("mgs_ctx_create: no CUDA device");
    return MGS_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= count) {
    set_last_error("mgs_ctx_create: device %d out of range [0, %d)", device, count);
    return MGS_ERR_NO_DEVICE;
  }
  DeviceGuard g(device);
  mgs_ctx* ctx = new (std::nothrow) mgs_ctx();
  if (!ctx) return invalid("mgs_ctx_create: out of host memory");
  Context& c = ctx->impl;
  c.device = device;
  cudaDeviceGetAttribute(&c.sm_count, cudaDevAttrMultiProcessorCount, device);
  cudaError_t e = cudaStreamCreateWithFlags(&c.compute, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c.h2d, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c.d2h, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&c.d_status, 256);
  if (e == cudaSuccess) e = cudaMemset(c.d_status, 0, 256);
  if (e == cudaSuccess) e = cudaMallocHost(&c.h_status, 256);
  if (e == cudaSuccess) c.h_status64 = reinterpret_cast<uint64_t*>(reinterpret_cast<char*>(c.h_status) + 64);
  if (e == cudaSuccess && arena_bytes > 0) e = c.reserve(arena_bytes);
  if (e != cudaSuccess) {
    int rc = cuda_fail(e, "mgs_ctx_create");
    mgs_ctx_destroy(ctx);
    return rc;
  }
  *out = ctx;
  mgs::clear_last_error();
  return MGS_OK;
}

int mgs_ctx_destroy(mgs_ctx* ctx) {
  if (!ctx) return MGS_OK;
  Context& c = ctx->impl;
  {
    DeviceGuard g(c.device);
    if (c.compute) cudaStreamSynchronize(c.compute);
    if (c.h2d) cudaStreamSynchronize(c.h2d);
    if (c.d2h) cudaStreamSynchronize(c.d2h);
    if (c.arena) cudaFree(c.arena);
    if (c.d_status) cudaFree(c.d_status);
    if (c.h_status) cudaFreeHost(c.h_status);
    if (c.host_arena) cudaFreeHost(c.host_arena);
    if (c.compute) cudaStreamDestroy(c.compute);
    if (c.h2d) cudaStreamDestroy(c.h2d);
    if (c.d2h) cudaStreamDestroy(c.d2h);
    delete ctx;
  }
  mgs::clear_last_error();
  return MGS_OK;
}

int mgs_ctx_synchronize(mgs_ctx* ctx) {
  if (!ctx) return invalid("mgs_ctx_synchronize: ctx is null");
  Context& c = ctx->impl;
  DeviceGuard g(c.device);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_fail(e, "mgs_ctx_synchronize");
  uint32_t status = 0;
  e = c.take_status(c.compute, &status);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_ctx_synchronize: status read");
  int rc = status_to_code(status);
  if (rc == MGS_OK) mgs::clear_last_error();
  return rc;
}

int mgs_ctx_arena_bytes(mgs_ctx* ctx, size_t* bytes) {
  if (!ctx || !bytes) return invalid("mgs_ctx_arena_bytes: null argument");
  *bytes = ctx->impl.arena_bytes;
  return MGS_OK;
}

int mgs_ctx_set_profiling(mgs_ctx* ctx, int enabled) {
  if (!ctx) return invalid("mgs_ctx_set_profiling: ctx is null");
  ctx->impl.recorder.set_enabled(enabled != 0);
  return MGS_OK;
}

int mgs_ctx_kernel_times(mgs_ctx* ctx, mgs_kernel_time* out, int capacity, int* count) {
  if (!ctx || !count || (capacity > 0 && !out)) return invalid("mgs_ctx_kernel_times: null argument");
  DeviceGuard g(ctx->impl.device);
  std::vector<std::pair<std::string, std::pair<uint64_t, double>>> rows;
  cudaError_t e = ctx->impl.recorder.collect(&rows);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_ctx_kernel_times");
  *count = int(rows.size());
  for (int i = 0; i < capacity && i < int(rows.size()); ++i) {
    std::memset(out[i].name, 0, sizeof(out[i].name));
    std::strncpy(out[i].name, rows[i].first.c_str(), sizeof(out[i].name) - 1);
    out[i].launches = rows[i].second.first;
    out[i].total_ms = rows[i].second.second;
  }
  return MGS_OK;
}

int mgs_ctx_launch_count(mgs_ctx* ctx, uint64_t* launches, int reset) {
  if (!ctx || !launches) return invalid("mgs_ctx_launch_count: null argument");
  *launches = ctx->impl.recorder.launches();
  if (reset) ctx->impl.recorder.reset_launches();
  return MGS_OK;
}

int mgs_host_alloc(size_t bytes, void** out) {
  if (!out) return invalid("mgs_host_alloc: out is null");
  *out = nullptr;
  if (bytes == 0) return MGS_OK;
  cudaError_t e = cudaMallocHost(out, bytes);
  if (e != cudaSuccess) {
    *out = nullptr;
    cudaGetLastError();
    set_last_error("mgs_host_alloc(%zu): %s", bytes, cudaGetErrorString(e));
    return MGS_ERR_OOM;
  }
  return MGS_OK;
}

int mgs_host_free(void* ptr) {
  if (!ptr) return MGS_OK;
  cudaError_t e = cudaFreeHost(ptr);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_host_free");
  return MGS_OK;
}

int mgs_sort_temp_bytes(int dtype, size_t n, size_t* bytes) {
  if (!bytes) return invalid("mgs_sort_temp_bytes: bytes is null");
  if (mgs::dtype_bytes(dtype) == 0) return invalid("mgs_sort_temp_bytes: unknown dtype");
  if (n > kMaxDeviceSortKeys) return invalid("mgs_sort_temp_bytes: n must be below 2^32");
  *bytes = mgs::radix_sort_temp_bytes(dtype, n);
  return MGS_OK;
}

int mgs_sort_device(mgs_ctx* ctx, int dtype, void* d_keys, size_t n, void* d_temp, size_t temp_bytes,
                    void* stream) {
  if (!ctx) return invalid("mgs_sort_device: ctx is null");
  const size_t w = mgs::dtype_bytes(dtype);
  if (w == 0) return invalid("mgs_sort_device: unknown dtype");
  if (n == 0) return MGS_OK;
  if (!d_keys) return invalid("mgs_sort_device: d_keys is null");
  if (reinterpret_cast<uintptr_t>(d_keys) % w != 0) return invalid("mgs_sort_device: d_keys is not key-aligned");
  if (n > kMaxDeviceSortKeys) return invalid("mgs_sort_device: n must be below 2^32 (use the chunked entry points)");
  Context& c = ctx->impl;
  DeviceGuard g(c.device);
  const size_t need = mgs::radix_sort_temp_bytes(dtype, n);
  if (d_temp == nullptr) {
    cudaError_t e = c.reserve(need);
    if (e != cudaSuccess) return cuda_fail(e, "mgs_sort_device: arena");
    d_temp = c.arena;
    temp_bytes = c.arena_bytes;
  } else if (temp_bytes < need) {
    set_last_error("mgs_sort_device: d_temp holds %zu bytes, %zu needed", temp_bytes, need);
    return MGS_ERR_INVALID;
  }
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c.compute;
  cudaError_t e = mgs::radix_sort(dtype, d_keys, n, d_temp, temp_bytes, s, c.d_status, &c.recorder);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_sort_device");
  mgs::clear_last_error();
  return MGS_OK;
}

int mgs_sort_pairs_temp_bytes(int dtype, size_t value_bytes, size_t n, size_t* bytes) {
  if (!bytes) return invalid("mgs_sort_pairs_temp_bytes: bytes is null");
  if (mgs::dtype_bytes(dtype) == 0) return invalid("mgs_sort_pairs_temp_bytes: unknown dtype");
  if (value_bytes != 4 && value_bytes != 8) return invalid("mgs_sort_pairs_temp_bytes: value_bytes must be 4 or 8");
  *bytes = n ? mgs::radix_sort_pairs_temp_bytes(dtype, value_bytes, n) : 0;
  return MGS_OK;
}

// Shared argument checks and scratch choice of the key-value entry points.
static int pairs_call(mgs_ctx* ctx, const char* what, int dtype, void* d_keys, void* d_values, size_t value_bytes,
                      size_t n, void* d_temp, size_t temp_bytes, void* stream, bool argsort) {
  if (!ctx) return invalid("key-value sort: ctx is null");
  const size_t w = mgs::dtype_bytes(dtype);
  if (w == 0) {
    set_last_error("%s: unknown dtype", what);
    return MGS_ERR_INVALID;
  }
  if (value_bytes != 4 && value_bytes != 8) {
    set_last_error("%s: value_bytes must be 4 or 8", what);
    return MGS_ERR_INVALID;
  }
  if (n == 0) return MGS_OK;
  if (!d_keys || !d_values) {
    set_last_error("%s: null pointer", what);
    return MGS_ERR_INVALID;
  }
  if (reinterpret_cast<uintptr_t>(d_keys) % w != 0 || reinterpret_cast<uintptr_t>(d_values) % value_bytes != 0) {
    set_last_error("%s: keys or values are not aligned to their size", what);
    return MGS_ERR_INVALID;
  }
  if (n > kMaxDeviceSortKeys) {
    set_last_error("%s: n must be below 2^32", what);
    return MGS_ERR_INVALID;
  }
  Context& c = ctx->impl;
  DeviceGuard g(c.device);
  const size_t need = mgs::radix_sort_pairs_temp_bytes(dtype, value_bytes, n);
  if (d_temp == nullptr) {
    cudaError_t e = c.reserve(need);
    if (e != cudaSuccess) return cuda_fail(e, what);
    d_temp = c.arena;
    temp_bytes = c.arena_bytes;
  } else if (temp_bytes < need) {
    set_last_error("%s: d_temp holds %zu bytes, %zu needed", what, temp_bytes, need);
    return MGS_ERR_INVALID;
  }
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c.compute;
  const cudaError_t e =
      argsort ? mgs::radix_argsort(dtype, d_keys, d_values, value_bytes, n, d_temp, temp_bytes, s, c.d_status,
                                   &c.recorder)
              : mgs::radix_sort_pairs(dtype, d_keys, d_values, value_bytes, n, d_temp, temp_bytes, s, c.d_status,
                                      &c.recorder);
  if (e != cudaSuccess) return cuda_fail(e, what);
  mgs::clear_last_error();
  return MGS_OK;
}

int mgs_sort_pairs_device(mgs_ctx* ctx, int dtype, void* d_keys, void* d_values, size_t value_bytes, size_t n,
                          void* d_temp, size_t temp_bytes, void* stream) {
  return pairs_call(ctx, "mgs_sort_pairs_device", dtype, d_keys, d_values, value_bytes, n, d_temp, temp_bytes, stream,
                    false);
}

int mgs_argsort_device(mgs_ctx* ctx, int dtype, void* d_keys, void* d_indices, size_t index_bytes, size_t n,
                       void* d_temp, size_t temp_bytes, void* stream) {
  return pairs_call(ctx, "mgs_argsort_device", dtype, d_keys, d_indices, index_bytes, n, d_temp, temp_bytes, stream,
                    true);
}

int mgs_sort_range_device(mgs_ctx* ctx, int dtype, void* d_keys, void* d_values, size_t value_bytes, size_t n,
                          int begin_bit, int end_bit, int descending, void* d_temp, size_t temp_bytes, void* stream) {
  if (!ctx) return invalid("mgs_sort_range_device: ctx is null");
  const size_t w = mgs::dtype_bytes(dtype);
  if (w == 0) return invalid("mgs_sort_range_device: unknown dtype");
  if (value_bytes != 0 && value_bytes != 4 && value_bytes != 8)
    return invalid("mgs_sort_range_device: value_bytes must be 0, 4 or 8");
  if (begin_bit < 0 || begin_bit > end_bit || end_bit > int(8 * w))
    return invalid("mgs_sort_range_device: need 0 <= begin_bit <= end_bit <= key bits");
  if (n == 0) return MGS_OK;
  if (!d_keys || (value_bytes && !d_values)) return invalid("mgs_sort_range_device: null pointer");
  if (reinterpret_cast<uintptr_t>(d_keys) % w != 0 ||
      (value_bytes && reinterpret_cast<uintptr_t>(d_values) % value_bytes != 0))
    return invalid("mgs_sort_range_device: keys or values are not aligned to their size");
  if (n > kMaxDeviceSortKeys) return invalid("mgs_sort_range_device: n must be below 2^32");
  Context& c = ctx->impl;
  DeviceGuard g(c.device);
  const size_t need =
      value_bytes ? mgs::radix_sort_pairs_temp_bytes(dtype, value_bytes, n) : mgs::radix_sort_temp_bytes(dtype, n);
  if (d_temp == nullptr) {
    cudaError_t e = c.reserve(need);
    if (e != cudaSuccess) return cuda_fail(e, "mgs_sort_range_device: arena");
    d_temp = c.arena;
    temp_bytes = c.arena_bytes;
  } else if (temp_bytes < need) {
    set_last_error("mgs_sort_range_device: d_temp holds %zu bytes, %zu needed", temp_bytes, need);
    return MGS_ERR_INVALID;
  }
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c.compute;
  const cudaError_t e = mgs::radix_sort_range(dtype, d_keys, d_values, value_bytes, n, begin_bit, end_bit, descending,
                                              d_temp, temp_bytes, s, c.d_status, &c.recorder);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_sort_range_device");
  mgs::clear_last_error();
  return MGS_OK;
}

namespace {
// Phases of one TanasicSort-style call, named like the reference's TimeDurations
// keys (src/tanasic_sort.cuh:229-298): memory_allocation = time spent growing
// the context arena in this call (0 once it is large enough), sort_phase = the
// rest of the call (copies, sorts and merges); the arena is kept, so there is
// no deallocation phase.
struct CallPhases {
  Context& c;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  explicit CallPhases(Context& ctx) : c(ctx) { c.reserve_s = 0; }
  ~CallPhases() {
    const double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    c.phase_s[0] = c.reserve_s;
    c.phase_s[1] = total > c.reserve_s ? total - c.reserve_s : 0.0;
    c.phase_s[2] = 0;
    c.phase_s[3] = 0;
  }
};
}  // namespace

int mgs_sort_host(mgs_ctx* ctx, int dtype, void* h_keys, size_t n) {
  if (!ctx) return invalid("mgs_sort_host: ctx is null");
  const size_t w = mgs::dtype_bytes(dtype);
  if (w == 0) return invalid("mgs_sort_host: unknown dtype");
  if (n == 0) return MGS_OK;  // src/tanasic_sort.cuh:225-227
  if (!h_keys) return invalid("mgs_sort_host: h_keys is null");
  if (n > kMaxDeviceSortKeys) return invalid("mgs_sort_host: n must be below 2^32");
  Context& c = ctx->impl;
  DeviceGuard g(c.device);
  CallPhases phases(c);
  if (mgs::plan_staged(n, w).slabs > 1) {
    // Copies overlapped with slab sorts and a windowed merge; needs room for
    // two copies of the keys, else the plain path below runs.
    cudaError_t e = mgs::staged_host_sort(c, dtype, h_keys, n);
    if (e == cudaSuccess) {
      uint32_t status = 0;
      e = c.take_status(c.compute, &status);
      if (e != cudaSuccess) return cuda_fail(e, "mgs_sort_host: synchronize");
      int rc = status_to_code(status);
      if (rc == MGS_OK) mgs::clear_last_error();
      return rc;
    }
    if (e != cudaErrorMemoryAllocation) return cuda_fail(e, "mgs_sort_host: staged sort");
    cudaGetLastError();
  }
  const size_t bytes = n * w;
  const size_t keys_bytes = align256(bytes);
  const size_t temp = mgs::radix_sort_temp_bytes(dtype, n);
  cudaError_t e = c.reserve(keys_bytes + temp);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_sort_host: arena");
  char* base = static_cast<char*>(c.arena);
  void* d_keys = base;
  void* d_temp = base + keys_bytes;
  e = cudaMemcpyAsync(d_keys, h_keys, bytes, cudaMemcpyHostToDevice, c.compute);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_sort_host: H2D");
  e = mgs::radix_sort(dtype, d_keys, n, d_temp, c.arena_bytes - keys_bytes, c.compute, c.d_status, &c.recorder);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_sort_host: sort");
  e = cudaMemcpyAsync(h_keys, d_keys, bytes, cudaMemcpyDeviceToHost, c.compute);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_sort_host: D2H");
  uint32_t status = 0;
  e = c.take_status(c.compute, &status);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_sort_host: synchronize");
  int rc = status_to_code(status);
  if (rc == MGS_OK) mgs::clear_last_error();
  return rc;
}

static int finish_sync(Context& c, const char* what) {
  uint32_t status = 0;
  cudaError_t e = c.take_status(c.compute, &status);
  if (e != cudaSuccess) return cuda_fail(e, what);
  int rc = status_to_code(status);
  if (rc == MGS_OK) mgs::clear_last_error();
  return rc;
}

static int check_chunks(int num_chunks) {
  if (num_chunks < 1 || (num_chunks & (num_chunks - 1)) != 0 || num_chunks > 2 * mgs::kMaxPivotHalf) return 0;
  return 1;
}

int mgs_tanasic_sort(mgs_ctx* ctx, int dtype, void* h_keys, size_t n, int num_chunks) {
  if (!ctx) return invalid("mgs_tanasic_sort: ctx is null");
  if (mgs::dtype_bytes(dtype) == 0) return invalid("mgs_tanasic_sort: unknown dtype");
  if (!check_chunks(num_chunks)) return invalid("mgs_tanasic_sort: num_chunks must be a power of two in [1, 128]");
  if (n == 0) return MGS_OK;  // src/tanasic_sort.cuh:225-227
  if (!h_keys) return invalid("mgs_tanasic_sort: h_keys is null");
  if (num_chunks == 1) return mgs_sort_host(ctx, dtype, h_keys, n);
  Context& c = ctx->impl;
  DeviceGuard g(c.device);
  CallPhases phases(c);
  const mgs::ChunkPlan plan = mgs::plan_chunks(n, num_chunks);
  if (plan.chunk > kMaxDeviceSortKeys) return invalid("mgs_tanasic_sort: chunks must hold fewer than 2^32 keys");
  const size_t temp = mgs::chunk_sort_temp_bytes(dtype, n, num_chunks);
  cudaError_t e = c.reserve(temp);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_tanasic_sort: arena");
  e = mgs::chunk_sort(c, dtype, h_keys, h_keys, nullptr, n, num_chunks, c.arena, c.arena_bytes, c.compute);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_tanasic_sort");
  return finish_sync(c, "mgs_tanasic_sort: synchronize");
}

int mgs_tanasic_sort_device(mgs_ctx* ctx, int dtype, void* d_keys, size_t n, int num_chunks) {
  if (!ctx) return invalid("mgs_tanasic_sort_device: ctx is null");
  const size_t w = mgs::dtype_bytes(dtype);
  if (w == 0) return invalid("mgs_tanasic_sort_device: unknown dtype");
  if (!check_chunks(num_chunks)) return invalid("mgs_tanasic_sort_device: num_chunks must be a power of two in [1, 128]");
  if (n == 0) return MGS_OK;
  if (!d_keys) return invalid("mgs_tanasic_sort_device: d_keys is null");
  Context& c = ctx->impl;
  DeviceGuard g(c.device);
  const mgs::ChunkPlan plan = mgs::plan_chunks(n, num_chunks);
  if (plan.chunk > kMaxDeviceSortKeys) return invalid("mgs_tanasic_sort_device: chunks must hold fewer than 2^32 keys");
  const size_t temp = mgs::chunk_sort_temp_bytes(dtype, n, num_chunks);
  cudaError_t e = c.reserve(temp);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_tanasic_sort_device: arena");
  e = mgs::chunk_sort(c, dtype, nullptr, nullptr, d_keys, n, num_chunks, c.arena, c.arena_bytes, c.compute);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_tanasic_sort_device");
  return finish_sync(c, "mgs_tanasic_sort_device: synchronize");
}

int mgs_find_pivot_device(mgs_ctx* ctx, int dtype, const void* const* d_left, const void* const* d_right, int half,
                          size_t chunk_size, size_t* pivot) {
  if (!ctx || !d_left || !d_right || !pivot) return invalid("mgs_find_pivot_device: null argument");
  if (mgs::dtype_bytes(dtype) == 0) return invalid("mgs_find_pivot_device: unknown dtype");
  if (half < 1 || half > mgs::kMaxPivotHalf || chunk_size == 0)
    return invalid("mgs_find_pivot_device: half must be in [1, 64] and chunk_size > 0");
  Context& c = ctx->impl;
  DeviceGuard g(c.device);
  cudaError_t e = c.reserve(256);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_find_pivot_device: arena");
  uint64_t* d_pivot = static_cast<uint64_t*>(c.arena);
  e = mgs::pivot_search(dtype, d_left, d_right, half, chunk_size, d_pivot, c.compute, &c.recorder);
  if (e == cudaSuccess) e = cudaMemcpyAsync(c.h_status64, d_pivot, 8, cudaMemcpyDeviceToHost, c.compute);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.compute);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_find_pivot_device");
  *pivot = size_t(*c.h_status64);
  mgs::clear_last_error();
  return MGS_OK;
}

int mgs_merge_temp_bytes(int dtype, int k, size_t total, size_t* bytes) {
  if (!bytes) return invalid("mgs_merge_temp_bytes: bytes is null");
  if (mgs::dtype_bytes(dtype) == 0) return invalid("mgs_merge_temp_bytes: unknown dtype");
  if (k < 1 || k > mgs::kMaxKwayRuns) return invalid("mgs_merge_temp_bytes: k must be in [1, 1024]");
  *bytes = mgs::kway_merge_temp_bytes(dtype, k, total);
  return MGS_OK;
}

int mgs_kway_merge_device(mgs_ctx* ctx, int dtype, const void* const* d_runs, const size_t* lens, int k, void* d_out,
                          void* d_temp, size_t temp_bytes, void* stream) {
  if (!ctx) return invalid("mgs_kway_merge_device: ctx is null");
  const size_t w = mgs::dtype_bytes(dtype);
  if (w == 0) return invalid("mgs_kway_merge_device: unknown dtype");
  if (k < 1 || k > mgs::kMaxKwayRuns) return invalid("mgs_kway_merge_device: k must be in [1, 1024]");
  if (!d_runs || !lens) return invalid("mgs_kway_merge_device: null run table");
  size_t total = 0;
  for (int r = 0; r < k; ++r) {
    if (lens[r] > 0 && !d_runs[r]) return invalid("mgs_kway_merge_device: null run pointer");
    total += lens[r];
  }
  if (total == 0) return MGS_OK;
  if (!d_out) return invalid("mgs_kway_merge_device: d_out is null");
  Context& c = ctx->impl;
  DeviceGuard g(c.device);
  const size_t need = mgs::kway_merge_temp_bytes(dtype, k, total);
  if (d_temp == nullptr) {
    cudaError_t e = c.reserve(need);
    if (e != cudaSuccess) return cuda_fail(e, "mgs_kway_merge_device: arena");
    d_temp = c.arena;
    temp_bytes = c.arena_bytes;
  } else if (temp_bytes < need) {
    set_last_error("mgs_kway_merge_device: d_temp holds %zu bytes, %zu needed", temp_bytes, need);
    return MGS_ERR_INVALID;
  }
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c.compute;
  cudaError_t e = mgs::kway_merge(dtype, d_runs, lens, k, d_out, d_temp, temp_bytes, s, &c.recorder);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_kway_merge_device");
  mgs::clear_last_error();
  return MGS_OK;
}

int mgs_merge_device(mgs_ctx* ctx, int dtype, const void* d_a, size_t na, const void* d_b, size_t nb, void* d_out,
                     void* d_temp, size_t temp_bytes, void* stream) {
  const void* runs[2] = {d_a, d_b};
  const size_t lens[2] = {na, nb};
  return mgs_kway_merge_device(ctx, dtype, runs, lens, 2, d_out, d_temp, temp_bytes, stream);
}

int mgs_segmented_sort_temp_bytes(int dtype, size_t n, size_t num_segments, size_t* bytes) {
  if (!bytes) return invalid("mgs_segmented_sort_temp_bytes: bytes is null");
  if (mgs::dtype_bytes(dtype) == 0) return invalid("mgs_segmented_sort_temp_bytes: unknown dtype");
  if (n > kMaxDeviceSortKeys || num_segments >= kMaxDeviceSortKeys)
    return invalid("mgs_segmented_sort_temp_bytes: n and num_segments must be below 2^32");
  *bytes = mgs::segmented_sort_temp_bytes(dtype, n, num_segments);
  return MGS_OK;
}

int mgs_segmented_sort_device(mgs_ctx* ctx, int dtype, void* d_keys, size_t n, const uint64_t* d_offsets,
                              size_t num_segments, void* d_temp, size_t temp_bytes, void* stream) {
  if (!ctx) return invalid("mgs_segmented_sort_device: ctx is null");
  const size_t w = mgs::dtype_bytes(dtype);
  if (w == 0) return invalid("mgs_segmented_sort_device: unknown dtype");
  if (n == 0 || num_segments == 0) return MGS_OK;
  if (!d_keys || !d_offsets) return invalid("mgs_segmented_sort_device: null pointer");
  if (reinterpret_cast<uintptr_t>(d_keys) % w != 0) return invalid("mgs_segmented_sort_device: d_keys is not key-aligned");
  if (n > kMaxDeviceSortKeys || num_segments >= kMaxDeviceSortKeys)
    return invalid("mgs_segmented_sort_device: n and num_segments must be below 2^32");
  Context& c = ctx->impl;
  DeviceGuard g(c.device);
  const size_t need = mgs::segmented_sort_temp_bytes(dtype, n, num_segments);
  if (d_temp == nullptr) {
    cudaError_t e = c.reserve(need);
    if (e != cudaSuccess) return cuda_fail(e, "mgs_segmented_sort_device: arena");
    d_temp = c.arena;
    temp_bytes = c.arena_bytes;
  } else if (temp_bytes < need) {
    set_last_error("mgs_segmented_sort_device: d_temp holds %zu bytes, %zu needed", temp_bytes, need);
    return MGS_ERR_INVALID;
  }
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c.compute;
  cudaError_t e = mgs::segmented_sort(dtype, d_keys, n, d_offsets, num_segments, d_temp, temp_bytes, s, c.d_status,
                                      &c.recorder);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_segmented_sort_device");
  mgs::clear_last_error();
  return MGS_OK;
}

int mgs_plan_sort_create(mgs_ctx* ctx, int dtype, void* d_keys, size_t n, void* d_temp, size_t temp_bytes,
                         mgs_plan** out) {
  if (!ctx || !out) return invalid("mgs_plan_sort_create: null argument");
  *out = nullptr;
  const size_t w = mgs::dtype_bytes(dtype);
  if (w == 0) return invalid("mgs_plan_sort_create: unknown dtype");
  if (n > 0 && !d_keys) return invalid("mgs_plan_sort_create: d_keys is null");
  if (reinterpret_cast<uintptr_t>(d_keys) % w != 0) return invalid("mgs_plan_sort_create: d_keys is not key-aligned");
  if (n > kMaxDeviceSortKeys) return invalid("mgs_plan_sort_create: n must be below 2^32");
  const size_t need = n ? mgs::radix_sort_temp_bytes(dtype, n) : 0;
  return plan_record(ctx, "mgs_plan_sort_create", need, d_temp, temp_bytes,
                     [&](void* t, size_t tb, cudaStream_t s, mgs::LaunchRecorder* rec) {
                       return mgs::radix_sort(dtype, d_keys, n, t, tb, s, ctx->impl.d_status, rec);
                     },
                     out);
}

int mgs_plan_segmented_create(mgs_ctx* ctx, int dtype, void* d_keys, size_t n, const uint64_t* d_offsets,
                              size_t num_segments, void* d_temp, size_t temp_bytes, mgs_plan** out) {
  if (!ctx || !out) return invalid("mgs_plan_segmented_create: null argument");
  *out = nullptr;
  const size_t w = mgs::dtype_bytes(dtype);
  if (w == 0) return invalid("mgs_plan_segmented_create: unknown dtype");
  const bool empty = (n == 0 || num_segments == 0);
  if (!empty && (!d_keys || !d_offsets)) return invalid("mgs_plan_segmented_create: null pointer");
  if (reinterpret_cast<uintptr_t>(d_keys) % w != 0)
    return invalid("mgs_plan_segmented_create: d_keys is not key-aligned");
  if (n > kMaxDeviceSortKeys || num_segments >= kMaxDeviceSortKeys)
    return invalid("mgs_plan_segmented_create: n and num_segments must be below 2^32");
  const size_t need = empty ? 0 : mgs::segmented_sort_temp_bytes(dtype, n, num_segments);
  return plan_record(ctx, "mgs_plan_segmented_create", need, d_temp, temp_bytes,
                     [&](void* t, size_t tb, cudaStream_t s, mgs::LaunchRecorder* rec) {
                       if (empty) return cudaSuccess;
                       return mgs::segmented_sort(dtype, d_keys, n, d_offsets, num_segments, t, tb, s,
                                                  ctx->impl.d_status, rec);
                     },
                     out);
}

int mgs_plan_launch(mgs_plan* plan, void* stream) {
  if (!plan) return invalid("mgs_plan_launch: plan is null");
  Context& c = plan->ctx->impl;
  DeviceGuard g(c.device);
  const cudaError_t e = cudaGraphLaunch(plan->exec, stream ? static_cast<cudaStream_t>(stream) : c.compute);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_plan_launch");
  c.recorder.add_launches(plan->launches);
  mgs::clear_last_error();
  return MGS_OK;
}

int mgs_plan_launch_count(mgs_plan* plan, uint64_t* launches) {
  if (!plan || !launches) return invalid("mgs_plan_launch_count: null argument");
  *launches = plan->launches;
  return MGS_OK;
}

int mgs_plan_destroy(mgs_plan* plan) {
  if (!plan) return MGS_OK;
  DeviceGuard g(plan->ctx->impl.device);
  cudaDeviceSynchronize();  // a replay may still run on any stream: let it finish before its graph and scratch go
  plan_release(plan);
  mgs::clear_last_error();
  return MGS_OK;
}

int mgs_tune_get(int dtype, size_t n, int* shape, int* rank_mode) {
  const size_t w = mgs::dtype_bytes(dtype);
  if (w == 0 || !shape || !rank_mode) return invalid("mgs_tune_get: unknown dtype or null argument");
  const mgs::SortVariant v = mgs::sort_variant(int(w), n);
  *shape = v.shape;
  *rank_mode = v.mode;
  return MGS_OK;
}

int mgs_tune_set(int dtype, int size_class, int shape, int rank_mode) {
  const size_t w = mgs::dtype_bytes(dtype);
  if (w == 0) return invalid("mgs_tune_set: unknown dtype");
  if (!mgs::set_sort_variant(int(w), size_class, mgs::SortVariant{shape, rank_mode})) {
    set_last_error("mgs_tune_set: size_class must be in [0, %d), shape in [0, 7), rank_mode 2 or 3",
                   mgs::kSizeClasses);
    return MGS_ERR_INVALID;
  }
  mgs::clear_last_error();
  return MGS_OK;
}

int mgs_tune_load(const char* path) {
  if (!path) return invalid("mgs_tune_load: path is null");
  const int r = mgs::load_tuning_file(path);
  if (r == -1) {
    set_last_error("mgs_tune_load: cannot open '%s'", path);
    return MGS_ERR_INVALID;
  }
  if (r == -2) {
    set_last_error("mgs_tune_load: '%s' has malformed or out-of-range lines (the valid ones were applied)", path);
    return MGS_ERR_INVALID;
  }
  mgs::clear_last_error();
  return MGS_OK;
}

int mgs_tune_save(const char* path) {
  if (!path) return invalid("mgs_tune_save: path is null");
  if (!mgs::save_tuning_file(path)) {
    set_last_error("mgs_tune_save: cannot write '%s'", path);
    return MGS_ERR_INVALID;
  }
  mgs::clear_last_error();
  return MGS_OK;
}

int mgs_autotune(mgs_ctx* ctx, int dtype, size_t max_n, int reps, mgs_tune_sample* out, int capacity, int* count) {
  if (!ctx) return invalid("mgs_autotune: ctx is null");
  if (mgs::dtype_bytes(dtype) == 0) return invalid("mgs_autotune: unknown dtype");
  if (reps < 1 || reps > 100) return invalid("mgs_autotune: reps must be in [1, 100]");
  if (capacity > 0 && !out) return invalid("mgs_autotune: out is null");
  Context& c = ctx->impl;
  DeviceGuard g(c.device);
  std::vector<mgs::TuneSample> samples;
  const cudaError_t e = mgs::autotune(dtype, max_n, reps, &samples);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_autotune");
  for (size_t i = 0; i < samples.size() && int(i) < capacity; ++i) {
    const mgs::TuneSample& t = samples[i];
    out[i] = mgs_tune_sample{t.key_bytes, t.size_class, t.n, t.variant.shape, t.variant.mode, t.ms, t.chosen ? 1 : 0};
  }
  if (count) *count = int(samples.size());
  mgs::clear_last_error();
  return MGS_OK;
}

int mgs_gowanlock_sort(mgs_ctx* ctx, int dtype, void* h_keys, size_t n, size_t chunk_size, size_t merge_group_size,
                       size_t num_buffers, int merge_mode) {
  if (!ctx) return invalid("mgs_gowanlock_sort: ctx is null");
  const size_t w = mgs::dtype_bytes(dtype);
  if (w == 0) return invalid("mgs_gowanlock_sort: unknown dtype");
  if (num_buffers != 2 && num_buffers != 3) return invalid("mgs_gowanlock_sort: num_buffers must be 2 or 3");
  if (merge_mode != MGS_MERGE_GPU && merge_mode != MGS_MERGE_CPU)
    return invalid("mgs_gowanlock_sort: merge_mode must be MGS_MERGE_GPU or MGS_MERGE_CPU");
  (void)merge_group_size;  // 0 = automatic; the merge is one k-way pass (see mgs.h)
  if (n == 0) return MGS_OK;  // src/gowanlock_sort.cuh:398-400
  if (!h_keys) return invalid("mgs_gowanlock_sort: h_keys is null");
  Context& c = ctx->impl;
  DeviceGuard g(c.device);
  size_t free_b = 0, total_b = 0;
  cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_gowanlock_sort: cudaMemGetInfo");
  const size_t budget = (free_b + c.arena_bytes) / 10 * 8;
  const mgs::OocPlan plan = mgs::plan_out_of_core(dtype, n, chunk_size, int(num_buffers), 0, budget);
  if (merge_mode == MGS_MERGE_GPU && plan.num_chunks > size_t(mgs::kMaxKwayRuns))
    return invalid("mgs_gowanlock_sort: more than 1024 chunks; use a larger chunk_size");
  const auto t0 = std::chrono::steady_clock::now();
  if (plan.num_chunks > 1) {
    e = c.reserve_host(n * w);
    if (e != cudaSuccess) return cuda_fail(e, "mgs_gowanlock_sort: pinned secondary buffer");
  }
  const double host_alloc_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  mgs::OocTimes t;
  e = mgs::out_of_core_sort(c, dtype, h_keys, n, plan, merge_mode == MGS_MERGE_CPU, c.host_arena, &t);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_gowanlock_sort");
  c.phase_s[0] = host_alloc_s + t.allocation_s;
  c.phase_s[1] = t.sort_s + t.merge_s;
  c.phase_s[2] = t.merge_s;
  c.phase_s[3] = 0;
  return finish_sync(c, "mgs_gowanlock_sort: synchronize");
}

int mgs_ctx_phase_seconds(mgs_ctx* ctx, const char* phase, double* seconds) {
  if (!ctx || !phase || !seconds) return invalid("mgs_ctx_phase_seconds: null argument");
  static const char* names[4] = {"memory_allocation", "sort_phase", "merge_phase", "memory_deallocation"};
  for (int i = 0; i < 4; ++i) {
    if (std::strcmp(phase, names[i]) == 0) {
      *seconds = ctx->impl.phase_s[i];
      return MGS_OK;
    }
  }
  set_last_error("mgs_ctx_phase_seconds: unknown phase '%s'", phase);
  return MGS_ERR_INVALID;
}

int mgs_generate(int dtype, const char* distribution, uint32_t seed, void* out, size_t n) {
  if (!distribution) return invalid("mgs_generate: distribution is null");
  if (mgs::dtype_bytes(dtype) == 0) return invalid("mgs_generate: unknown dtype");
  if (n == 0) return MGS_OK;
  if (!out) return invalid("mgs_generate: out is null");
  if (!mgs::generate_keys(dtype, distribution, seed, out, n)) {
    set_last_error("mgs_generate: unknown distribution '%s' for this dtype", distribution);
    return MGS_ERR_INVALID;
  }
  mgs::clear_last_error();
  return MGS_OK;
}

int mgs_generate_device(mgs_ctx* ctx, int dtype, const char* distribution, uint32_t seed, void* d_out, size_t n) {
  if (!ctx) return invalid("mgs_generate_device: ctx is null");
  if (!distribution) return invalid("mgs_generate_device: distribution is null");
  size_t need = 0;
  std::string why;
  if (!mgs::generate_device_temp_bytes(dtype, distribution, n, &need, &why)) {
    set_last_error("mgs_generate_device: %s", why.c_str());
    return MGS_ERR_INVALID;
  }
  if (n == 0) return MGS_OK;
  const size_t w = mgs::dtype_bytes(dtype);
  if (!d_out) return invalid("mgs_generate_device: d_out is null");
  if (reinterpret_cast<uintptr_t>(d_out) % w != 0) return invalid("mgs_generate_device: d_out is not key-aligned");
  if (n > kMaxDeviceSortKeys) return invalid("mgs_generate_device: n must be below 2^32");
  Context& c = ctx->impl;
  DeviceGuard g(c.device);
  if (need > 0) {
    cudaError_t e = c.reserve(need);
    if (e != cudaSuccess) return cuda_fail(e, "mgs_generate_device: arena");
  }
  cudaError_t e = mgs::generate_device(dtype, distribution, seed, d_out, n, c.arena, c.arena_bytes, c.compute,
                                       c.d_status, &c.recorder);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_generate_device");
  return finish_sync(c, "mgs_generate_device: synchronize");
}

int mgs_test_set_waits(int device, uint32_t lookback_spins, uint32_t tma_polls, uint32_t hold_tile) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    set_last_error("mgs_test_set_waits: no CUDA device %d", device);
    return MGS_ERR_NO_DEVICE;
  }
  DeviceGuard g(device);
  const cudaError_t e = mgs::set_wait_control(lookback_spins, tma_polls, hold_tile);
  if (e != cudaSuccess) return cuda_fail(e, "mgs_test_set_waits");
  mgs::clear_last_error();
  return MGS_OK;
}

int mgs_test_fail_device_allocations(int count) {
  if (count < 0) return invalid("mgs_test_fail_device_allocations: count must be >= 0");
  mgs::fail_next_arena_reservations(count);
  mgs::clear_last_error();
  return MGS_OK;
}

}  // extern "C"
