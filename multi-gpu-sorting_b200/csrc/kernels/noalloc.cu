// Device sort for callers that cannot allocate device memory.
//
// Some callers of a sort cannot call cudaMalloc: code that runs while a
// memory pool or arena owns all of the device memory, allocators and
// runtimes that must not re-enter the CUDA allocator, and hosts that forbid
// allocation once they start serving. For them, mgs_sort_device_noalloc sorts
// with a fixed scratch area that is part of this library's device image: a
// file-scope __device__ array, created when the library's module is loaded on
// a GPU and held by that GPU until the process exits. The caller passes the
// keys (in and out); nothing else is allocated.
//
// Limits and behaviour:
//   * Scratch is kNoAllocScratchBytes (32 MiB) per GPU. A call sorts at most
//     2^22 (4,194,304) keys of 4 bytes or 2^21 (2,097,152) keys of 8 bytes
//     (their scratch need, mgs_sort_temp_bytes, stays below 20 MiB); larger n is
//     rejected with MGS_ERR_INVALID.
//   * Every call on a GPU shares the one array. Calls whose work overlaps on
//     that GPU (different streams, or several host threads) race on it; order
//     them on one stream or serialize them.
//   * The array keeps the last call's contents. Everything the sort needs to
//     start at zero (digit counts, tile counters, look-back status words) is
//     cleared by each call on its stream before use.
//   * The first call on a device resolves the array's device address for that
//     device (cudaGetSymbolAddress, with that device current) and caches it.
//     Make that first call before any stream capture on the device. The cache
//     is keyed by the device's current CUDA context (its unique context id):
//     after cudaDeviceReset, or any other teardown of the device's context,
//     the library's module is loaded again and the array may sit at a new
//     address, so the next call resolves it again (that call is then a first
//     call once more, and must come before any stream capture too).
//   * Asynchronous on `stream`; device-side wait timeouts are not reported
//     (there is no context status word), the result is then unspecified.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "engine_types.h"
#include "mgs.h"
#include "radix_sort.cuh"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
constexpr size_t kNoAllocMaxBytesOfKeys = size_t(16) << 20;  // 2^22 4-byte keys or 2^21 8-byte keys
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_mutex;
void* g_scratch_ptr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};  // id of the context the cached address belongs to

// Unique id of the calling thread's current CUDA context (ids are never reused
// within a process), through the driver entry points the runtime exposes; 0
// when it cannot be read, which forces a fresh address lookup.
unsigned long long current_context_id() {
  using GetCurrentFn = CUresult (*)(CUcontext*);
  using GetIdFn = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrentFn get_current = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<GetCurrentFn>(f);
  }();
  static GetIdFn get_id = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<GetIdFn>(f);
  }();
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (get_current == nullptr || get_id == nullptr || get_current(&c) != CUDA_SUCCESS || c == nullptr ||
      get_id(c, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

// Device address of g_noalloc_scratch on `device` (which is current), looked
// up again whenever the device's context is not the one the cached address
// came from.
cudaError_t scratch_address(int device, void** out) {
  std::lock_guard<std::mutex> lock(g_mutex);
  const unsigned long long ctx_id = current_context_id();
  if (g_scratch_ptr[device] == nullptr || ctx_id == 0 || g_scratch_ctx[device] != ctx_id) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[device] = p;
    g_scratch_ctx[device] = ctx_id;
  }
  *out = g_scratch_ptr[device];
  return cudaSuccess;
}

}  // namespace

namespace mgs {
void set_last_error(const char* fmt, ...);
void clear_last_error();
}  // namespace mgs

extern "C" int mgs_sort_device_noalloc(int dtype, void* d_keys, size_t n, void* stream) {
  const size_t w = mgs::dtype_bytes(dtype);
  if (w == 0) {
    mgs::set_last_error("mgs_sort_device_noalloc: unknown dtype");
    return MGS_ERR_INVALID;
  }
  if (n == 0) return MGS_OK;
  if (d_keys == nullptr || reinterpret_cast<uintptr_t>(d_keys) % w != 0) {
    mgs::set_last_error("mgs_sort_device_noalloc: d_keys is null or not key-aligned");
    return MGS_ERR_INVALID;
  }
  const size_t max_keys = kNoAllocMaxBytesOfKeys / w;
  if (n > max_keys || mgs::radix_sort_temp_bytes(dtype, n) > kNoAllocScratchBytes) {
    mgs::set_last_error(
        "mgs_sort_device_noalloc: %zu keys exceed the static scratch (%zu bytes): at most %zu keys of %zu bytes", n,
        kNoAllocScratchBytes, max_keys, w);
    return MGS_ERR_INVALID;
  }
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e == cudaSuccess && (device < 0 || device >= kMaxDevices)) e = cudaErrorInvalidDevice;
  void* scratch = nullptr;
  if (e == cudaSuccess) e = scratch_address(device, &scratch);
  if (e == cudaSuccess)
    e = mgs::radix_sort(dtype, d_keys, n, scratch, kNoAllocScratchBytes, static_cast<cudaStream_t>(stream), nullptr,
                        nullptr);
  if (e != cudaSuccess) {
    mgs::set_last_error("mgs_sort_device_noalloc: %s", cudaGetErrorString(e));
    cudaGetLastError();
    return MGS_ERR_CUDA;
  }
  mgs::clear_last_error();
  return MGS_OK;
}
