#include "staged_sort.h"

#include <algorithm>
#include <vector>

#include "../kernels/engine_types.h"
#include "../kernels/merge.cuh"
#include "../kernels/radix_sort.cuh"

namespace mgs {
namespace {

inline size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// Below 2^24 keys the copies take about a millisecond each way and the sort
// a few hundred microseconds: staging would save less than its extra launches.
constexpr size_t kMinStagedKeys = size_t(1) << 24;
constexpr size_t kMinSlabKeys = size_t(1) << 22;
constexpr int kMaxSlabs = 8;
constexpr int kWindows = 8;
constexpr size_t kSlabAlignKeys = 64;  // slab starts on 256-byte boundaries (TMA staging of the radix sort)

struct StagedLayout {
  size_t in_off, out_off, sort_off, sort_bytes, merge_off, merge_bytes, total;
};

StagedLayout staged_layout(int dtype, size_t n, const StagedPlan& p) {
  const size_t w = dtype_bytes(dtype);
  StagedLayout L;
  size_t off = 0;
  L.in_off = off;
  off += align256(n * w);
  L.out_off = off;
  off += align256(n * w);
  L.sort_off = off;
  L.sort_bytes = align256(radix_sort_temp_bytes(dtype, p.slab_keys));
  off += L.sort_bytes;
  L.merge_off = off;
  L.merge_bytes = align256(kway_merge_temp_bytes(dtype, p.slabs, n));
  off += L.merge_bytes;
  L.total = off;
  return L;
}

struct Events {
  cudaEvent_t ready = nullptr, slab = nullptr, window = nullptr;
  cudaError_t create() {
    for (cudaEvent_t* e : {&ready, &slab, &window}) {
      const cudaError_t r = cudaEventCreateWithFlags(e, cudaEventDisableTiming);
      if (r != cudaSuccess) return r;
    }
    return cudaSuccess;
  }
  ~Events() {
    for (cudaEvent_t e : {ready, slab, window})
      if (e) cudaEventDestroy(e);
  }
};

}  // namespace

StagedPlan plan_staged(size_t n, size_t w) {
  (void)w;
  StagedPlan p;
  if (n < kMinStagedKeys) {
    p.slabs = 1;
    p.slab_keys = n;
    p.window_keys = n;
    return p;
  }
  const size_t want = std::min<size_t>(kMaxSlabs, n / kMinSlabKeys);
  p.slab_keys = ((n + want - 1) / want + kSlabAlignKeys - 1) / kSlabAlignKeys * kSlabAlignKeys;
  p.slabs = int((n + p.slab_keys - 1) / p.slab_keys);
  p.window_keys = (n + kWindows - 1) / kWindows;
  return p;
}

size_t staged_sort_device_bytes(int dtype, size_t n) {
  const size_t w = dtype_bytes(dtype);
  if (w == 0) return 0;
  return staged_layout(dtype, n, plan_staged(n, w)).total;
}

cudaError_t staged_host_sort(Context& c, int dtype, void* h_keys, size_t n) {
  const size_t w = dtype_bytes(dtype);
  if (w == 0 || h_keys == nullptr) return cudaErrorInvalidValue;
  const StagedPlan p = plan_staged(n, w);
  if (p.slabs < 2) return cudaErrorInvalidValue;
  const StagedLayout L = staged_layout(dtype, n, p);
  cudaError_t e = c.reserve(L.total);
  if (e != cudaSuccess) return e;
  Events ev;
  e = ev.create();
  if (e != cudaSuccess) return e;

  char* base = static_cast<char*>(c.arena);
  char* d_in = base + L.in_off;
  char* d_out = base + L.out_off;
  char* h = static_cast<char*>(h_keys);

  // Earlier asynchronous work of the context may still read the arena.
  e = cudaEventRecord(ev.ready, c.compute);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(c.h2d, ev.ready, 0);
  if (e != cudaSuccess) return e;

  std::vector<const void*> runs(size_t(p.slabs));
  std::vector<size_t> lens(size_t(p.slabs));
  for (int i = 0; i < p.slabs; ++i) {
    const size_t first = size_t(i) * p.slab_keys;
    const size_t len = std::min(p.slab_keys, n - first);
    runs[size_t(i)] = d_in + first * w;
    lens[size_t(i)] = len;
    e = cudaMemcpyAsync(d_in + first * w, h + first * w, len * w, cudaMemcpyHostToDevice, c.h2d);
    if (e == cudaSuccess) e = cudaEventRecord(ev.slab, c.h2d);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c.compute, ev.slab, 0);
    if (e == cudaSuccess)
      e = radix_sort(dtype, d_in + first * w, len, base + L.sort_off, L.sort_bytes, c.compute, c.d_status,
                     &c.recorder);
    if (e != cudaSuccess) return e;
  }

  const MergeWindowFn to_host = [&](size_t first, size_t count) -> cudaError_t {
    cudaError_t r = cudaEventRecord(ev.window, c.compute);
    if (r == cudaSuccess) r = cudaStreamWaitEvent(c.d2h, ev.window, 0);
    if (r == cudaSuccess)
      r = cudaMemcpyAsync(h + first * w, d_out + first * w, count * w, cudaMemcpyDeviceToHost, c.d2h);
    return r;
  };
  e = kway_merge_windowed(dtype, runs.data(), lens.data(), p.slabs, d_out, base + L.merge_off, L.merge_bytes,
                          p.window_keys, to_host, c.compute, &c.recorder);
  // Whatever was enqueued must finish before the host buffer is handed back.
  const cudaError_t s1 = cudaStreamSynchronize(c.d2h);
  const cudaError_t s2 = cudaStreamSynchronize(c.h2d);
  if (e != cudaSuccess) return e;
  return s1 != cudaSuccess ? s1 : s2;
}

}  // namespace mgs
