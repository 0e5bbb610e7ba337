// Out-of-core sort: GowanlockSort (HET sort, src/gowanlock_sort.cuh:127-483 of
// the reference) on one GPU.
//
// Phase A (chunk sort): the keys stream through a ring of `num_buffers` device
// chunk buffers. Chunk i is copied H2D on the context's h2d stream (one copy
// engine), radix-sorted on the compute stream, and copied D2H on the d2h stream
// (the other copy engine); CUDA events order the three, so with three buffers
// the H2D of chunk i+1, the sort of chunk i and the D2H of chunk i-1 overlap
// (the reference's 3-buffer mode gets the same overlap from InplaceMemcpy,
// src/inplace_memcpy.cuh:7-69; its 2-buffer mode, src/gowanlock_sort.cuh:127-230,
// corresponds to num_buffers = 2 here).
// Phase B (merge): the sorted runs are merged into the caller's buffer, either
//   * on the GPU (default): the output is produced in windows; the exact split
//     of every window boundary over the runs is computed on the host
//     (multi-sequence selection, stable by run index), the window's pieces of
//     every run are copied H2D, merged by the k-way merge kernel and copied D2H,
//     with consecutive windows pipelined over two buffer sets; or
//   * on the CPU with __gnu_parallel::multiway_merge and std::less<T>, the
//     reference's own merge (src/gowanlock_sort.cuh:73-74,91-92).
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <parallel/algorithm>
#include <vector>

#include "../kernels/device_common.cuh"
#include "../kernels/dispatch.cuh"
#include "../kernels/merge.cuh"
#include "../kernels/radix_sort.cuh"
#include "context.h"
#include "out_of_core.h"

namespace mgs {
namespace {

inline size_t align256(size_t x) { return (x + 255) / 256 * 256; }

struct EventRing {
  std::vector<cudaEvent_t> ev;
  explicit EventRing(size_t n) : ev(n, nullptr) {
    for (auto& e : ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  }
  ~EventRing() {
    for (auto e : ev)
      if (e) cudaEventDestroy(e);
  }
};

// Split of the first d outputs of the stable k-way merge of sorted host runs:
// split[r] = number of keys taken from run r (ties go to the lower run index).
// Bisection over the radix-order key space with every run's index window
// narrowed as the value window shrinks, then equal keys split in run order.
template <class Tr>
void host_kway_split(const typename Tr::Bits* const* runs, const size_t* lens, int k, size_t d, size_t* split) {
  using Bits = typename Tr::Bits;
  size_t total = 0;
  for (int r = 0; r < k; ++r) total += lens[r];
  if (d >= total) {
    for (int r = 0; r < k; ++r) split[r] = lens[r];
    return;
  }
  std::vector<size_t> a(k, 0), b(lens, lens + k), u(k);
  auto upper = [&](int r, size_t lo, size_t hi, Bits v) {
    while (lo < hi) {
      const size_t mid = (lo + hi) / 2;
      if (Tr::Ordered(runs[r][mid]) <= v) lo = mid + 1; else hi = mid;
    }
    return lo;
  };
  auto lower = [&](int r, size_t lo, size_t hi, Bits v) {
    while (lo < hi) {
      const size_t mid = (lo + hi) / 2;
      if (Tr::Ordered(runs[r][mid]) < v) lo = mid + 1; else hi = mid;
    }
    return lo;
  };
  Bits vlo = 0, vhi = ~Bits(0);
  while (vlo < vhi) {
    size_t width = 0;
    for (int r = 0; r < k; ++r) width += b[r] - a[r];
    if (width == 0) break;
    const Bits vmid = vlo + (vhi - vlo) / 2;
    size_t le = 0;
    for (int r = 0; r < k; ++r) {
      u[r] = upper(r, a[r], b[r], vmid);
      le += u[r];
    }
    if (le > d) {
      vhi = vmid;
      b = u;
    } else {
      vlo = vmid + 1;
      a = u;
    }
  }
  size_t lt_sum = 0;
  std::vector<size_t> lt(k), eq(k);
  for (int r = 0; r < k; ++r) {
    lt[r] = lower(r, 0, b[r], vlo);
    eq[r] = upper(r, std::max(a[r], lt[r]), lens[r], vlo) - lt[r];
    lt_sum += lt[r];
  }
  size_t rem = d - lt_sum;
  for (int r = 0; r < k; ++r) {
    const size_t take = std::min(rem, eq[r]);
    split[r] = lt[r] + take;
    rem -= take;
  }
}

template <typename T>
void cpu_multiway_merge(const T* src, const std::vector<size_t>& offs, const std::vector<size_t>& lens, T* out,
                        size_t n) {
  std::vector<std::pair<T*, T*>> pairs;
  for (size_t r = 0; r < lens.size(); ++r) {
    T* b = const_cast<T*>(src) + offs[r];
    pairs.emplace_back(b, b + lens[r]);
  }
  __gnu_parallel::multiway_merge(pairs.begin(), pairs.end(), out, n, std::less<T>());
}

void cpu_merge_dispatch(int dtype, const void* src, const std::vector<size_t>& offs, const std::vector<size_t>& lens,
                        void* out, size_t n) {
  switch (dtype) {
    case 0: cpu_multiway_merge(static_cast<const uint32_t*>(src), offs, lens, static_cast<uint32_t*>(out), n); break;
    case 1: cpu_multiway_merge(static_cast<const int32_t*>(src), offs, lens, static_cast<int32_t*>(out), n); break;
    case 2: cpu_multiway_merge(static_cast<const float*>(src), offs, lens, static_cast<float*>(out), n); break;
    case 3: cpu_multiway_merge(static_cast<const uint64_t*>(src), offs, lens, static_cast<uint64_t*>(out), n); break;
    case 4: cpu_multiway_merge(static_cast<const int64_t*>(src), offs, lens, static_cast<int64_t*>(out), n); break;
    default: cpu_multiway_merge(static_cast<const double*>(src), offs, lens, static_cast<double*>(out), n); break;
  }
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

OocPlan plan_out_of_core(int dtype, size_t n, size_t chunk, int num_buffers, size_t window, size_t device_budget) {
  const size_t w = dtype_bytes(dtype);
  OocPlan p{};
  p.num_buffers = num_buffers < 2 ? 2 : (num_buffers > 3 ? 3 : num_buffers);
  if (chunk == 0) {
    // Default: the whole input when it fits the budget (the reference's
    // chunk_size = n / num_gpus, src/gowanlock_sort.cuh:402-404), else the
    // largest chunk whose ring of buffers and sort scratch fit.
    const size_t per_key = w * (p.num_buffers + 1) + 1;
    chunk = std::max<size_t>(1, device_budget / per_key);
    chunk = std::min(chunk, n);
  }
  chunk = std::min(chunk, (size_t(1) << 32) - 1);
  p.chunk = chunk;
  p.num_chunks = (n + chunk - 1) / chunk;
  p.window = window ? window : std::min<size_t>(n, (size_t(512) << 20) / w);
  p.phase_a_bytes = size_t(p.num_buffers) * align256(chunk * w) + align256(radix_sort_temp_bytes(dtype, chunk));
  const int k = int(std::min<size_t>(p.num_chunks, size_t(kMaxKwayRuns)));
  p.phase_b_bytes = 4 * align256(p.window * w) + align256(kway_merge_temp_bytes(dtype, k, p.window));
  return p;
}

cudaError_t out_of_core_sort(Context& c, int dtype, void* h_keys, size_t n, const OocPlan& p, int merge_on_cpu,
                             void* h_secondary, OocTimes* times) {
  const size_t w = dtype_bytes(dtype);
  const size_t C = p.chunk;
  const size_t k = p.num_chunks;
  char* h = static_cast<char*>(h_keys);
  char* sec = static_cast<char*>(h_secondary);
  const auto t0 = std::chrono::steady_clock::now();
  cudaError_t e = c.reserve(std::max(p.phase_a_bytes, k > 1 && !merge_on_cpu ? p.phase_b_bytes : 0));
  if (e != cudaSuccess) return e;
  if (times) times->allocation_s = seconds_since(t0);
  char* arena = static_cast<char*>(c.arena);

  // ---- phase A: chunk sort ring ----
  const auto ta = std::chrono::steady_clock::now();
  {
    const int NB = p.num_buffers;
    std::vector<char*> buf(NB);
    for (int i = 0; i < NB; ++i) buf[i] = arena + size_t(i) * align256(C * w);
    char* radix_temp = arena + size_t(NB) * align256(C * w);
    const size_t radix_bytes = align256(radix_sort_temp_bytes(dtype, C));
    char* dst = (k == 1) ? h : sec;  // one chunk: straight back in place
    EventRing h2d_done(NB), sort_done(NB), d2h_done(NB);
    for (size_t i = 0; i < k && e == cudaSuccess; ++i) {
      const int b = int(i % NB);
      const size_t off = i * C;
      const size_t len = std::min(C, n - off);
      if (i >= size_t(NB)) e = cudaStreamWaitEvent(c.h2d, d2h_done.ev[b], 0);
      if (e == cudaSuccess) e = cudaMemcpyAsync(buf[b], h + off * w, len * w, cudaMemcpyHostToDevice, c.h2d);
      if (e == cudaSuccess) e = cudaEventRecord(h2d_done.ev[b], c.h2d);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(c.compute, h2d_done.ev[b], 0);
      if (e == cudaSuccess) e = radix_sort(dtype, buf[b], len, radix_temp, radix_bytes, c.compute, c.d_status, &c.recorder);
      if (e == cudaSuccess) e = cudaEventRecord(sort_done.ev[b], c.compute);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(c.d2h, sort_done.ev[b], 0);
      if (e == cudaSuccess) e = cudaMemcpyAsync(dst + off * w, buf[b], len * w, cudaMemcpyDeviceToHost, c.d2h);
      if (e == cudaSuccess) e = cudaEventRecord(d2h_done.ev[b], c.d2h);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.d2h);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.compute);
    if (e != cudaSuccess) return e;
  }
  if (times) times->sort_s = seconds_since(ta);
  if (k == 1) {
    if (times) times->merge_s = 0;
    return cudaSuccess;
  }

  // ---- phase B: merge the k sorted runs (sec) into the caller's buffer (h) ----
  const auto tb = std::chrono::steady_clock::now();
  std::vector<size_t> offs(k), lens(k);
  for (size_t r = 0; r < k; ++r) {
    offs[r] = r * C;
    lens[r] = std::min(C, n - r * C);
  }
  if (merge_on_cpu) {
    cpu_merge_dispatch(dtype, sec, offs, lens, h, n);
    if (times) times->merge_s = seconds_since(tb);
    return cudaSuccess;
  }
  if (k > size_t(kMaxKwayRuns)) return cudaErrorInvalidValue;
  const size_t W = p.window;
  const size_t nwin = (n + W - 1) / W;
  // Exact window boundaries over the runs (host multi-sequence selection).
  std::vector<size_t> split((nwin + 1) * k);
  dispatch_dtype(dtype, [&](auto tr) {
    using Tr = decltype(tr);
    using Bits = typename Tr::Bits;
    std::vector<const Bits*> runs(k);
    for (size_t r = 0; r < k; ++r) runs[r] = reinterpret_cast<const Bits*>(sec) + offs[r];
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t wi = 0; wi <= nwin; ++wi)
      host_kway_split<Tr>(runs.data(), lens.data(), int(k), std::min(wi * W, n), &split[wi * k]);
  });
  char* in[2] = {arena, arena + align256(W * w)};
  char* out[2] = {arena + 2 * align256(W * w), arena + 3 * align256(W * w)};
  char* kway_temp = arena + 4 * align256(W * w);
  const size_t kway_bytes = align256(kway_merge_temp_bytes(dtype, int(k), W));
  EventRing h2d_done(2), merge_done(2), d2h_done(2);
  std::vector<const void*> wruns(k);
  std::vector<size_t> wlens(k);
  for (size_t wi = 0; wi < nwin && e == cudaSuccess; ++wi) {
    const int b = int(wi & 1);
    if (wi >= 2) e = cudaStreamWaitEvent(c.h2d, merge_done.ev[b], 0);  // in[b] consumed by window wi-2
    size_t pos = 0;
    for (size_t r = 0; r < k && e == cudaSuccess; ++r) {
      const size_t s0 = split[wi * k + r], s1 = split[(wi + 1) * k + r];
      wruns[r] = in[b] + pos * w;
      wlens[r] = s1 - s0;
      if (s1 > s0)
        e = cudaMemcpyAsync(in[b] + pos * w, sec + (offs[r] + s0) * w, (s1 - s0) * w, cudaMemcpyHostToDevice, c.h2d);
      pos += s1 - s0;
    }
    if (e == cudaSuccess) e = cudaEventRecord(h2d_done.ev[b], c.h2d);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c.compute, h2d_done.ev[b], 0);
    if (e == cudaSuccess && wi >= 2) e = cudaStreamWaitEvent(c.compute, d2h_done.ev[b], 0);  // out[b] drained
    if (e == cudaSuccess)
      e = kway_merge(dtype, wruns.data(), wlens.data(), int(k), out[b], kway_temp, kway_bytes, c.compute, &c.recorder);
    if (e == cudaSuccess) e = cudaEventRecord(merge_done.ev[b], c.compute);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c.d2h, merge_done.ev[b], 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h + wi * W * w, out[b], pos * w, cudaMemcpyDeviceToHost, c.d2h);
    if (e == cudaSuccess) e = cudaEventRecord(d2h_done.ev[b], c.d2h);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.d2h);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.compute);
  if (times) times->merge_s = seconds_since(tb);
  return e;
}

}  // namespace mgs
