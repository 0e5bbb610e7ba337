#include "context.h"

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>

namespace mgs {

namespace {
thread_local std::string g_last_error;
std::atomic<int> g_failing_reservations{0};  // arena growths still to fail (test hook)
}

void fail_next_arena_reservations(int count) { g_failing_reservations.store(count > 0 ? count : 0); }

void set_last_error(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}
void clear_last_error() { g_last_error.clear(); }
const char* last_error() { return g_last_error.c_str(); }

EventRecorder::~EventRecorder() {
  for (auto& p : pending_) {
    cudaEventDestroy(p.start);
    cudaEventDestroy(p.stop);
  }
  for (auto e : free_events_) cudaEventDestroy(e);
  if (open_start_) cudaEventDestroy(open_start_);
}

cudaEvent_t EventRecorder::take_event() {
  if (!free_events_.empty()) {
    cudaEvent_t e = free_events_.back();
    free_events_.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

void EventRecorder::before(const char* name, cudaStream_t stream) {
  (void)name;
  ++launches_;
  if (!enabled_) return;
  open_start_ = take_event();
  cudaEventRecord(open_start_, stream);
}

void EventRecorder::after(const char* name, cudaStream_t stream) {
  if (!enabled_ || open_start_ == nullptr) return;
  cudaEvent_t stop = take_event();
  cudaEventRecord(stop, stream);
  pending_.push_back({name, open_start_, stop});
  open_start_ = nullptr;
}

cudaError_t EventRecorder::collect(std::vector<std::pair<std::string, std::pair<uint64_t, double>>>* out) {
  std::map<std::string, std::pair<uint64_t, double>> agg;
  cudaError_t first = cudaSuccess;
  for (auto& p : pending_) {
    cudaError_t e = cudaEventSynchronize(p.stop);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, p.start, p.stop);
    if (e != cudaSuccess && first == cudaSuccess) first = e;
    auto& a = agg[p.name];
    a.first += 1;
    a.second += ms;
    free_events_.push_back(p.start);
    free_events_.push_back(p.stop);
  }
  pending_.clear();
  out->assign(agg.begin(), agg.end());
  return first;
}

cudaError_t Context::reserve(size_t bytes) {
  if (bytes <= arena_bytes) return cudaSuccess;
  for (int left = g_failing_reservations.load(); left > 0;) {
    if (g_failing_reservations.compare_exchange_weak(left, left - 1)) return cudaErrorMemoryAllocation;
  }
  const auto t0 = std::chrono::steady_clock::now();
  struct Timed {
    double& acc;
    std::chrono::steady_clock::time_point t0;
    ~Timed() { acc += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
  } timed{reserve_s, t0};
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return e;
  if (arena) cudaFree(arena);
  arena = nullptr;
  arena_bytes = 0;
  // Grow with headroom so that a sequence of slightly larger requests does not
  // reallocate every time.
  const size_t want = bytes + bytes / 16;
  e = cudaMalloc(&arena, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    e = cudaMalloc(&arena, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      arena = nullptr;
      return cudaErrorMemoryAllocation;
    }
    arena_bytes = bytes;
    return cudaSuccess;
  }
  arena_bytes = want;
  return cudaSuccess;
}

cudaError_t Context::reserve_host(size_t bytes) {
  if (bytes <= host_arena_bytes) return cudaSuccess;
  if (host_arena) cudaFreeHost(host_arena);
  host_arena = nullptr;
  host_arena_bytes = 0;
  cudaError_t e = cudaHostAlloc(&host_arena, bytes, cudaHostAllocDefault);
  if (e != cudaSuccess) {
    cudaGetLastError();
    host_arena = nullptr;
    return cudaErrorMemoryAllocation;
  }
  host_arena_bytes = bytes;
  return cudaSuccess;
}

cudaError_t Context::take_status(cudaStream_t stream, uint32_t* status) {
  cudaError_t e = cudaMemcpyAsync(h_status, d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return e;
  *status = *h_status;
  if (*status != 0) {
    e = cudaMemsetAsync(d_status, 0, sizeof(uint32_t), stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  }
  return e;
}

}  // namespace mgs
