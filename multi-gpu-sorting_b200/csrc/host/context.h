// Engine context: one per device. Owns the streams, a grow-only device arena,
// the device status word and the launch recorder (launch counting and optional
// per-kernel CUDA-event timing).
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../kernels/launch.cuh"

namespace mgs {

// Failure injection for tests: the next `count` growths of any context's
// device arena fail as if cudaMalloc had run out of memory.
void fail_next_arena_reservations(int count);

// Thread-local last error message of the C ABI.
void set_last_error(const char* fmt, ...);
void clear_last_error();
const char* last_error();

class EventRecorder : public LaunchRecorder {
 public:
  ~EventRecorder() override;
  void before(const char* name, cudaStream_t stream) override;
  void after(const char* name, cudaStream_t stream) override;
  void set_enabled(bool on) { enabled_ = on; }
  bool enabled() const { return enabled_; }
  uint64_t launches() const { return launches_; }
  void reset_launches() { launches_ = 0; }
  void add_launches(uint64_t n) { launches_ += n; }  // launches replayed from a recorded plan
  // Synchronizes on the recorded events and folds them into per-name totals.
  cudaError_t collect(std::vector<std::pair<std::string, std::pair<uint64_t, double>>>* out);

 private:
  cudaEvent_t take_event();
  struct Pending {
    std::string name;
    cudaEvent_t start, stop;
  };
  bool enabled_ = false;
  uint64_t launches_ = 0;
  std::vector<cudaEvent_t> free_events_;
  std::vector<Pending> pending_;
  cudaEvent_t open_start_ = nullptr;
};

struct Context {
  int device = 0;
  int sm_count = 148;
  cudaStream_t compute = nullptr;  // kernels
  cudaStream_t h2d = nullptr;      // host->device copy engine stream
  cudaStream_t d2h = nullptr;      // device->host copy engine stream
  void* arena = nullptr;
  size_t arena_bytes = 0;
  uint32_t* d_status = nullptr;  // device status word (DeviceStatus bits)
  uint32_t* h_status = nullptr;  // pinned mirror used by status reads
  uint64_t* h_status64 = nullptr;  // pinned 8-byte word (pivot readback), inside the h_status block
  EventRecorder recorder;
  void* host_arena = nullptr;  // grow-only pinned host buffer (out-of-core sorted runs)
  size_t host_arena_bytes = 0;
  double phase_s[4] = {0, 0, 0, 0};  // last call's memory_allocation, sort_phase, merge_phase, memory_deallocation
  double reserve_s = 0;              // seconds spent growing the arena since the counter was last reset

  // Ensures the pinned host arena holds at least `bytes`.
  cudaError_t reserve_host(size_t bytes);

  // Ensures the arena holds at least `bytes` (synchronizes before growing).
  cudaError_t reserve(size_t bytes);
  // Reads and clears the device status word on `stream` (synchronizes it).
  cudaError_t take_status(cudaStream_t stream, uint32_t* status);
};

}  // namespace mgs

struct mgs_ctx {
  mgs::Context impl;
};
