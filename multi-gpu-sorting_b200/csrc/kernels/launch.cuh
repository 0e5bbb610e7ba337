// Kernel launch helper: every launch of the engine goes through launch_kernel so
// that the context can count launches and, when profiling is on, bracket each
// launch with CUDA events on its stream.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <utility>

namespace mgs {

class LaunchRecorder {
 public:
  virtual ~LaunchRecorder() = default;
  virtual void before(const char* name, cudaStream_t stream) = 0;
  virtual void after(const char* name, cudaStream_t stream) = 0;
};

// Dynamic shared memory above 48 KB needs a per-kernel attribute, and the
// attribute belongs to the device's context: ensure() raises it once for each
// device (ordinals 0..63; others set it on every call) that launches the kernel.
class SmemLimitOnce {
 public:
  template <typename... KArgs>
  cudaError_t ensure(void (*kernel)(KArgs...), size_t bytes) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t bit = (dev >= 0 && dev < 64) ? (uint64_t(1) << dev) : 0;
    if (bit && (done_.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
    if (e == cudaSuccess && bit) done_.fetch_or(bit, std::memory_order_acq_rel);
    return e;
  }

 private:
  std::atomic<uint64_t> done_{0};
};

#ifdef __CUDACC__
template <typename... KArgs, typename... Args>
inline cudaError_t launch_kernel(LaunchRecorder* rec, const char* name, void (*kernel)(KArgs...), dim3 grid,
                                 dim3 block, size_t smem, cudaStream_t stream, Args&&... args) {
  if (grid.x == 0 || grid.y == 0 || grid.z == 0) return cudaSuccess;
  if (rec) rec->before(name, stream);
  kernel<<<grid, block, smem, stream>>>(std::forward<Args>(args)...);
  cudaError_t err = cudaGetLastError();
  if (rec) rec->after(name, stream);
  return err;
}
#endif

}  // namespace mgs
