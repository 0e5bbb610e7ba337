// Kernel launch helper: every launch of the engine goes through launch_kernel so
// that the context can count launches and, when profiling is on, bracket each
// launch with CUDA events on its stream.
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace mgs {

class LaunchRecorder {
 public:
  virtual ~LaunchRecorder() = default;
  virtual void before(const char* name, cudaStream_t stream) = 0;
  virtual void after(const char* name, cudaStream_t stream) = 0;
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
