// ORACLE build shim — test infrastructure only.
// thrust 2.8.2 (CUDA 12.9) no longer ships the experimental pinned_allocator
// that the reference's HostVector alias names (src/host_vector.cuh:4-7). This
// header provides the same name as a pinned-host-memory allocator so that the
// reference's headers compile unchanged for the oracle.
#pragma once
#include <thrust/mr/allocator.h>
#include <thrust/system/cuda/memory_resource.h>

namespace thrust {
namespace system {
namespace cuda {
namespace experimental {
template <typename T>
using pinned_allocator =
    thrust::mr::stateless_resource_allocator<T, thrust::system::cuda::universal_host_pinned_memory_resource>;
}  // namespace experimental
}  // namespace cuda
}  // namespace system
}  // namespace thrust
