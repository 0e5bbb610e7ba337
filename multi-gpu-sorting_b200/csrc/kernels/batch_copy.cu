// Gather / scatter kernels of the serving loop's coalesced batches. One CTA
// per request (grid-stride over requests); each CTA streams its request's keys
// with plain coalesced loads and stores, inverting the top bit when the
// request holds signed keys that share a batch with unsigned ones.
#include "batch_copy.cuh"

#include <algorithm>

#include "launch.cuh"

namespace mgs {
namespace {

constexpr int kCopyBlock = 256;

template <typename T, bool IN>
__global__ __launch_bounds__(kCopyBlock) void batch_stage_kernel(T* __restrict__ staging,
                                                                 const BatchEntry* __restrict__ entries,
                                                                 uint32_t count) {
  constexpr T kTop = T(1) << (sizeof(T) * 8 - 1);
  for (uint32_t e = blockIdx.x; e < count; e += gridDim.x) {
    const BatchEntry en = entries[e];
    const T flip = en.flip ? kTop : T(0);
    T* stage = staging + en.offset;
    T* dev = static_cast<T*>(en.device);
    if (dev == nullptr) {
      if (flip == T(0)) continue;  // a host entry without a transform: nothing to do on the device
      for (uint64_t i = threadIdx.x; i < en.n; i += kCopyBlock) stage[i] ^= flip;
    } else if (IN) {
      for (uint64_t i = threadIdx.x; i < en.n; i += kCopyBlock) stage[i] = dev[i] ^ flip;
    } else {
      for (uint64_t i = threadIdx.x; i < en.n; i += kCopyBlock) dev[i] = stage[i] ^ flip;
    }
  }
}

template <bool IN>
cudaError_t stage(void* staging, const BatchEntry* entries, uint32_t count, int key_bytes, cudaStream_t stream,
                  LaunchRecorder* rec) {
  const dim3 grid(std::min<unsigned>(count, 1024u));
  const char* name = IN ? "batch_stage_in" : "batch_stage_out";
  if (key_bytes == 4)
    return launch_kernel(rec, name, batch_stage_kernel<uint32_t, IN>, grid, dim3(kCopyBlock), 0, stream,
                         static_cast<uint32_t*>(staging), entries, count);
  if (key_bytes == 8)
    return launch_kernel(rec, name, batch_stage_kernel<unsigned long long, IN>, grid, dim3(kCopyBlock), 0, stream,
                         static_cast<unsigned long long*>(staging), entries, count);
  return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t batch_stage_in(void* staging, const BatchEntry* entries, uint32_t count, int key_bytes,
                           cudaStream_t stream, LaunchRecorder* rec) {
  return stage<true>(staging, entries, count, key_bytes, stream, rec);
}

cudaError_t batch_stage_out(void* staging, const BatchEntry* entries, uint32_t count, int key_bytes,
                            cudaStream_t stream, LaunchRecorder* rec) {
  return stage<false>(staging, entries, count, key_bytes, stream, rec);
}

}  // namespace mgs
