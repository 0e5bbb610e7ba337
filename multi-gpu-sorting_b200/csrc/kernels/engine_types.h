// Plain (host and device) definitions shared by the engine's C++ and CUDA code.
#pragma once

#include <stddef.h>
#include <stdint.h>

namespace mgs {

// Bytes per key of an mgs_dtype (u32, i32, f32 -> 4; u64, i64, f64 -> 8).
inline size_t dtype_bytes(int dtype) {
  return (dtype >= 0 && dtype <= 2) ? 4u : (dtype >= 3 && dtype <= 5) ? 8u : 0u;
}

// Device status bits (OR-ed into a status word that the host reads back).
enum DeviceStatus : uint32_t {
  kStatusLookbackTimeout = 1u,
  kStatusTmaTimeout = 2u,
  kStatusQueueTimeout = 4u,
  kStatusBadInput = 8u,
};

}  // namespace mgs
