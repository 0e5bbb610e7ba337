// Device input generator: the distributions of the host generator
// (csrc/host/data_generator.cpp: the reference's DataGenerator,
// src/data_generator.cuh:18-211, plus the engine's workload distributions)
// produced in device memory, byte for byte the same as the host produces them.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <string>

#include "launch.cuh"

namespace mgs {

// Bytes of device scratch generate_device needs. Returns false, with the
// reason in *why, for a distribution that is unknown for the dtype or that the
// device does not reproduce bit for bit ("normal", "nearly-sorted" and
// "normal0" take the host C library's log / cos).
bool generate_device_temp_bytes(int dtype, const char* distribution, size_t n, size_t* bytes, std::string* why);

// Fills d_out[0..n) on `stream` with the bytes mgs_generate writes for the same
// (dtype, distribution, seed, n). Entries the host generator leaves untouched
// (staggered and bucket-sorted with n < 10) are left untouched here too.
// Synchronizes `stream` before returning (host tables are uploaded from
// pageable memory).
cudaError_t generate_device(int dtype, const char* distribution, uint32_t seed, void* d_out, size_t n, void* d_temp,
                            size_t temp_bytes, cudaStream_t stream, uint32_t* d_status, LaunchRecorder* rec);

}  // namespace mgs
