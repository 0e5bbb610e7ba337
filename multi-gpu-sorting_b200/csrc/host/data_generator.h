// Host input generator (the reference's DataGenerator plus the engine's
// workload distributions) and the pieces of it that the device generator
// (csrc/kernels/generate.cu) reuses so that both produce the same bytes.
#pragma once

#include <stddef.h>
#include <stdint.h>

#include <vector>

namespace mgs {

// Fills out[0..n) on the host; false for an unknown distribution.
bool generate_keys(int dtype, const char* distribution, uint32_t seed, void* out, size_t n);

// Logical generator threads of the reference scheme (src/data_generator.cuh:210).
constexpr int kGeneratorThreads = 128;

// Index block [*begin, *end) of logical thread t when n iterations are split
// as OpenMP schedule(static) splits them over kGeneratorThreads threads.
void generator_static_block(size_t n, int t, size_t* begin, size_t* end);

// The 624 state words, before the first twist, of the std::mt19937 that the
// generator seeds with `seed` (seed sequence of src/data_generator.cuh:193-205).
bool mt19937_seed_state(uint32_t seed, uint32_t* state624);

// Zipf(kZipfExponent) over kZipfDistinct ranks: the normalised CDF and the key
// of every rank (key_bytes = dtype size bytes per rank, native layout).
constexpr double kZipfExponent = 1.1;
constexpr size_t kZipfDistinct = size_t(1) << 20;
bool zipf_tables(int dtype, uint32_t seed, std::vector<double>* cdf, std::vector<unsigned char>* values);

}  // namespace mgs
