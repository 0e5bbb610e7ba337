// Autotuner and tuning files for the onesweep variant table (tile shape x
// ranking mode per key width and size class, radix_sort.cuh).
//
// Tuning file: text, one entry per line, '#' starts a comment:
//   <key_bytes 4|8> <size_class 0..5> <shape 0..6> <rank_mode 2|3>
// The library reads MGS_TUNE_FILE if that variable is set, else
// tuning/b200.tune beside the directory of libmgs.so, on the first sort.
#include <dlfcn.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "engine_types.h"
#include "radix_sort.cuh"

namespace mgs {
namespace {

// Uniformly random keys: splitmix64 (Steele, Lea, Flood, "Fast splittable
// pseudorandom number generators", 2014) of seed + index, truncated to 32 bits
// for 4-byte keys.
__global__ void fill_random_kernel(void* out, size_t n, int key_bytes, unsigned long long seed) {
  const size_t stride = size_t(gridDim.x) * blockDim.x;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    unsigned long long z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    if (key_bytes == 8) {
      static_cast<unsigned long long*>(out)[i] = z;
    } else {
      static_cast<uint32_t*>(out)[i] = uint32_t(z);
    }
  }
}

struct DeviceBuffers {
  void* keys = nullptr;
  void* pristine = nullptr;
  void* temp = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t start = nullptr, stop = nullptr;
  ~DeviceBuffers() {
    if (stream) cudaStreamSynchronize(stream);
    if (keys) cudaFree(keys);
    if (pristine) cudaFree(pristine);
    if (temp) cudaFree(temp);
    if (start) cudaEventDestroy(start);
    if (stop) cudaEventDestroy(stop);
    if (stream) cudaStreamDestroy(stream);
  }
};

}  // namespace

cudaError_t autotune(int dtype, size_t max_n, int reps, std::vector<TuneSample>* out) {
  const size_t w = dtype_bytes(dtype);
  if (w == 0 || reps < 1 || reps > 100) return cudaErrorInvalidValue;
  size_t nmax = 0;
  for (int c = 0; c < kSizeClasses; ++c)
    if (size_class_sample(c) <= max_n) nmax = std::max(nmax, size_class_sample(c));
  if (nmax == 0) return cudaSuccess;

  DeviceBuffers b;
  const size_t temp_bytes = radix_sort_temp_bytes(dtype, nmax);
  cudaError_t e = cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&b.start);
  if (e == cudaSuccess) e = cudaEventCreate(&b.stop);
  if (e == cudaSuccess) e = cudaMalloc(&b.keys, nmax * w);
  if (e == cudaSuccess) e = cudaMalloc(&b.pristine, nmax * w);
  if (e == cudaSuccess) e = cudaMalloc(&b.temp, temp_bytes);
  if (e != cudaSuccess) return e;
  fill_random_kernel<<<1184, 256, 0, b.stream>>>(b.pristine, nmax, int(w), 0x5EEDull);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;

  for (int c = 0; c < kSizeClasses; ++c) {
    const size_t n = size_class_sample(c);
    if (n > max_n) continue;
    SortVariant best{-1, -1};
    double best_ms = 1e30;
    const size_t first = out ? out->size() : 0;
    for (int mode = 2; mode <= 3; ++mode) {
      for (int shape = 0; shape < 7; ++shape) {
        const SortVariant v{shape, mode};
        if (!set_sort_variant(int(w), c, v)) continue;
        std::vector<float> t;
        for (int r = 0; r <= reps; ++r) {
          e = cudaMemcpyAsync(b.keys, b.pristine, n * w, cudaMemcpyDeviceToDevice, b.stream);
          if (e == cudaSuccess) e = cudaEventRecord(b.start, b.stream);
          if (e == cudaSuccess) e = radix_sort(dtype, b.keys, n, b.temp, temp_bytes, b.stream, nullptr, nullptr);
          if (e == cudaSuccess) e = cudaEventRecord(b.stop, b.stream);
          if (e == cudaSuccess) e = cudaEventSynchronize(b.stop);
          float ms = 0.f;
          if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, b.start, b.stop);
          if (e != cudaSuccess) return e;
          if (r > 0) t.push_back(ms);  // the first sort of a variant warms it up
        }
        std::nth_element(t.begin(), t.begin() + t.size() / 2, t.end());
        const double med = t[t.size() / 2];
        if (out) out->push_back(TuneSample{int(w), c, n, v, med, false});
        if (med < best_ms) {
          best_ms = med;
          best = v;
        }
      }
    }
    set_sort_variant(int(w), c, best);
    if (out)
      for (size_t i = first; i < out->size(); ++i)
        (*out)[i].chosen = ((*out)[i].variant.shape == best.shape && (*out)[i].variant.mode == best.mode);
  }
  return cudaStreamSynchronize(b.stream);
}

namespace {

int read_tuning_file(const char* path) {
  FILE* f = std::fopen(path, "r");
  if (!f) return -1;
  char line[256];
  int entries = 0, bad = 0;
  while (std::fgets(line, sizeof(line), f)) {
    if (char* hash = std::strchr(line, '#')) *hash = 0;
    int kb, c, shape, mode;
    char extra;
    const int got = std::sscanf(line, "%d %d %d %d %c", &kb, &c, &shape, &mode, &extra);
    if (got <= 0) continue;  // blank or comment line
    if (got == 4 && store_sort_variant(kb, c, SortVariant{shape, mode})) {
      ++entries;
    } else {
      ++bad;
    }
  }
  std::fclose(f);
  return bad ? -2 : entries;
}

}  // namespace

int load_tuning_file(const char* path) {
  ensure_default_tuning();
  return read_tuning_file(path);
}

bool save_tuning_file(const char* path) {
  FILE* f = std::fopen(path, "w");
  if (!f) return false;
  std::fprintf(f, "# mgs onesweep variants: key_bytes size_class shape rank_mode\n");
  std::fprintf(f, "# size classes: 0 n<2^16, 1 n<2^18, 2 n<2^20, 3 n<2^22, 4 n<2^26, 5 larger\n");
  for (int kb : {4, 8}) {
    for (int c = 0; c < kSizeClasses; ++c) {
      const SortVariant v = table_variant(kb, c);
      std::fprintf(f, "%d %d %d %d\n", kb, c, v.shape, v.mode);
    }
  }
  return std::fclose(f) == 0;
}

void load_default_tuning() {
  if (const char* env = std::getenv("MGS_TUNE_FILE")) {
    read_tuning_file(env);
    return;
  }
  Dl_info info;
  if (dladdr(reinterpret_cast<void*>(&load_default_tuning), &info) == 0 || info.dli_fname == nullptr) return;
  std::string dir(info.dli_fname);
  const size_t slash = dir.find_last_of('/');
  dir = (slash == std::string::npos) ? std::string(".") : dir.substr(0, slash);
  read_tuning_file((dir + "/../tuning/b200.tune").c_str());
}

}  // namespace mgs
