// ORACLE — test infrastructure only. Not part of the product.
//
// C entry points around the reference's own code (hpides/multi-gpu-sorting),
// compiled from the reference's headers where they lie (see oracle/Makefile)
// into oracle/_ref/libref.so. Each function calls the reference's code path
// unchanged:
//   ref_generate          DataGenerator::ComputeDistribution<T>   src/data_generator.cuh:18-36
//   ref_tanasic_sort      SetupTanasicSort + TanasicSort<T>        src/tanasic_sort.cuh:206-299
//   ref_gowanlock_sort    SetupGowanlockSort + GowanlockSort<T>    src/gowanlock_sort.cuh:117-125,395-483
//   ref_gnu_parallel_sort the "gnu_parallel" algorithm branch      src/sort_benchmark.cu:103-108
//   ref_multiway_merge    __gnu_parallel::multiway_merge call      src/local_cpu_multiway_merge_benchmark.cu:70-71
//   ref_cub_sort_device_ms cub::DeviceRadixSort::SortKeys on device keys, the
//                          library call the reference times in
//                          src/local_gpu_sort_algorithm_benchmark.cu:51-67 (CUDA events)
//   ref_phase_seconds     TimeDurations phase                       src/time_durations.cuh
//   ref_cub_sort_range    cub::DeviceRadixSort with begin_bit / end_bit, ascending
//                         or descending, keys or pairs
//   ref_thrust_sort_by_key thrust::sort_by_key on device keys and 4- or 8-byte
//                          values: the library the reference sorts with
//                          (src/tanasic_sort.cuh:264), in its key-value form
#include <omp.h>

#include <cub/cub.cuh>
#include <thrust/execution_policy.h>
#include <thrust/sort.h>

#include <cstdint>
#include <cstdio>
#include <exception>
#include <cstring>
#include <parallel/algorithm>
#include <string>
#include <utility>
#include <vector>

#include "data_generator.cuh"
#include "gowanlock_sort.cuh"
#include "host_vector.cuh"
#include "tanasic_sort.cuh"
#include "time_durations.cuh"

namespace {

template <typename Fn>
int dispatch(int dtype, Fn&& fn) {
  switch (dtype) {
    case 0: fn(uint32_t{}); return 0;
    case 1: fn(int{}); return 0;
    case 2: fn(float{}); return 0;
    case 3: fn(uint64_t{}); return 0;
    case 4: fn(long{}); return 0;
    case 5: fn(double{}); return 0;
    default: return 1;
  }
}

// Runs one wrapper body: clears the runtime's last error first (the reference
// ignores CUDA errors in release builds, src/cuda_error.cuh:5-10, so a failed
// call inside it can leave a non-sticky error that thrust would later report as
// its own), turns C++ exceptions (thrust::system_error, std::bad_alloc) into a
// return code with the message on stderr instead of terminating the process,
// and clears what the body itself left behind.
template <typename R, typename F>
R guarded(R on_error, F&& body) {
  cudaGetLastError();
  try {
    R r = body();
    cudaGetLastError();
    return r;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "libref: %s\n", e.what());
  } catch (...) {
    std::fprintf(stderr, "libref: unknown exception\n");
  }
  cudaGetLastError();
  return on_error;
}

}  // namespace

extern "C" {

int ref_generate(int dtype, const char* distribution, uint32_t seed, void* out, size_t n) {
  return dispatch(dtype, [&](auto tag) {
    using T = decltype(tag);
    DataGenerator generator(seed);
    // Value-initialised like the benchmark's HostVector input (src/sort_benchmark.cu:280); a plain
    // vector so that generation needs no CUDA driver.
    std::vector<T> elements(n);
    if (n > 0) generator.ComputeDistribution<T>(elements.data(), elements.size(), distribution);
    if (n > 0) std::memcpy(out, elements.data(), n * sizeof(T));
  });
}

int ref_tanasic_sort(int dtype, void* keys, size_t n, int device) {
  return guarded(9, [&] { return dispatch(dtype, [&](auto tag) {
    using T = decltype(tag);
    std::vector<int> gpus{device};
    HostVector<T> elements(static_cast<T*>(keys), static_cast<T*>(keys) + n);
    SetupTanasicSort(gpus);
    TanasicSort<T>(&elements, gpus);
    if (n > 0) std::memcpy(keys, thrust::raw_pointer_cast(elements.data()), n * sizeof(T));
  }); });
}

int ref_gowanlock_sort(int dtype, void* keys, size_t n, size_t chunk_size, size_t merge_group_size,
                       size_t num_buffers, int device, int num_threads) {
  return guarded(9, [&] { return dispatch(dtype, [&](auto tag) {
    using T = decltype(tag);
    std::vector<int> gpus{device};
    HostVector<T> elements(static_cast<T*>(keys), static_cast<T*>(keys) + n);
    SetupGowanlockSort(gpus, num_threads);
    GowanlockSort<T>(&elements, chunk_size, merge_group_size, num_buffers, gpus);
    if (n > 0) std::memcpy(keys, thrust::raw_pointer_cast(elements.data()), n * sizeof(T));
  }); });
}

int ref_gnu_parallel_sort(int dtype, void* keys, size_t n, int num_threads) {
  return dispatch(dtype, [&](auto tag) {
    using T = decltype(tag);
    T* p = static_cast<T*>(keys);
    omp_set_num_threads(num_threads);
    TimeDurations::Get()->Tic("sort_phase");
    __gnu_parallel::sort(p, p + n);
    TimeDurations::Get()->Toc("sort_phase");
  });
}

int ref_multiway_merge(int dtype, const void* const* runs, const size_t* lens, int k, void* out, int num_threads) {
  return dispatch(dtype, [&](auto tag) {
    using T = decltype(tag);
    omp_set_num_threads(num_threads);
    std::vector<std::pair<T*, T*>> iterator_pairs;
    size_t total = 0;
    for (int i = 0; i < k; ++i) {
      T* b = const_cast<T*>(static_cast<const T*>(runs[i]));
      iterator_pairs.emplace_back(b, b + lens[i]);
      total += lens[i];
    }
    TimeDurations::Get()->Tic("merge_phase");
    __gnu_parallel::multiway_merge(iterator_pairs.begin(), iterator_pairs.end(), static_cast<T*>(out), total,
                                   std::less<T>());
    TimeDurations::Get()->Toc("merge_phase");
  });
}

// Sorts d_keys[0..n) (device) with cub::DeviceRadixSort::SortKeys, in place as the reference's
// benchmark does (same pointer for input and output), and returns the CUDA-event time in ms of
// the sort alone. d_temp must hold the bytes CUB asks for; temp_bytes 0 = query them (returned
// through *need).
// cub::DeviceRadixSort::SortKeys[Descending] / SortPairs[Descending] with begin_bit / end_bit, in place
// on device buffers (value_bytes 0 = keys only). Allocates its own output and scratch buffers.
int ref_cub_sort_range(int dtype, void* d_keys, void* d_values, size_t value_bytes, size_t n, int begin_bit,
                       int end_bit, int descending) {
  if (value_bytes != 0 && value_bytes != 4 && value_bytes != 8) return 1;
  return guarded(9, [&] {
  int rc = 0;
  dispatch(dtype, [&](auto tag) {
    using T = decltype(tag);
    T* k = static_cast<T*>(d_keys);
    T* k_out = nullptr;
    void* v_out = nullptr;
    void* temp = nullptr;
    size_t bytes = 0;
    if (cudaMalloc(&k_out, n * sizeof(T) + 16) != cudaSuccess) {
      rc = 2;
      return;
    }
    if (value_bytes) cudaMalloc(&v_out, n * value_bytes + 16);
    auto run = [&](auto* v_in, auto* v_o) {
      for (int pass = 0; pass < 2; ++pass) {  // size query, then the sort
        if (value_bytes == 0) {
          if (descending)
            cub::DeviceRadixSort::SortKeysDescending(temp, bytes, k, k_out, n, begin_bit, end_bit);
          else
            cub::DeviceRadixSort::SortKeys(temp, bytes, k, k_out, n, begin_bit, end_bit);
        } else {
          if (descending)
            cub::DeviceRadixSort::SortPairsDescending(temp, bytes, k, k_out, v_in, v_o, n, begin_bit, end_bit);
          else
            cub::DeviceRadixSort::SortPairs(temp, bytes, k, k_out, v_in, v_o, n, begin_bit, end_bit);
        }
        if (pass == 0 && cudaMalloc(&temp, bytes + 16) != cudaSuccess) {
          rc = 3;
          return;
        }
      }
    };
    if (value_bytes == 8) {
      run(static_cast<uint64_t*>(d_values), static_cast<uint64_t*>(v_out));
    } else {
      run(static_cast<uint32_t*>(d_values), static_cast<uint32_t*>(v_out));
    }
    if (rc == 0 && cudaDeviceSynchronize() != cudaSuccess) rc = 4;
    if (rc == 0) cudaMemcpy(d_keys, k_out, n * sizeof(T), cudaMemcpyDeviceToDevice);
    if (rc == 0 && value_bytes) cudaMemcpy(d_values, v_out, n * value_bytes, cudaMemcpyDeviceToDevice);
    cudaFree(k_out);
    if (v_out) cudaFree(v_out);
    if (temp) cudaFree(temp);
  });
  return rc;
  });
}

int ref_thrust_sort_by_key(int dtype, void* d_keys, void* d_values, size_t value_bytes, size_t n) {
  if (value_bytes != 4 && value_bytes != 8) return 1;
  return guarded(9, [&] {
  int rc = 0;
  dispatch(dtype, [&](auto tag) {
    using T = decltype(tag);
    T* k = static_cast<T*>(d_keys);
    if (value_bytes == 4) {
      uint32_t* v = static_cast<uint32_t*>(d_values);
      thrust::sort_by_key(thrust::device, k, k + n, v);
    } else {
      uint64_t* v = static_cast<uint64_t*>(d_values);
      thrust::sort_by_key(thrust::device, k, k + n, v);
    }
    rc = cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
  });
  return rc;
  });
}

// Out of place, as CUB requires (its key ranges must not overlap): d_keys_in is
// read, d_keys_out receives the sorted keys.
double ref_cub_sort_device_ms(int dtype, const void* d_keys_in, void* d_keys_out, size_t n, void* d_temp,
                              size_t temp_bytes, size_t* need) {
  return guarded(-2.0, [&] {
  double ms = -1.0;
  dispatch(dtype, [&](auto tag) {
    using T = decltype(tag);
    const T* in = static_cast<const T*>(d_keys_in);
    T* out = static_cast<T*>(d_keys_out);
    size_t bytes = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, bytes, in, out, n, 0, int(sizeof(T) * 8));
    if (need) *need = bytes;
    if (temp_bytes < bytes || d_temp == nullptr || in == nullptr || out == nullptr) return;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a);
    cub::DeviceRadixSort::SortKeys(d_temp, bytes, in, out, n, 0, int(sizeof(T) * 8));
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    ms = t;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  });
  return ms;
  });
}

double ref_phase_seconds(const char* phase) { return TimeDurations::Get()->durations[phase].count(); }

int ref_num_procs(void) { return omp_get_num_procs(); }

}  // extern "C"
