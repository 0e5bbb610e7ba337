// Shared runtime of the C++ compat headers: one engine context per device,
// created on first use and destroyed at exit, and the error convention.
//
// The reference's CheckCudaError (src/cuda_error.cuh:5-17) ignores errors in
// release builds and, with -DDEBUG, prints "Error: <message> <file> <line>" and
// exits with the error code. The compat layer always checks: a failing engine
// call prints "Error: <message>" and exits with the engine status.
#pragma once

#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>

#include "mgs.h"

namespace mgs_compat {

inline void check(int status, const char* what) {
  if (status != MGS_OK) {
    std::printf("Error: %s: %s\n", what, mgs_last_error_string());
    std::exit(status);
  }
}

class Contexts {
 public:
  static mgs_ctx* get(int device) {
    static Contexts instance;
    std::lock_guard<std::mutex> lock(instance.mutex_);
    auto it = instance.ctx_.find(device);
    if (it != instance.ctx_.end()) return it->second;
    mgs_ctx* c = nullptr;
    check(mgs_ctx_create(device, 0, &c), "mgs_ctx_create");
    instance.ctx_[device] = c;
    return c;
  }
  ~Contexts() {
    for (auto& kv : ctx_) mgs_ctx_destroy(kv.second);
  }

 private:
  std::mutex mutex_;
  std::map<int, mgs_ctx*> ctx_;
};

template <typename T>
struct DType;
template <>
struct DType<unsigned> { static constexpr int value = MGS_U32; };
template <>
struct DType<int> { static constexpr int value = MGS_I32; };
template <>
struct DType<float> { static constexpr int value = MGS_F32; };
template <>
struct DType<unsigned long> { static constexpr int value = MGS_U64; };
template <>
struct DType<long> { static constexpr int value = MGS_I64; };
template <>
struct DType<double> { static constexpr int value = MGS_F64; };

}  // namespace mgs_compat
