// HostVector<T>: the reference's pinned host vector (src/host_vector.cuh:7, a
// thrust::host_vector with a pinned allocator), here a minimal vector over
// page-locked memory from mgs_host_alloc. Elements are value-initialised. On a
// machine without a CUDA device the memory is ordinary pageable memory, so
// that the CLI's CPU sorts still run; engine calls on such a machine fail.
#pragma once

#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <utility>

#include "mgs_runtime.h"

template <typename T>
class HostVector {
 public:
  using value_type = T;
  using iterator = T*;
  using const_iterator = const T*;

  HostVector() = default;
  explicit HostVector(size_t n) { resize(n); }
  HostVector(const HostVector&) = delete;
  HostVector& operator=(const HostVector&) = delete;
  HostVector(HostVector&& o) noexcept { swap(o); }
  HostVector& operator=(HostVector&& o) noexcept {
    swap(o);
    return *this;
  }
  ~HostVector() { release(); }

  void resize(size_t n) {
    if (n > capacity_) {
      void* p = nullptr;
      bool pinned = true;
      const int rc = mgs_host_alloc(n * sizeof(T), &p);
      if (rc != MGS_OK) {
        int devices = 0;
        if (mgs_device_count(&devices) == MGS_OK && devices > 0) mgs_compat::check(rc, "HostVector");
        p = std::malloc(n * sizeof(T));  // no CUDA device: pageable memory
        pinned = false;
        if (p == nullptr) mgs_compat::check(MGS_ERR_OOM, "HostVector");
      }
      if (data_) std::memcpy(p, data_, size_ * sizeof(T));
      release();
      data_ = static_cast<T*>(p);
      pinned_ = pinned;
      capacity_ = n;
    }
    for (size_t i = size_; i < n; ++i) data_[i] = T();
    size_ = n;
  }
  void clear() { size_ = 0; }
  void shrink_to_fit() {
    if (size_ == 0 && data_) {
      release();
      capacity_ = 0;
    }
  }
  size_t size() const { return size_; }
  bool empty() const { return size_ == 0; }
  T* data() { return data_; }
  const T* data() const { return data_; }
  T& operator[](size_t i) { return data_[i]; }
  const T& operator[](size_t i) const { return data_[i]; }
  T* begin() { return data_; }
  T* end() { return data_ + size_; }
  const T* begin() const { return data_; }
  const T* end() const { return data_ + size_; }

 private:
  void release() {
    if (data_) {
      if (pinned_) mgs_host_free(data_); else std::free(data_);
    }
    data_ = nullptr;
  }
  void swap(HostVector& o) {
    std::swap(data_, o.data_);
    std::swap(size_, o.size_);
    std::swap(capacity_, o.capacity_);
    std::swap(pinned_, o.pinned_);
  }
  T* data_ = nullptr;
  bool pinned_ = true;
  size_t size_ = 0;
  size_t capacity_ = 0;
};
