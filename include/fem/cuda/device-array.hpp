// fem::cuda::DeviceArray (drop-in for the reference's
// include/cuda/device-array.hpp): a move-only owner of a device allocation
// with explicit, synchronous host <-> device copies, over libfem_b200's
// memory entry points.  Failures throw std::runtime_error.
#pragma once
#include <cstddef>
#include <stdexcept>
#include <type_traits>
#include <vector>

#include "../fem-b200-detail.hpp"

namespace fem::cuda {

template <class T>
class DeviceArray {
  static_assert(std::is_trivially_copyable_v<T>, "DeviceArray elements are copied as raw bytes");

 public:
  DeviceArray() = default;
  explicit DeviceArray(std::size_t n) { allocate(n); }
  explicit DeviceArray(const std::vector<T>& host) : DeviceArray(host.size()) { copy_from_host(host); }
  ~DeviceArray() { release(); }

  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  DeviceArray(DeviceArray&& other) noexcept : data_(other.data_), size_(other.size_) {
    other.data_ = nullptr;
    other.size_ = 0;
  }
  DeviceArray& operator=(DeviceArray&& other) noexcept {
    if (this != &other) {
      release();
      data_ = other.data_, size_ = other.size_;
      other.data_ = nullptr, other.size_ = 0;
    }
    return *this;
  }

  T* data() { return data_; }
  const T* data() const { return data_; }
  std::size_t size() const { return size_; }
  std::size_t bytes() const { return size_ * sizeof(T); }
  bool empty() const { return size_ == 0; }

  // New allocation of n entries (contents not kept); no-op for the same size.
  void resize(std::size_t n) {
    if (n == size_) return;
    release();
    allocate(n);
  }
  void zero() {
    if (size_) fem::detail::check(fem_b200_memset_zero(data_, bytes(), nullptr));
  }
  void copy_from_host(const std::vector<T>& host) {
    if (host.size() != size_) throw std::invalid_argument("DeviceArray::copy_from_host: size mismatch");
    if (size_) fem::detail::check(fem_b200_memcpy(data_, host.data(), bytes(), 0, nullptr));
  }
  void copy_to_host(std::vector<T>& host) const {
    host.resize(size_);
    if (size_) fem::detail::check(fem_b200_memcpy(host.data(), data_, bytes(), 1, nullptr));
  }
  std::vector<T> to_host() const {
    std::vector<T> host;
    copy_to_host(host);
    return host;
  }

 private:
  void allocate(std::size_t n) {
    if (n == 0) return;
    void* p = nullptr;
    fem::detail::check(fem_b200_malloc(&p, n * sizeof(T)));
    data_ = static_cast<T*>(p);
    size_ = n;
  }
  void release() noexcept {
    if (data_) (void)fem_b200_free(data_);
    data_ = nullptr;
    size_ = 0;
  }
  T* data_ = nullptr;
  std::size_t size_ = 0;
};

}  // namespace fem::cuda
