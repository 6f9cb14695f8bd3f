// Internal helpers of the C++ drop-in headers: the ABI status -> exception
// mapping, and a move-only device buffer over fem_b200_malloc/free.  Every
// computation of the drop-in runs on the GPU through libfem_b200.
#pragma once
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../fem_b200.h"

namespace fem::detail {

// FEM_B200_ERROR_ARGUMENT -> std::invalid_argument, anything else ->
// std::runtime_error: the reference's exception split.
inline void check(int rc) {
  if (rc == FEM_B200_SUCCESS) return;
  const std::string msg = fem_b200_last_error();
  if (rc == FEM_B200_ERROR_ARGUMENT) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

template <class T>
class DevBuffer {
 public:
  DevBuffer() = default;
  explicit DevBuffer(std::size_t n) { resize(n); }
  explicit DevBuffer(const std::vector<T>& host) { upload(host); }
  ~DevBuffer() { reset(); }
  DevBuffer(const DevBuffer&) = delete;
  DevBuffer& operator=(const DevBuffer&) = delete;
  DevBuffer(DevBuffer&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr, o.n_ = 0; }
  DevBuffer& operator=(DevBuffer&& o) noexcept {
    if (this != &o) {
      reset();
      p_ = o.p_, n_ = o.n_;
      o.p_ = nullptr, o.n_ = 0;
    }
    return *this;
  }
  void resize(std::size_t n) {
    if (n == n_) return;
    reset();
    void* p = nullptr;
    check(fem_b200_malloc(&p, n * sizeof(T)));
    p_ = static_cast<T*>(p), n_ = n;
  }
  void upload(const T* host, std::size_t n) {
    resize(n);
    if (n) check(fem_b200_memcpy(p_, host, n * sizeof(T), 0, nullptr));
  }
  void upload(const std::vector<T>& host) { upload(host.data(), host.size()); }
  void download(T* host, std::size_t n) const {
    if (n) check(fem_b200_memcpy(host, p_, n * sizeof(T), 1, nullptr));
  }
  void zero() {
    if (n_) check(fem_b200_memset_zero(p_, n_ * sizeof(T), nullptr));
  }
  T* get() const { return p_; }
  std::size_t size() const { return n_; }

 private:
  void reset() noexcept {
    if (p_) (void)fem_b200_free(p_);
    p_ = nullptr, n_ = 0;
  }
  T* p_ = nullptr;
  std::size_t n_ = 0;
};

inline int64_t int_pow(int64_t b, int e) {
  int64_t r = 1;
  for (int i = 0; i < e; ++i) r *= b;
  return r;
}

}  // namespace fem::detail
