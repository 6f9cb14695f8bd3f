// Shared host-side plumbing of libfem_b200: status codes, the thread-local
// error message, CUDA error checks, and the try/catch shell every C entry
// point runs in.
#pragma once
#include <cuda_runtime_api.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "fem_b200.h"

namespace fem_b200 {

// Argument errors (the reference throws std::invalid_argument).
struct arg_error : std::invalid_argument {
  using std::invalid_argument::invalid_argument;
};
// A configuration the device path does not implement (no CPU fallback).
struct unsupported_error : std::runtime_error {
  using std::runtime_error::runtime_error;
};
// A failed CUDA runtime call or kernel status.
struct cuda_error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void set_last_error(const std::string& msg);

// Throws cuda_error with file:line and clears the (non-sticky) error, so the
// next check does not blame the wrong call (the reference's CUDA_CHECK
// semantics, include/cuda/cuda-check.hpp:17-32).
inline void cuda_check(cudaError_t err, const char* expr, const char* file, int line) {
  if (err == cudaSuccess) return;
  (void)cudaGetLastError();
  throw cuda_error(std::string(file) + ":" + std::to_string(line) + ": " + expr + " failed: " +
                   cudaGetErrorName(err) + " (" + cudaGetErrorString(err) + ")");
}

template <class F>
int guarded(F&& f) {
  try {
    f();
    return FEM_B200_SUCCESS;
  } catch (const arg_error& e) {
    set_last_error(e.what());
    return FEM_B200_ERROR_ARGUMENT;
  } catch (const std::invalid_argument& e) {
    set_last_error(e.what());
    return FEM_B200_ERROR_ARGUMENT;
  } catch (const unsupported_error& e) {
    set_last_error(e.what());
    return FEM_B200_ERROR_UNSUPPORTED;
  } catch (const cuda_error& e) {
    set_last_error(e.what());
    return FEM_B200_ERROR_CUDA;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return FEM_B200_ERROR_CUDA;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return FEM_B200_ERROR_CUDA;
  }
}

inline void require(bool ok, const std::string& msg) {
  if (!ok) throw arg_error(msg);
}

inline int64_t ipow(int64_t b, int e) {
  int64_t r = 1;
  for (int i = 0; i < e; ++i) r *= b;
  return r;
}

}  // namespace fem_b200

#define FEM_CUDA_CHECK(expr) ::fem_b200::cuda_check((expr), #expr, __FILE__, __LINE__)
