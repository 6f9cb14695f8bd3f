// CUDA_CHECK for code that calls the CUDA runtime itself (drop-in for the
// reference's include/cuda/cuda-check.hpp; needs cuda_runtime_api.h and the
// CUDA runtime at link time, unlike the rest of the drop-in headers).
#pragma once
#include <cuda_runtime_api.h>

#include <stdexcept>
#include <string>

namespace fem::cuda {

// Throws std::runtime_error naming the call and its file:line, after
// clearing the (non-sticky) error so the next check does not report it again.
inline void check(cudaError_t err, const char* expr, const char* file, int line) {
  if (err == cudaSuccess) return;
  (void)cudaGetLastError();
  throw std::runtime_error(std::string(file) + ":" + std::to_string(line) + ": " + expr + " failed: " +
                           cudaGetErrorName(err) + " (" + cudaGetErrorString(err) + ")");
}

}  // namespace fem::cuda

#define CUDA_CHECK(expr) ::fem::cuda::check((expr), #expr, __FILE__, __LINE__)
#define CUDA_CHECK_LAUNCH() CUDA_CHECK(cudaGetLastError())
