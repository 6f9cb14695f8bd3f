// fem::cuda device queries (drop-in for the reference's
// include/cuda/device-info.hpp).
#pragma once
#include <cstddef>
#include <sstream>
#include <stdexcept>
#include <string>

#include "../fem-b200-detail.hpp"

namespace fem::cuda {

struct DeviceInfo {
  int id = 0;
  std::string name;
  int cc_major = 0, cc_minor = 0;
  int sm_count = 0;
  int warp_size = 0;
  int max_threads_per_block = 0;
  int regs_per_block = 0;
  std::size_t shared_mem_per_block = 0;
  std::size_t shared_mem_per_block_optin = 0;
  std::size_t shared_mem_per_sm = 0;
  std::size_t total_global_mem = 0;
  std::size_t free_global_mem = 0;
};

inline int device_count() { return fem_b200_device_count(); }

// src/cuda/device-info.cpp:28-56: std::invalid_argument for a bad id.
inline DeviceInfo device_info(int device = 0) {
  if (device < 0 || device >= device_count()) throw std::invalid_argument("device_info: no such CUDA device");
  char name[256];
  int ints[6];
  int64_t sizes[5];
  fem::detail::check(fem_b200_device_info(device, name, sizeof(name), ints, sizes));
  DeviceInfo d;
  d.id = device;
  d.name = name;
  d.cc_major = ints[0], d.cc_minor = ints[1], d.sm_count = ints[2], d.warp_size = ints[3];
  d.max_threads_per_block = ints[4], d.regs_per_block = ints[5];
  d.shared_mem_per_block = std::size_t(sizes[0]), d.shared_mem_per_block_optin = std::size_t(sizes[1]);
  d.shared_mem_per_sm = std::size_t(sizes[2]), d.total_global_mem = std::size_t(sizes[3]);
  d.free_global_mem = std::size_t(sizes[4]);
  return d;
}

inline std::string to_string(const DeviceInfo& info) {
  constexpr double KiB = 1024.0, MiB = 1024.0 * 1024.0;
  std::ostringstream s;
  s << "device " << info.id << ": " << info.name << " (compute capability " << info.cc_major << "." << info.cc_minor
    << ")\n  SMs: " << info.sm_count << ", warp size: " << info.warp_size
    << ", max threads/block: " << info.max_threads_per_block << ", registers/block: " << info.regs_per_block
    << "\n  shared memory: " << info.shared_mem_per_block / KiB << " KiB/block (opt-in "
    << info.shared_mem_per_block_optin / KiB << "), " << info.shared_mem_per_sm / KiB << " KiB/SM"
    << "\n  global memory: " << info.free_global_mem / MiB << " MiB free of " << info.total_global_mem / MiB << " MiB";
  return s.str();
}

}  // namespace fem::cuda
