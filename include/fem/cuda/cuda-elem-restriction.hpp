// fem::cuda element restriction (drop-in for the reference's
// include/cuda/cuda-elem-restriction.hpp): the index arrays live in
// DeviceArrays owned by the struct, copied once at create; the kernels are
// libfem_b200's (coalesced gather / atomic scatter-add through a shared-memory
// transpose of the offsets tile, and the transpose-map reduction).
#pragma once
#include <array>
#include <vector>

#include "../elem-restriction.hpp"
#include "../transpose-mode.hpp"
#include "device-array.hpp"

namespace fem::cuda {

// How Transpose resolves the race on shared L-vector entries:
//   Atomic         atomic adds, order varies between runs;
//   Deterministic  one thread per used L-node sums its E-entries in a fixed
//                  order through the transpose map: bitwise reproducible.
enum class ScatterMode { Atomic, Deterministic };

// CSR inverse of the offsets: used L-nodes ascending; for node n the E-nodes
// t_indices[t_offsets[n] .. t_offsets[n+1]) as i + e*elem_size, increasing.
struct TransposeMap {
  std::vector<int> l_vec_indices;
  std::vector<int> t_offsets;
  std::vector<int> t_indices;
};

// src/cuda/cuda-elem-restriction.cu:149-177 (host).
inline void build_transpose_map(const fem::ElemRestriction& restriction, TransposeMap& map) {
  if (restriction.type != RestrictionType::Offset)
    throw std::invalid_argument("build_transpose_map: only for Offset restrictions");
  const std::size_t n_t = static_cast<std::size_t>(restriction.num_elem) * restriction.elem_size;
  std::vector<int> lvi(static_cast<std::size_t>(restriction.l_size)), to(lvi.size() + 1), ti(n_t);
  int n = 0;
  fem::detail::check(fem_b200_transpose_map(restriction.num_elem, restriction.elem_size, restriction.l_size,
                                            restriction.offsets.data(), lvi.data(), to.data(), ti.data(), &n));
  lvi.resize(static_cast<std::size_t>(n));
  to.resize(static_cast<std::size_t>(n) + 1);
  map.l_vec_indices = std::move(lvi);
  map.t_offsets = std::move(to);
  map.t_indices = std::move(ti);
}

struct ElemRestriction {
  RestrictionType type = RestrictionType::Offset;
  int num_elem = 0, elem_size = 0, num_comp = 0, comp_stride = 0;
  int l_size = 0, e_size = 0;
  std::array<int, 3> strides{};
  ScatterMode scatter_mode = ScatterMode::Atomic;
  DeviceArray<int> offsets;
  int num_nodes = 0;
  DeviceArray<int> l_vec_indices, t_offsets, t_indices;
};

// src/cuda/cuda-elem-restriction.cu:188-215: `restriction` is replaced only on success.
inline void elem_restriction_create(const fem::ElemRestriction& host, ScatterMode scatter_mode,
                                    ElemRestriction& restriction) {
  ElemRestriction r;
  r.type = host.type;
  r.num_elem = host.num_elem, r.elem_size = host.elem_size, r.num_comp = host.num_comp;
  r.comp_stride = host.comp_stride, r.l_size = host.l_size, r.e_size = host.e_size;
  r.strides = host.strides;
  r.scatter_mode = scatter_mode;
  if (host.type == RestrictionType::Offset) {
    if (host.offsets.size() != static_cast<std::size_t>(host.num_elem) * host.elem_size)
      throw std::invalid_argument("cuda::elem_restriction_create: offsets size != num_elem * elem_size");
    r.offsets = DeviceArray<int>(host.offsets);
    if (scatter_mode == ScatterMode::Deterministic) {
      TransposeMap map;
      build_transpose_map(host, map);
      r.num_nodes = static_cast<int>(map.l_vec_indices.size());
      r.l_vec_indices = DeviceArray<int>(map.l_vec_indices);
      r.t_offsets = DeviceArray<int>(map.t_offsets);
      r.t_indices = DeviceArray<int>(map.t_indices);
    }
  }
  restriction = std::move(r);
}

// NoTranspose: out resized to e_size and overwritten.  Transpose: out must
// already have l_size entries; the result is added into it.  Asynchronous on
// the default stream (the result is visible after the next synchronising call).
// src/cuda/cuda-elem-restriction.cu:230-273.
inline void elem_restriction_apply(const ElemRestriction& restriction, ContractMode t_mode,
                                   const DeviceArray<double>& in, DeviceArray<double>& out) {
  const ElemRestriction& r = restriction;
  const bool tr = t_mode == ContractMode::Transpose;
  if (static_cast<int>(in.size()) != (tr ? r.e_size : r.l_size))
    throw std::invalid_argument("cuda::elem_restriction_apply: in has the wrong size");
  if (tr) {
    if (static_cast<int>(out.size()) != r.l_size)
      throw std::invalid_argument(
          "cuda::elem_restriction_apply: Transpose adds into out, which must already have l_size entries");
  } else {
    out.resize(static_cast<std::size_t>(r.e_size));
  }
  if (static_cast<std::size_t>(r.num_elem) * r.elem_size == 0) return;
  using fem::detail::check;
  if (r.type == RestrictionType::Strided) {
    check(fem_b200_strided_apply(tr, r.num_elem, r.elem_size, r.num_comp, r.strides.data(), in.data(), out.data(),
                                 nullptr));
  } else if (!tr) {
    check(fem_b200_offset_gather(r.num_elem, r.elem_size, r.num_comp, r.comp_stride, r.offsets.data(), in.data(),
                                 out.data(), nullptr));
  } else if (r.scatter_mode == ScatterMode::Atomic) {
    check(fem_b200_offset_scatter_add(r.num_elem, r.elem_size, r.num_comp, r.comp_stride, r.offsets.data(),
                                      in.data(), out.data(), nullptr));
  } else {
    check(fem_b200_transpose_scatter_add(r.num_nodes, r.num_elem, r.elem_size, r.num_comp, r.comp_stride,
                                         r.l_vec_indices.data(), r.t_offsets.data(), r.t_indices.data(), in.data(),
                                         out.data(), nullptr));
  }
}

}  // namespace fem::cuda
