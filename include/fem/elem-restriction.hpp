// Element restriction (drop-in for the reference's include/elem-restriction.hpp).
// Validation is libfem_b200's host set-up; applies run on the GPU: the
// host vectors are copied in and out around the device kernels.
#pragma once
#include <array>
#include <vector>

#include "fem-b200-detail.hpp"
#include "transpose-mode.hpp"

namespace fem {

enum class RestrictionType { Offset, Strided };

struct ElemRestriction {
  RestrictionType type = RestrictionType::Offset;
  int num_elem;
  int elem_size;
  int num_comp;
  int comp_stride;
  int l_size;
  int e_size;
  std::vector<int> offsets;        // Offset: [num_elem][elem_size]
  std::array<int, 3> strides{};    // Strided: (node, component, element)
  bool has_backend_strides = false;
};

// src/elem-restriction.cpp:102-138 (the same checks and messages).
inline void elem_restriction_create(const int num_elem, const int elem_size, const int num_comp,
                                    const int comp_stride, const int l_size, const std::vector<int>& offsets,
                                    ElemRestriction& restriction) {
  detail::check(fem_b200_restriction_check_offset(num_elem, elem_size, num_comp, comp_stride, l_size, offsets.data(),
                                                  static_cast<int64_t>(offsets.size())));
  restriction.type = RestrictionType::Offset;
  restriction.num_elem = num_elem;
  restriction.elem_size = elem_size;
  restriction.num_comp = num_comp;
  restriction.comp_stride = comp_stride;
  restriction.l_size = l_size;
  restriction.e_size = num_comp * elem_size * num_elem;
  restriction.offsets = offsets;
  restriction.strides = {};
  restriction.has_backend_strides = false;
}

// src/elem-restriction.cpp:155-181, user strides.
inline void elem_restriction_create_strided(const int num_elem, const int elem_size, const int num_comp,
                                            const int l_size, const std::array<int, 3>& strides,
                                            ElemRestriction& restriction) {
  detail::check(fem_b200_restriction_check_strided(num_elem, elem_size, num_comp, l_size, strides.data()));
  restriction.type = RestrictionType::Strided;
  restriction.num_elem = num_elem;
  restriction.elem_size = elem_size;
  restriction.num_comp = num_comp;
  restriction.comp_stride = 0;
  restriction.l_size = l_size;
  restriction.e_size = num_comp * elem_size * num_elem;
  restriction.offsets.clear();
  restriction.strides = strides;
  restriction.has_backend_strides = false;
}

// src/elem-restriction.cpp:200-204, backend strides {num_elem, elem_size*num_elem, 1}.
inline void elem_restriction_create_strided(const int num_elem, const int elem_size, const int num_comp,
                                            const int l_size, ElemRestriction& restriction) {
  elem_restriction_create_strided(num_elem, elem_size, num_comp, l_size, {num_elem, elem_size * num_elem, 1},
                                  restriction);
  restriction.has_backend_strides = true;
}

namespace detail {
// Runs one restriction on device arrays already holding `in` / `out`.
inline void restriction_apply_device(const ElemRestriction& r, ContractMode t_mode, const double* in, double* out,
                                     const int* d_offsets) {
  const int tr = t_mode == ContractMode::Transpose;
  if (r.type == RestrictionType::Strided) {
    check(fem_b200_strided_apply(tr, r.num_elem, r.elem_size, r.num_comp, r.strides.data(), in, out, nullptr));
  } else if (!tr) {
    check(fem_b200_offset_gather(r.num_elem, r.elem_size, r.num_comp, r.comp_stride, d_offsets, in, out, nullptr));
  } else {
    check(fem_b200_offset_scatter_add(r.num_elem, r.elem_size, r.num_comp, r.comp_stride, d_offsets, in, out,
                                      nullptr));
  }
}
}  // namespace detail

// NoTranspose: out (resized to e_size) = E in.  Transpose: out (resized to
// l_size if needed, NOT zeroed) += E^T in.  src/elem-restriction.cpp:34-83.
// The scatter-add is atomic, so sums of shared nodes may differ from the
// reference in the last bits; fem::cuda with ScatterMode::Deterministic sums
// in the reference's order.
inline void elem_restriction_apply(const ElemRestriction& restriction, ContractMode t_mode,
                                   const std::vector<double>& in, std::vector<double>& out) {
  const ElemRestriction& r = restriction;
  const bool tr = t_mode == ContractMode::Transpose;
  if (in.size() != static_cast<std::size_t>(tr ? r.e_size : r.l_size))
    throw std::invalid_argument("elem_restriction_apply: in has the wrong size");
  out.resize(tr ? r.l_size : r.e_size);
  if (out.empty()) return;
  detail::DevBuffer<double> d_in(in), d_out;
  if (tr)
    d_out.upload(out);
  else
    d_out.resize(out.size());
  detail::DevBuffer<int> d_offs;
  if (r.type == RestrictionType::Offset) d_offs.upload(r.offsets);
  detail::restriction_apply_device(r, t_mode, d_in.get(), d_out.get(), d_offs.get());
  d_out.download(out.data(), out.size());
}

// multiplicity = E^T (E 1), resized to l_size (src/elem-restriction.cpp:215-227).
inline void elem_restriction_get_multiplicity(const ElemRestriction& restriction, std::vector<double>& multiplicity) {
  std::vector<double> ones(restriction.l_size, 1.0), e;
  elem_restriction_apply(restriction, ContractMode::NoTranspose, ones, e);
  std::vector<double> m(restriction.l_size, 0.0);
  elem_restriction_apply(restriction, ContractMode::Transpose, e, m);
  multiplicity = std::move(m);
}

}  // namespace fem
