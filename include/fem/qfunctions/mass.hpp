// Mass-operator QFunctions (drop-in for the reference's
// include/qfunctions/mass.hpp).  Same signatures and [size][Q] layouts; the
// bodies run on the GPU (the host arrays are copied in and out), and
// operator_apply recognises them by address and fuses them into its kernels.
#pragma once
#include "../fem-b200-detail.hpp"

namespace fem::qfunctions {

struct BuildMassContext {
  int dim;
};

// The number of components the vector mass applies to (no reference counterpart).
struct ApplyMassVectorContext {
  int num_comp;
};

// qdata = det(J) * w; in[0] "dx" [d][c][p] (size dim*dim, Grad), in[1]
// "weights" (Weight), out[0] "qdata" (None).  include/qfunctions/mass.hpp:17-40.
inline int build_mass(void* ctx, int Q, const double* const* in, double* const* out) {
  if (!ctx || Q <= 0) return 1;
  const int dim = static_cast<const BuildMassContext*>(ctx)->dim;
  if (dim < 1 || dim > 3) return 1;
  try {
    detail::DevBuffer<double> J, w, q(static_cast<std::size_t>(Q));
    J.upload(in[0], static_cast<std::size_t>(dim) * dim * Q);
    w.upload(in[1], static_cast<std::size_t>(Q));
    detail::check(fem_b200_qfunction_build_mass(dim, Q, J.get(), w.get(), q.get(), nullptr));
    q.download(out[0], static_cast<std::size_t>(Q));
  } catch (...) {
    return 2;
  }
  return 0;
}

// v = qdata * u on the first Q entries (component 0 only, as the reference's
// loop, include/qfunctions/mass.hpp:45-51).
inline int apply_mass(void* /*ctx*/, int Q, const double* const* in, double* const* out) {
  if (Q <= 0) return 1;
  try {
    detail::DevBuffer<double> u, qd, v(static_cast<std::size_t>(Q));
    u.upload(in[0], static_cast<std::size_t>(Q));
    qd.upload(in[1], static_cast<std::size_t>(Q));
    detail::check(fem_b200_qfunction_apply_mass(Q, u.get(), qd.get(), v.get(), nullptr));
    v.download(out[0], static_cast<std::size_t>(Q));
  } catch (...) {
    return 2;
  }
  return 0;
}

// v_k = qdata * u_k for every component k (context ApplyMassVectorContext;
// in[0] "u" [comp][Q], in[1] "qdata", out[0] "v" [comp][Q]).
inline int apply_mass_vector(void* ctx, int Q, const double* const* in, double* const* out) {
  if (!ctx || Q <= 0) return 1;
  const int nc = static_cast<const ApplyMassVectorContext*>(ctx)->num_comp;
  if (nc < 1) return 1;
  try {
    detail::DevBuffer<double> u, qd, v(static_cast<std::size_t>(nc) * Q);
    u.upload(in[0], static_cast<std::size_t>(nc) * Q);
    qd.upload(in[1], static_cast<std::size_t>(Q));
    for (int k = 0; k < nc; ++k)
      detail::check(fem_b200_qfunction_apply_mass(Q, u.get() + static_cast<std::size_t>(k) * Q, qd.get(),
                                                  v.get() + static_cast<std::size_t>(k) * Q, nullptr));
    v.download(out[0], static_cast<std::size_t>(nc) * Q);
  } catch (...) {
    return 2;
  }
  return 0;
}

}  // namespace fem::qfunctions
