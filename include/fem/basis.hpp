// 1D rules and the tensor-product H1 Lagrange basis (drop-in for the
// reference's include/basis.hpp).  The data is built by libfem_b200's host
// set-up, bitwise equal to the reference's.
#pragma once
#include <vector>

#include "fem-b200-detail.hpp"

namespace fem {

// Q Gauss-Legendre points / weights on [-1, 1] (src/basis.cpp:16-68).
inline void gauss_legendre_quadrature(int Q, std::vector<double>& q_ref_1d, std::vector<double>& q_weight_1d) {
  std::vector<double> x(Q > 0 ? Q : 1), w(Q > 0 ? Q : 1);
  detail::check(fem_b200_gauss_legendre(Q, x.data(), w.data()));
  q_ref_1d = std::move(x);
  q_weight_1d = std::move(w);
}

// Q Gauss-Lobatto points (ascending), weights if requested (src/basis.cpp:81-144).
inline void gauss_lobatto_points(int Q, std::vector<double>& q_ref_1d, std::vector<double>* q_weight_1d = nullptr) {
  std::vector<double> x(Q > 1 ? Q : 1), w(Q > 1 ? Q : 1);
  detail::check(fem_b200_gauss_lobatto(Q, x.data(), q_weight_1d ? w.data() : nullptr));
  q_ref_1d = std::move(x);
  if (q_weight_1d) *q_weight_1d = std::move(w);
}

// Lagrange interpolation / derivative matrices [M][P] (src/basis.cpp:156-186).
inline void lagrange_basis_matrix(const std::vector<double>& nodes, const std::vector<double>& eval_points,
                                  std::vector<double>& interp_1d, std::vector<double>& grad_1d) {
  const int P = static_cast<int>(nodes.size()), M = static_cast<int>(eval_points.size());
  interp_1d.assign(static_cast<std::size_t>(M) * P, 0.0);
  grad_1d.assign(static_cast<std::size_t>(M) * P, 0.0);
  if (P == 0) return;
  detail::check(
      fem_b200_lagrange_basis_matrix(P, nodes.data(), M, eval_points.data(), interp_1d.data(), grad_1d.data()));
}

// Quadrature of the tensor basis; nodes are always Gauss-Lobatto.
enum class QuadMode { Gauss, GaussLobatto };

struct TensorBasis {
  int dim;
  int num_comp;
  int P_1d;  // nodes per dimension
  int Q_1d;  // quadrature points per dimension

  std::vector<double> q_ref_1d;     // Q_1d
  std::vector<double> q_weight_1d;  // Q_1d
  std::vector<double> interp_1d;    // Q_1d * P_1d, row-major [q][p]
  std::vector<double> grad_1d;      // Q_1d * P_1d

  // src/basis.cpp:202-228: dim 1..3, num_comp 1..3, P_1d >= 2, Q_1d >= 1.
  static TensorBasis create_tensor_H1_lagrange(int dim, int num_comp, int P_1d, int Q_1d,
                                               QuadMode quad_mode = QuadMode::Gauss) {
    const std::size_t q = Q_1d > 0 ? std::size_t(Q_1d) : 1, qp = q * (P_1d > 0 ? std::size_t(P_1d) : 1);
    std::vector<double> x(q), w(q), B(qp), G(qp);
    detail::check(fem_b200_tensor_h1_lagrange(dim, num_comp, P_1d, Q_1d,
                                              quad_mode == QuadMode::Gauss ? FEM_B200_QUAD_GAUSS
                                                                           : FEM_B200_QUAD_GAUSS_LOBATTO,
                                              x.data(), w.data(), B.data(), G.data()));
    return TensorBasis{dim, num_comp, P_1d, Q_1d, x, w, B, G};
  }
};

namespace detail {
// A device basis built from a TensorBasis's own arrays.
struct BasisHandle {
  fem_b200_basis h = nullptr;
  explicit BasisHandle(const TensorBasis& b) {
    if (b.q_weight_1d.size() != std::size_t(b.Q_1d) || b.interp_1d.size() != std::size_t(b.Q_1d) * b.P_1d ||
        b.grad_1d.size() != std::size_t(b.Q_1d) * b.P_1d)
      throw std::invalid_argument("TensorBasis: array sizes do not match P_1d / Q_1d");
    check(fem_b200_basis_create_from(b.dim, b.num_comp, b.P_1d, b.Q_1d, b.q_weight_1d.data(), b.interp_1d.data(),
                                     b.grad_1d.data(), &h));
  }
  ~BasisHandle() {
    if (h) (void)fem_b200_basis_destroy(h);
  }
  BasisHandle(const BasisHandle&) = delete;
  BasisHandle& operator=(const BasisHandle&) = delete;
};
}  // namespace detail

}  // namespace fem
