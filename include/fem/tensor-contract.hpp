// Sum-factorised basis action (drop-in for the reference's
// include/tensor-contract.hpp), computed on the GPU.
#pragma once
#include <vector>

#include "basis.hpp"
#include "eval-mode.hpp"
#include "fem-b200-detail.hpp"
#include "transpose-mode.hpp"

namespace fem {

// v[(a*J + j)*C + c] (+)= sum_b t(j,b) u[(a*B + b)*C + c]; t(j,b) = t[j*B + b]
// (NoTranspose) or t[b*J + j] (Transpose); add = false resizes and
// overwrites v.  src/tensor-contract.cpp:35-59.
inline void tensor_contract_apply(int A, int B, int C, int J, const std::vector<double>& t, ContractMode t_mode,
                                  bool add, const std::vector<double>& u, std::vector<double>& v) {
  const std::size_t n = static_cast<std::size_t>(A) * J * C;
  if (t.size() < static_cast<std::size_t>(J) * B || u.size() < static_cast<std::size_t>(A) * B * C)
    throw std::invalid_argument("tensor_contract_apply: t or u is too small");
  v.resize(n);  // add: entries beyond the old size start at 0, as in the reference
  if (n == 0) return;
  detail::DevBuffer<double> dt(t), du(u), dv;
  if (add)
    dv.upload(v);
  else
    dv.resize(n);
  detail::check(fem_b200_contract(A, B, C, J, dt.get(), t_mode == ContractMode::Transpose ? FEM_B200_TRANSPOSE
                                                                                          : FEM_B200_NOTRANSPOSE,
                                  add ? 1 : 0, du.get(), dv.get(), nullptr));
  dv.download(v.data(), n);
}

namespace detail {
inline void basis_apply_host(const TensorBasis& basis, int num_elem, ContractMode t_mode, EvalMode eval_mode,
                             const std::vector<double>& u, std::vector<double>& v) {
  const int64_t pn = int_pow(basis.P_1d, basis.dim) * basis.num_comp * num_elem;
  const int64_t qn = int_pow(basis.Q_1d, basis.dim) * basis.num_comp * num_elem;
  const bool tr = t_mode == ContractMode::Transpose;
  int64_t n_u = 0, n_v = 0;
  int mode = FEM_B200_EVAL_INTERP;
  switch (eval_mode) {
    case EvalMode::Interp: n_u = tr ? qn : pn, n_v = tr ? pn : qn; break;
    case EvalMode::Grad:
      mode = FEM_B200_EVAL_GRAD;
      n_u = tr ? basis.dim * qn : pn, n_v = tr ? pn : basis.dim * qn;
      break;
    case EvalMode::Weight:
      if (tr) throw std::invalid_argument("EvalMode::Weight is incompatible with ContractMode::Transpose");
      mode = FEM_B200_EVAL_WEIGHT;
      n_v = int_pow(basis.Q_1d, basis.dim) * num_elem;
      break;
    default: throw std::invalid_argument("tensor_basis_apply: unknown eval_mode");
  }
  if (mode != FEM_B200_EVAL_WEIGHT && static_cast<int64_t>(u.size()) != n_u)
    throw std::invalid_argument("tensor_basis_apply: u has the wrong size");
  BasisHandle b(basis);
  DevBuffer<double> du, dv(static_cast<std::size_t>(n_v));
  if (mode != FEM_B200_EVAL_WEIGHT) du.upload(u);
  check(fem_b200_basis_apply(b.h, num_elem, tr ? FEM_B200_TRANSPOSE : FEM_B200_NOTRANSPOSE, mode, du.get(), n_u,
                             dv.get(), n_v, nullptr));
  v.resize(static_cast<std::size_t>(n_v));
  dv.download(v.data(), v.size());
}
}  // namespace detail

// Values at the quadrature points (NoTranspose) or the adjoint
// (Transpose), all elements batched.  src/tensor-contract.cpp:74-91.
inline void tensor_basis_apply_interp(const TensorBasis& basis, int num_elem, ContractMode t_mode,
                                      const std::vector<double>& u, std::vector<double>& v) {
  detail::basis_apply_host(basis, num_elem, t_mode, EvalMode::Interp, u, v);
}

// Gradients, v = [dim][comp][q][e] (NoTranspose) or the adjoint.
// src/tensor-contract.cpp:111-156.  Transpose overwrites v (the reference
// adds into whatever v held; on a zeroed or empty v both agree).
inline void tensor_basis_apply_grad(const TensorBasis& basis, int num_elem, ContractMode t_mode,
                                    const std::vector<double>& u, std::vector<double>& v) {
  detail::basis_apply_host(basis, num_elem, t_mode, EvalMode::Grad, u, v);
}

// Tensor-product weights v[q*num_elem + e].  src/tensor-contract.cpp:169-192.
inline void tensor_basis_apply_weight(const TensorBasis& basis, int num_elem, ContractMode t_mode,
                                      std::vector<double>& v) {
  detail::basis_apply_host(basis, num_elem, t_mode, EvalMode::Weight, {}, v);
}

// Dispatch by eval_mode.  src/tensor-contract.cpp:207-222.
inline void tensor_basis_apply(const TensorBasis& basis, int num_elem, ContractMode t_mode, EvalMode eval_mode,
                               const std::vector<double>& u, std::vector<double>& v) {
  detail::basis_apply_host(basis, num_elem, t_mode, eval_mode, u, v);
}

}  // namespace fem
