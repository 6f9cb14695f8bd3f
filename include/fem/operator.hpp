// Operator (drop-in for the reference's include/operator.hpp).
//
// Fields, validation and ownership are the reference's (src/operator.cpp:
// 21-136).  operator_apply runs on the GPU through libfem_b200 for the
// library's mass QFunctions:
//   * apply_mass / apply_mass_vector with fields (Interp "u", None "qdata") ->
//     (Interp "v"): one fused gather / interp / QFunction / interp^T /
//     scatter-add kernel;
//   * build_mass with fields (Grad "dx", Weight) -> (None "qdata"): one fused
//     geometric-factor kernel.
// The device plan (restriction, basis, the plan's copy of qdata) is built on
// the first apply and kept in the Operator.  Other QFunctions have no device
// implementation: operator_apply throws std::runtime_error for them (there is
// no CPU fallback).
#pragma once
#include <memory>
#include <optional>
#include <string>
#include <vector>

#include "basis.hpp"
#include "elem-restriction.hpp"
#include "fem-b200-detail.hpp"
#include "qfunction.hpp"
#include "qfunctions/mass.hpp"

namespace fem {

enum class VectorKind { Active, Passive, None };

struct FieldVector {
  VectorKind kind = VectorKind::None;
  std::vector<double> data;  // Passive only
};
inline FieldVector vector_active() { return {VectorKind::Active, {}}; }
inline FieldVector vector_none() { return {VectorKind::None, {}}; }
inline FieldVector vector_passive(std::vector<double> data) { return {VectorKind::Passive, std::move(data)}; }

struct OperatorField {
  std::string name;
  EvalMode eval_mode;
  int size;
  std::optional<ElemRestriction> restriction;
  std::optional<TensorBasis> basis;
  FieldVector vector;
};

namespace detail {
struct OperatorPlan;
}

struct Operator {
  QFunction qf;
  std::vector<std::optional<OperatorField>> inputs;
  std::vector<std::optional<OperatorField>> outputs;
  int num_elem = 0;
  int num_qpts = 0;
  int active_in_l_size = 0;
  int active_out_l_size = 0;
  // The device plan, built by the first operator_apply (shared by copies).
  std::shared_ptr<detail::OperatorPlan> device_plan;
};

// src/operator.cpp:21-27
inline void operator_create(const QFunction& qf, Operator& op) {
  if (!qf.user) throw std::invalid_argument("operator_create: QFunction has no user function");
  op = Operator{};
  op.qf = qf;
  op.inputs.resize(qf.inputs.size());
  op.outputs.resize(qf.outputs.size());
}

// src/operator.cpp:44-117: the field must exist and be unset; restriction,
// basis and vector must fit its EvalMode and size and agree with the fields
// already set (num_elem, quadrature points, active l_size).
inline void operator_set_field(Operator& op, const std::string& name, std::optional<ElemRestriction> restriction,
                               std::optional<TensorBasis> basis, FieldVector vector) {
  auto err = [&](const std::string& msg) {
    return std::invalid_argument("operator_set_field '" + name + "': " + msg);
  };
  const QFunctionField* qf_field = nullptr;
  std::optional<OperatorField>* slot = nullptr;
  bool is_input = true;
  for (std::size_t f = 0; f < op.qf.inputs.size() && !qf_field; ++f)
    if (op.qf.inputs[f].name == name) qf_field = &op.qf.inputs[f], slot = &op.inputs[f];
  for (std::size_t f = 0; f < op.qf.outputs.size() && !qf_field; ++f)
    if (op.qf.outputs[f].name == name) qf_field = &op.qf.outputs[f], slot = &op.outputs[f], is_input = false;
  if (!qf_field) throw err("the QFunction has no field with this name");
  if (slot->has_value()) throw err("already set");
  const EvalMode mode = qf_field->eval_mode;
  const int size = qf_field->size;
  switch (mode) {
    case EvalMode::Weight:
      if (restriction) throw err("EvalMode::Weight takes no restriction");
      if (!basis) throw err("EvalMode::Weight needs a basis (for its quadrature weights)");
      if (vector.kind != VectorKind::None) throw err("EvalMode::Weight takes vector_none()");
      break;
    case EvalMode::None:
      if (!restriction) throw err("EvalMode::None needs a restriction");
      if (basis) throw err("EvalMode::None takes no basis");
      if (restriction->num_comp != size) throw err("restriction num_comp must equal the field size");
      break;
    case EvalMode::Interp:
    case EvalMode::Grad: {
      if (!restriction) throw err("EvalMode::Interp/Grad needs a restriction");
      if (!basis) throw err("EvalMode::Interp/Grad needs a basis");
      const int expected = mode == EvalMode::Interp ? basis->num_comp : basis->num_comp * basis->dim;
      if (size != expected)
        throw err(mode == EvalMode::Interp ? "field size must equal basis num_comp"
                                           : "field size must equal basis num_comp * dim");
      if (restriction->num_comp != basis->num_comp) throw err("restriction and basis num_comp differ");
      if (restriction->elem_size != detail::int_pow(basis->P_1d, basis->dim))
        throw err("restriction elem_size must equal basis P_1d^dim");
      break;
    }
  }
  if (mode != EvalMode::Weight && vector.kind == VectorKind::None)
    throw err("needs vector_active() or vector_passive(...)");
  if (!is_input && vector.kind != VectorKind::Active) throw err("output fields must be active");
  if (vector.kind == VectorKind::Passive && static_cast<int>(vector.data.size()) != restriction->l_size)
    throw err("passive vector size must equal restriction l_size");
  const int num_qpts = basis ? int(detail::int_pow(basis->Q_1d, basis->dim)) : restriction->elem_size;
  if (op.num_qpts != 0 && num_qpts != op.num_qpts)
    throw err("number of quadrature points differs from previously set fields");
  if (restriction && op.num_elem != 0 && restriction->num_elem != op.num_elem)
    throw err("num_elem differs from previously set fields");
  if (vector.kind == VectorKind::Active) {
    int& active = is_input ? op.active_in_l_size : op.active_out_l_size;
    if (active != 0 && restriction->l_size != active)
      throw err("active fields share one vector, so their restrictions need the same l_size");
    active = restriction->l_size;
  }
  op.num_qpts = num_qpts;
  if (restriction) op.num_elem = restriction->num_elem;
  *slot = OperatorField{name, mode, size, std::move(restriction), std::move(basis), std::move(vector)};
  op.device_plan.reset();
}

// src/operator.cpp:126-136
inline void operator_check_ready(const Operator& op) {
  for (std::size_t f = 0; f < op.inputs.size(); ++f)
    if (!op.inputs[f]) throw std::invalid_argument("operator_check_ready: field '" + op.qf.inputs[f].name + "' is not set");
  for (std::size_t f = 0; f < op.outputs.size(); ++f)
    if (!op.outputs[f])
      throw std::invalid_argument("operator_check_ready: field '" + op.qf.outputs[f].name + "' is not set");
  if (op.num_elem == 0) throw std::invalid_argument("operator_check_ready: no field has a restriction");
}

namespace detail {

inline bool same_restriction(const ElemRestriction& a, const ElemRestriction& b) {
  return a.type == b.type && a.num_elem == b.num_elem && a.elem_size == b.elem_size && a.num_comp == b.num_comp &&
         a.comp_stride == b.comp_stride && a.l_size == b.l_size && a.offsets == b.offsets && a.strides == b.strides;
}
inline bool same_basis(const TensorBasis& a, const TensorBasis& b) {
  return a.dim == b.dim && a.num_comp == b.num_comp && a.P_1d == b.P_1d && a.Q_1d == b.Q_1d &&
         a.q_weight_1d == b.q_weight_1d && a.interp_1d == b.interp_1d && a.grad_1d == b.grad_1d;
}

struct RestrictionHandle {
  fem_b200_restriction h = nullptr;
  explicit RestrictionHandle(const ElemRestriction& r) {
    if (r.type != RestrictionType::Offset) throw std::runtime_error("operator_apply: expected an offset restriction");
    check(fem_b200_restriction_create_offset(r.num_elem, r.elem_size, r.num_comp, r.comp_stride, r.l_size,
                                             r.offsets.data(), FEM_B200_SCATTER_ATOMIC, &h));
  }
  ~RestrictionHandle() {
    if (h) (void)fem_b200_restriction_destroy(h);
  }
  RestrictionHandle(const RestrictionHandle&) = delete;
  RestrictionHandle& operator=(const RestrictionHandle&) = delete;
};

// Gathers a None-field L-vector through its restriction into the [q][e]
// layout the device plans use.
inline DevBuffer<double> qpoint_vector(const ElemRestriction& r, const std::vector<double>& l_vec) {
  DevBuffer<double> d_l(l_vec), d_e(static_cast<std::size_t>(r.e_size));
  DevBuffer<int> d_offs;
  if (r.type == RestrictionType::Offset) d_offs.upload(r.offsets);
  restriction_apply_device(r, ContractMode::NoTranspose, d_l.get(), d_e.get(), d_offs.get());
  return d_e;
}

struct OperatorPlan {
  enum Kind { Mass, Build } kind = Mass;
  std::unique_ptr<RestrictionHandle> r;
  std::unique_ptr<BasisHandle> b;
  fem_b200_mass mass = nullptr;
  ElemRestriction out_restriction;  // Build: where qdata goes
  int l_size = 0;
  ~OperatorPlan() {
    if (mass) (void)fem_b200_mass_destroy(mass);
  }
};

inline std::shared_ptr<OperatorPlan> build_plan(const Operator& op) {
  auto plan = std::make_shared<OperatorPlan>();
  const QFunctionUser user = op.qf.user;
  const bool mass = user == &qfunctions::apply_mass || user == &qfunctions::apply_mass_vector;
  const bool build = user == &qfunctions::build_mass;
  const char* shape_msg =
      "operator_apply: the device path runs apply_mass / apply_mass_vector with fields (Interp u, None qdata) -> "
      "(Interp v), and build_mass with (Grad dx, Weight) -> (None qdata)";
  if (!mass && !build)
    throw std::runtime_error("operator_apply: this QFunction has no device implementation (the device path runs "
                             "fem::qfunctions::apply_mass, apply_mass_vector and build_mass)");
  if (op.inputs.size() != 2 || op.outputs.size() != 1) throw std::runtime_error(shape_msg);
  const OperatorField& in0 = *op.inputs[0];
  const OperatorField& in1 = *op.inputs[1];
  const OperatorField& out0 = *op.outputs[0];
  if (mass) {
    if (in0.eval_mode != EvalMode::Interp || in0.vector.kind != VectorKind::Active ||
        in1.eval_mode != EvalMode::None || in1.vector.kind != VectorKind::Passive || in1.size != 1 ||
        out0.eval_mode != EvalMode::Interp)
      throw std::runtime_error(shape_msg);
    if (!same_restriction(*in0.restriction, *out0.restriction) || !same_basis(*in0.basis, *out0.basis))
      throw std::runtime_error("operator_apply: the device mass operator needs the same restriction and basis for u and v");
    int qf = FEM_B200_QF_APPLY_MASS;
    if (user == &qfunctions::apply_mass_vector) {
      qfunctions::ApplyMassVectorContext c{};
      if (op.qf.ctx.size() != sizeof(c)) throw std::runtime_error("apply_mass_vector needs an ApplyMassVectorContext");
      std::memcpy(&c, op.qf.ctx.data(), sizeof(c));
      if (c.num_comp != in0.basis->num_comp)
        throw std::runtime_error("apply_mass_vector: context num_comp differs from the basis num_comp");
      qf = FEM_B200_QF_APPLY_MASS_VECTOR;
    }
    plan->kind = OperatorPlan::Mass;
    plan->r = std::make_unique<RestrictionHandle>(*in0.restriction);
    plan->b = std::make_unique<BasisHandle>(*in0.basis);
    DevBuffer<double> qd = qpoint_vector(*in1.restriction, in1.vector.data);
    check(fem_b200_mass_create(plan->r->h, plan->b->h, qd.get(), static_cast<int64_t>(qd.size()), qf, &plan->mass));
    plan->l_size = in0.restriction->l_size;
  } else {
    if (in0.eval_mode != EvalMode::Grad || in0.vector.kind != VectorKind::Active ||
        in1.eval_mode != EvalMode::Weight || out0.eval_mode != EvalMode::None || out0.size != 1)
      throw std::runtime_error(shape_msg);
    qfunctions::BuildMassContext c{};
    if (op.qf.ctx.size() != sizeof(c)) throw std::runtime_error("build_mass needs a BuildMassContext");
    std::memcpy(&c, op.qf.ctx.data(), sizeof(c));
    if (c.dim != in0.basis->dim || in0.basis->num_comp != c.dim)
      throw std::runtime_error("build_mass: the coordinate basis must have dim == num_comp == context dim");
    if (in1.basis->q_weight_1d != in0.basis->q_weight_1d || in1.basis->Q_1d != in0.basis->Q_1d ||
        in1.basis->dim != in0.basis->dim)
      throw std::runtime_error("build_mass: the weights basis must match the coordinate basis's quadrature");
    plan->kind = OperatorPlan::Build;
    plan->r = std::make_unique<RestrictionHandle>(*in0.restriction);
    plan->b = std::make_unique<BasisHandle>(*in0.basis);
    plan->out_restriction = *out0.restriction;
    plan->l_size = out0.restriction->l_size;
  }
  return plan;
}

}  // namespace detail

// out = A(in): out resized to active_out_l_size, zeroed, then summed into.
// src/operator.cpp:148-182.
inline void operator_apply(Operator& op, const std::vector<double>& in, std::vector<double>& out) {
  operator_check_ready(op);
  if (op.active_in_l_size > 0 && static_cast<int>(in.size()) != op.active_in_l_size)
    throw std::invalid_argument("operator_apply: input vector size does not match active_in_l_size");
  if (!op.device_plan) op.device_plan = detail::build_plan(op);
  detail::OperatorPlan& p = *op.device_plan;
  out.assign(static_cast<std::size_t>(op.active_out_l_size), 0.0);
  if (p.kind == detail::OperatorPlan::Mass) {
    detail::check(fem_b200_mass_apply_host(p.mass, in.data(), static_cast<int64_t>(in.size()), out.data(),
                                           static_cast<int64_t>(out.size()), nullptr));
    return;
  }
  // build_mass: qdata in the [q][e] layout, then through the output restriction
  const int64_t nq = static_cast<int64_t>(op.num_qpts) * op.num_elem;
  detail::DevBuffer<double> x(in), qd(static_cast<std::size_t>(nq)), l_out(out.size());
  detail::check(fem_b200_mass_build(p.r->h, p.b->h, x.get(), static_cast<int64_t>(in.size()), qd.get(), nq, nullptr));
  l_out.zero();
  detail::DevBuffer<int> offs;
  if (p.out_restriction.type == RestrictionType::Offset) offs.upload(p.out_restriction.offsets);
  detail::restriction_apply_device(p.out_restriction, ContractMode::Transpose, qd.get(), l_out.get(), offs.get());
  l_out.download(out.data(), out.size());
}

}  // namespace fem
