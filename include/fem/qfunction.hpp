// QFunctions (drop-in for the reference's include/qfunction.hpp).
//
// A QFunction is a plain function pointer with named fields, laid out
// [size][Q].  The library's own QFunctions (fem::qfunctions::apply_mass,
// apply_mass_vector, build_mass) are recognised by address and run on the
// GPU; operator_apply runs them fused with the rest of the operator.  Any
// other user function is user code: qfunction_apply calls it as given, and
// operator_apply rejects it (there is no device version of it).
#pragma once
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "eval-mode.hpp"
#include "fem-b200-detail.hpp"

namespace fem {

using QFunctionUser = int (*)(void* ctx, int Q, const double* const* in, double* const* out);

struct QFunctionField {
  std::string name;
  int size;  // num_comp (Interp/None), num_comp*dim (Grad), 1 (Weight)
  EvalMode eval_mode;
};

struct QFunction {
  QFunctionUser user = nullptr;
  std::vector<QFunctionField> inputs;
  std::vector<QFunctionField> outputs;
  std::vector<unsigned char> ctx;  // byte copy of a trivially copyable context
};

// src/qfunction.cpp:14-22
inline void qfunction_create(QFunctionUser user, QFunction& qf) {
  if (!user) throw std::invalid_argument("QFunction user function pointer is null");
  qf = QFunction{};
  qf.user = user;
}

namespace detail {
// Names are unique across inputs and outputs (src/qfunction.cpp:26-37).
inline void check_qf_field(const QFunction& qf, const std::string& name, int size, EvalMode eval_mode,
                           const char* who) {
  if (size <= 0) throw std::invalid_argument(std::string(who) + ": size must be positive");
  if (eval_mode == EvalMode::Weight && size != 1)
    throw std::invalid_argument(std::string(who) + ": an EvalMode::Weight field must have size 1");
  for (const auto* fields : {&qf.inputs, &qf.outputs})
    for (const QFunctionField& f : *fields)
      if (f.name == name) throw std::invalid_argument(std::string(who) + ": duplicate field name '" + name + "'");
}
}  // namespace detail

// src/qfunction.cpp:48-51
inline void qfunction_add_input(QFunction& qf, const std::string& name, int size, EvalMode eval_mode) {
  detail::check_qf_field(qf, name, size, eval_mode, "qfunction_add_input");
  qf.inputs.push_back({name, size, eval_mode});
}

// src/qfunction.cpp:63-69
inline void qfunction_add_output(QFunction& qf, const std::string& name, int size, EvalMode eval_mode) {
  if (eval_mode == EvalMode::Weight) throw std::invalid_argument("qfunction_add_output: EvalMode::Weight is input-only");
  detail::check_qf_field(qf, name, size, eval_mode, "qfunction_add_output");
  qf.outputs.push_back({name, size, eval_mode});
}

// include/qfunction.hpp:49-54: a byte copy, not a pointer.
template <class T>
void qfunction_set_context(QFunction& qf, const T& data) {
  static_assert(std::is_trivially_copyable_v<T>, "QFunction context must be trivially copyable");
  qf.ctx.resize(sizeof(T));
  std::memcpy(qf.ctx.data(), &data, sizeof(T));
}

// Validate, size the outputs ([size][Q], resized, existing values kept),
// run the function; a non-zero return throws std::runtime_error.
// src/qfunction.cpp:81-111.
inline void qfunction_apply(QFunction& qf, int Q, const std::vector<std::vector<double>>& in,
                            std::vector<std::vector<double>>& out) {
  if (Q <= 0) throw std::invalid_argument("qfunction_apply: Q must be positive");
  if (in.size() != qf.inputs.size())
    throw std::invalid_argument("qfunction_apply: number of input fields does not match QFunction");
  for (std::size_t f = 0; f < in.size(); ++f)
    if (in[f].size() != static_cast<std::size_t>(qf.inputs[f].size) * Q)
      throw std::invalid_argument("qfunction_apply: input field " + qf.inputs[f].name + " has incorrect size");
  out.resize(qf.outputs.size());
  for (std::size_t f = 0; f < out.size(); ++f) out[f].resize(static_cast<std::size_t>(qf.outputs[f].size) * Q);
  std::vector<const double*> ip(in.size());
  std::vector<double*> op(out.size());
  for (std::size_t f = 0; f < in.size(); ++f) ip[f] = in[f].data();
  for (std::size_t f = 0; f < out.size(); ++f) op[f] = out[f].data();
  void* ctx = qf.ctx.empty() ? nullptr : qf.ctx.data();
  if (qf.user(ctx, Q, ip.data(), op.data()) != 0)
    throw std::runtime_error("qfunction_apply: user function returned non-zero error code");
}

}  // namespace fem
