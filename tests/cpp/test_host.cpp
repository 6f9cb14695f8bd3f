// Drop-in C++ API, host side (no GPU): the reference's known answers and
// validation matrix through include/fem/*.hpp.  Values restate the
// reference's tests (file:line cited per case).
#include <cmath>

#include "basis.hpp"
#include "cuda/cuda-elem-restriction.hpp"
#include "elem-restriction.hpp"
#include "harness.hpp"
#include "operator.hpp"
#include "qfunction.hpp"
#include "qfunctions/mass.hpp"

using harness::Approx;
using fem::EvalMode;

namespace {
fem::QFunction mass_qf() {
  fem::QFunction qf;
  fem::qfunction_create(fem::qfunctions::apply_mass, qf);
  fem::qfunction_add_input(qf, "u", 1, EvalMode::Interp);
  fem::qfunction_add_input(qf, "qdata", 1, EvalMode::None);
  fem::qfunction_add_output(qf, "v", 1, EvalMode::Interp);
  return qf;
}
fem::QFunction build_qf(int dim) {
  fem::QFunction qf;
  fem::qfunction_create(fem::qfunctions::build_mass, qf);
  fem::qfunction_add_input(qf, "dx", dim * dim, EvalMode::Grad);
  fem::qfunction_add_input(qf, "weights", 1, EvalMode::Weight);
  fem::qfunction_add_output(qf, "qdata", 1, EvalMode::None);
  fem::qfunction_set_context(qf, fem::qfunctions::BuildMassContext{dim});
  return qf;
}
int noop(void*, int, const double* const*, double* const*) { return 0; }
int sum_diff(void*, int Q, const double* const* in, double* const* out) {
  for (int p = 0; p < Q; p++) {
    const double a = in[0][p], b = in[0][Q + p];
    out[0][p] = a + b;
    out[0][Q + p] = a - b;
  }
  return 0;
}
int check_null_ctx(void* ctx, int Q, const double* const*, double* const* out) {
  for (int p = 0; p < Q; p++) out[0][p] = ctx == nullptr ? 1.0 : 0.0;
  return 0;
}
int fail(void*, int, const double* const*, double* const*) { return 3; }
}  // namespace

// tests/test-basis.cpp:12-59
TEST_CASE("Gauss-Legendre: weights sum to 2, sorted, exact to degree 2Q-1", "[basis]") {
  for (int Q = 1; Q <= 5; ++Q) {
    std::vector<double> x, w;
    fem::gauss_legendre_quadrature(Q, x, w);
    REQUIRE(x.size() == std::size_t(Q));
    double s = 0;
    for (double wi : w) s += wi;
    REQUIRE(s == Approx(2.0).margin(1e-12));
    for (int i = 1; i < Q; ++i) REQUIRE(x[i] > x[i - 1]);
    for (int k = 0; k <= 2 * Q - 1; ++k) {
      double integral = 0;
      for (int i = 0; i < Q; ++i) integral += w[i] * std::pow(x[i], k);
      REQUIRE(integral == Approx(k % 2 == 0 ? 2.0 / (k + 1) : 0.0).margin(1e-10));
    }
  }
  std::vector<double> x, w;
  REQUIRE_THROWS_AS(fem::gauss_legendre_quadrature(0, x, w), std::invalid_argument);
}

// tests/test-basis.cpp:65-107
TEST_CASE("Gauss-Lobatto: endpoints, sorted, weights, P=3 is {-1,0,1}", "[basis]") {
  for (int P = 2; P <= 5; ++P) {
    std::vector<double> x, w;
    fem::gauss_lobatto_points(P, x, &w);
    REQUIRE(x.front() == Approx(-1.0).margin(1e-12));
    REQUIRE(x.back() == Approx(1.0).margin(1e-12));
    double s = 0;
    for (double wi : w) s += wi;
    REQUIRE(s == Approx(2.0).margin(1e-12));
  }
  std::vector<double> x;
  fem::gauss_lobatto_points(3, x);
  REQUIRE(x[1] == Approx(0.0).margin(1e-12));
  REQUIRE_THROWS_AS(fem::gauss_lobatto_points(1, x), std::invalid_argument);
}

// tests/test-basis.cpp:113-162, 181-206
TEST_CASE("Lagrange matrices and the linear reference stiffness", "[basis]") {
  std::vector<double> B, G;
  fem::lagrange_basis_matrix({-1.0, 0.0, 1.0}, {-1.0, 0.0, 1.0}, B, G);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) REQUIRE(B[i * 3 + j] == Approx(i == j ? 1.0 : 0.0).margin(1e-10));
  fem::lagrange_basis_matrix({-1.0, -0.3, 0.4, 1.0}, {-1.0, -0.6, 0.0, 0.55, 1.0}, B, G);
  for (int i = 0; i < 5; ++i) {
    double sb = 0, sg = 0;
    for (int j = 0; j < 4; ++j) sb += B[i * 4 + j], sg += G[i * 4 + j];
    REQUIRE(sb == Approx(1.0).margin(1e-10));
    REQUIRE(sg == Approx(0.0).margin(1e-10));
  }
  auto basis = fem::TensorBasis::create_tensor_H1_lagrange(1, 1, 2, 2);
  double K[2][2] = {{0, 0}, {0, 0}};
  for (int q = 0; q < 2; ++q)
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) K[i][j] += basis.q_weight_1d[q] * basis.grad_1d[q * 2 + i] * basis.grad_1d[q * 2 + j];
  REQUIRE(K[0][0] == Approx(0.5).margin(1e-10));
  REQUIRE(K[0][1] == Approx(-0.5).margin(1e-10));
  REQUIRE_THROWS_AS(fem::TensorBasis::create_tensor_H1_lagrange(4, 1, 2, 2), std::invalid_argument);
  REQUIRE_THROWS_AS(fem::TensorBasis::create_tensor_H1_lagrange(3, 1, 1, 2), std::invalid_argument);
}

// tests/test-elem-restriction.cpp:123-173
TEST_CASE("elem_restriction_create: fields and the validation matrix", "[elem-restriction]") {
  fem::ElemRestriction r;
  fem::elem_restriction_create(2, 2, 3, 10, 30, {0, 1, 1, 2}, r);
  REQUIRE(r.e_size == 12);
  REQUIRE(r.offsets == std::vector<int>({0, 1, 1, 2}));
  const std::vector<int> ok = {0, 1, 1, 2};
  REQUIRE_THROWS_AS(fem::elem_restriction_create(0, 2, 1, 1, 3, {}, r), std::invalid_argument);
  REQUIRE_THROWS_AS(fem::elem_restriction_create(2, 0, 1, 1, 3, {}, r), std::invalid_argument);
  REQUIRE_THROWS_AS(fem::elem_restriction_create(2, 2, 0, 1, 3, ok, r), std::invalid_argument);
  REQUIRE_THROWS_AS(fem::elem_restriction_create(2, 2, 1, 1, 0, ok, r), std::invalid_argument);
  REQUIRE_THROWS_AS(fem::elem_restriction_create(2, 2, 2, 0, 200, ok, r), std::invalid_argument);
  REQUIRE_NOTHROW(fem::elem_restriction_create(2, 2, 1, 0, 3, ok, r));
  REQUIRE_THROWS_AS(fem::elem_restriction_create(2, 2, 1, 1, 3, {0, 1, 1}, r), std::invalid_argument);
  REQUIRE_THROWS_AS(fem::elem_restriction_create(2, 2, 1, 1, 3, {0, 1, 1, 3}, r), std::invalid_argument);
  REQUIRE_THROWS_AS(fem::elem_restriction_create(2, 2, 1, 1, 3, {0, -1, 1, 2}, r), std::invalid_argument);
  REQUIRE_THROWS_AS(fem::elem_restriction_create(1, 2, 2, 100, 3, {0, 1}, r), std::invalid_argument);
  REQUIRE_NOTHROW(fem::elem_restriction_create(1, 2, 2, 2, 4, {0, 1}, r));
  REQUIRE_THROWS_AS(fem::elem_restriction_create(1, 2, 2, 2, 3, {0, 1}, r), std::invalid_argument);
}

// tests/test-elem-restriction.cpp:245-296
TEST_CASE("elem_restriction_create_strided: backend and user strides", "[elem-restriction]") {
  fem::ElemRestriction r;
  fem::elem_restriction_create_strided(3, 4, 2, 24, r);
  REQUIRE(r.type == fem::RestrictionType::Strided);
  REQUIRE(r.has_backend_strides);
  REQUIRE(r.strides == std::array<int, 3>({3, 12, 1}));
  fem::elem_restriction_create_strided(2, 3, 2, 12, {1, 3, 6}, r);
  REQUIRE_FALSE(r.has_backend_strides);
  REQUIRE_THROWS_AS(fem::elem_restriction_create_strided(2, 4, 2, 15, r), std::invalid_argument);
  REQUIRE_THROWS_AS(fem::elem_restriction_create_strided(2, 3, 2, 11, {1, 3, 6}, r), std::invalid_argument);
  REQUIRE_THROWS_AS(fem::elem_restriction_create_strided(2, 3, 2, 12, {-1, 3, 6}, r), std::invalid_argument);
  fem::elem_restriction_create(2, 2, 1, 1, 3, {0, 1, 1, 2}, r);
  REQUIRE(r.type == fem::RestrictionType::Offset);
  REQUIRE_FALSE(r.has_backend_strides);
}

// tests/cuda/test-cuda-elem-restriction.cu:87-128
TEST_CASE("build_transpose_map known answers", "[transpose-map]") {
  fem::ElemRestriction r;
  fem::elem_restriction_create(2, 2, 1, 1, 3, {0, 1, 1, 2}, r);
  fem::cuda::TransposeMap map;
  fem::cuda::build_transpose_map(r, map);
  REQUIRE(map.l_vec_indices == std::vector<int>({0, 1, 2}));
  REQUIRE(map.t_offsets == std::vector<int>({0, 1, 3, 4}));
  REQUIRE(map.t_indices == std::vector<int>({0, 1, 2, 3}));
  fem::elem_restriction_create(2, 2, 1, 1, 6, {2, 4, 5, 2}, r);
  fem::cuda::build_transpose_map(r, map);
  REQUIRE(map.l_vec_indices == std::vector<int>({2, 4, 5}));
  REQUIRE(map.t_offsets == std::vector<int>({0, 2, 3, 4}));
  REQUIRE(map.t_indices == std::vector<int>({0, 3, 1, 2}));
  fem::elem_restriction_create_strided(2, 3, 1, 6, r);
  REQUIRE_THROWS_AS(fem::cuda::build_transpose_map(r, map), std::invalid_argument);
}

// tests/test-qfunction.cpp:18-77, 129-213 (user QFunctions are user code)
TEST_CASE("qfunction bookkeeping, context copy, user functions", "[qfunction]") {
  fem::QFunction qf = mass_qf();
  REQUIRE(qf.user == &fem::qfunctions::apply_mass);
  REQUIRE(qf.inputs.size() == 2);
  REQUIRE(qf.outputs[0].name == "v");
  REQUIRE(qf.ctx.empty());
  REQUIRE_THROWS_AS(fem::qfunction_create(nullptr, qf), std::invalid_argument);
  fem::qfunction_create(noop, qf);
  REQUIRE_THROWS_AS(fem::qfunction_add_input(qf, "u", 0, EvalMode::Interp), std::invalid_argument);
  REQUIRE_THROWS_AS(fem::qfunction_add_input(qf, "w", 2, EvalMode::Weight), std::invalid_argument);
  REQUIRE_THROWS_AS(fem::qfunction_add_output(qf, "w", 1, EvalMode::Weight), std::invalid_argument);
  fem::qfunction_add_input(qf, "u", 1, EvalMode::Interp);
  REQUIRE_THROWS_AS(fem::qfunction_add_output(qf, "u", 1, EvalMode::Interp), std::invalid_argument);
  fem::qfunctions::BuildMassContext ctx{2};
  fem::qfunction_set_context(qf, ctx);
  ctx.dim = 99;
  fem::qfunctions::BuildMassContext stored;
  std::memcpy(&stored, qf.ctx.data(), sizeof(stored));
  REQUIRE(stored.dim == 2);
  fem::qfunction_create(sum_diff, qf);
  fem::qfunction_add_input(qf, "u", 2, EvalMode::Interp);
  fem::qfunction_add_output(qf, "v", 2, EvalMode::Interp);
  std::vector<std::vector<double>> out;
  fem::qfunction_apply(qf, 3, {{1, 2, 3, 10, 20, 30}}, out);
  REQUIRE(out[0] == std::vector<double>({11, 22, 33, -9, -18, -27}));
  fem::qfunction_create(check_null_ctx, qf);
  fem::qfunction_add_output(qf, "flag", 1, EvalMode::None);
  fem::qfunction_apply(qf, 2, {}, out);
  REQUIRE(out[0] == std::vector<double>({1, 1}));
  fem::qfunction_create(fail, qf);
  REQUIRE_THROWS_AS(fem::qfunction_apply(qf, 1, {}, out), std::runtime_error);
  qf = mass_qf();
  REQUIRE_THROWS_AS(fem::qfunction_apply(qf, 2, {{1, 2}}, out), std::invalid_argument);
  REQUIRE_THROWS_AS(fem::qfunction_apply(qf, 2, {{1, 2}, {3}}, out), std::invalid_argument);
  REQUIRE_THROWS_AS(fem::qfunction_apply(qf, 0, {{}, {}}, out), std::invalid_argument);
}

// tests/test-operator.cpp:129-250
TEST_CASE("operator_set_field validation and bookkeeping", "[operator]") {
  auto basis = fem::TensorBasis::create_tensor_H1_lagrange(1, 1, 2, 3);
  fem::ElemRestriction rstr, q_rstr;
  fem::elem_restriction_create(2, 2, 1, 1, 3, {0, 1, 1, 2}, rstr);
  fem::elem_restriction_create_strided(2, 3, 1, 6, q_rstr);
  std::vector<double> qdata(6, 0.5);
  fem::Operator op;
  fem::operator_create(mass_qf(), op);
  fem::operator_set_field(op, "u", rstr, basis, fem::vector_active());
  REQUIRE_THROWS_AS(fem::operator_check_ready(op), std::invalid_argument);
  REQUIRE_THROWS_AS(fem::operator_set_field(op, "u", rstr, basis, fem::vector_active()), std::invalid_argument);
  REQUIRE_THROWS_AS(fem::operator_set_field(op, "w", rstr, basis, fem::vector_active()), std::invalid_argument);
  REQUIRE_THROWS_AS(fem::operator_set_field(op, "qdata", q_rstr, basis, fem::vector_passive(qdata)),
                    std::invalid_argument);
  REQUIRE_THROWS_AS(fem::operator_set_field(op, "qdata", q_rstr, std::nullopt, fem::vector_passive({1, 2, 3, 4, 5})),
                    std::invalid_argument);
  fem::operator_set_field(op, "qdata", q_rstr, std::nullopt, fem::vector_passive(qdata));
  REQUIRE_THROWS_AS(fem::operator_set_field(op, "v", rstr, basis, fem::vector_passive({1, 2, 3})),
                    std::invalid_argument);
  fem::operator_set_field(op, "v", rstr, basis, fem::vector_active());
  REQUIRE_NOTHROW(fem::operator_check_ready(op));
  REQUIRE(op.num_elem == 2);
  REQUIRE(op.num_qpts == 3);
  REQUIRE(op.active_in_l_size == 3);
  REQUIRE(op.active_out_l_size == 3);
  fem::Operator b;
  fem::operator_create(build_qf(1), b);
  REQUIRE_THROWS_AS(fem::operator_set_field(b, "weights", rstr, basis, fem::vector_none()), std::invalid_argument);
  REQUIRE_THROWS_AS(fem::operator_set_field(b, "weights", std::nullopt, std::nullopt, fem::vector_none()),
                    std::invalid_argument);
  REQUIRE_NOTHROW(fem::operator_set_field(b, "weights", std::nullopt, basis, fem::vector_none()));
  fem::Operator b2;
  fem::operator_create(build_qf(2), b2);
  REQUIRE_THROWS_AS(fem::operator_set_field(b2, "dx", rstr, basis, fem::vector_active()), std::invalid_argument);
  fem::Operator none;
  REQUIRE_THROWS_AS(fem::operator_create(fem::QFunction{}, none), std::invalid_argument);
}
