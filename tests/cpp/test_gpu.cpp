// Drop-in C++ API on the GPU: the reference's operator, restriction,
// tensor-contraction, QFunction and fem::cuda tests (file:line cited per
// case), run through include/fem/*.hpp and libfem_b200.  Tagged [gpu].
#include <cmath>
#include <cstdlib>

#include "basis.hpp"
#include "cuda/cuda-elem-restriction.hpp"
#include "cuda/device-array.hpp"
#include "cuda/device-info.hpp"
#include "elem-restriction.hpp"
#include "harness.hpp"
#include "operator.hpp"
#include "qfunction.hpp"
#include "qfunctions/mass.hpp"
#include "tensor-contract.hpp"

using harness::Approx;
using fem::ContractMode;
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
double dot(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0;
  for (std::size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
  return s;
}
double sum(const std::vector<double>& a) {
  double s = 0;
  for (double x : a) s += x;
  return s;
}
std::vector<double> ramp(std::size_t n, double scale) {
  std::vector<double> v(n);
  for (std::size_t i = 0; i < n; ++i) v[i] = scale * (0.37 * i - 1.3 + 0.01 * (i % 7) * (i % 5));
  return v;
}

// tests/test-operator.cpp:57-83: 2 linear elements, P=2, Q=3
struct Mesh1D {
  fem::TensorBasis basis = fem::TensorBasis::create_tensor_H1_lagrange(1, 1, 2, 3);
  fem::ElemRestriction rstr, q_rstr;
  Mesh1D() {
    fem::elem_restriction_create(2, 2, 1, 1, 3, {0, 1, 1, 2}, rstr);
    fem::elem_restriction_create_strided(2, 3, 1, 6, q_rstr);
  }
  std::vector<double> qdata(double h0, double h1) const {
    std::vector<double> w;
    fem::tensor_basis_apply_weight(basis, 2, ContractMode::NoTranspose, w);
    for (int q = 0; q < 3; ++q) w[q * 2 + 0] *= h0 / 2, w[q * 2 + 1] *= h1 / 2;
    return w;
  }
  fem::Operator mass(const std::vector<double>& qd) const {
    fem::Operator op;
    fem::operator_create(mass_qf(), op);
    fem::operator_set_field(op, "u", rstr, basis, fem::vector_active());
    fem::operator_set_field(op, "qdata", q_rstr, std::nullopt, fem::vector_passive(qd));
    fem::operator_set_field(op, "v", rstr, basis, fem::vector_active());
    return op;
  }
};

// tests/test-operator.cpp:90-121: distorted 2-quad mesh of area 5
struct Mesh2D {
  fem::TensorBasis mesh_basis = fem::TensorBasis::create_tensor_H1_lagrange(2, 2, 2, 3);
  fem::TensorBasis sol_basis = fem::TensorBasis::create_tensor_H1_lagrange(2, 1, 2, 3);
  fem::ElemRestriction coord_rstr, sol_rstr, q_rstr;
  std::vector<double> coords = {0, 1, 3, 0.5, 1, 2.5, 0, 0, 0, 2, 2, 2};
  Mesh2D() {
    const std::vector<int> offsets = {0, 1, 3, 4, 1, 2, 4, 5};
    fem::elem_restriction_create(2, 4, 2, 6, 12, offsets, coord_rstr);
    fem::elem_restriction_create(2, 4, 1, 1, 6, offsets, sol_rstr);
    fem::elem_restriction_create_strided(2, 9, 1, 18, q_rstr);
  }
  std::vector<double> build_qdata() const {
    fem::Operator op;
    fem::operator_create(build_qf(2), op);
    fem::operator_set_field(op, "dx", coord_rstr, mesh_basis, fem::vector_active());
    fem::operator_set_field(op, "weights", std::nullopt, mesh_basis, fem::vector_none());
    fem::operator_set_field(op, "qdata", q_rstr, std::nullopt, fem::vector_active());
    std::vector<double> q;
    fem::operator_apply(op, coords, q);
    return q;
  }
  fem::Operator mass(const std::vector<double>& qd) const {
    fem::Operator op;
    fem::operator_create(mass_qf(), op);
    fem::operator_set_field(op, "u", sol_rstr, sol_basis, fem::vector_active());
    fem::operator_set_field(op, "qdata", q_rstr, std::nullopt, fem::vector_passive(qd));
    fem::operator_set_field(op, "v", sol_rstr, sol_basis, fem::vector_active());
    return op;
  }
};
}  // namespace

// tests/test-operator.cpp:256-271
TEST_CASE("operator_apply: 1D mass matrix (h/6)[2 1; 1 2]", "[gpu][operator]") {
  Mesh1D m;
  fem::Operator op = m.mass(m.qdata(1, 1));
  std::vector<double> v;
  fem::operator_apply(op, {1, 1, 1}, v);
  REQUIRE(v.size() == 3);
  REQUIRE(v[0] == Approx(0.5));
  REQUIRE(v[1] == Approx(1.0));
  REQUIRE(v[2] == Approx(0.5));
  fem::operator_apply(op, {0, 1, 2}, v);
  REQUIRE(v[0] == Approx(1.0 / 6));
  REQUIRE(v[1] == Approx(1.0));
  REQUIRE(v[2] == Approx(5.0 / 6));
}

// tests/test-operator.cpp:273-286
TEST_CASE("operator_apply: 1D build operator gives qdata = w * J", "[gpu][operator]") {
  Mesh1D m;
  fem::Operator op;
  fem::operator_create(build_qf(1), op);
  fem::operator_set_field(op, "dx", m.rstr, m.basis, fem::vector_active());
  fem::operator_set_field(op, "weights", std::nullopt, m.basis, fem::vector_none());
  fem::operator_set_field(op, "qdata", m.q_rstr, std::nullopt, fem::vector_active());
  std::vector<double> qdata;
  fem::operator_apply(op, {0, 1, 3}, qdata);
  const auto expected = m.qdata(1, 2);
  REQUIRE(qdata.size() == expected.size());
  for (std::size_t i = 0; i < expected.size(); ++i) REQUIRE(qdata[i] == Approx(expected[i]));
}

// tests/test-operator.cpp:288-297, 320-329
TEST_CASE("operator_apply: 2D area of a distorted mesh, symmetry", "[gpu][operator]") {
  Mesh2D m;
  const auto qdata = m.build_qdata();
  REQUIRE(sum(qdata) == Approx(5.0));
  fem::Operator op = m.mass(qdata);
  std::vector<double> v;
  fem::operator_apply(op, std::vector<double>(6, 1.0), v);
  REQUIRE(sum(v) == Approx(5.0));
  const auto u = ramp(6, 1.0), w = ramp(6, -0.7);
  std::vector<double> Mu, Mw;
  fem::operator_apply(op, u, Mu);
  fem::operator_apply(op, w, Mw);
  REQUIRE(dot(w, Mu) == Approx(dot(u, Mw)).margin(1e-12));
}

// tests/test-operator.cpp:299-318
TEST_CASE("operator_apply equals the hand-composed restrict/basis/QFunction chain", "[gpu][operator]") {
  Mesh1D m;
  const auto qdata = m.qdata(1, 2);
  fem::Operator op = m.mass(qdata);
  const std::vector<double> u = {0.3, -1.2, 2.5};
  std::vector<double> e_u, q_u, e_v, expected(3, 0.0);
  fem::elem_restriction_apply(m.rstr, ContractMode::NoTranspose, u, e_u);
  fem::tensor_basis_apply_interp(m.basis, 2, ContractMode::NoTranspose, e_u, q_u);
  fem::QFunction qf = mass_qf();
  std::vector<std::vector<double>> q_out;
  fem::qfunction_apply(qf, 6, {q_u, qdata}, q_out);
  fem::tensor_basis_apply_interp(m.basis, 2, ContractMode::Transpose, q_out[0], e_v);
  fem::elem_restriction_apply(m.rstr, ContractMode::Transpose, e_v, expected);
  std::vector<double> v;
  fem::operator_apply(op, u, v);
  for (std::size_t i = 0; i < v.size(); ++i) REQUIRE(v[i] == Approx(expected[i]).margin(1e-14));
}

// tests/test-operator.cpp:331-352
TEST_CASE("operator_apply overwrites out and rejects bad calls", "[gpu][operator]") {
  Mesh1D m;
  fem::Operator op = m.mass(m.qdata(1, 1));
  std::vector<double> v(10, 99.0);
  fem::operator_apply(op, {1, 1, 1}, v);
  REQUIRE(v.size() == 3);
  REQUIRE(v[1] == Approx(1.0));
  REQUIRE_THROWS_AS(fem::operator_apply(op, {1, 1}, v), std::invalid_argument);
  fem::Operator incomplete;
  fem::operator_create(mass_qf(), incomplete);
  fem::operator_set_field(incomplete, "u", m.rstr, m.basis, fem::vector_active());
  REQUIRE_THROWS_AS(fem::operator_apply(incomplete, {1, 1, 1}, v), std::invalid_argument);
}

TEST_CASE("operator_apply rejects a QFunction without a device implementation", "[gpu][operator]") {
  Mesh1D m;
  fem::QFunction qf;
  fem::qfunction_create([](void*, int, const double* const*, double* const*) { return 0; }, qf);
  fem::qfunction_add_input(qf, "u", 1, EvalMode::Interp);
  fem::qfunction_add_input(qf, "qdata", 1, EvalMode::None);
  fem::qfunction_add_output(qf, "v", 1, EvalMode::Interp);
  fem::Operator op;
  fem::operator_create(qf, op);
  fem::operator_set_field(op, "u", m.rstr, m.basis, fem::vector_active());
  fem::operator_set_field(op, "qdata", m.q_rstr, std::nullopt, fem::vector_passive(m.qdata(1, 1)));
  fem::operator_set_field(op, "v", m.rstr, m.basis, fem::vector_active());
  std::vector<double> v;
  REQUIRE_THROWS_AS(fem::operator_apply(op, {1, 1, 1}, v), std::runtime_error);
}

// tests/test-elem-restriction.cpp:21-116, 180-228
TEST_CASE("elem_restriction_apply known answers and multiplicity", "[gpu][elem-restriction]") {
  fem::ElemRestriction r;
  fem::elem_restriction_create(2, 2, 1, 1, 3, {0, 1, 1, 2}, r);
  std::vector<double> E;
  fem::elem_restriction_apply(r, ContractMode::NoTranspose, {10.0, 20.0, 30.0}, E);
  REQUIRE(E == std::vector<double>({10, 20, 20, 30}));
  std::vector<double> L(3, 0.0);
  fem::elem_restriction_apply(r, ContractMode::Transpose, {10.0, 20.0, 20.0, 30.0}, L);
  REQUIRE(L == std::vector<double>({10, 40, 30}));
  L = {100, 200, 300};
  fem::elem_restriction_apply(r, ContractMode::Transpose, {10.0, 20.0, 20.0, 30.0}, L);
  REQUIRE(L == std::vector<double>({110, 240, 330}));
  fem::elem_restriction_create(2, 2, 2, 100, 200, {0, 1, 2, 3}, r);
  std::vector<double> Lg(200);
  for (int i = 0; i < 200; ++i) Lg[i] = i;
  fem::elem_restriction_apply(r, ContractMode::NoTranspose, Lg, E);
  REQUIRE(E == std::vector<double>({0, 2, 1, 3, 100, 102, 101, 103}));
  std::vector<int> offs;
  for (int e = 0; e < 3; ++e)
    for (int j = 0; j < 4; ++j) offs.push_back(e * 3 + j);
  fem::elem_restriction_create(3, 4, 1, 1, 10, offs, r);
  std::vector<double> mult;
  fem::elem_restriction_get_multiplicity(r, mult);
  for (int i = 0; i < 10; ++i) REQUIRE(mult[i] == ((i > 0 && i < 9 && i % 3 == 0) ? 2.0 : 1.0));
  fem::elem_restriction_create(2, 2, 2, 5, 12, {0, 1, 1, 2}, r);
  fem::elem_restriction_get_multiplicity(r, mult);
  REQUIRE(mult == std::vector<double>({1, 2, 1, 0, 0, 1, 2, 1, 0, 0, 0, 0}));
  // strided: user strides gather, backend identity, accumulate (:302-345)
  fem::elem_restriction_create_strided(2, 3, 2, 12, {1, 3, 6}, r);
  std::vector<double> L12(12);
  for (int i = 0; i < 12; ++i) L12[i] = i;
  fem::elem_restriction_apply(r, ContractMode::NoTranspose, L12, E);
  REQUIRE(E == std::vector<double>({0, 6, 1, 7, 2, 8, 3, 9, 4, 10, 5, 11}));
  fem::elem_restriction_create_strided(2, 2, 1, 4, r);
  std::vector<double> L4 = {10, 20, 30, 40};
  fem::elem_restriction_apply(r, ContractMode::Transpose, {1, 2, 3, 4}, L4);
  REQUIRE(L4 == std::vector<double>({11, 22, 33, 44}));
}

// tests/test-tensor-contract.cpp:19-104
TEST_CASE("tensor_contract_apply known answers", "[gpu][tensor-contract]") {
  const std::vector<double> t = {1, 2, 3, 4, 5, 6};
  std::vector<double> v;
  fem::tensor_contract_apply(1, 3, 1, 2, t, ContractMode::NoTranspose, false, {2, -1, 3}, v);
  REQUIRE(v == std::vector<double>({9, 21}));
  fem::tensor_contract_apply(1, 3, 2, 2, t, ContractMode::NoTranspose, false, {2, 1, -1, 1, 3, 1}, v);
  REQUIRE(v == std::vector<double>({9, 6, 21, 15}));
  v = {100, 200};
  fem::tensor_contract_apply(1, 3, 1, 2, t, ContractMode::NoTranspose, true, {2, -1, 3}, v);
  REQUIRE(v == std::vector<double>({109, 221}));
  std::vector<double> w;
  fem::tensor_contract_apply(1, 2, 1, 3, t, ContractMode::Transpose, false, {9, 21}, w);
  REQUIRE(w == std::vector<double>({93, 123, 153}));
}

// tests/test-tensor-contract.cpp:268-309: P = Q = 16, spectral accuracy
TEST_CASE("tensor_basis_apply_grad matches an analytic gradient in 3D", "[gpu][tensor-contract]") {
  const int P = 16, Q = 16;
  auto basis = fem::TensorBasis::create_tensor_H1_lagrange(3, 1, P, Q);
  std::vector<double> nodes;
  fem::gauss_lobatto_points(P, nodes);
  std::vector<double> u(P * P * P);
  for (int iz = 0; iz < P; ++iz)
    for (int iy = 0; iy < P; ++iy)
      for (int ix = 0; ix < P; ++ix) {
        const double x = nodes[ix], y = nodes[iy], z = nodes[iz];
        u[(iz * P + iy) * P + ix] = std::sin(x) + std::cos(x * y) + x * y * z;
      }
  std::vector<double> v;
  fem::tensor_basis_apply_grad(basis, 1, ContractMode::NoTranspose, u, v);
  const int Q3 = Q * Q * Q;
  REQUIRE(v.size() == std::size_t(3 * Q3));
  for (int jz = 0; jz < Q; ++jz)
    for (int jy = 0; jy < Q; ++jy)
      for (int jx = 0; jx < Q; ++jx) {
        const double x = basis.q_ref_1d[jx], y = basis.q_ref_1d[jy], z = basis.q_ref_1d[jz];
        const int q = (jz * Q + jy) * Q + jx;
        REQUIRE(v[q] == Approx(std::cos(x) - y * std::sin(x * y) + y * z).margin(1e-11));
        REQUIRE(v[Q3 + q] == Approx(-x * std::sin(x * y) + x * z).margin(1e-11));
        REQUIRE(v[2 * Q3 + q] == Approx(x * y).margin(1e-11));
      }
}

// tests/test-tensor-contract.cpp:543-633
TEST_CASE("basis adjoint identities and weights", "[gpu][tensor-contract]") {
  const int dim = 3, nc = 3, ne = 2, P = 3, Q = 5;
  auto basis = fem::TensorBasis::create_tensor_H1_lagrange(dim, nc, P, Q);
  std::srand(33);
  std::vector<double> u(nc * 27 * ne), w(nc * 125 * ne), g(dim * nc * 125 * ne);
  for (auto& x : u) x = double(std::rand()) / RAND_MAX - 0.5;
  for (auto& x : w) x = double(std::rand()) / RAND_MAX - 0.5;
  for (auto& x : g) x = double(std::rand()) / RAND_MAX - 0.5;
  std::vector<double> Bu, BTw, Gu, GTg;
  fem::tensor_basis_apply_interp(basis, ne, ContractMode::NoTranspose, u, Bu);
  fem::tensor_basis_apply_interp(basis, ne, ContractMode::Transpose, w, BTw);
  REQUIRE(dot(Bu, w) == Approx(dot(u, BTw)).margin(1e-10));
  fem::tensor_basis_apply_grad(basis, ne, ContractMode::NoTranspose, u, Gu);
  fem::tensor_basis_apply_grad(basis, ne, ContractMode::Transpose, g, GTg);
  REQUIRE(dot(Gu, g) == Approx(dot(u, GTg)).margin(1e-10));
  for (int d = 1; d <= 3; ++d) {
    auto b = fem::TensorBasis::create_tensor_H1_lagrange(d, 3, 3, 5);
    std::vector<double> wt;
    fem::tensor_basis_apply(b, 2, ContractMode::NoTranspose, EvalMode::Weight, {}, wt);
    REQUIRE(sum(wt) == Approx(2 * std::pow(2.0, d)).margin(1e-12));
  }
  std::vector<double> wt;
  REQUIRE_THROWS_AS(fem::tensor_basis_apply(basis, 3, ContractMode::Transpose, EvalMode::Weight, {}, wt),
                    std::invalid_argument);
}

// tests/test-qfunction.cpp:84-127: the library QFunctions on the device
TEST_CASE("qfunction_apply: apply_mass and build_mass det(J) w", "[gpu][qfunction]") {
  fem::QFunction qf = mass_qf();
  std::vector<std::vector<double>> out;
  fem::qfunction_apply(qf, 5, {{1, 2, 3, 4, 5}, {0.5, -1, 2, 0, 10}}, out);
  REQUIRE(out[0] == std::vector<double>({0.5, -2, 6, 0, 50}));
  const std::vector<double> w = {0.5, 2.0};
  struct Case {
    int dim;
    std::vector<double> J;
    double d0, d1;
  };
  const std::vector<Case> cases = {{1, {3.0, -2.0}, 3.0, -2.0},
                                   {2, {2, 1, 1, 2, 0, 3, 3, 4}, 6.0, -2.0},
                                   {3, {1, 2, 0, 0, 0, 1, 0, 1, 2, 3, 0, 0, 0, 0, 0, 1, 3, 4}, 6.0, 25.0}};
  for (const Case& c : cases) {
    fem::QFunction b = build_qf(c.dim);
    fem::qfunction_apply(b, 2, {c.J, w}, out);
    REQUIRE(out[0][0] == Approx(c.d0 * w[0]));
    REQUIRE(out[0][1] == Approx(c.d1 * w[1]));
  }
}

// tests/cuda/test-cuda-elem-restriction.cu:134-233
TEST_CASE("fem::cuda restriction: create, size checks, deterministic reproducibility", "[gpu][cuda]") {
  fem::ElemRestriction host;
  fem::elem_restriction_create(2, 2, 1, 1, 3, {0, 1, 1, 2}, host);
  fem::cuda::ElemRestriction dev;
  fem::cuda::elem_restriction_create(host, fem::cuda::ScatterMode::Deterministic, dev);
  REQUIRE(dev.offsets.to_host() == host.offsets);
  REQUIRE(dev.num_nodes == 3);
  REQUIRE(dev.t_indices.to_host() == std::vector<int>({0, 1, 2, 3}));
  fem::cuda::DeviceArray<double> out;
  REQUIRE_THROWS_AS(fem::cuda::elem_restriction_apply(dev, ContractMode::NoTranspose, fem::cuda::DeviceArray<double>(4), out),
                    std::invalid_argument);
  REQUIRE_THROWS_AS(fem::cuda::elem_restriction_apply(dev, ContractMode::Transpose, fem::cuda::DeviceArray<double>(3), out),
                    std::invalid_argument);
  REQUIRE_THROWS_AS(fem::cuda::elem_restriction_apply(dev, ContractMode::Transpose, fem::cuda::DeviceArray<double>(4), out),
                    std::invalid_argument);
  fem::cuda::DeviceArray<double> l(std::vector<double>{10, 20, 30}), e;
  fem::cuda::elem_restriction_apply(dev, ContractMode::NoTranspose, l, e);
  REQUIRE(e.to_host() == std::vector<double>({10, 20, 20, 30}));
  // a 16^3 quadratic mesh, 3 interleaved components: 5 runs bitwise equal
  const int n = 16, P = 3, N = n * (P - 1) + 1;
  std::vector<int> offs;
  for (int ez = 0; ez < n; ++ez)
    for (int ey = 0; ey < n; ++ey)
      for (int ex = 0; ex < n; ++ex)
        for (int iz = 0; iz < P; ++iz)
          for (int iy = 0; iy < P; ++iy)
            for (int ix = 0; ix < P; ++ix)
              offs.push_back(((ex * (P - 1) + ix) + N * ((ey * (P - 1) + iy) + N * (ez * (P - 1) + iz))) * 3);
  fem::elem_restriction_create(n * n * n, P * P * P, 3, 1, N * N * N * 3, offs, host);
  fem::cuda::elem_restriction_create(host, fem::cuda::ScatterMode::Deterministic, dev);
  std::vector<double> eh(host.e_size);
  for (int i = 0; i < host.e_size; ++i) eh[i] = std::sin(0.37 * i + 0.3) + 1e-3 * std::cos(11.0 * i);
  fem::cuda::DeviceArray<double> ed(eh);
  std::vector<double> first;
  for (int run = 0; run < 5; ++run) {
    fem::cuda::DeviceArray<double> lo(host.l_size);
    lo.zero();
    fem::cuda::elem_restriction_apply(dev, ContractMode::Transpose, ed, lo);
    auto res = lo.to_host();
    if (run == 0)
      first = res;
    else
      REQUIRE(res == first);
  }
}

// tests/cuda/test-device.cu:26-102
TEST_CASE("DeviceArray round trip, zero, resize, move; device_info", "[gpu][cuda]") {
  const std::vector<double> h = {1.5, -2.0, 3.25, 0.0, 1e-300, 7.0};
  fem::cuda::DeviceArray<double> d(h);
  REQUIRE(d.size() == h.size());
  REQUIRE(d.to_host() == h);
  d.zero();
  REQUIRE(d.to_host() == std::vector<double>(6, 0.0));
  REQUIRE_THROWS_AS(d.copy_from_host(std::vector<double>(4)), std::invalid_argument);
  const double* before = d.data();
  d.resize(6);
  REQUIRE(d.data() == before);
  fem::cuda::DeviceArray<double> a(std::vector<double>{1, 2, 3});
  const double* p = a.data();
  fem::cuda::DeviceArray<double> b(std::move(a));
  REQUIRE(b.data() == p);
  REQUIRE(a.data() == nullptr);  // NOLINT(bugprone-use-after-move)
  fem::cuda::DeviceArray<double> empty;
  REQUIRE(empty.empty());
  REQUIRE(fem::cuda::device_count() >= 1);
  const auto info = fem::cuda::device_info(0);
  REQUIRE(!info.name.empty());
  REQUIRE(info.warp_size == 32);
  REQUIRE(info.sm_count >= 1);
  REQUIRE(info.free_global_mem <= info.total_global_mem);
  REQUIRE_THROWS_AS(fem::cuda::device_info(-1), std::invalid_argument);
}
