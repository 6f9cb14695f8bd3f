// ref_driver.cpp -- a C entry layer around the UNMODIFIED reference library
// (fe-demo-cpp src/*.cpp, compiled from where it lies by oracle/Makefile).
//
// TEST INFRASTRUCTURE ONLY.  It drives the reference through its own public
// C++ API (operator_create / operator_set_field / operator_apply, ...) so that
// tests can pin the C restatement (fem_oracle.c) against the reference's own
// outputs, tests/golden/make_golden.py can write fixtures, and bench.py can
// time the reference CPU path (the "reference" arm and cpu_baseline).  The
// product library never links or calls it.
#include <algorithm>
#include <cstring>
#include <exception>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "basis.hpp"
#include "elem-restriction.hpp"
#include "operator.hpp"
#include "qfunction.hpp"
#include "qfunctions/mass.hpp"
#include "tensor-contract.hpp"

namespace {

thread_local std::string g_err;

template <class F>
int guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::invalid_argument& e) {
    g_err = e.what();
    return 1;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 2;
  }
}

int ipow(int b, int e) {
  int r = 1;
  for (int i = 0; i < e; ++i) r *= b;
  return r;
}

fem::QFunction apply_mass_qf(int size) {
  fem::QFunction qf;
  fem::qfunction_create(fem::qfunctions::apply_mass, qf);
  fem::qfunction_add_input(qf, "u", size, fem::EvalMode::Interp);
  fem::qfunction_add_input(qf, "qdata", 1, fem::EvalMode::None);
  fem::qfunction_add_output(qf, "v", size, fem::EvalMode::Interp);
  return qf;
}

fem::QFunction build_mass_qf(int dim) {
  fem::QFunction qf;
  fem::qfunction_create(fem::qfunctions::build_mass, qf);
  fem::qfunction_add_input(qf, "dx", dim * dim, fem::EvalMode::Grad);
  fem::qfunction_add_input(qf, "weights", 1, fem::EvalMode::Weight);
  fem::qfunction_add_output(qf, "qdata", 1, fem::EvalMode::None);
  fem::qfunction_set_context(qf, fem::qfunctions::BuildMassContext{dim});
  return qf;
}

fem::Operator make_mass_op(int dim, int ne, int P, int Q, int nc, int comp_stride, int l_size,
                           const std::vector<int>& offsets, const std::vector<double>& qdata) {
  const int nq = ipow(Q, dim);
  fem::TensorBasis basis = fem::TensorBasis::create_tensor_H1_lagrange(dim, nc, P, Q);
  fem::ElemRestriction r, qr;
  fem::elem_restriction_create(ne, ipow(P, dim), nc, comp_stride, l_size, offsets, r);
  fem::elem_restriction_create_strided(ne, nq, 1, nq * ne, qr);
  fem::Operator op;
  fem::operator_create(apply_mass_qf(nc), op);
  fem::operator_set_field(op, "u", r, basis, fem::vector_active());
  fem::operator_set_field(op, "qdata", qr, std::nullopt, fem::vector_passive(qdata));
  fem::operator_set_field(op, "v", r, basis, fem::vector_active());
  return op;
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

int ref_gauss_legendre(int Q, double* x, double* w) {
  return guarded([&] {
    std::vector<double> xv, wv;
    fem::gauss_legendre_quadrature(Q, xv, wv);
    std::copy(xv.begin(), xv.end(), x);
    std::copy(wv.begin(), wv.end(), w);
  });
}

int ref_gauss_lobatto(int Q, double* x, double* w) {
  return guarded([&] {
    std::vector<double> xv, wv;
    fem::gauss_lobatto_points(Q, xv, w ? &wv : nullptr);
    std::copy(xv.begin(), xv.end(), x);
    if (w) std::copy(wv.begin(), wv.end(), w);
  });
}

int ref_tensor_h1_lagrange(int dim, int nc, int P, int Q, int quad_mode, double* q_ref, double* q_weight,
                           double* interp, double* grad) {
  return guarded([&] {
    auto b = fem::TensorBasis::create_tensor_H1_lagrange(
        dim, nc, P, Q, quad_mode == 0 ? fem::QuadMode::Gauss : fem::QuadMode::GaussLobatto);
    std::copy(b.q_ref_1d.begin(), b.q_ref_1d.end(), q_ref);
    std::copy(b.q_weight_1d.begin(), b.q_weight_1d.end(), q_weight);
    std::copy(b.interp_1d.begin(), b.interp_1d.end(), interp);
    std::copy(b.grad_1d.begin(), b.grad_1d.end(), grad);
  });
}

// tensor_basis_apply on a zeroed (fresh) output; n_v is the expected size.
int ref_basis_apply(int dim, int nc, int P, int Q, int quad_mode, int ne, int t_mode, int eval_mode, const double* u,
                    long n_u, double* v, long n_v) {
  return guarded([&] {
    auto b = fem::TensorBasis::create_tensor_H1_lagrange(
        dim, nc, P, Q, quad_mode == 0 ? fem::QuadMode::Gauss : fem::QuadMode::GaussLobatto);
    std::vector<double> uv(u, u + n_u), out;
    fem::tensor_basis_apply(b, ne, t_mode ? fem::ContractMode::Transpose : fem::ContractMode::NoTranspose,
                            static_cast<fem::EvalMode>(eval_mode), uv, out);
    if (static_cast<long>(out.size()) != n_v) throw std::runtime_error("ref_basis_apply: unexpected output size");
    std::copy(out.begin(), out.end(), v);
  });
}

// elem_restriction_apply on an offset restriction.  Transpose adds into v.
int ref_offset_apply(int ne, int es, int nc, int comp_stride, int l_size, const int* offsets, int t_mode,
                     const double* in, double* out) {
  return guarded([&] {
    fem::ElemRestriction r;
    fem::elem_restriction_create(ne, es, nc, comp_stride, l_size, std::vector<int>(offsets, offsets + (long)ne * es),
                                 r);
    if (t_mode == 0) {
      std::vector<double> l(in, in + l_size), e;
      fem::elem_restriction_apply(r, fem::ContractMode::NoTranspose, l, e);
      std::copy(e.begin(), e.end(), out);
    } else {
      std::vector<double> e(in, in + r.e_size), l(out, out + l_size);
      fem::elem_restriction_apply(r, fem::ContractMode::Transpose, e, l);
      std::copy(l.begin(), l.end(), out);
    }
  });
}

int ref_multiplicity(int ne, int es, int nc, int comp_stride, int l_size, const int* offsets, double* mult) {
  return guarded([&] {
    fem::ElemRestriction r;
    fem::elem_restriction_create(ne, es, nc, comp_stride, l_size, std::vector<int>(offsets, offsets + (long)ne * es),
                                 r);
    std::vector<double> m;
    fem::elem_restriction_get_multiplicity(r, m);
    std::copy(m.begin(), m.end(), mult);
  });
}

// qdata = build_mass through operator_apply; coords is the dim-component
// L-vector (component k of node n at offsets[...] + k*comp_stride).
int ref_mass_build(int dim, int ne, int P, int Q, int comp_stride, int l_size, const int* offsets, const double* coords,
                   double* qdata) {
  return guarded([&] {
    const int nq = ipow(Q, dim);
    fem::TensorBasis mesh_basis = fem::TensorBasis::create_tensor_H1_lagrange(dim, dim, P, Q);
    fem::ElemRestriction xr, qr;
    fem::elem_restriction_create(ne, ipow(P, dim), dim, comp_stride, l_size,
                                 std::vector<int>(offsets, offsets + (long)ne * ipow(P, dim)), xr);
    fem::elem_restriction_create_strided(ne, nq, 1, nq * ne, qr);
    fem::Operator op;
    fem::operator_create(build_mass_qf(dim), op);
    fem::operator_set_field(op, "dx", xr, mesh_basis, fem::vector_active());
    fem::operator_set_field(op, "weights", std::nullopt, mesh_basis, fem::vector_none());
    fem::operator_set_field(op, "qdata", qr, std::nullopt, fem::vector_active());
    std::vector<double> x(coords, coords + l_size), q;
    fem::operator_apply(op, x, q);
    std::copy(q.begin(), q.end(), qdata);
  });
}

// v = M u with the reference apply_mass QFunction (component 0 only when
// nc > 1, which is what the reference computes).
int ref_mass_apply(int dim, int ne, int P, int Q, int nc, int comp_stride, int l_size, const int* offsets,
                   const double* qdata, const double* u, double* v) {
  return guarded([&] {
    const int nq = ipow(Q, dim);
    fem::Operator op = make_mass_op(dim, ne, P, Q, nc, comp_stride, l_size,
                                    std::vector<int>(offsets, offsets + (long)ne * ipow(P, dim)),
                                    std::vector<double>(qdata, qdata + (long)nq * ne));
    std::vector<double> uv(u, u + l_size), out;
    fem::operator_apply(op, uv, out);
    std::copy(out.begin(), out.end(), v);
  });
}

// Vector mass as nc scalar reference applies, one per component view
// (offsets + k*comp_stride), summed; each L entry belongs to one component.
int ref_mass_apply_vector(int dim, int ne, int P, int Q, int nc, int comp_stride, int l_size, const int* offsets,
                          const double* qdata, const double* u, double* v) {
  return guarded([&] {
    const int nq = ipow(Q, dim), es = ipow(P, dim);
    std::vector<double> total(l_size, 0.0), uv(u, u + l_size), vk;
    for (int k = 0; k < nc; ++k) {
      std::vector<int> offs(offsets, offsets + (long)ne * es);
      for (int& o : offs) o += k * comp_stride;
      fem::Operator op =
          make_mass_op(dim, ne, P, Q, 1, 1, l_size, offs, std::vector<double>(qdata, qdata + (long)nq * ne));
      fem::operator_apply(op, uv, vk);
      for (int l = 0; l < l_size; ++l) total[l] += vk[l];
    }
    std::copy(total.begin(), total.end(), v);
  });
}

// ---------------------------------------------------------------------------
// Threaded, element-chunked reference mass apply (the CPU baseline).  The
// reference is single-threaded; a CPU user runs it per element chunk, each
// chunk with its own compact L-numbering (so operator_apply zeroes only the
// chunk's nodes and int32 sizes stay valid), then adds the chunk results.
// Chunk results are added in chunk order.  Nodes inside one chunk get the same
// sum as the unchunked reference; nodes on a chunk boundary differ only by the
// grouping of their (at most 8) element contributions.
// ---------------------------------------------------------------------------
struct RefChunk {
  std::vector<int> nodes;  // global L index of each local node (sorted)
  fem::Operator op;
  std::vector<double> u_loc, v_loc;
};

struct RefPlan {
  std::vector<RefChunk> chunks;
  long l_size = 0;
};

// qdata == nullptr: each chunk builds its own qdata from the coordinates
// (blocked, component k at k*l_size) with the reference build operator.
void* ref_plan_create(int dim, long ne, int P, int Q, long l_size, const int* offsets, const double* qdata,
                      const double* coords, int n_chunks) {
  RefPlan* plan = nullptr;
  int rc = guarded([&] {
    auto p = std::make_unique<RefPlan>();
    p->l_size = l_size;
    const int es = ipow(P, dim), nq = ipow(Q, dim);
    n_chunks = std::max<int>(1, std::min<long>(n_chunks, ne));
    p->chunks.resize(n_chunks);
    std::vector<std::thread> th;
    for (int c = 0; c < n_chunks; ++c) {
      th.emplace_back([&, c] {
        const long e0 = ne * c / n_chunks, e1 = ne * (c + 1) / n_chunks, nce = e1 - e0;
        RefChunk& ch = p->chunks[c];
        std::vector<int> all(offsets + e0 * es, offsets + e1 * es);
        ch.nodes = all;
        std::sort(ch.nodes.begin(), ch.nodes.end());
        ch.nodes.erase(std::unique(ch.nodes.begin(), ch.nodes.end()), ch.nodes.end());
        for (int& o : all) o = int(std::lower_bound(ch.nodes.begin(), ch.nodes.end(), o) - ch.nodes.begin());
        std::vector<double> qd((long)nq * nce);
        const int n_loc = int(ch.nodes.size());
        if (qdata) {
          for (int q = 0; q < nq; ++q)
            for (long e = 0; e < nce; ++e) qd[q * nce + e] = qdata[(long)q * ne + e0 + e];
        } else {
          std::vector<double> x((long)dim * n_loc);
          for (int k = 0; k < dim; ++k)
            for (int j = 0; j < n_loc; ++j) x[(long)k * n_loc + j] = coords[k * l_size + ch.nodes[j]];
          if (ref_mass_build(dim, int(nce), P, Q, n_loc, dim * n_loc, all.data(), x.data(), qd.data()) != 0)
            throw std::runtime_error(g_err);
        }
        ch.op = make_mass_op(dim, int(nce), P, Q, 1, 1, n_loc, all, qd);
        ch.u_loc.resize(ch.nodes.size());
      });
    }
    for (auto& t : th) t.join();
    plan = p.release();
  });
  return rc == 0 ? plan : nullptr;
}

int ref_plan_apply(void* handle, const double* u, double* v) {
  return guarded([&] {
    RefPlan& p = *static_cast<RefPlan*>(handle);
    std::vector<std::thread> th;
    for (auto& ch : p.chunks) {
      th.emplace_back([&ch, u] {
        for (size_t j = 0; j < ch.nodes.size(); ++j) ch.u_loc[j] = u[ch.nodes[j]];
        fem::operator_apply(ch.op, ch.u_loc, ch.v_loc);
      });
    }
    for (auto& t : th) t.join();
    std::fill(v, v + p.l_size, 0.0);
    for (auto& ch : p.chunks)
      for (size_t j = 0; j < ch.nodes.size(); ++j) v[ch.nodes[j]] += ch.v_loc[j];
  });
}

void ref_plan_destroy(void* handle) { delete static_cast<RefPlan*>(handle); }

}  // extern "C"
