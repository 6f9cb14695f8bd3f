// Host set-up of libfem_b200: 1D quadrature rules, Lagrange matrices, tensor
// basis data, restriction validation and the transpose map.  Runs once per
// basis / restriction, never per apply, and needs no GPU.
//
// The 1D rules use the published algorithms the reference uses (Newton on the
// Legendre three-term recurrence from Chebyshev / Chebyshev-Lobatto guesses;
// Fornberg's 1998 recurrence for the Lagrange matrices), with the same
// arithmetic, so the basis matrices come out bitwise equal to the reference's
// (src/basis.cpp:16-228); the device operator then differs from the
// reference only by the kernels' own rounding.
#include <cfloat>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.hpp"
#include "host_setup.hpp"

namespace fem_b200 {

namespace {

// P_n(x) by recurrence; returns P_n and stores P_{n-1}.  For n < 2 the value
// is reported as 0, as the reference's "P2 = 0" start does (src/basis.cpp:36-43).
struct LegendrePair {
  double pn, pn1;
};
LegendrePair legendre(int n, double x) {
  double prev = 1.0, cur = x, next = 0.0;
  for (int j = 2; j <= n; j++) {
    next = ((2.0 * j - 1.0) * x * cur - (j - 1.0) * prev) / j;
    prev = cur;
    cur = next;
  }
  return {next, prev};
}

const double kPi = 4.0 * std::atan(1.0);
const double kTol = 10 * DBL_EPSILON;

}  // namespace

void gauss_legendre(int Q, double* x, double* w) {
  require(Q > 0, "gauss_legendre_quadrature: Q must be positive");
  for (int i = 0; i <= Q / 2; i++) {
    double t = std::cos(kPi * (2.0 * i + 1.0) / (2.0 * Q));
    LegendrePair p = legendre(Q, t);
    double slope = (t * p.pn - p.pn1) * Q / (t * t - 1.0);
    t = t - p.pn / slope;
    for (int it = 0; it < 100 && std::fabs(p.pn) > kTol; it++) {
      p = legendre(Q, t);
      slope = (t * p.pn - p.pn1) * Q / (t * t - 1.0);
      t -= p.pn / slope;
    }
    const double weight = 2.0 / ((1.0 - t * t) * slope * slope);
    x[i] = -t;
    x[Q - 1 - i] = t;
    w[i] = weight;
    w[Q - 1 - i] = weight;
  }
}

void gauss_lobatto(int Q, double* x, double* w) {
  require(Q > 1, "Cannot create Lobatto quadrature with Q <= 1");
  x[0] = -1.0;
  x[Q - 1] = 1.0;
  if (w) w[0] = w[Q - 1] = 2.0 / (Q * (Q - 1));
  for (int i = 1; i <= (Q - 1) / 2; i++) {
    double t = std::cos(kPi * i / (Q - 1));
    LegendrePair p = legendre(Q - 1, t);
    double d1 = (t * p.pn - p.pn1) * Q / (t * t - 1.0);
    double d2 = (2 * t * d1 - (Q * (Q - 1)) * p.pn) / (1.0 - t * t);
    t -= d1 / d2;
    for (int it = 0; it < 100 && std::fabs(d1) > kTol; it++) {
      p = legendre(Q - 1, t);
      d1 = (t * p.pn - p.pn1) * Q / (t * t - 1.0);
      d2 = (2 * t * d1 - (Q * (Q - 1)) * p.pn) / (1.0 - t * t);
      t -= d1 / d2;
    }
    x[i] = -t;
    x[Q - 1 - i] = t;
    if (w) w[i] = w[Q - 1 - i] = 2.0 / ((Q * (Q - 1)) * p.pn * p.pn);
  }
}

void lagrange_matrices(int P, const double* nodes, int M, const double* pts, double* interp, double* grad) {
  std::memset(interp, 0, sizeof(double) * size_t(M) * P);
  std::memset(grad, 0, sizeof(double) * size_t(M) * P);
  for (int m = 0; m < M; m++) {
    double* L = interp + size_t(m) * P;
    double* D = grad + size_t(m) * P;
    double prod_prev = 1.0;                   // prod_{k<j-1} (x_{j-1} - x_k)
    double dist = nodes[0] - pts[m];          // x_j - xi, updated per j
    L[0] = 1.0;
    for (int j = 1; j < P; j++) {
      double prod = 1.0;
      const double dist_prev = dist;
      dist = nodes[j] - pts[m];
      for (int k = 0; k < j; k++) {
        const double gap = nodes[j] - nodes[k];
        prod *= gap;
        if (k == j - 1) {
          D[j] = prod_prev * (L[k] - dist_prev * D[k]) / prod;
          L[j] = -prod_prev * dist_prev * L[k] / prod;
        }
        D[k] = (dist * D[k] - L[k]) / gap;
        L[k] = dist * L[k] / gap;
      }
      prod_prev = prod;
    }
  }
}

BasisData make_basis(int dim, int num_comp, int P, int Q, int quad_mode) {
  require(dim >= 1 && dim <= 3, "create_tensor_H1_lagrange: dim must be 1, 2, or 3");
  require(num_comp >= 1 && num_comp <= 3, "create_tensor_H1_lagrange: num_comp must be 1, 2, or 3");
  require(P >= 2, "create_tensor_H1_lagrange: P_1d must be >= 2");
  require(Q >= 1, "create_tensor_H1_lagrange: Q_1d must be >= 1");
  require(quad_mode == FEM_B200_QUAD_GAUSS || quad_mode == FEM_B200_QUAD_GAUSS_LOBATTO,
          "create_tensor_H1_lagrange: unknown quad_mode");
  BasisData b;
  b.dim = dim;
  b.num_comp = num_comp;
  b.P = P;
  b.Q = Q;
  b.quad_mode = quad_mode;
  std::vector<double> nodes(P);
  gauss_lobatto(P, nodes.data(), nullptr);
  b.q_ref.resize(Q);
  b.q_weight.resize(Q);
  if (quad_mode == FEM_B200_QUAD_GAUSS)
    gauss_legendre(Q, b.q_ref.data(), b.q_weight.data());
  else
    gauss_lobatto(Q, b.q_ref.data(), b.q_weight.data());
  b.interp.resize(size_t(Q) * P);
  b.grad.resize(size_t(Q) * P);
  lagrange_matrices(P, nodes.data(), Q, b.q_ref.data(), b.interp.data(), b.grad.data());
  return b;
}

void check_offset(int num_elem, int elem_size, int num_comp, int comp_stride, int l_size, const int* offsets,
                  int64_t n_offsets) {
  require(num_elem > 0, "elem_restriction_create: num_elem must be positive");
  require(elem_size > 0, "elem_restriction_create: elem_size must be at least 1");
  require(num_comp > 0, "elem_restriction_create: num_comp must be at least 1");
  require(!(num_comp > 1 && comp_stride <= 0),
          "elem_restriction_create: comp_stride must be at least 1 when num_comp > 1");
  require(l_size > 0, "elem_restriction_create: l_size must be positive");
  require(n_offsets == int64_t(num_elem) * elem_size, "elem_restriction_create: offsets size must be num_elem * elem_size");
  require(offsets != nullptr, "elem_restriction_create: offsets is NULL");
  const int64_t span = int64_t(num_comp - 1) * comp_stride;
  for (int64_t t = 0; t < n_offsets; ++t) {
    const int64_t o = offsets[t];
    if (o < 0 || o + span >= l_size)
      throw arg_error(
          "elem_restriction_create: offsets (including component offsets) must be in the range [0, l_size - 1]");
  }
}

void check_strided(int num_elem, int elem_size, int num_comp, int l_size, const int* strides) {
  require(num_elem > 0, "elem_restriction_create_strided: num_elem must be positive");
  require(elem_size > 0, "elem_restriction_create_strided: elem_size must be at least 1");
  require(num_comp > 0, "elem_restriction_create_strided: num_comp must be at least 1");
  require(l_size > 0, "elem_restriction_create_strided: l_size must be positive");
  int64_t s[3] = {num_elem, int64_t(elem_size) * num_elem, 1};
  if (strides) {
    for (int i = 0; i < 3; ++i) {
      require(strides[i] >= 0, "elem_restriction_create_strided: strides must be non-negative");
      s[i] = strides[i];
    }
  }
  const int64_t max_index = int64_t(elem_size - 1) * s[0] + int64_t(num_comp - 1) * s[1] + int64_t(num_elem - 1) * s[2];
  require(max_index < l_size, "elem_restriction_create_strided: strided indices must be in the range [0, l_size - 1]");
}

int transpose_map(int num_elem, int elem_size, int l_size, const int* offsets, int* l_vec_indices, int* t_offsets,
                  int* t_indices) {
  const int64_t n_t = int64_t(num_elem) * elem_size;
  // Mark the used L-nodes, then number them in increasing L order.
  std::vector<int> slot(size_t(l_size), -1);
  for (int64_t t = 0; t < n_t; ++t) slot[offsets[t]] = 0;
  int n = 0;
  for (int l = 0; l < l_size; ++l)
    if (slot[l] == 0) {
      slot[l] = n;
      l_vec_indices[n++] = l;
    }
  // Row lengths, prefix sum, then rows filled in increasing t (so sorted).
  std::fill(t_offsets, t_offsets + n + 1, 0);
  for (int64_t t = 0; t < n_t; ++t) ++t_offsets[slot[offsets[t]] + 1];
  for (int r = 0; r < n; ++r) t_offsets[r + 1] += t_offsets[r];
  std::vector<int> cursor(t_offsets, t_offsets + n);
  for (int64_t t = 0; t < n_t; ++t) t_indices[cursor[slot[offsets[t]]]++] = int(t);
  return n;
}

}  // namespace fem_b200
