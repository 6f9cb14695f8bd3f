// Host set-up routines of libfem_b200 (see host_setup.cpp).
#pragma once
#include <cstdint>
#include <vector>

namespace fem_b200 {

struct BasisData {
  int dim = 0, num_comp = 0, P = 0, Q = 0, quad_mode = 0;
  std::vector<double> q_ref, q_weight;  // Q
  std::vector<double> interp, grad;     // [Q][P]
};

void gauss_legendre(int Q, double* x, double* w);
void gauss_lobatto(int Q, double* x, double* w);
void lagrange_matrices(int P, const double* nodes, int M, const double* pts, double* interp, double* grad);
BasisData make_basis(int dim, int num_comp, int P, int Q, int quad_mode);

void check_offset(int num_elem, int elem_size, int num_comp, int comp_stride, int l_size, const int* offsets,
                  int64_t n_offsets);
void check_strided(int num_elem, int elem_size, int num_comp, int l_size, const int* strides);
int transpose_map(int num_elem, int elem_size, int l_size, const int* offsets, int* l_vec_indices, int* t_offsets,
                  int* t_indices);

}  // namespace fem_b200
