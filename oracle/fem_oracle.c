/*
 * fem_oracle.c -- CPU restatement of fe-demo-cpp's matrix-free mass path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke()
 * entry and the cpu_baseline leg of bench.py may load it; the product library
 * (fe_demo_cpp_b200/) never links, calls or falls back to it.
 *
 * Every function restates one piece of the reference algorithm with the same
 * arithmetic order, so that when compiled as ISO C (no FMA contraction, no
 * -march) its results are bitwise equal to the reference's own CPU build.
 * That equality is checked against fixtures generated from the compiled
 * reference (tests/golden/) and against the known answers in the reference's
 * tests.  Indices are 64-bit here, so the int32 limits of the reference
 * (src/operator.cpp:154, src/tensor-contract.cpp:43) do not apply.
 *
 * Layouts (reference conventions):
 *   E-vector  E[(k*elem_size + i)*num_elem + e]    include/elem-restriction.hpp:49-51
 *   Q-vector  [comp][q][e]; grad output [d][comp][q][e]  include/tensor-contract.hpp:30-33
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef int64_t idx;

enum { ORC_NOTRANSPOSE = 0, ORC_TRANSPOSE = 1 };
enum { ORC_GAUSS = 0, ORC_GAUSS_LOBATTO = 1 };

static idx ipow(idx b, int e) {
  idx r = 1;
  for (int i = 0; i < e; ++i) r *= b;
  return r;
}

/* ------------------------------------------------------------------------ */
/* 1D rules: src/basis.cpp                                                    */
/* ------------------------------------------------------------------------ */

/* Legendre P_n(x) by the three-term recurrence, keeping P_{n-1} in *pm1.
 * The reference starts its recurrence with "P2 = 0" and never enters the loop
 * for n < 2, so P_n(x) reads as 0 there (src/basis.cpp:36-43); kept as is. */
static double legendre_rec(int n, double x, double *pm1) {
  double p0 = 1.0, p1 = x, p2 = 0.0;
  for (int j = 2; j <= n; j++) {
    p2 = ((2.0 * j - 1.0) * x * p1 - (j - 1.0) * p0) / j;
    p0 = p1;
    p1 = p2;
  }
  *pm1 = p0;
  return p2;
}

/* Gauss-Legendre points and weights by Newton on P_Q from Chebyshev guesses.
 * src/basis.cpp:16-68 (gauss_legendre_quadrature). */
int orc_gauss_legendre(int Q, double *x, double *w) {
  if (Q <= 0) return 1;
  const double pi = 4.0 * atan(1.0);
  const double tol = 10 * DBL_EPSILON;
  for (int i = 0; i <= Q / 2; i++) {
    double xi = cos(pi * (2.0 * i + 1.0) / (2.0 * Q));
    double pm1;
    double pq = legendre_rec(Q, xi, &pm1);
    double dp = (xi * pq - pm1) * Q / (xi * xi - 1.0);
    xi = xi - pq / dp;
    for (int k = 0; k < 100 && fabs(pq) > tol; k++) {
      pq = legendre_rec(Q, xi, &pm1);
      dp = (xi * pq - pm1) * Q / (xi * xi - 1.0);
      xi -= pq / dp;
    }
    const double wi = 2.0 / ((1.0 - xi * xi) * dp * dp);
    w[i] = wi;
    w[Q - 1 - i] = wi;
    x[i] = -xi;
    x[Q - 1 - i] = xi;
  }
  return 0;
}

/* Gauss-Lobatto points (and optionally weights): the endpoints plus Newton on
 * the scaled P'_{Q-1} / P''_{Q-1} pair of the reference.
 * src/basis.cpp:81-144 (gauss_lobatto_points). w may be NULL. */
int orc_gauss_lobatto(int Q, double *x, double *w) {
  if (Q <= 1) return 1;
  const double pi = 4.0 * atan(1.0);
  const double tol = 10 * DBL_EPSILON;
  x[0] = -1.0;
  x[Q - 1] = 1.0;
  if (w) {
    const double we = 2.0 / (Q * (Q - 1));
    w[0] = we;
    w[Q - 1] = we;
  }
  for (int i = 1; i <= (Q - 1) / 2; i++) {
    double xi = cos(pi * i / (Q - 1));
    double pm1;
    double p = legendre_rec(Q - 1, xi, &pm1);
    double dp = (xi * p - pm1) * Q / (xi * xi - 1.0);
    double d2p = (2 * xi * dp - (Q * (Q - 1)) * p) / (1.0 - xi * xi);
    xi -= dp / d2p;
    for (int k = 0; k < 100 && fabs(dp) > tol; k++) {
      p = legendre_rec(Q - 1, xi, &pm1);
      dp = (xi * p - pm1) * Q / (xi * xi - 1.0);
      d2p = (2 * xi * dp - (Q * (Q - 1)) * p) / (1.0 - xi * xi);
      xi -= dp / d2p;
    }
    x[i] = -xi;
    x[Q - 1 - i] = xi;
    if (w) {
      const double wi = 2.0 / ((Q * (Q - 1)) * p * p);
      w[i] = wi;
      w[Q - 1 - i] = wi;
    }
  }
  return 0;
}

/* Lagrange interpolation and derivative matrices, row-major [M][P], by
 * Fornberg's recurrence.  src/basis.cpp:156-186 (lagrange_basis_matrix). */
void orc_lagrange_matrices(int P, const double *nodes, int M, const double *pts, double *interp, double *grad) {
  memset(interp, 0, sizeof(double) * (size_t)M * P);
  memset(grad, 0, sizeof(double) * (size_t)M * P);
  for (int i = 0; i < M; i++) {
    double *b = interp + (size_t)i * P, *g = grad + (size_t)i * P;
    double c1 = 1.0, c3 = nodes[0] - pts[i];
    b[0] = 1.0;
    for (int j = 1; j < P; j++) {
      double c2 = 1.0;
      const double c4 = c3;
      c3 = nodes[j] - pts[i];
      for (int k = 0; k < j; k++) {
        const double dx = nodes[j] - nodes[k];
        c2 *= dx;
        if (k == j - 1) {
          g[j] = c1 * (b[k] - c4 * g[k]) / c2;
          b[j] = -c1 * c4 * b[k] / c2;
        }
        g[k] = (c3 * g[k] - b[k]) / dx;
        b[k] = c3 * b[k] / dx;
      }
      c1 = c2;
    }
  }
}

/* TensorBasis::create_tensor_H1_lagrange: GLL nodes, Gauss or GLL quadrature.
 * src/basis.cpp:202-228.  Outputs sized Q, Q, Q*P, Q*P. */
int orc_tensor_h1_lagrange(int dim, int num_comp, int P, int Q, int quad_mode, double *q_ref, double *q_weight,
                           double *interp, double *grad) {
  if (dim < 1 || dim > 3 || num_comp < 1 || num_comp > 3 || P < 2 || Q < 1) return 1;
  double nodes[64];
  if (P > 64) return 1;
  orc_gauss_lobatto(P, nodes, NULL);
  if (quad_mode == ORC_GAUSS) {
    orc_gauss_legendre(Q, q_ref, q_weight);
  } else if (quad_mode == ORC_GAUSS_LOBATTO) {
    if (orc_gauss_lobatto(Q, q_ref, q_weight)) return 1;
  } else {
    return 1;
  }
  orc_lagrange_matrices(P, nodes, Q, q_ref, interp, grad);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Element restriction: src/elem-restriction.cpp                             */
/* ------------------------------------------------------------------------ */

/* Offset gather (NoTranspose) and scatter-add (Transpose), element-outer,
 * component, node-inner loop order.  src/elem-restriction.cpp:64-82.
 * Transpose ADDS into l (it does not zero it). */
void orc_offset_apply(int t_mode, idx num_elem, int elem_size, int num_comp, idx comp_stride, const int *offsets,
                      const double *in, double *out) {
  for (idx e = 0; e < num_elem; e++)
    for (int k = 0; k < num_comp; k++)
      for (int i = 0; i < elem_size; i++) {
        const idx l = (idx)offsets[e * elem_size + i] + k * comp_stride;
        const idx ev = ((idx)k * elem_size + i) * num_elem + e;
        if (t_mode == ORC_NOTRANSPOSE)
          out[ev] = in[l];
        else
          out[l] += in[ev];
      }
}

/* Strided gather / scatter-add with (node, comp, elem) strides.
 * src/elem-restriction.cpp:40-60. */
void orc_strided_apply(int t_mode, idx num_elem, int elem_size, int num_comp, const idx strides[3], const double *in,
                       double *out) {
  for (idx e = 0; e < num_elem; e++)
    for (int k = 0; k < num_comp; k++)
      for (int i = 0; i < elem_size; i++) {
        const idx l = i * strides[0] + k * strides[1] + e * strides[2];
        const idx ev = ((idx)k * elem_size + i) * num_elem + e;
        if (t_mode == ORC_NOTRANSPOSE)
          out[ev] = in[l];
        else
          out[l] += in[ev];
      }
}

/* Multiplicity E^T (E 1) of an offset restriction; mult sized l_size.
 * src/elem-restriction.cpp:215-227. */
void orc_offset_multiplicity(idx num_elem, int elem_size, int num_comp, idx comp_stride, idx l_size,
                             const int *offsets, double *mult) {
  const idx e_size = (idx)num_comp * elem_size * num_elem;
  double *ev = (double *)malloc(sizeof(double) * (size_t)(e_size ? e_size : 1));
  for (idx l = 0; l < l_size; l++) mult[l] = 1.0;
  orc_offset_apply(ORC_NOTRANSPOSE, num_elem, elem_size, num_comp, comp_stride, offsets, mult, ev);
  for (idx l = 0; l < l_size; l++) mult[l] = 0.0;
  orc_offset_apply(ORC_TRANSPOSE, num_elem, elem_size, num_comp, comp_stride, offsets, ev, mult);
  free(ev);
}

/* CSR inverse of the offsets (deterministic scatter map): used L-nodes in
 * increasing order, each row listing t = i + e*elem_size in increasing order.
 * src/cuda/cuda-elem-restriction.cu:149-177 (build_transpose_map).
 * Caller sizes: l_vec_indices and t_offsets hold up to l_size (+1) entries,
 * t_indices num_elem*elem_size.  Returns the number of used nodes. */
idx orc_transpose_map(idx num_elem, int elem_size, idx l_size, const int *offsets, int *l_vec_indices, int *t_offsets,
                      int *t_indices) {
  const idx n_t = num_elem * elem_size;
  idx *node_of = (idx *)malloc(sizeof(idx) * (size_t)(l_size ? l_size : 1));
  for (idx l = 0; l < l_size; l++) node_of[l] = -1;
  for (idx t = 0; t < n_t; t++) node_of[offsets[t]] = 0;
  idx n = 0;
  for (idx l = 0; l < l_size; l++)
    if (node_of[l] == 0) {
      node_of[l] = n;
      l_vec_indices[n++] = (int)l;
    }
  for (idx r = 0; r <= n; r++) t_offsets[r] = 0;
  for (idx t = 0; t < n_t; t++) t_offsets[node_of[offsets[t]] + 1]++;
  for (idx r = 0; r < n; r++) t_offsets[r + 1] += t_offsets[r];
  int *next = (int *)malloc(sizeof(int) * (size_t)(n ? n : 1));
  for (idx r = 0; r < n; r++) next[r] = t_offsets[r];
  for (idx t = 0; t < n_t; t++) t_indices[next[node_of[offsets[t]]]++] = (int)t;
  free(next);
  free(node_of);
  return n;
}

/* ------------------------------------------------------------------------ */
/* Sum-factorised basis action: src/tensor-contract.cpp                      */
/* ------------------------------------------------------------------------ */

/* v[(a*J + j)*C + c] (+)= sum_b t(j,b) u[(a*B + b)*C + c], the sum formed in a
 * local accumulator in increasing b, then added to v.
 * src/tensor-contract.cpp:35-59 (tensor_contract_apply). */
void orc_contract(idx A, int B, idx C, int J, const double *t, int t_mode, int add, const double *u, double *v) {
  const idx s0 = (t_mode == ORC_NOTRANSPOSE) ? B : 1;
  const idx s1 = (t_mode == ORC_NOTRANSPOSE) ? 1 : J;
  if (!add) memset(v, 0, sizeof(double) * (size_t)(A * J * C));
  for (idx a = 0; a < A; ++a)
    for (int j = 0; j < J; ++j)
      for (idx c = 0; c < C; ++c) {
        double sum = 0.0;
        for (int b = 0; b < B; ++b) sum += t[j * s0 + b * s1] * u[(a * B + b) * C + c];
        v[(a * J + j) * C + c] += sum;
      }
}

/* Interp (NoTranspose: nodes -> points; Transpose: points -> nodes), dim
 * chained contractions with ping-pong scratch.  src/tensor-contract.cpp:74-91. */
void orc_interp(int dim, int num_comp, int P1, int Q1, const double *interp_1d, idx num_elem, int t_mode,
                const double *u, double *v) {
  int P = P1, Q = Q1;
  if (t_mode == ORC_TRANSPOSE) {
    P = Q1;
    Q = P1;
  }
  idx pre = num_comp * ipow(P, dim - 1), post = num_elem;
  const idx big = num_comp * ipow(P1 > Q1 ? P1 : Q1, dim) * num_elem;
  double *tmp[2] = {(double *)malloc(sizeof(double) * (size_t)big), (double *)malloc(sizeof(double) * (size_t)big)};
  for (int d = 0; d < dim; d++) {
    const double *src = (d == 0) ? u : tmp[d % 2];
    double *dst = (d == dim - 1) ? v : tmp[(d + 1) % 2];
    orc_contract(pre, P, post, Q, interp_1d, t_mode, 0, src, dst);
    pre /= P;
    post *= Q;
  }
  free(tmp[0]);
  free(tmp[1]);
}

/* Grad.  NoTranspose: v is [d][comp][q][e], block d uses grad_1d on axis d and
 * interp_1d elsewhere.  Transpose: the dim passes ADD into v (which the
 * reference does not clear; callers pass a zeroed v to get A^T w).
 * src/tensor-contract.cpp:111-156. */
void orc_grad(int dim, int num_comp, int P1, int Q1, const double *interp_1d, const double *grad_1d, idx num_elem,
              int t_mode, const double *u, double *v) {
  int P = P1, Q = Q1;
  const idx qblock = num_comp * ipow(Q1, dim) * num_elem; /* one d-axis block at the quadrature points */
  if (t_mode == ORC_TRANSPOSE) {
    P = Q1;
    Q = P1;
  }
  const idx big = num_comp * ipow(P1 > Q1 ? P1 : Q1, dim) * num_elem;
  double *tmp[2] = {(double *)malloc(sizeof(double) * (size_t)big), (double *)malloc(sizeof(double) * (size_t)big)};
  for (int ax = 0; ax < dim; ++ax) {
    idx pre = num_comp * ipow(P, dim - 1), post = num_elem;
    for (int d = 0; d < dim; ++d) {
      const double *mat = (d == ax) ? grad_1d : interp_1d;
      const int last = (d == dim - 1);
      const double *src = (d == 0) ? (t_mode == ORC_TRANSPOSE ? u + ax * qblock : u) : tmp[d % 2];
      double *dst = last ? (t_mode == ORC_TRANSPOSE ? v : v + ax * qblock) : tmp[(d + 1) % 2];
      orc_contract(pre, P, post, Q, mat, t_mode, last && t_mode == ORC_TRANSPOSE, src, dst);
      pre /= P;
      post *= Q;
    }
  }
  free(tmp[0]);
  free(tmp[1]);
}

/* Tensor-product weights, v[q*num_elem + e] = w_z*(w_y*w_x) (that product
 * order).  src/tensor-contract.cpp:169-192 (tensor_basis_apply_weight). */
void orc_weight(int dim, int Q, const double *q_weight_1d, idx num_elem, double *v) {
  for (int d = 0; d < dim; d++) {
    const idx pre = ipow(Q, dim - d - 1), post = ipow(Q, d);
    for (idx i = 0; i < pre; i++)
      for (int j = 0; j < Q; j++)
        for (idx k = 0; k < post; k++) {
          const idx base = ((i * Q + j) * post + k) * num_elem;
          const double wv = q_weight_1d[j] * (d == 0 ? 1 : v[base]);
          for (idx e = 0; e < num_elem; e++) v[base + e] = wv;
        }
  }
}

/* ------------------------------------------------------------------------ */
/* Mass QFunctions: include/qfunctions/mass.hpp                               */
/* ------------------------------------------------------------------------ */

/* qdata = det(J) * w, J laid out [d][c][p].  include/qfunctions/mass.hpp:17-40. */
int orc_build_mass_qf(int dim, idx Q, const double *J, const double *w, double *qdata) {
#define JJ(d, c, p) J[((idx)(d) * dim + (c)) * Q + (p)]
  for (idx p = 0; p < Q; p++) {
    double det;
    switch (dim) {
      case 1: det = JJ(0, 0, p); break;
      case 2: det = JJ(0, 0, p) * JJ(1, 1, p) - JJ(0, 1, p) * JJ(1, 0, p); break;
      case 3:
        det = JJ(0, 0, p) * (JJ(1, 1, p) * JJ(2, 2, p) - JJ(1, 2, p) * JJ(2, 1, p)) -
              JJ(0, 1, p) * (JJ(1, 0, p) * JJ(2, 2, p) - JJ(1, 2, p) * JJ(2, 0, p)) +
              JJ(0, 2, p) * (JJ(1, 0, p) * JJ(2, 1, p) - JJ(1, 1, p) * JJ(2, 0, p));
        break;
      default: return 1;
    }
    qdata[p] = det * w[p];
  }
#undef JJ
  return 0;
}

/* v = qdata * u over the first Q entries only (component 0).
 * include/qfunctions/mass.hpp:45-51. */
void orc_apply_mass_qf(idx Q, const double *u, const double *qdata, double *v) {
  for (idx p = 0; p < Q; p++) v[p] = qdata[p] * u[p];
}

/* ------------------------------------------------------------------------ */
/* Operator: src/operator.cpp:148-182 composed for the two mass operators     */
/* ------------------------------------------------------------------------ */

/* Mass apply with the reference's apply_mass QFunction and an offset
 * restriction for u / v, backend-strided qdata ([q][e]).  out = 0, then the
 * scatter-add.  For num_comp > 1 the reference QFunction writes component 0
 * only and the other components of the Q-vector stay 0 (q_out is freshly
 * resized, src/qfunction.cpp:94-97), so v gets nothing there: kept.
 * comp_only < 0: as the reference.  comp_only = k >= 0: a scalar mass on
 * component k alone (used to restate the vector mass as num_comp scalar
 * applies, each adding into out).  Returns nonzero on a bad argument. */
int orc_mass_apply(int dim, idx num_elem, int P, int Q, int num_comp, idx comp_stride, idx l_size, const int *offsets,
                   const double *interp_1d, const double *qdata, const double *u, double *out, int zero_out,
                   int comp_only) {
  const int es = (int)ipow(P, dim);
  const idx nq = ipow(Q, dim);
  const idx Qtot = nq * num_elem;
  const int nc = comp_only >= 0 ? 1 : num_comp;
  const idx cs = comp_only >= 0 ? 0 : comp_stride;
  const idx shift = comp_only >= 0 ? comp_only * comp_stride : 0;
  double *e_vec = (double *)malloc(sizeof(double) * (size_t)(nc * es * num_elem));
  double *q_u = (double *)malloc(sizeof(double) * (size_t)(nc * Qtot));
  double *q_v = (double *)calloc((size_t)(nc * Qtot), sizeof(double));
  if (!e_vec || !q_u || !q_v) return 2;
  /* gather with a shifted view of u for the single-component restatement */
  orc_offset_apply(ORC_NOTRANSPOSE, num_elem, es, nc, cs, offsets, u + shift, e_vec);
  orc_interp(dim, nc, P, Q, interp_1d, num_elem, ORC_NOTRANSPOSE, e_vec, q_u);
  /* the strided (backend) qdata gather is the identity copy */
  orc_apply_mass_qf(Qtot, q_u, qdata, q_v);
  if (zero_out)
    for (idx l = 0; l < l_size; l++) out[l] = 0.0;
  orc_interp(dim, nc, P, Q, interp_1d, num_elem, ORC_TRANSPOSE, q_v, e_vec);
  orc_offset_apply(ORC_TRANSPOSE, num_elem, es, nc, cs, offsets, e_vec, out + shift);
  free(e_vec);
  free(q_u);
  free(q_v);
  return 0;
}

/* Vector mass (v_k = M u_k for every component) restated as num_comp scalar
 * applies on the shifted component views, as the reference would be driven
 * with its scalar apply_mass. */
int orc_mass_apply_vector(int dim, idx num_elem, int P, int Q, int num_comp, idx comp_stride, idx l_size,
                          const int *offsets, const double *interp_1d, const double *qdata, const double *u,
                          double *out) {
  for (idx l = 0; l < l_size; l++) out[l] = 0.0;
  for (int k = 0; k < num_comp; k++) {
    int rc = orc_mass_apply(dim, num_elem, P, Q, num_comp, comp_stride, l_size, offsets, interp_1d, qdata, u, out, 0,
                            k);
    if (rc) return rc;
  }
  return 0;
}

/* Geometric factors: the build operator with "dx" (Grad of the coordinates,
 * num_comp = dim), "weights" (Weight) and "qdata" (None, backend strided).
 * qdata out is [q][e], sized Q^dim * num_elem.  src/operator.cpp:148-182 with
 * include/qfunctions/mass.hpp:17-40. */
int orc_mass_build(int dim, idx num_elem, int P, int Q, idx comp_stride, const int *offsets, const double *interp_1d,
                   const double *grad_1d, const double *q_weight_1d, const double *coords, double *qdata) {
  const int es = (int)ipow(P, dim);
  const idx nq = ipow(Q, dim);
  const idx Qtot = nq * num_elem;
  double *e_vec = (double *)malloc(sizeof(double) * (size_t)(dim * es * num_elem));
  double *jac = (double *)malloc(sizeof(double) * (size_t)(dim * dim * Qtot));
  double *wts = (double *)malloc(sizeof(double) * (size_t)Qtot);
  double *qd = (double *)malloc(sizeof(double) * (size_t)Qtot);
  if (!e_vec || !jac || !wts || !qd) return 2;
  orc_offset_apply(ORC_NOTRANSPOSE, num_elem, es, dim, comp_stride, offsets, coords, e_vec);
  orc_grad(dim, dim, P, Q, interp_1d, grad_1d, num_elem, ORC_NOTRANSPOSE, e_vec, jac);
  orc_weight(dim, Q, q_weight_1d, num_elem, wts);
  int rc = orc_build_mass_qf(dim, Qtot, jac, wts, qd);
  /* out = 0 then the backend-strided scatter-add: 0 + x */
  for (idx p = 0; p < Qtot; p++) qdata[p] = 0.0 + qd[p];
  free(e_vec);
  free(jac);
  free(wts);
  free(qd);
  return rc;
}
