// Standalone element-restriction and basis kernels (sm_100a).
//
// Restriction layouts are the reference's (src/elem-restriction.cpp:34-83):
//   E[(k*elem_size + i)*num_elem + e]  <->  L[offsets[e*elem_size + i] + k*comp_stride]
// The offsets are row-major [e][i] (i fastest) while the E-vector has e
// fastest, so a direct thread mapping coalesces only one side (the
// reference's kernels, src/cuda/cuda-elem-restriction.cu:37-67, coalesce the
// offsets).  Here a 32-element x 32-node tile of offsets is staged through
// shared memory, so both the offsets reads and the E-vector accesses are
// contiguous across a warp.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "transpose_scatter.cuh"

namespace fem_b200 {

constexpr int kTile = 32;

// mode 0: gather  E = L[offsets]        (out = E, overwritten)
// mode 1: scatter L[offsets] += E       (atomic)
// mode 2: count   L[offsets] += 1.0     (multiplicity numerator, E unused)
template <int MODE>
__global__ void __launch_bounds__(kTile * 8) offset_tile_kernel(const int* __restrict__ offsets, int num_elem,
                                                               int elem_size, int num_comp, int64_t comp_stride,
                                                               const double* __restrict__ in, double* __restrict__ out) {
  __shared__ int so[kTile][kTile + 1];
  const int i0 = blockIdx.x * kTile;
  const int64_t e0 = int64_t(blockIdx.y) * kTile;
  const int tx = threadIdx.x, ty = threadIdx.y;
  // read: lanes along the node index (contiguous offsets)
  for (int r = ty; r < kTile; r += 8) {
    const int64_t e = e0 + r;
    const int i = i0 + tx;
    so[r][tx] = (e < num_elem && i < elem_size) ? offsets[e * elem_size + i] : -1;
  }
  __syncthreads();
  // write: lanes along the element index (contiguous E-vector)
  const int64_t e = e0 + tx;
  if (e >= num_elem) return;
  for (int c = ty; c < kTile; c += 8) {
    const int i = i0 + c;
    if (i >= elem_size) break;
    const int64_t off = so[tx][c];
    for (int k = 0; k < num_comp; ++k) {
      const int64_t ev = (int64_t(k) * elem_size + i) * num_elem + e;
      const int64_t lv = off + k * comp_stride;
      if (MODE == 0)
        out[ev] = __ldg(in + lv);
      else if (MODE == 1)
        atomicAdd(out + lv, __ldg(in + ev));
      else
        atomicAdd(out + lv, 1.0);
    }
  }
}

// Strided gather (mode 0) / scatter-add (mode 1), one thread per E entry in
// E order; with backend strides both sides are the same contiguous array.
template <int MODE>
__global__ void strided_kernel(int num_elem, int elem_size, int num_comp, int64_t s0, int64_t s1, int64_t s2,
                               const double* __restrict__ in, double* __restrict__ out) {
  const int64_t n = int64_t(num_elem) * elem_size * num_comp;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t e = t % num_elem, rest = t / num_elem;
    const int64_t i = rest % elem_size, k = rest / elem_size;
    const int64_t l = i * s0 + k * s1 + e * s2;
    if (MODE == 0)
      out[t] = in[l];
    else
      out[l] += in[t];
  }
}

// One pass of the batched 1D contraction (the reference's single primitive,
// src/tensor-contract.cpp:35-59):
//   v[(a*J + j)*C + c] (+)= sum_b t(j,b) u[(a*B + b)*C + c]
// one thread per output, c fastest (c runs over the already-contracted axes
// and the elements, so warps read and write contiguous runs).
// t(j,b) = t[j*B + b] (NoTranspose) or t[b*J + j] (Transpose).
__global__ void contract_kernel(int64_t A, int B, int64_t C, int J, const double* __restrict__ t, int transpose,
                                int add, const double* __restrict__ u, double* __restrict__ v) {
  const int64_t n = A * J * C;
  const int64_t s0 = transpose ? 1 : B, s1 = transpose ? J : 1;
  for (int64_t o = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; o < n; o += int64_t(gridDim.x) * blockDim.x) {
    const int64_t c = o % C, rest = o / C;
    const int64_t j = rest % J, a = rest / J;
    const double* up = u + a * B * C + c;
    double s = 0.0;
    for (int b = 0; b < B; ++b) s += __ldg(t + j * s0 + b * s1) * __ldg(up + b * C);
    if (add)
      v[o] += s;
    else
      v[o] = s;
  }
}

// Tensor-product quadrature weights v[q*num_elem + e] = prod_d w[q_d], formed
// in the reference's order w_z*(w_y*w_x) (src/tensor-contract.cpp:169-192).
__global__ void weight_kernel(int dim, int Q, const double* __restrict__ w1, int num_elem, double* __restrict__ v) {
  int nq = 1;
  for (int d = 0; d < dim; ++d) nq *= Q;
  const int64_t n = int64_t(nq) * num_elem;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n; t += int64_t(gridDim.x) * blockDim.x) {
    int q = int(t / num_elem);
    double w = 1.0;
    for (int d = 0; d < dim; ++d) {
      w = w1[q % Q] * (d == 0 ? 1.0 : w);
      q /= Q;
    }
    v[t] = w;
  }
}

// Pointwise mass QFunctions over Q points (include/qfunctions/mass.hpp):
// v = qdata * u (component 0), and qdata = det(J) * w with J laid out
// [d][c][p] and the reference's cofactor expansion.
__global__ void qf_apply_mass_kernel(int64_t Q, const double* __restrict__ u, const double* __restrict__ qdata,
                                     double* __restrict__ v) {
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < Q; p += int64_t(gridDim.x) * blockDim.x)
    v[p] = qdata[p] * u[p];
}

__global__ void qf_build_mass_kernel(int dim, int64_t Q, const double* __restrict__ J, const double* __restrict__ w,
                                     double* __restrict__ qdata) {
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < Q; p += int64_t(gridDim.x) * blockDim.x) {
    auto j = [&](int d, int c) { return J[(int64_t(d) * dim + c) * Q + p]; };
    double det;
    if (dim == 1)
      det = j(0, 0);
    else if (dim == 2)
      det = j(0, 0) * j(1, 1) - j(0, 1) * j(1, 0);
    else
      det = j(0, 0) * (j(1, 1) * j(2, 2) - j(1, 2) * j(2, 1)) - j(0, 1) * (j(1, 0) * j(2, 2) - j(1, 2) * j(2, 0)) +
            j(0, 2) * (j(1, 0) * j(2, 1) - j(1, 1) * j(2, 0));
    qdata[p] = det * w[p];
  }
}

}  // namespace fem_b200
