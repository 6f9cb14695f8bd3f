// dim = 3 mass apply with one element per thread (sm_100a), for the lowest
// orders: an element's nodal values and the partial contractions of one
// quadrature plane (qz) at a time fit in registers (P <= 3) -- no shared
// memory, no barriers.  Per plane: z, y, x, qdata, x^T, y^T, and the plane's
// z^T terms added to the element's nodal sums (in qz order, as a z^T sum).
// Lane t of a CTA takes element blockIdx.x * 128 + t; through the plan's
// tiled layout ([tile][i][e], 8 elements a tile) a warp's loads of one local
// node or point are four contiguous 32-byte pieces.  The contractions run in
// the one-tile kernel's order (z, y, x, x^T, y^T, z^T, each sum in ascending
// index), so results agree with it to the last bit.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "mass_kernels.cuh"

namespace fem_b200 {

// l2_ahead > 0: the first warp of CTA b has the qdata and offsets of CTA
// b + l2_ahead's 16 tiles prefetched into L2 (one lane a block).
template <int P, int Q>
__global__ void __launch_bounds__(128) mass3d_apply_element_kernel(const __grid_constant__ Mat1D<P, Q> m,
                                                                  const int* __restrict__ offs,
                                                                  const double* __restrict__ qd,
                                                                  const double* __restrict__ u,
                                                                  double* __restrict__ v, double* __restrict__ ev,
                                                                  int num_elem, int num_comp_run,
                                                                  int64_t comp_stride, int64_t l2_ahead = 0) {
  constexpr int TE = 8, ES = P * P * P, NQ = Q * Q * Q;
  if (l2_ahead > 0 && threadIdx.x < 32) {
    const int64_t n_tiles = (int64_t(num_elem) + TE - 1) / TE;
    const int64_t t = (int64_t(blockIdx.x) + l2_ahead) * (128 / TE) + (threadIdx.x & 15);
    if (t < n_tiles) {
      if (threadIdx.x < 16)
        l2_prefetch_bulk(qd + t * (int64_t(NQ) * TE), unsigned(NQ * TE * 8));
      else
        l2_prefetch_bulk(offs + t * (int64_t(ES) * TE), unsigned(ES * TE * 4));
    }
  }
  const int64_t eg = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (eg >= num_elem) return;
  const int64_t tile = eg / TE;
  const int el = int(eg % TE);
  int off[ES];
  const int* ot = offs + tile * (int64_t(ES) * TE) + el;
#pragma unroll
  for (int i = 0; i < ES; ++i) off[i] = __ldg(ot + i * TE);
  const double* qt = qd + tile * (int64_t(NQ) * TE) + el;
  for (int k = 0; k < num_comp_run; ++k) {
    const int64_t ks = k * comp_stride;
    double x[ES], acc[ES];  // the element's u, and its z^T sums
#pragma unroll
    for (int i = 0; i < ES; ++i) x[i] = __ldg(u + off[i] + ks), acc[i] = 0.0;
    // P = 3: one quadrature plane at a time keeps the live set in registers;
    // P = 2: all planes unrolled (86 -> 124 registers, faster: more loads in flight)
#pragma unroll(P == 2 ? Q : 1)
    for (int qz = 0; qz < Q; ++qz) {
      double a1[P][P];
#pragma unroll
      for (int py = 0; py < P; ++py)
#pragma unroll
        for (int px = 0; px < P; ++px) {
          double s = 0.0;
#pragma unroll
          for (int pz = 0; pz < P; ++pz) s += m.B[qz * P + pz] * x[(pz * P + py) * P + px];
          a1[py][px] = s;
        }
      double a2[Q][P];
#pragma unroll
      for (int px = 0; px < P; ++px)
#pragma unroll
        for (int qy = 0; qy < Q; ++qy) {
          double s = 0.0;
#pragma unroll
          for (int py = 0; py < P; ++py) s += m.B[qy * P + py] * a1[py][px];
          a2[qy][px] = s;
        }
      double a3[Q][P];
#pragma unroll
      for (int qy = 0; qy < Q; ++qy) {
        double r[Q];
#pragma unroll
        for (int qx = 0; qx < Q; ++qx) {
          double s = 0.0;
#pragma unroll
          for (int px = 0; px < P; ++px) s += m.B[qx * P + px] * a2[qy][px];
          r[qx] = __ldg(qt + (qx * (Q * Q) + qz * Q + qy) * TE) * s;
        }
#pragma unroll
        for (int px = 0; px < P; ++px) {
          double s = 0.0;
#pragma unroll
          for (int qx = 0; qx < Q; ++qx) s += m.B[qx * P + px] * r[qx];
          a3[qy][px] = s;
        }
      }
#pragma unroll
      for (int px = 0; px < P; ++px)
#pragma unroll
        for (int py = 0; py < P; ++py) {
          double s = 0.0;
#pragma unroll
          for (int qy = 0; qy < Q; ++qy) s += m.B[qy * P + py] * a3[qy][px];
#pragma unroll
          for (int pz = 0; pz < P; ++pz) acc[(pz * P + py) * P + px] += m.B[qz * P + pz] * s;
        }
    }
#pragma unroll
    for (int i = 0; i < ES; ++i) {
      if (ev)
        ev[(int64_t(k) * ES + i) * num_elem + eg] = acc[i];
      else
        atomicAdd(v + off[i] + ks, acc[i]);
    }
  }
}

}  // namespace fem_b200
