// dim = 3 mass apply with two elements per thread (sm_100a).
//
// Same per-element algorithm and column roles as mass3d_apply_kernel, but a
// CTA takes 16 elements (two of the plan's 8-element tiles) and thread
// (pair, col) works on the adjacent elements 2*pair and 2*pair+1.  Every
// offsets / qdata load and every shared-memory access is then a 16-byte
// vector (int2 / double2) for both elements at once, and the address and
// index arithmetic is shared by the two.  A quarter-warp is one column of 8
// pairs, i.e. 128 contiguous bytes: shared memory needs no padding to be
// conflict-free.  Only the u gather and the scatter-add stay scalar.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "mass_kernels.cuh"

namespace fem_b200 {

template <int P, int Q>
struct Mass3DX2 {
  static constexpr int E = 16;             // elements per CTA (two 8-element plan tiles)
  static constexpr int TE = 8;             // elements per plan tile
  static constexpr int NPAIR = E / 2;      // threads per column
  static constexpr int NT = NPAIR * Q * Q;
  static constexpr int PS1 = P * Q * E;    // S1[py][qz*P+px][e]
  static constexpr int PS2 = Q * Q * E;    // S2[px][qz*Q+qy][e]
  static constexpr int PS3 = P * Q * E;    // S3[qy][qz*P+px][e]
  static constexpr int PS4 = P * P * E;    // S4[qz][py*P+px][e]
  static constexpr int SA = cmax(P * PS1, Q * PS3);
  static constexpr int SB = cmax(P * PS2, Q * PS4);
  static constexpr int SMEM = (SA + SB) * 8;
  static constexpr int ES = P * P * P, NQ = Q * Q * Q;
};

template <int P, int Q>
__global__ void __launch_bounds__(Mass3DX2<P, Q>::NT) mass3d_apply_x2_kernel(
    const __grid_constant__ Mat1D<P, Q> m, const int* __restrict__ offs, const double* __restrict__ qd,
    const double* __restrict__ u, double* __restrict__ v, double* __restrict__ ev, int num_elem, int num_comp_run,
    int64_t comp_stride) {
  using L = Mass3DX2<P, Q>;
  constexpr int E = L::E, TE = L::TE;
  extern __shared__ __align__(16) double smem[];
  double* sa = smem;
  double* sb = smem + L::SA;
  const int t = threadIdx.x, pr = t % L::NPAIR, col = t / L::NPAIR;
  const int e2 = 2 * pr;                      // first of the thread's two elements within the CTA
  const int64_t tile8 = int64_t(blockIdx.x) * 2 + (e2 / TE);  // plan tile holding both
  const int el = e2 % TE;                     // position inside that plan tile
  const int64_t eg0 = tile8 * TE + el;        // global element of the pair's first
  const bool valid0 = eg0 < num_elem, valid1 = eg0 + 1 < num_elem;
  const bool nodal = col < P * P;
  const bool mixed = col < P * Q;

  double2 qv[Q];
  {
    const double* qt = qd + tile8 * (int64_t(L::NQ) * TE) + col * TE + el;
#pragma unroll
    for (int qx = 0; qx < Q; ++qx) qv[qx] = __ldg(reinterpret_cast<const double2*>(qt + qx * (Q * Q * TE)));
  }
  int2 off[P];
  if (nodal) {
    const int* ot = offs + tile8 * (int64_t(L::ES) * TE) + col * TE + el;
#pragma unroll
    for (int pz = 0; pz < P; ++pz) off[pz] = __ldg(reinterpret_cast<const int2*>(ot + pz * (P * P * TE)));
  }

  for (int k = 0; k < num_comp_run; ++k) {
    const double* uk = u + k * comp_stride;
    if (nodal) {  // phase A: z
      double2 x[P];
#pragma unroll
      for (int pz = 0; pz < P; ++pz) x[pz] = make_double2(__ldg(uk + off[pz].x), __ldg(uk + off[pz].y));
      const int px = col % P, py = col / P;
#pragma unroll
      for (int qz = 0; qz < Q; ++qz) {
        double2 s = make_double2(0.0, 0.0);
#pragma unroll
        for (int pz = 0; pz < P; ++pz) {
          const double b = m.B[qz * P + pz];
          s.x += b * x[pz].x;
          s.y += b * x[pz].y;
        }
        *reinterpret_cast<double2*>(sa + py * L::PS1 + (qz * P + px) * E + e2) = s;
      }
    }
    __syncthreads();
    if (mixed) {  // phase B: y
      double2 y[P];
#pragma unroll
      for (int py = 0; py < P; ++py) y[py] = *reinterpret_cast<const double2*>(sa + py * L::PS1 + col * E + e2);
      const int px = col % P, qz = col / P;
#pragma unroll
      for (int qy = 0; qy < Q; ++qy) {
        double2 s = make_double2(0.0, 0.0);
#pragma unroll
        for (int py = 0; py < P; ++py) {
          const double b = m.B[qy * P + py];
          s.x += b * y[py].x;
          s.y += b * y[py].y;
        }
        *reinterpret_cast<double2*>(sb + px * L::PS2 + (qz * Q + qy) * E + e2) = s;
      }
    }
    __syncthreads();
    {  // phase C: x, pointwise mass, x^T
      double2 w[P];
#pragma unroll
      for (int px = 0; px < P; ++px) w[px] = *reinterpret_cast<const double2*>(sb + px * L::PS2 + col * E + e2);
      double2 r[Q];
#pragma unroll
      for (int qx = 0; qx < Q; ++qx) {
        double2 s = make_double2(0.0, 0.0);
#pragma unroll
        for (int px = 0; px < P; ++px) {
          const double b = m.B[qx * P + px];
          s.x += b * w[px].x;
          s.y += b * w[px].y;
        }
        r[qx] = make_double2(qv[qx].x * s.x, qv[qx].y * s.y);
      }
      const int qy = col % Q, qz = col / Q;
#pragma unroll
      for (int px = 0; px < P; ++px) {
        double2 s = make_double2(0.0, 0.0);
#pragma unroll
        for (int qx = 0; qx < Q; ++qx) {
          const double b = m.B[qx * P + px];
          s.x += b * r[qx].x;
          s.y += b * r[qx].y;
        }
        *reinterpret_cast<double2*>(sa + qy * L::PS3 + (qz * P + px) * E + e2) = s;
      }
    }
    __syncthreads();
    if (mixed) {  // phase F: y^T
      double2 y[Q];
#pragma unroll
      for (int qy = 0; qy < Q; ++qy) y[qy] = *reinterpret_cast<const double2*>(sa + qy * L::PS3 + col * E + e2);
      const int px = col % P, qz = col / P;
#pragma unroll
      for (int py = 0; py < P; ++py) {
        double2 s = make_double2(0.0, 0.0);
#pragma unroll
        for (int qy = 0; qy < Q; ++qy) {
          const double b = m.B[qy * P + py];
          s.x += b * y[qy].x;
          s.y += b * y[qy].y;
        }
        *reinterpret_cast<double2*>(sb + qz * L::PS4 + (py * P + px) * E + e2) = s;
      }
    }
    __syncthreads();
    if (nodal) {  // phase G: z^T and the scatter
      double2 z[Q];
#pragma unroll
      for (int qz = 0; qz < Q; ++qz) z[qz] = *reinterpret_cast<const double2*>(sb + qz * L::PS4 + col * E + e2);
      double* vk = v + k * comp_stride;
#pragma unroll
      for (int pz = 0; pz < P; ++pz) {
        double2 s = make_double2(0.0, 0.0);
#pragma unroll
        for (int qz = 0; qz < Q; ++qz) {
          const double b = m.B[qz * P + pz];
          s.x += b * z[qz].x;
          s.y += b * z[qz].y;
        }
        if (ev) {
          const int64_t row = (int64_t(k) * L::ES + pz * P * P + col) * num_elem;
          if (valid0) ev[row + eg0] = s.x;
          if (valid1) ev[row + eg0 + 1] = s.y;
        } else {
          if (valid0) atomicAdd(vk + off[pz].x, s.x);
          if (valid1) atomicAdd(vk + off[pz].y, s.y);
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace fem_b200
