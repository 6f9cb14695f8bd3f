// dim = 3 mass apply with four elements per CTA ("narrow", sm_100a).
//
// Same per-element algorithm, column roles and arithmetic as
// mass3d_apply_kernel (so the results are the same to the last bit), but a
// CTA takes half of one of the plan's 8-element tiles: 4*Q*Q threads.  At
// high order the one-tile CTA has 8*Q*Q = 512..800 threads and its register
// budget (65536 / threads) forces spills; half the threads leave each thread
// twice the registers.  Two CTAs per plan tile (blockIdx.x = 2*tile + half).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "mass_kernels.cuh"

namespace fem_b200 {

template <int P, int Q>
struct Narrow3D {
  static constexpr int E = 4;   // elements per CTA
  static constexpr int TE = 8;  // elements per plan tile
  static constexpr int NT = E * Q * Q;
  static constexpr int PS1 = plane_stride(P * Q * E, E);  // S1[py][qz*P+px][e]
  static constexpr int PS2 = plane_stride(Q * Q * E, E);  // S2[px][qz*Q+qy][e]
  static constexpr int PS3 = plane_stride(P * Q * E, E);  // S3[qy][qz*P+px][e]
  static constexpr int PS4 = plane_stride(P * P * E, E);  // S4[qz][py*P+px][e]
  static constexpr int SA = cmax(P * PS1, Q * PS3);
  static constexpr int SB = cmax(P * PS2, Q * PS4);
  static constexpr int SMEM = (SA + SB) * 8;
  static constexpr int ES = P * P * P, NQ = Q * Q * Q;
};

template <int P, int Q, int MINB>
__global__ void __launch_bounds__(Narrow3D<P, Q>::NT, MINB) mass3d_apply_narrow_kernel(
    const __grid_constant__ Mat1D<P, Q> m, const int* __restrict__ offs, const double* __restrict__ qd,
    const double* __restrict__ u, double* __restrict__ v, double* __restrict__ ev, int num_elem, int num_comp_run,
    int64_t comp_stride) {
  using L = Narrow3D<P, Q>;
  constexpr int E = L::E, TE = L::TE;
  extern __shared__ __align__(16) double smem[];
  double* sa = smem;
  double* sb = smem + L::SA;
  const int t = threadIdx.x, e = t % E, col = t / E;
  const int64_t tile = blockIdx.x / 2;
  const int el = int(blockIdx.x % 2) * E + e;  // position in the plan tile
  const int64_t eg = tile * TE + el;
  const bool valid = eg < num_elem;
  const bool nodal = col < P * P, mixed = col < P * Q;
  double qv[Q];
  {
    const double* qt = qd + tile * (int64_t(L::NQ) * TE) + col * TE + el;
#pragma unroll
    for (int qx = 0; qx < Q; ++qx) qv[qx] = __ldg(qt + qx * (Q * Q * TE));
  }
  int off[P];
  if (nodal) {
    const int* ot = offs + tile * (int64_t(L::ES) * TE) + col * TE + el;
#pragma unroll
    for (int pz = 0; pz < P; ++pz) off[pz] = __ldg(ot + pz * (P * P * TE));
  }
  for (int k = 0; k < num_comp_run; ++k) {
    const int64_t ks = k * comp_stride;
    if (nodal) {  // z
      double x[P];
#pragma unroll
      for (int pz = 0; pz < P; ++pz) x[pz] = __ldg(u + off[pz] + ks);
      const int px = col % P, py = col / P;
#pragma unroll
      for (int qz = 0; qz < Q; ++qz) {
        double s = 0.0;
#pragma unroll
        for (int pz = 0; pz < P; ++pz) s += m.B[qz * P + pz] * x[pz];
        sa[py * L::PS1 + (qz * P + px) * E + e] = s;
      }
    }
    __syncthreads();
    if (mixed) {  // y
      double y[P];
#pragma unroll
      for (int py = 0; py < P; ++py) y[py] = sa[py * L::PS1 + col * E + e];
      const int px = col % P, qz = col / P;
#pragma unroll
      for (int qy = 0; qy < Q; ++qy) {
        double s = 0.0;
#pragma unroll
        for (int py = 0; py < P; ++py) s += m.B[qy * P + py] * y[py];
        sb[px * L::PS2 + (qz * Q + qy) * E + e] = s;
      }
    }
    __syncthreads();
    {  // x, pointwise mass, x^T
      double w[P];
#pragma unroll
      for (int px = 0; px < P; ++px) w[px] = sb[px * L::PS2 + col * E + e];
      double r[Q];
#pragma unroll
      for (int qx = 0; qx < Q; ++qx) {
        double s = 0.0;
#pragma unroll
        for (int px = 0; px < P; ++px) s += m.B[qx * P + px] * w[px];
        r[qx] = qv[qx] * s;
      }
      const int qy = col % Q, qz = col / Q;
#pragma unroll
      for (int px = 0; px < P; ++px) {
        double s = 0.0;
#pragma unroll
        for (int qx = 0; qx < Q; ++qx) s += m.B[qx * P + px] * r[qx];
        sa[qy * L::PS3 + (qz * P + px) * E + e] = s;
      }
    }
    __syncthreads();
    if (mixed) {  // y^T
      double y[Q];
#pragma unroll
      for (int qy = 0; qy < Q; ++qy) y[qy] = sa[qy * L::PS3 + col * E + e];
      const int px = col % P, qz = col / P;
#pragma unroll
      for (int py = 0; py < P; ++py) {
        double s = 0.0;
#pragma unroll
        for (int qy = 0; qy < Q; ++qy) s += m.B[qy * P + py] * y[qy];
        sb[qz * L::PS4 + (py * P + px) * E + e] = s;
      }
    }
    __syncthreads();
    if (nodal) {  // z^T and the scatter
      double z[Q];
#pragma unroll
      for (int qz = 0; qz < Q; ++qz) z[qz] = sb[qz * L::PS4 + col * E + e];
#pragma unroll
      for (int pz = 0; pz < P; ++pz) {
        double s = 0.0;
#pragma unroll
        for (int qz = 0; qz < Q; ++qz) s += m.B[qz * P + pz] * z[qz];
        if (valid) {
          if (ev)
            ev[(int64_t(k) * L::ES + pz * P * P + col) * num_elem + eg] = s;
          else
            atomicAdd(v + off[pz] + ks, s);
        }
      }
    }
    // the next component's z pass writes buffer A after the barrier that
    // ended its last readers (y^T); its y pass writes B after the next one
  }
}

}  // namespace fem_b200
