// Fused dim-3 tensor basis applies (sm_100a): interp and grad, NoTranspose
// and Transpose, between the reference's E-vector [k][i][e] and Q-vector
// [k][q][e] (grad: [d][k][q][e]) layouts, element innermost over the whole
// mesh (src/tensor-contract.cpp:74-156, include/tensor-contract.hpp:21-33).
//
// One CTA takes 8 consecutive elements with 8*Q*Q threads, the column roles
// of the fused mass apply (mass_kernels.cuh): the contraction along z runs
// in a thread's registers, x and y exchange through padded shared memory, so
// every input value is read once and every output value written once, in
// 64-byte element-contiguous pieces.  No scratch in global memory.
//   NoTranspose: A (px,py) z -> B (px,qz) y -> C (qy,qz) x -> output
//   Transpose:   C (qy,qz) x^T -> F (px,qz) y^T -> G (px,py) z^T -> output
// Grad contracts one axis with G and the others with B: d = 0 is d/dx
// (the first axis of the reference's contraction order), d = 2 is d/dz.
// The transpose of grad sums its three directions into one E-vector and
// overwrites the output (the reference adds into a stale v,
// src/tensor-contract.cpp:115-145; declined).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "mass_kernels.cuh"

namespace fem_b200 {

template <int P, int Q>
struct Basis3D {
  static constexpr int E = 8;
  static constexpr int NT = E * Q * Q;
  static constexpr int PS1 = plane_stride(P * Q * E, E);  // [py][qz*P+px][e]
  static constexpr int PS2 = plane_stride(Q * Q * E, E);  // [px][qz*Q+qy][e]
  static constexpr int PS3 = plane_stride(P * Q * E, E);  // [qy][qz*P+px][e]
  static constexpr int PS4 = plane_stride(P * P * E, E);  // [qz][py*P+px][e]
  static constexpr int S1 = P * PS1, S2 = P * PS2, S3 = Q * PS3, S4 = Q * PS4;
  static constexpr int P3 = P * P * P, Q3 = Q * Q * Q;
  // doubles of shared memory per mode
  static constexpr int SMEM_INTERP = cmax(S1, S3) + cmax(S2, S4);
  static constexpr int SMEM_GRAD_N = 2 * S1 + 3 * S2;
  static constexpr int SMEM_GRAD_T = 3 * S3 + 2 * S4;
  // the grad kernels ask for two resident CTAs where that leaves >= 96
  // registers a thread (left alone they take ~170 at P=5: one CTA per SM)
  static constexpr int MINB_GRAD = 65536 / (2 * NT) >= 96 ? 2 : 1;
};

// The 1D matrices read from a shared-memory copy at every use (like SharedB):
// at high order the compiler would hold all 2*P*Q entries in registers.
struct SharedBG {
  const volatile double* B;
  const volatile double* G;
};

// Runs body(m) with m the kernel's matrix parameter or (SB) a shared copy of
// its B and G made by the whole CTA.
template <bool SB, int P, int Q, class F>
__device__ __forceinline__ void with_matrix(const Mat1D<P, Q>& mp, F&& body) {
  if constexpr (SB) {
    __shared__ double bg[2 * P * Q];
    for (int i = threadIdx.x; i < 2 * P * Q; i += blockDim.x) bg[i] = i < P * Q ? mp.B[i] : mp.G[i - P * Q];
    __syncthreads();
    body(SharedBG{bg, bg + P * Q});
  } else {
    body(mp);
  }
}

// v[k][q][e] = (B x B x B) u[k][i][e].  EO: the even-odd contractions
// (eo_fwd; centro-symmetric B, the parameter matrix, not with SB).
template <int P, int Q, bool SB = false, bool EO = false>
__global__ void __launch_bounds__(Basis3D<P, Q>::NT) basis3d_interp_kernel(const __grid_constant__ Mat1D<P, Q> mp,
                                                                          const double* __restrict__ u,
                                                                          double* __restrict__ v, int num_elem,
                                                                          int num_comp) {
  static_assert(!(SB && EO), "the even-odd folds live in the parameter matrix");
  with_matrix<SB>(mp, [&](const auto& m) {
  using L = Basis3D<P, Q>;
  constexpr int E = L::E;
  extern __shared__ __align__(16) double smem[];
  double* sa = smem;
  double* sb = smem + cmax(L::S1, L::S3);
  const int t = threadIdx.x, e = t % E, col = t / E;
  const int64_t eg = int64_t(blockIdx.x) * E + e, ne = num_elem;
  const bool valid = eg < num_elem;
  for (int k = 0; k < num_comp; ++k) {
    if (col < P * P) {  // A: z
      const int px = col % P, py = col / P;
      double x[P];
#pragma unroll
      for (int pz = 0; pz < P; ++pz)
        x[pz] = valid ? __ldg(u + (int64_t(k) * L::P3 + (pz * P + py) * P + px) * ne + eg) : 0.0;
      if constexpr (EO) {
        double o[Q];
        eo_fwd<P, Q>(m, x, o);
#pragma unroll
        for (int qz = 0; qz < Q; ++qz) sa[py * L::PS1 + (qz * P + px) * E + e] = o[qz];
      } else {
#pragma unroll
        for (int qz = 0; qz < Q; ++qz) {
          double s = 0.0;
#pragma unroll
          for (int pz = 0; pz < P; ++pz) s += m.B[qz * P + pz] * x[pz];
          sa[py * L::PS1 + (qz * P + px) * E + e] = s;
        }
      }
    }
    __syncthreads();
    if (col < P * Q) {  // B: y
      const int px = col % P, qz = col / P;
      double y[P];
#pragma unroll
      for (int py = 0; py < P; ++py) y[py] = sa[py * L::PS1 + col * E + e];
      if constexpr (EO) {
        double o[Q];
        eo_fwd<P, Q>(m, y, o);
#pragma unroll
        for (int qy = 0; qy < Q; ++qy) sb[px * L::PS2 + (qz * Q + qy) * E + e] = o[qy];
      } else {
#pragma unroll
        for (int qy = 0; qy < Q; ++qy) {
          double s = 0.0;
#pragma unroll
          for (int py = 0; py < P; ++py) s += m.B[qy * P + py] * y[py];
          sb[px * L::PS2 + (qz * Q + qy) * E + e] = s;
        }
      }
    }
    __syncthreads();
    {  // C: x, and the output row (qy, qz)
      const int qy = col % Q, qz = col / Q;
      double w[P];
#pragma unroll
      for (int px = 0; px < P; ++px) w[px] = sb[px * L::PS2 + col * E + e];
      double* out = v + (int64_t(k) * L::Q3 + (qz * Q + qy) * Q) * ne + eg;
      if constexpr (EO) {
        double o[Q];
        eo_fwd<P, Q>(m, w, o);
#pragma unroll
        for (int qx = 0; qx < Q; ++qx)
          if (valid) out[qx * ne] = o[qx];
      } else {
#pragma unroll
        for (int qx = 0; qx < Q; ++qx) {
          double s = 0.0;
#pragma unroll
          for (int px = 0; px < P; ++px) s += m.B[qx * P + px] * w[px];
          if (valid) out[qx * ne] = s;
        }
      }
    }
    // the next component's A writes sa, last read by B before the barrier
    // above; its B writes sb after its own barrier, which every C has passed
  }
  });
}

// v[k][i][e] = (B^T x B^T x B^T) u[k][q][e].  EO: the even-odd contractions
// (eo_bwd), as for interp.
template <int P, int Q, bool SB = false, bool EO = false>
__global__ void __launch_bounds__(Basis3D<P, Q>::NT) basis3d_interp_t_kernel(const __grid_constant__ Mat1D<P, Q> mp,
                                                                            const double* __restrict__ u,
                                                                            double* __restrict__ v, int num_elem,
                                                                            int num_comp) {
  static_assert(!(SB && EO), "the even-odd folds live in the parameter matrix");
  with_matrix<SB>(mp, [&](const auto& m) {
  using L = Basis3D<P, Q>;
  constexpr int E = L::E;
  extern __shared__ __align__(16) double smem[];
  double* sa = smem;
  double* sb = smem + cmax(L::S1, L::S3);
  const int t = threadIdx.x, e = t % E, col = t / E;
  const int64_t eg = int64_t(blockIdx.x) * E + e, ne = num_elem;
  const bool valid = eg < num_elem;
  for (int k = 0; k < num_comp; ++k) {
    {  // C^T: x
      const int qy = col % Q, qz = col / Q;
      const double* in = u + (int64_t(k) * L::Q3 + (qz * Q + qy) * Q) * ne + eg;
      double r[Q];
#pragma unroll
      for (int qx = 0; qx < Q; ++qx) r[qx] = valid ? __ldg(in + qx * ne) : 0.0;
      if constexpr (EO) {
        double o[P];
        eo_bwd<P, Q>(m, r, o);
#pragma unroll
        for (int px = 0; px < P; ++px) sa[qy * L::PS3 + (qz * P + px) * E + e] = o[px];
      } else {
#pragma unroll
        for (int px = 0; px < P; ++px) {
          double s = 0.0;
#pragma unroll
          for (int qx = 0; qx < Q; ++qx) s += m.B[qx * P + px] * r[qx];
          sa[qy * L::PS3 + (qz * P + px) * E + e] = s;
        }
      }
    }
    __syncthreads();
    if (col < P * Q) {  // F: y^T
      const int px = col % P, qz = col / P;
      double y[Q];
#pragma unroll
      for (int qy = 0; qy < Q; ++qy) y[qy] = sa[qy * L::PS3 + col * E + e];
      if constexpr (EO) {
        double o[P];
        eo_bwd<P, Q>(m, y, o);
#pragma unroll
        for (int py = 0; py < P; ++py) sb[qz * L::PS4 + (py * P + px) * E + e] = o[py];
      } else {
#pragma unroll
        for (int py = 0; py < P; ++py) {
          double s = 0.0;
#pragma unroll
          for (int qy = 0; qy < Q; ++qy) s += m.B[qy * P + py] * y[qy];
          sb[qz * L::PS4 + (py * P + px) * E + e] = s;
        }
      }
    }
    __syncthreads();
    if (col < P * P) {  // G: z^T, and the output column (px, py)
      double z[Q];
#pragma unroll
      for (int qz = 0; qz < Q; ++qz) z[qz] = sb[qz * L::PS4 + col * E + e];
      double zo[P];
      if constexpr (EO) eo_bwd<P, Q>(m, z, zo);
#pragma unroll
      for (int pz = 0; pz < P; ++pz) {
        double s = 0.0;
        if constexpr (EO) {
          s = zo[pz];
        } else {
#pragma unroll
          for (int qz = 0; qz < Q; ++qz) s += m.B[qz * P + pz] * z[qz];
        }
        if (valid) v[(int64_t(k) * L::P3 + pz * P * P + col) * ne + eg] = s;
      }
    }
  }
  });
}

// v[d][k][q][e] = d/dX_d of u[k][i][e] at the points (G on axis d, B on the others)
template <int P, int Q, bool SB = false>
__global__ void __launch_bounds__(Basis3D<P, Q>::NT, Basis3D<P, Q>::MINB_GRAD) basis3d_grad_kernel(const __grid_constant__ Mat1D<P, Q> mp,
                                                                        const double* __restrict__ u,
                                                                        double* __restrict__ v, int num_elem,
                                                                        int num_comp) {
  with_matrix<SB>(mp, [&](const auto& m) {
  using L = Basis3D<P, Q>;
  constexpr int E = L::E;
  extern __shared__ __align__(16) double smem[];
  double* s1b = smem;
  double* s1g = smem + L::S1;
  double* sbb = smem + 2 * L::S1;
  double* sgb = sbb + L::S2;
  double* sbg = sgb + L::S2;
  const int t = threadIdx.x, e = t % E, col = t / E;
  const int64_t eg = int64_t(blockIdx.x) * E + e, ne = num_elem;
  const bool valid = eg < num_elem;
  const int64_t dstride = int64_t(num_comp) * L::Q3 * ne;
  for (int k = 0; k < num_comp; ++k) {
    if (col < P * P) {  // A: z with B and with G
      const int px = col % P, py = col / P;
      double x[P];
#pragma unroll
      for (int pz = 0; pz < P; ++pz)
        x[pz] = valid ? __ldg(u + (int64_t(k) * L::P3 + (pz * P + py) * P + px) * ne + eg) : 0.0;
#pragma unroll
      for (int qz = 0; qz < Q; ++qz) {
        double sbz = 0.0, sgz = 0.0;
#pragma unroll
        for (int pz = 0; pz < P; ++pz) {
          sbz += m.B[qz * P + pz] * x[pz];
          sgz += m.G[qz * P + pz] * x[pz];
        }
        s1b[py * L::PS1 + (qz * P + px) * E + e] = sbz;
        s1g[py * L::PS1 + (qz * P + px) * E + e] = sgz;
      }
    }
    __syncthreads();
    if (col < P * Q) {  // B: y -> B_y B_z, G_y B_z (from the B_z column), B_y G_z (from the G_z column)
      const int px = col % P, qz = col / P;
      {
        double yb[P];
#pragma unroll
        for (int py = 0; py < P; ++py) yb[py] = s1b[py * L::PS1 + col * E + e];
#pragma unroll
        for (int qy = 0; qy < Q; ++qy) {
          double bb = 0.0, gb = 0.0;
#pragma unroll
          for (int py = 0; py < P; ++py) {
            bb += m.B[qy * P + py] * yb[py];
            gb += m.G[qy * P + py] * yb[py];
          }
          const int idx = px * L::PS2 + (qz * Q + qy) * E + e;
          sbb[idx] = bb, sgb[idx] = gb;
        }
      }
      double yg[P];
#pragma unroll
      for (int py = 0; py < P; ++py) yg[py] = s1g[py * L::PS1 + col * E + e];
#pragma unroll
      for (int qy = 0; qy < Q; ++qy) {
        double bg = 0.0;
#pragma unroll
        for (int py = 0; py < P; ++py) bg += m.B[qy * P + py] * yg[py];
        sbg[px * L::PS2 + (qz * Q + qy) * E + e] = bg;
      }
    }
    __syncthreads();
    {  // C: x -> the three derivatives of row (qy, qz), one direction at a time
      const int qy = col % Q, qz = col / Q;
      double* out = v + (int64_t(k) * L::Q3 + (qz * Q + qy) * Q) * ne + eg;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double* src = d == 0 ? sbb : d == 1 ? sgb : sbg;
        const auto mx = d == 0 ? m.G : m.B;  // d/dx contracts x with G
        double w[P];
#pragma unroll
        for (int px = 0; px < P; ++px) w[px] = src[px * L::PS2 + col * E + e];
#pragma unroll
        for (int qx = 0; qx < Q; ++qx) {
          double s = 0.0;
#pragma unroll
          for (int px = 0; px < P; ++px) s += mx[qx * P + px] * w[px];
          if (valid) out[d * dstride + qx * ne] = s;
        }
      }
    }
  }
  });
}

// v[k][i][e] = sum_d (d/dX_d)^T u[d][k][q][e]
template <int P, int Q, bool SB = false>
__global__ void __launch_bounds__(Basis3D<P, Q>::NT, Basis3D<P, Q>::MINB_GRAD) basis3d_grad_t_kernel(const __grid_constant__ Mat1D<P, Q> mp,
                                                                          const double* __restrict__ u,
                                                                          double* __restrict__ v, int num_elem,
                                                                          int num_comp) {
  with_matrix<SB>(mp, [&](const auto& m) {
  using L = Basis3D<P, Q>;
  constexpr int E = L::E;
  extern __shared__ __align__(16) double smem[];
  double* s0 = smem;
  double* s1 = smem + L::S3;
  double* s2 = smem + 2 * L::S3;
  double* sa = smem + 3 * L::S3;
  double* sz = sa + L::S4;
  const int t = threadIdx.x, e = t % E, col = t / E;
  const int64_t eg = int64_t(blockIdx.x) * E + e, ne = num_elem;
  const bool valid = eg < num_elem;
  const int64_t dstride = int64_t(num_comp) * L::Q3 * ne;
  for (int k = 0; k < num_comp; ++k) {
    {  // C^T: x with G for d = 0, B for d = 1, 2
      const int qy = col % Q, qz = col / Q;
      const double* in = u + (int64_t(k) * L::Q3 + (qz * Q + qy) * Q) * ne + eg;
      double r0[Q], r1[Q], r2[Q];
#pragma unroll
      for (int qx = 0; qx < Q; ++qx) {
        r0[qx] = valid ? __ldg(in + qx * ne) : 0.0;
        r1[qx] = valid ? __ldg(in + dstride + qx * ne) : 0.0;
        r2[qx] = valid ? __ldg(in + 2 * dstride + qx * ne) : 0.0;
      }
#pragma unroll
      for (int px = 0; px < P; ++px) {
        double a = 0.0, b = 0.0, c = 0.0;
#pragma unroll
        for (int qx = 0; qx < Q; ++qx) {
          a += m.G[qx * P + px] * r0[qx];
          b += m.B[qx * P + px] * r1[qx];
          c += m.B[qx * P + px] * r2[qx];
        }
        const int idx = qy * L::PS3 + (qz * P + px) * E + e;
        s0[idx] = a, s1[idx] = b, s2[idx] = c;
      }
    }
    __syncthreads();
    if (col < P * Q) {  // F: y^T -> (B_y^T d0 + G_y^T d1) and B_y^T d2
      const int px = col % P, qz = col / P;
      double y0[Q], y1[Q], y2[Q];
#pragma unroll
      for (int qy = 0; qy < Q; ++qy) {
        const int idx = qy * L::PS3 + col * E + e;
        y0[qy] = s0[idx], y1[qy] = s1[idx], y2[qy] = s2[idx];
      }
#pragma unroll
      for (int py = 0; py < P; ++py) {
        double a = 0.0, c = 0.0;
#pragma unroll
        for (int qy = 0; qy < Q; ++qy) {
          a += m.B[qy * P + py] * y0[qy] + m.G[qy * P + py] * y1[qy];
          c += m.B[qy * P + py] * y2[qy];
        }
        const int idx = qz * L::PS4 + (py * P + px) * E + e;
        sa[idx] = a, sz[idx] = c;
      }
    }
    __syncthreads();
    if (col < P * P) {  // G: z^T -> B_z^T (first) + G_z^T (second)
      double za[Q], zc[Q];
#pragma unroll
      for (int qz = 0; qz < Q; ++qz) {
        za[qz] = sa[qz * L::PS4 + col * E + e];
        zc[qz] = sz[qz * L::PS4 + col * E + e];
      }
#pragma unroll
      for (int pz = 0; pz < P; ++pz) {
        double s = 0.0;
#pragma unroll
        for (int qz = 0; qz < Q; ++qz) s += m.B[qz * P + pz] * za[qz] + m.G[qz * P + pz] * zc[qz];
        if (valid) v[(int64_t(k) * L::P3 + pz * P * P + col) * ne + eg] = s;
      }
    }
    __syncthreads();  // the next component's C^T rewrites s0..s2 (read by F) and F rewrites sa, sz (read by G)
  }
  });
}

}  // namespace fem_b200
