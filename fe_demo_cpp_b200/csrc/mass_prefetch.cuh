// Persistent dim = 3 mass apply with prefetch (sm_100a).
//
// Same per-element algorithm, thread roles and contraction buffers as
// mass3d_apply_kernel.  CTAs walk tiles blockIdx.x, +gridDim.x, ... and keep
// the next tiles' inputs moving while the current one computes:
//   * qdata: thread 0 bulk-copies whole tiles (cp.async.bulk, mbarrier
//     completion, no multicast) into a 2-slot shared-memory ring, two tiles
//     ahead; phase C reads it from there;
//   * offsets: the next tile's are loaded into registers at the top of the
//     current tile;
//   * u: the next tile's column is gathered into registers after phase C.
// Waits are bounded (pipe::mbar_wait); one that runs out sets *status, waits
// (bounded) for the copies still in flight and returns.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "mass_kernels.cuh"
#include "mass_pipe.cuh"

namespace fem_b200 {

template <int P, int Q>
struct Prefetch3D {
  using M = Mass3D<P, Q>;
  static constexpr int QD_TILE = M::NQ * M::E;  // doubles per tile
  static constexpr int SMEM = (M::SA + M::SB) * 8 + 2 * QD_TILE * 8 + 2 * 8;
};

template <int P, int Q>
__global__ void __launch_bounds__(Mass3D<P, Q>::NT) mass3d_apply_prefetch_kernel(
    const __grid_constant__ Mat1D<P, Q> m, const int* __restrict__ offs, const double* __restrict__ qd,
    const double* __restrict__ u, double* __restrict__ v, double* __restrict__ ev, int num_elem, int num_comp_run,
    int64_t comp_stride, int n_tiles, int* __restrict__ status) {
  using L = Mass3D<P, Q>;
  constexpr int E = L::E;
  constexpr int OFF_TILE = L::ES * E, QD_TILE = Prefetch3D<P, Q>::QD_TILE;
  extern __shared__ __align__(128) double smem[];
  double* sa = smem;
  double* sb = smem + L::SA;
  double* qring = smem + L::SA + L::SB;  // [2][QD_TILE]
  uint64_t* bar = reinterpret_cast<uint64_t*>(qring + 2 * QD_TILE);
  const int t = threadIdx.x, e = t % E, col = t / E;
  const bool nodal = col < P * P;  // (px, py) = (col % P, col / P)
  const bool mixed = col < P * Q;  // (px, qz) = (col % P, col / P)
  const int* op = offs + col * E + e;  // this thread's view of the tiled offsets
  const int grid = gridDim.x;

  auto issue_qd = [&](int it) {  // thread 0: tile blockIdx.x + it*grid into slot it % 2
    const int tl = int(blockIdx.x) + it * grid;
    if (tl >= n_tiles) return;
    pipe::mbar_expect_tx(&bar[it & 1], QD_TILE * 8);
    pipe::bulk_copy_g2s(qring + (it & 1) * QD_TILE, qd + int64_t(tl) * QD_TILE, QD_TILE * 8, &bar[it & 1]);
  };
  auto drain = [&](int it) {  // error exit: the copies for it and it+1 may still be in flight
    if (t == 0) atomicOr(status, 1);
    for (int j = it; j <= it + 1; ++j)
      if (int(blockIdx.x) + j * grid < n_tiles) (void)pipe::mbar_wait(&bar[j & 1], uint32_t((j >> 1) & 1));
  };

  if (t == 0) {
    pipe::mbar_init(&bar[0], 1);
    pipe::mbar_init(&bar[1], 1);
    pipe::mbar_init_fence();
  }
  __syncthreads();
  if (t == 0) {
    issue_qd(0);
    issue_qd(1);
  }

  int tile = blockIdx.x;
  int off[P];
  double x[P];
  if (nodal) {
#pragma unroll
    for (int pz = 0; pz < P; ++pz) off[pz] = __ldg(op + int64_t(tile) * OFF_TILE + pz * (P * P * E));
#pragma unroll
    for (int pz = 0; pz < P; ++pz) x[pz] = __ldg(u + off[pz]);
  }

  for (int it = 0; tile < n_tiles; tile += grid, ++it) {
    const int next = tile + grid;
    const bool has_next = next < n_tiles;
    const int64_t eg = int64_t(tile) * E + e;
    const bool valid = eg < num_elem;
    const double* qs = qring + (it & 1) * QD_TILE + col * E + e;
    int off_n[P];
#pragma unroll
    for (int pz = 0; pz < P; ++pz) off_n[pz] = 0;
    if (nodal && has_next) {
#pragma unroll
      for (int pz = 0; pz < P; ++pz) off_n[pz] = __ldg(op + int64_t(next) * OFF_TILE + pz * (P * P * E));
    }
    for (int k = 0; k < num_comp_run; ++k) {
      const int64_t ks = k * comp_stride;
      if (nodal) {  // phase A: z
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
      if (mixed) {  // phase B: y
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
      if (k == 0) {  // this tile's qdata (issued two tiles ago) doubles as the B -> C barrier
        if (!__syncthreads_and(pipe::mbar_wait(&bar[it & 1], uint32_t((it >> 1) & 1)))) {
          drain(it);
          return;
        }
      } else {
        __syncthreads();
      }
      {  // phase C: x, pointwise mass, x^T
        double w[P];
#pragma unroll
        for (int px = 0; px < P; ++px) w[px] = sb[px * L::PS2 + col * E + e];
        double r[Q];
#pragma unroll
        for (int qx = 0; qx < Q; ++qx) {
          double s = 0.0;
#pragma unroll
          for (int px = 0; px < P; ++px) s += m.B[qx * P + px] * w[px];
          r[qx] = qs[qx * (Q * Q * E)] * s;
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
      // the next work item's column: lands during phases F and G
      double xn[P];
      if (nodal) {
        if (k + 1 < num_comp_run) {
#pragma unroll
          for (int pz = 0; pz < P; ++pz) xn[pz] = __ldg(u + off[pz] + ks + comp_stride);
        } else if (has_next) {
#pragma unroll
          for (int pz = 0; pz < P; ++pz) xn[pz] = __ldg(u + off_n[pz]);
        } else {
#pragma unroll
          for (int pz = 0; pz < P; ++pz) xn[pz] = 0.0;
        }
      }
      __syncthreads();
      // every thread is past its last read of this tile's qdata slot: refill it
      if (t == 0 && k + 1 == num_comp_run) issue_qd(it + 2);
      if (mixed) {  // phase F: y^T
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
      if (nodal) {  // phase G: z^T and the scatter
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
#pragma unroll
        for (int pz = 0; pz < P; ++pz) x[pz] = xn[pz];
      }
      // the next phase A writes buffer A (last read in phase F, before the
      // barrier above); its phase B writes B after a barrier all G readers pass
    }
    if (nodal) {
#pragma unroll
      for (int pz = 0; pz < P; ++pz) off[pz] = off_n[pz];
    }
  }
}

}  // namespace fem_b200
