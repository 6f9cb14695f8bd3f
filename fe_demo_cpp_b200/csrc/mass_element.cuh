// dim = 3 mass apply with one element per thread (sm_100a), for the lowest
// orders: an element's nodal values and the partial contractions of one
// quadrature plane (qz) at a time fit in registers (P <= 3) -- no barriers
// in the element's work.  Per plane: z, y, x, qdata, x^T, y^T, and the
// plane's z^T terms added to the element's nodal sums (in qz order, as a z^T
// sum).  Lane t of a CTA takes element blockIdx.x * CTA size + t; through the
// plan's tiled layout ([tile][i][e], 8 elements a tile) a warp's loads of one
// local node or point are four contiguous 32-byte pieces.  The contractions
// run in the one-tile kernel's order (z, y, x, x^T, y^T, z^T, each sum in
// ascending index), so results agree with it to the last bit.
//
// Two forms:
//   * mass3d_apply_element_kernel: offsets and qdata read from global memory
//     where they are used (one plane's qdata at a time);
//   * mass3d_apply_element_staged_kernel: the CTA's tiles of offsets and
//     qdata are copied into shared memory first, by 1D bulk copies (no
//     multicast) all issued at the start and completing on one mbarrier, so
//     the only global loads left on an element's path are its gather of u.
//     One wait a CTA, bounded: if it runs out, bit 0 of *status is set, the
//     CTA waits (bounded again) for the copies and returns.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "mass_kernels.cuh"
#include "mass_pipe.cuh"

namespace fem_b200 {

// An element's node offsets: held in registers (the unstaged kernel) ...
template <int ES>
struct OffRegs {
  int o[ES];
  __device__ __forceinline__ int operator[](int i) const { return o[i]; }
};
// ... or read from the shared-memory slot at each use (the staged kernel:
// 27 fewer live registers at P = 3).
struct OffShared {
  const int* p;  // node i at p[i * 8]
  __device__ __forceinline__ int operator[](int i) const { return p[i * 8]; }
};

// One element's apply for every component: off[i] = its node i's L-vector
// offset, qt = its qdata column (entry (qx, qy, qz) at
// qt[(qx * Q * Q + qz * Q + qy) * 8]), global (__ldg) or shared memory.
template <int P, int Q, bool SHARED_QD, class Off>
__device__ __forceinline__ void element_apply(const Mat1D<P, Q>& m, const Off& off,
                                              const double* __restrict__ qt, const double* __restrict__ u,
                                              double* __restrict__ v, double* __restrict__ ev, int num_elem,
                                              int num_comp_run, int64_t comp_stride, int64_t eg) {
  constexpr int TE = 8, ES = P * P * P;
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
          const int qi = (qx * (Q * Q) + qz * Q + qy) * TE;
          r[qx] = (SHARED_QD ? qt[qi] : __ldg(qt + qi)) * s;
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
  OffRegs<ES> off;
  const int* ot = offs + tile * (int64_t(ES) * TE) + el;
#pragma unroll
  for (int i = 0; i < ES; ++i) off.o[i] = __ldg(ot + i * TE);
  element_apply<P, Q, false>(m, off, qd + tile * (int64_t(NQ) * TE) + el, u, v, ev, num_elem, num_comp_run,
                             comp_stride, eg);
}

// Shared-memory layout of the staged kernel for CT threads (CT / 8 tiles):
// per tile a slot of qdata ([point][element], one row of padding where the
// point count is even) and one of offsets ([node][element], likewise), so
// that a warp's four tiles fall in different banks.  Bulk-copy sizes and
// slot strides are multiples of 16 bytes.
template <int P, int Q, int CT>
struct ElemStage {
  static constexpr int TE = 8, ES = P * P * P, NQ = Q * Q * Q, TILES = CT / TE;
  static constexpr int QD_SLOT = (NQ + (NQ % 2 == 0 ? 1 : 0)) * TE;  // doubles
  static constexpr int OFF_SLOT = (ES + (ES % 2 == 0 ? 1 : 0)) * TE;  // ints
  static constexpr int QD_BYTES = TILES * QD_SLOT * 8, OFF_BYTES = TILES * OFF_SLOT * 4;
  static constexpr int SMEM = QD_BYTES + OFF_BYTES + 16;
  static_assert(CT % 32 == 0 && (QD_SLOT * 8) % 16 == 0 && (OFF_SLOT * 4) % 16 == 0, "slot alignment");
};

// l2_ahead > 0: lanes of the first warp prefetch into L2 the qdata and
// offsets of CTA b + l2_ahead's tiles, as the unstaged kernel.  offs and qd
// must be 16-byte aligned and hold whole tiles (the plan's tiled layout).
template <int P, int Q, int CT>
__global__ void __launch_bounds__(CT) mass3d_apply_element_staged_kernel(
    const __grid_constant__ Mat1D<P, Q> m, const int* __restrict__ offs, const double* __restrict__ qd,
    const double* __restrict__ u, double* __restrict__ v, double* __restrict__ ev, int num_elem, int num_comp_run,
    int64_t comp_stride, int64_t l2_ahead, int* __restrict__ status) {
  using L = ElemStage<P, Q, CT>;
  constexpr int TE = L::TE, ES = L::ES, NQ = L::NQ;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* sq = reinterpret_cast<double*>(smem_raw);
  int* so = reinterpret_cast<int*>(smem_raw + L::QD_BYTES);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + L::QD_BYTES + L::OFF_BYTES);
  const int t = threadIdx.x;
  const int64_t n_tiles = (int64_t(num_elem) + TE - 1) / TE;
  const int64_t tile0 = int64_t(blockIdx.x) * L::TILES;
  const int nt = int(n_tiles - tile0 < L::TILES ? n_tiles - tile0 : L::TILES);  // >= 1: grid covers n_tiles
  if (t == 0) {
    pipe::mbar_init(bar, 1);
    pipe::mbar_init_fence();
  }
  __syncthreads();
  if (t == 0) {
    pipe::mbar_expect_tx(bar, uint32_t(nt) * uint32_t(NQ * TE * 8 + ES * TE * 4));
    for (int j = 0; j < nt; ++j) {
      pipe::bulk_copy_g2s(sq + j * L::QD_SLOT, qd + (tile0 + j) * (int64_t(NQ) * TE), NQ * TE * 8, bar);
      pipe::bulk_copy_g2s(so + j * L::OFF_SLOT, offs + (tile0 + j) * (int64_t(ES) * TE), ES * TE * 4, bar);
    }
  }
  if (l2_ahead > 0 && t < 32 && t < 2 * L::TILES) {
    const int64_t tp = (int64_t(blockIdx.x) + l2_ahead) * L::TILES + (t % L::TILES);
    if (tp < n_tiles) {
      if (t < L::TILES)
        l2_prefetch_bulk(qd + tp * (int64_t(NQ) * TE), unsigned(NQ * TE * 8));
      else
        l2_prefetch_bulk(offs + tp * (int64_t(ES) * TE), unsigned(ES * TE * 4));
    }
  }
  if (!__syncthreads_and(pipe::mbar_wait(bar, 0))) {
    if (t == 0) atomicOr(status, 1);
    (void)pipe::mbar_wait(bar, 0);  // bounded: no copy may still target this CTA's shared memory
    return;
  }
  const int64_t eg = tile0 * TE + t;
  if (eg >= num_elem) return;
  const int lt = t / TE, el = t % TE;
  element_apply<P, Q, true>(m, OffShared{so + lt * L::OFF_SLOT + el}, sq + lt * L::QD_SLOT + el, u, v, ev,
                            num_elem, num_comp_run, comp_stride, eg);
}

}  // namespace fem_b200
