// Persistent, software-pipelined dim = 3 mass apply (sm_100a).
//
// Same per-element algorithm and thread roles as mass3d_apply_kernel
// (mass_kernels.cuh), reorganised so that no global-memory latency sits on
// the critical path of a tile:
//
//   * each CTA walks tiles blockIdx.x, +gridDim.x, ... (grid = SMs x resident
//     CTAs);
//   * thread 0 copies whole tiles of the plan's tiled offsets / qdata into
//     shared memory with 1D bulk copies (cp.async.bulk, completion on an
//     mbarrier, no multicast): offsets three tiles deep, qdata two;
//   * at phase C of tile i every thread waits for tile i's qdata and tile
//     i+1's offsets (both issued an iteration earlier) and issues the gather of
//     tile i+1's u column into registers, which then lands while phases C, F
//     and G of tile i run.
//
// Every mbarrier wait is bounded; a wait that runs out sets bit 0 of
// *status, the CTA waits (bounded again) for its copies still in flight and
// returns.  The host reads the status word after a synchronising call.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "mass_kernels.cuh"

namespace fem_b200 {

namespace pipe {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// global -> shared bulk copy of `bytes` (16-byte aligned addresses, size a
// multiple of 16), completing `bytes` transactions on `bar`.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// A bounded wait: at most 2^22 polls (each poll may suspend the thread for a
// short, hardware-chosen time), i.e. seconds, never forever.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (uint32_t i = 0; i < (1u << 22); ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

}  // namespace pipe

template <int P, int Q>
struct Pipe3D {
  using M = Mass3D<P, Q>;
  static constexpr int E = M::E;
  static constexpr int NT = M::NT;
  static constexpr int NOFF = 3, NQD = 2;
  static constexpr int OFF_TILE = P * P * P * E;  // ints per tile
  static constexpr int QD_TILE = Q * Q * Q * E;   // doubles per tile
  static constexpr int QD_BYTES = NQD * QD_TILE * 8;
  static constexpr int AB_BYTES = (M::SA + M::SB) * 8;
  static constexpr int OFF_BYTES = NOFF * OFF_TILE * 4;
  static constexpr int SMEM = QD_BYTES + AB_BYTES + OFF_BYTES + 8 * (NOFF + NQD);
};

// EO: the even-odd contractions (eo_fwd / eo_bwd, centro-symmetric B) in
// place of the direct sums, in all six passes.
template <int P, int Q, bool EO = false>
__global__ void __launch_bounds__(Pipe3D<P, Q>::NT) mass3d_apply_pipe_kernel(
    const __grid_constant__ Mat1D<P, Q> m, const int* __restrict__ offs, const double* __restrict__ qd,
    const double* __restrict__ u, double* __restrict__ v, double* __restrict__ ev, int num_elem, int num_comp_run,
    int64_t comp_stride, int64_t n_tiles, int* __restrict__ status) {
  using L = Pipe3D<P, Q>;
  using M = Mass3D<P, Q>;
  constexpr int E = L::E;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* qds = reinterpret_cast<double*>(smem_raw);                        // [NQD][QD_TILE]
  double* sa = reinterpret_cast<double*>(smem_raw + L::QD_BYTES);           // contraction buffer A
  double* sb = sa + M::SA;                                                  // contraction buffer B
  int* ofs = reinterpret_cast<int*>(smem_raw + L::QD_BYTES + L::AB_BYTES);  // [NOFF][OFF_TILE]
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + L::QD_BYTES + L::AB_BYTES + L::OFF_BYTES);
  uint64_t* bar_off = bar;         // [NOFF]
  uint64_t* bar_qd = bar + L::NOFF;  // [NQD]

  const int t = threadIdx.x, e = t % E, col = t / E;
  const bool nodal = col < P * P;
  const bool mixed = col < P * Q;
  const int64_t grid = gridDim.x;
  const int64_t first = blockIdx.x;
  auto tile_of = [&](int64_t it) { return first + it * grid; };
  auto exists = [&](int64_t it) { return tile_of(it) < n_tiles; };

  // issue helpers (thread 0 only)
  auto issue_offs = [&](int64_t it) {
    if (!exists(it)) return;
    const int s = int(it % L::NOFF);
    pipe::mbar_expect_tx(&bar_off[s], L::OFF_TILE * 4);
    pipe::bulk_copy_g2s(ofs + s * L::OFF_TILE, offs + tile_of(it) * L::OFF_TILE, L::OFF_TILE * 4, &bar_off[s]);
  };
  auto issue_qd = [&](int64_t it) {
    if (!exists(it)) return;
    const int s = int(it % L::NQD);
    pipe::mbar_expect_tx(&bar_qd[s], L::QD_TILE * 8);
    pipe::bulk_copy_g2s(qds + s * L::QD_TILE, qd + tile_of(it) * L::QD_TILE, L::QD_TILE * 8, &bar_qd[s]);
  };
  auto wait_offs = [&](int64_t it) {
    return pipe::mbar_wait(&bar_off[it % L::NOFF], uint32_t((it / L::NOFF) & 1));
  };
  auto wait_qd = [&](int64_t it) { return pipe::mbar_wait(&bar_qd[it % L::NQD], uint32_t((it / L::NQD) & 1)); };
  // Error exit: flag it, then wait (bounded) for every copy issued but not yet
  // consumed, so no bulk copy still targets this CTA's shared memory.
  auto fail = [&](int64_t off_lo, int64_t off_hi, int64_t qd_lo, int64_t qd_hi) {
    if (t == 0) atomicOr(status, 1);
    for (int64_t j = off_lo; j <= off_hi; ++j)
      if (exists(j)) (void)wait_offs(j);
    for (int64_t j = qd_lo; j <= qd_hi; ++j)
      if (exists(j)) (void)wait_qd(j);
  };

  if (t == 0) {
    for (int i = 0; i < L::NOFF + L::NQD; ++i) pipe::mbar_init(&bar[i], 1);
    pipe::mbar_init_fence();
  }
  __syncthreads();
  if (t == 0) {
    issue_offs(0);
    issue_offs(1);
    issue_qd(0);
  }
  if (!__syncthreads_and(wait_offs(0))) {
    fail(0, 1, 0, 0);
    return;
  }
  double x[P];
  if (nodal) {
#pragma unroll
    for (int pz = 0; pz < P; ++pz) x[pz] = __ldg(u + ofs[pz * (P * P * E) + col * E + e]);
  }

  for (int64_t it = 0; exists(it); ++it) {
    const int64_t tile = tile_of(it);
    const int* os = ofs + int(it % L::NOFF) * L::OFF_TILE;
    const double* qs = qds + int(it % L::NQD) * L::QD_TILE;
    const int64_t eg = tile * E + e;
    const bool valid = eg < num_elem;
    if (t == 0) {
      issue_offs(it + 2);  // into the slot tile it-1 released
      issue_qd(it + 1);
    }
    for (int k = 0; k < num_comp_run; ++k) {
      const int64_t ks = k * comp_stride;
      if (nodal) {  // phase A: z
        const int px = col % P, py = col / P;
        double o[Q];
        if constexpr (EO) {
          eo_fwd<P, Q>(m, x, o);
        } else {
#pragma unroll
          for (int qz = 0; qz < Q; ++qz) {
            double s = 0.0;
#pragma unroll
            for (int pz = 0; pz < P; ++pz) s += m.B[qz * P + pz] * x[pz];
            o[qz] = s;
          }
        }
#pragma unroll
        for (int qz = 0; qz < Q; ++qz) sa[py * M::PS1 + (qz * P + px) * E + e] = o[qz];
      }
      __syncthreads();
      if (mixed) {  // phase B: y
        double y[P];
#pragma unroll
        for (int py = 0; py < P; ++py) y[py] = sa[py * M::PS1 + col * E + e];
        const int px = col % P, qz = col / P;
        double o[Q];
        if constexpr (EO) {
          eo_fwd<P, Q>(m, y, o);
        } else {
#pragma unroll
          for (int qy = 0; qy < Q; ++qy) {
            double s = 0.0;
#pragma unroll
            for (int py = 0; py < P; ++py) s += m.B[qy * P + py] * y[py];
            o[qy] = s;
          }
        }
#pragma unroll
        for (int qy = 0; qy < Q; ++qy) sb[px * M::PS2 + (qz * Q + qy) * E + e] = o[qy];
      }
      if (k == 0) {  // this tile's qdata and the next tile's offsets (issued an iteration ago)
        bool ok = wait_qd(it);
        if (exists(it + 1)) ok = wait_offs(it + 1) && ok;
        if (!__syncthreads_and(ok)) {
          fail(it + 1, it + 2, it, it + 1);
          return;
        }
      } else {
        __syncthreads();
      }
      // gather the next work item's column now; it lands during C, F and G
      double xn[P];
      if (nodal) {
        if (k + 1 < num_comp_run) {
#pragma unroll
          for (int pz = 0; pz < P; ++pz) xn[pz] = __ldg(u + os[pz * (P * P * E) + col * E + e] + ks + comp_stride);
        } else if (exists(it + 1)) {
          const int* on = ofs + int((it + 1) % L::NOFF) * L::OFF_TILE;
#pragma unroll
          for (int pz = 0; pz < P; ++pz) xn[pz] = __ldg(u + on[pz * (P * P * E) + col * E + e]);
        } else {
#pragma unroll
          for (int pz = 0; pz < P; ++pz) xn[pz] = 0.0;
        }
      }
      {  // phase C: x, pointwise mass, x^T
        double w[P];
#pragma unroll
        for (int px = 0; px < P; ++px) w[px] = sb[px * M::PS2 + col * E + e];
        double r[Q];
        const int qy = col % Q, qz = col / Q;
        if constexpr (EO) {
          double t[Q], o[P];
          eo_fwd<P, Q>(m, w, t);
#pragma unroll
          for (int qx = 0; qx < Q; ++qx) r[qx] = qs[(qx * Q * Q + col) * E + e] * t[qx];
          eo_bwd<P, Q>(m, r, o);
#pragma unroll
          for (int px = 0; px < P; ++px) sa[qy * M::PS3 + (qz * P + px) * E + e] = o[px];
        } else {
#pragma unroll
          for (int qx = 0; qx < Q; ++qx) {
            double s = 0.0;
#pragma unroll
            for (int px = 0; px < P; ++px) s += m.B[qx * P + px] * w[px];
            r[qx] = qs[(qx * Q * Q + col) * E + e] * s;
          }
#pragma unroll
          for (int px = 0; px < P; ++px) {
            double s = 0.0;
#pragma unroll
            for (int qx = 0; qx < Q; ++qx) s += m.B[qx * P + px] * r[qx];
            sa[qy * M::PS3 + (qz * P + px) * E + e] = s;
          }
        }
      }
      __syncthreads();
      if (mixed) {  // phase F: y^T
        double y[Q];
#pragma unroll
        for (int qy = 0; qy < Q; ++qy) y[qy] = sa[qy * M::PS3 + col * E + e];
        const int px = col % P, qz = col / P;
        double o[P];
        if constexpr (EO) {
          eo_bwd<P, Q>(m, y, o);
        } else {
#pragma unroll
          for (int py = 0; py < P; ++py) {
            double s = 0.0;
#pragma unroll
            for (int qy = 0; qy < Q; ++qy) s += m.B[qy * P + py] * y[qy];
            o[py] = s;
          }
        }
#pragma unroll
        for (int py = 0; py < P; ++py) sb[qz * M::PS4 + (py * P + px) * E + e] = o[py];
      }
      __syncthreads();
      if (nodal) {  // phase G: z^T and the scatter
        double z[Q];
#pragma unroll
        for (int qz = 0; qz < Q; ++qz) z[qz] = sb[qz * M::PS4 + col * E + e];
        double o[P];
        if constexpr (EO) {
          eo_bwd<P, Q>(m, z, o);
        } else {
#pragma unroll
          for (int pz = 0; pz < P; ++pz) {
            double s = 0.0;
#pragma unroll
            for (int qz = 0; qz < Q; ++qz) s += m.B[qz * P + pz] * z[qz];
            o[pz] = s;
          }
        }
#pragma unroll
        for (int pz = 0; pz < P; ++pz) {
          const double s = o[pz];
          if (valid) {
            if (ev)
              ev[(int64_t(k) * M::ES + pz * P * P + col) * num_elem + eg] = s;
            else
              atomicAdd(v + os[pz * (P * P * E) + col * E + e] + ks, s);
          }
        }
#pragma unroll
        for (int pz = 0; pz < P; ++pz) x[pz] = xn[pz];
      }
    }
    // Tile done: its offsets/qdata slots and both contraction buffers are free.
    __syncthreads();
  }
}

}  // namespace fem_b200
