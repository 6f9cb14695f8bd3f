// dim = 3 mass apply with its 1D contractions on the tensor cores (sm_100a,
// tcgen05.mma kind::tf32, FP32 accumulation in tensor memory), for high
// order: P = 6..8 with Q <= 8.
//
// Each of the six sum-factorised contractions of an 8-element tile
// (src/tensor-contract.cpp:74-91 chains them per axis; here x, y, z, then
// z^T, y^T, x^T) is one batched GEMM: the rows are (element, axis, axis)
// triples -- 8 rows a group, at most 512 rows, i.e. up to four M = 128
// blocks -- the K dimension is the contracted axis (padded to 8) and N = 16
// holds the interpolation matrix twice, as its TF32 part and its TF32
// residual, so that one MMA gives A * B to nearly FP32 accuracy in B.
//   S1 rows (e,pz,py) K=px  <- gather of u (own row)
//   S2 rows (e,pz,qx) K=py  <- S1 output, transposed
//   S3 rows (e,qx,qy) K=pz  <- S2 output, transposed
//   S4 rows (e,qx,qy) K=qz  <- S3 output times qdata (own row)
//   S5 rows (e,qx,pz) K=qy  <- S4 output, transposed
//   S6 rows (e,pz,py) K=qx  <- S5 output, transposed; then the scatter-add
// Operands live in shared memory in the canonical K-major no-swizzle layout
// (tc_ptx.cuh); a thread owns one TMEM lane (row) of each block, reads its
// 16 accumulator columns with tcgen05.ld and writes the next stage's operand
// (16-byte stores for its own row, 4-byte stores for a transpose).
//
// SPLIT (FP32 storage): every operand is written as its TF32 part plus the
// TF32 part of the rest, and two MMAs accumulate hi * [B_hi; B_lo] +
// lo * [B_hi; 0]: the product to about FP32 accuracy ("3xTF32").  Otherwise
// one MMA a block: the operands are rounded to TF32 (relative 2^-11) at every
// stage -- the BF16-storage apply, whose inputs carry 8 bits anyway.
//
// Padding: rows and K entries beyond an axis hold stale but finite values
// from other stages (the buffers are zeroed once per CTA), and the B
// operands are zero beyond the axes, so padding contributes exact zeros.
// Persistent CTAs taking tiles from a ticket, tensor memory allocated once
// per CTA; every wait on the tensor cores is bounded (status bit 2 on
// timeout).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "mass_kernels.cuh"
#include "tc_ptx.cuh"

namespace fem_b200 {

// The B operands of the six stages, as the 16 x 8 K-major shared-memory
// image (tc::kmajor_index): forward [q][p] and backward [p][q], each as
// {B_hi; B_lo} and {B_hi; 0}.
constexpr int kTcOpFloats = 2 * tc::kTcSboBytes / 4;  // 16 rows: two row groups
struct TcMats {
  float op[4][kTcOpFloats];  // 0 fwd split, 1 fwd hi, 2 bwd split, 3 bwd hi
};

template <int P, int Q>
struct TcMass3D {
  static constexpr int E = 8;
  static constexpr int NT = 128;
  static constexpr int ES = P * P * P;
  static constexpr int G = P > Q ? P : Q;
  static constexpr int NBLK = (E * G * 8 + 127) / 128;  // M blocks of the widest stage (<= 4)
  static constexpr int A_FLOATS = NBLK * tc::kTcBlockFloats;  // one operand buffer: NBLK x 128 rows x 8
  static constexpr int TMEM_COLS = NBLK * 16 <= 32 ? 32 : 64;
  // dynamic shared memory: the operand buffers and the B operands, padded so
  // that at most 512 / TMEM_COLS CTAs fit on an SM (tensor memory never runs
  // short, so no CTA waits in its allocation)
  static constexpr int smem(bool split) {
    const int need = ((split ? 2 : 1) * A_FLOATS + 4 * kTcOpFloats) * 4;
    const int cap = 512 / TMEM_COLS;  // CTAs a SM's tensor memory holds
    const int floor_bytes = 233472 / (cap + 1) + 1024;
    return need > floor_bytes ? need : floor_bytes;
  }
  static constexpr int nblk(int g) { return (E * g * 8 + 127) / 128; }
};

template <int P, int Q, bool SPLIT, class S>
__global__ void __launch_bounds__(128) mass3d_apply_tc_kernel(const __grid_constant__ TcMats mats,
                                                             const int* __restrict__ offs, const S* __restrict__ qd,
                                                             const S* __restrict__ u, float* __restrict__ v,
                                                             int num_elem, int num_comp_run, int64_t comp_stride,
                                                             int64_t n_tiles, int* __restrict__ ticket,
                                                             int* __restrict__ status) {
  using L = TcMass3D<P, Q>;
  static_assert(P <= 8 && Q <= 8, "one K = 8 step a contraction");
  extern __shared__ __align__(1024) unsigned char tc_smem_bytes[];
  float* smem = reinterpret_cast<float*>(tc_smem_bytes);
  float* a_hi = smem;
  float* a_lo = smem + L::A_FLOATS;                       // SPLIT only
  float* bops = smem + (SPLIT ? 2 : 1) * L::A_FLOATS;    // 4 operands
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t taddr_s;
  __shared__ int tile_s;
  const int tid = threadIdx.x, warp = tid >> 5;

  for (int i = tid; i < (SPLIT ? 2 : 1) * L::A_FLOATS; i += L::NT) smem[i] = 0.0f;
  for (int i = tid; i < 4 * kTcOpFloats; i += L::NT) bops[i] = mats.op[i / kTcOpFloats][i % kTcOpFloats];
  if (tid == 0) tc::mbar_init(&bar, 1);
  if (warp == 0) tc::tmem_alloc(&taddr_s, L::TMEM_COLS);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = taddr_s;
  const uint32_t lane_base = uint32_t(32 * warp) << 16;
  const uint32_t idesc = tc::idesc_tf32(128, 16);
  const uint32_t a_hi_addr = tc::smem_u32(a_hi), a_lo_addr = tc::smem_u32(a_lo), b_addr = tc::smem_u32(bops);
  uint32_t phase = 0;

  // all threads: operands written -> MMAs over nblk blocks -> accumulators ready
  auto mma_stage = [&](int nblk, int bwd) {
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      constexpr uint32_t op_bytes = kTcOpFloats * 4, blk_bytes = tc::kTcBlockFloats * 4;
      const uint64_t b_split = tc::kmajor_desc(b_addr + uint32_t(bwd) * 2 * op_bytes);
      const uint64_t b_hi = tc::kmajor_desc(b_addr + uint32_t(bwd) * 2 * op_bytes + op_bytes);
      for (int blk = 0; blk < nblk; ++blk) {
        tc::mma_tf32(tmem + uint32_t(blk) * 16, tc::kmajor_desc(a_hi_addr + uint32_t(blk) * blk_bytes), b_split, idesc,
                     0);
        if constexpr (SPLIT)
          tc::mma_tf32(tmem + uint32_t(blk) * 16, tc::kmajor_desc(a_lo_addr + uint32_t(blk) * blk_bytes), b_hi, idesc,
                       1);
      }
      tc::mma_commit(&bar);
    }
    if (!tc::mbar_wait(&bar, phase, 1 << 20)) atomicOr(status, 4);
    phase ^= 1u;
    tc::fence_after_sync();
  };
  // this thread's row of block blk: columns j and j + 8 summed (B_hi and B_lo)
  auto load_row = [&](int blk, float (&d)[8]) {
    float r[16];
    tc::tmem_ld16(tmem + lane_base + uint32_t(blk) * 16, r);
    tc::tmem_wait_ld();
#pragma unroll
    for (int j = 0; j < 8; ++j) d[j] = r[j] + r[j + 8];
  };
  auto put = [&](int R, int k, float x) {
    const int idx = (R >> 7) * tc::kTcBlockFloats + tc::kmajor_index(R & 127, k);
    const float hi = tc::to_tf32(x);
    a_hi[idx] = hi;
    if constexpr (SPLIT) a_lo[idx] = tc::to_tf32(x - hi);
  };
  auto put_row = [&](int R, const float (&x)[8]) {
    const int idx = (R >> 7) * tc::kTcBlockFloats + tc::kmajor_index(R & 127, 0);
    constexpr int K4 = tc::kTcLboBytes / 4;  // the second K half
    float h[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) h[k] = tc::to_tf32(x[k]);
    *reinterpret_cast<float4*>(a_hi + idx) = make_float4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<float4*>(a_hi + idx + K4) = make_float4(h[4], h[5], h[6], h[7]);
    if constexpr (SPLIT) {
      float l[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) l[k] = tc::to_tf32(x[k] - h[k]);
      *reinterpret_cast<float4*>(a_lo + idx) = make_float4(l[0], l[1], l[2], l[3]);
      *reinterpret_cast<float4*>(a_lo + idx + K4) = make_float4(l[4], l[5], l[6], l[7]);
    }
  };
  constexpr int NBP = L::nblk(P), NBQ = L::nblk(Q);

  // tiles from a ticket (zeroed before the launch): a CTA that becomes
  // resident late takes what is left, so the load stays balanced
  for (;;) {
    if (tid == 0) tile_s = atomicAdd(ticket, 1);
    __syncthreads();
    const int64_t tile = tile_s;
    if (tile >= n_tiles) break;
    for (int comp = 0; comp < num_comp_run; ++comp) {
      const int64_t ks = comp * comp_stride;
      // S1: gather, rows (e,pz,py), K = px
#pragma unroll
      for (int blk = 0; blk < NBP; ++blk) {
        const int R = blk * 128 + tid;
        const int e = R / (P * 8), pz = (R / 8) % P, py = R % 8;
        if (R < 64 * P && py < P) {
          float x[8] = {0, 0, 0, 0, 0, 0, 0, 0};
          if (tile * 8 + e < num_elem) {
            const int* ot = offs + (tile * L::ES + (pz * P + py) * P) * 8 + e;
#pragma unroll
            for (int px = 0; px < P; ++px) x[px] = load_as<float>(u + __ldg(ot + px * 8) + ks);
          }
          put_row(R, x);
        }
      }
      mma_stage(NBP, 0);
      // S2: (e,pz,py) x qx -> rows (e,pz,qx), K = py
#pragma unroll
      for (int blk = 0; blk < NBP; ++blk) {
        float d[8];
        load_row(blk, d);
        const int R = blk * 128 + tid;
        const int e = R / (P * 8), pz = (R / 8) % P, py = R % 8;
        if (R < 64 * P && py < P) {
#pragma unroll
          for (int j = 0; j < Q; ++j) put((e * P + pz) * 8 + j, py, d[j]);
        }
      }
      mma_stage(NBP, 0);
      // S3: (e,pz,qx) x qy -> rows (e,qx,qy), K = pz
#pragma unroll
      for (int blk = 0; blk < NBP; ++blk) {
        float d[8];
        load_row(blk, d);
        const int R = blk * 128 + tid;
        const int e = R / (P * 8), pz = (R / 8) % P, qx = R % 8;
        if (R < 64 * P && qx < Q) {
#pragma unroll
          for (int j = 0; j < Q; ++j) put((e * Q + qx) * 8 + j, pz, d[j]);
        }
      }
      mma_stage(NBQ, 0);
      // S4: (e,qx,qy) x qz times qdata -> the same rows, K = qz
#pragma unroll
      for (int blk = 0; blk < NBQ; ++blk) {
        float d[8];
        load_row(blk, d);
        const int R = blk * 128 + tid;
        const int e = R / (Q * 8), qx = (R / 8) % Q, qy = R % 8;
        if (R < 64 * Q && qy < Q) {
          float x[8] = {0, 0, 0, 0, 0, 0, 0, 0};
          if (tile * 8 + e < num_elem) {
            const S* qt = qd + ((tile * Q + qx) * (Q * Q) + qy) * 8 + e;
#pragma unroll
            for (int qz = 0; qz < Q; ++qz) x[qz] = load_as<float>(qt + qz * Q * 8) * d[qz];
          }
          put_row(R, x);
        }
      }
      mma_stage(NBQ, 1);
      // S5: (e,qx,qy) x pz -> rows (e,qx,pz), K = qy
#pragma unroll
      for (int blk = 0; blk < NBQ; ++blk) {
        float d[8];
        load_row(blk, d);
        const int R = blk * 128 + tid;
        const int e = R / (Q * 8), qx = (R / 8) % Q, qy = R % 8;
        if (R < 64 * Q && qy < Q) {
#pragma unroll
          for (int j = 0; j < P; ++j) put((e * Q + qx) * 8 + j, qy, d[j]);
        }
      }
      mma_stage(NBQ, 1);
      // S6: (e,qx,pz) x py -> rows (e,pz,py), K = qx
#pragma unroll
      for (int blk = 0; blk < NBQ; ++blk) {
        float d[8];
        load_row(blk, d);
        const int R = blk * 128 + tid;
        const int e = R / (Q * 8), qx = (R / 8) % Q, pz = R % 8;
        if (R < 64 * Q && pz < P) {
#pragma unroll
          for (int j = 0; j < P; ++j) put((e * P + pz) * 8 + j, qx, d[j]);
        }
      }
      mma_stage(NBP, 1);
      // scatter-add of (e,pz,py) x px
#pragma unroll
      for (int blk = 0; blk < NBP; ++blk) {
        float d[8];
        load_row(blk, d);
        const int R = blk * 128 + tid;
        const int e = R / (P * 8), pz = (R / 8) % P, py = R % 8;
        if (R < 64 * P && py < P && tile * 8 + e < num_elem) {
          const int* ot = offs + (tile * L::ES + (pz * P + py) * P) * 8 + e;
#pragma unroll
          for (int px = 0; px < P; ++px) atomicAdd(v + __ldg(ot + px * 8) + ks, d[px]);
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, L::TMEM_COLS);
}

}  // namespace fem_b200
