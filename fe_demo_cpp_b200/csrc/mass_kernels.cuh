// Fused sm_100a kernels of the mass operator and its geometric-factor build.
//
// One CTA owns a tile of E consecutive elements.  Lanes run over the tile's
// elements fastest (thread t -> element t % E, "column" t / E), so every
// global stream of the path -- offsets, the L-vector gather, qdata, the
// E-vector -- is read or written by consecutive lanes at consecutive element
// indices, the element-innermost layout of the reference
// (include/elem-restriction.hpp:49-51).  For dim = 3 a thread owns one
// column along the last axis in registers; the contractions along the other
// axes exchange through shared memory, padded so that a half-warp never has a
// bank conflict.  The 1D matrices live in the kernel's parameter bank
// (__grid_constant__), so each FMA reads its matrix entry as a constant
// operand: no shared-memory or register traffic for B or G.
//
// Algorithm (per element): the reference's operator_apply on the mass
// QFunction (src/operator.cpp:148-182): gather (src/elem-restriction.cpp:64-72),
// dim contractions with interp_1d (src/tensor-contract.cpp:74-91),
// v = qdata * u (include/qfunctions/mass.hpp:45-51), the transposed
// contractions, scatter-add (src/elem-restriction.cpp:73-82).  The axis order
// of the contractions differs (z first here, x first there), so results agree
// with the reference to rounding, not bitwise.
#pragma once
#include <cuda_runtime.h>

#include <cuda_bf16.h>

#include <type_traits>

#include <cstdint>

#include "apply_ext.cuh"

namespace fem_b200 {

// A value of storage type S as compute type T (S = T, or BF16 storage of u
// and qdata under FP32 arithmetic).
template <class T, class S>
__device__ __forceinline__ T as_t(S x) {
  if constexpr (std::is_same<S, __nv_bfloat16>::value)
    return T(__bfloat162float(x));
  else
    return T(x);
}
template <class T, class S>
__device__ __forceinline__ T load_as(const S* p) {
  return as_t<T>(__ldg(p));
}

template <int P, int Q, class T = double>
struct Mat1D {
  T B[Q * P];  // interp_1d, row-major [q][p]
  T G[Q * P];  // grad_1d (the diagonal kernels carry interp_1d squared here)
  T W[Q];      // q_weight_1d
  // Even-odd folds of B for the even-odd contractions (eo_fwd / eo_bwd),
  // filled by fill_eo: for q < ceil(Q/2), j < P/2,
  //   Ep[q][j] = (B[q][j] + B[q][P-1-j]) / 2,  Em[q][j] = (B[q][j] - B[q][P-1-j]) / 2.
  T Ep[((Q + 1) / 2) * (P / 2)];
  T Em[(Q / 2) * (P / 2)];
};

// Fills Mat1D::Ep / Em from B (host).
template <int P, int Q, class T>
void fill_eo(Mat1D<P, Q, T>& m) {
  constexpr int HP = P / 2;
  for (int q = 0; q < (Q + 1) / 2; ++q)
    for (int j = 0; j < HP; ++j) m.Ep[q * HP + j] = (m.B[q * P + j] + m.B[q * P + P - 1 - j]) / 2;
  for (int q = 0; q < Q / 2; ++q)
    for (int j = 0; j < HP; ++j) m.Em[q * HP + j] = (m.B[q * P + j] - m.B[q * P + P - 1 - j]) / 2;
}

// Even-odd forms of the 1D contractions, for a centro-symmetric B
// (B[Q-1-q][P-1-p] = B[q][p]: Lagrange bases on symmetric nodes evaluated at
// symmetric points, e.g. GLL nodes and Gauss points).  With xe = x[j] +
// x[P-1-j], xo = x[j] - x[P-1-j], the outputs q and Q-1-q are E + O and E - O
// with E = sum Ep xe (+ the middle column for odd P) and O = sum Em xo: about
// 17% fewer multiply-adds at P = 5, Q = 6, and dependency chains of P/2
// instead of P.  The sums are regrouped, so results agree with the direct
// contraction to rounding, not bitwise.
// out[q] = sum_p B[q][p] x[p]
template <int P, int Q, class T, class M>
__device__ __forceinline__ void eo_fwd(const M& m, const T (&x)[P], T (&out)[Q]) {
  constexpr int HP = P / 2, HQ = Q / 2;
  T xe[HP], xo[HP];
#pragma unroll
  for (int j = 0; j < HP; ++j) xe[j] = x[j] + x[P - 1 - j], xo[j] = x[j] - x[P - 1 - j];
#pragma unroll
  for (int q = 0; q < (Q + 1) / 2; ++q) {
    T e = (P & 1) ? m.B[q * P + HP] * x[HP] : T(0);
#pragma unroll
    for (int j = 0; j < HP; ++j) e += m.Ep[q * HP + j] * xe[j];
    if (q < HQ) {
      T o = T(0);
#pragma unroll
      for (int j = 0; j < HP; ++j) o += m.Em[q * HP + j] * xo[j];
      out[q] = e + o;
      out[Q - 1 - q] = e - o;
    } else {
      out[q] = e;  // the middle point of an odd Q: its odd part vanishes
    }
  }
}

// out[p] = sum_q B[q][p] y[q]
template <int P, int Q, class T, class M>
__device__ __forceinline__ void eo_bwd(const M& m, const T (&y)[Q], T (&out)[P]) {
  constexpr int HP = P / 2, HQ = Q / 2;
  T ye[HQ], yo[HQ];
#pragma unroll
  for (int i = 0; i < HQ; ++i) ye[i] = y[i] + y[Q - 1 - i], yo[i] = y[i] - y[Q - 1 - i];
#pragma unroll
  for (int p = 0; p < HP; ++p) {
    T e = (Q & 1) ? m.B[HQ * P + p] * y[HQ] : T(0);
#pragma unroll
    for (int i = 0; i < HQ; ++i) e += m.Ep[i * HP + p] * ye[i];
    T o = T(0);
#pragma unroll
    for (int i = 0; i < HQ; ++i) o += m.Em[i * HP + p] * yo[i];
    out[p] = e + o;
    out[P - 1 - p] = e - o;
  }
  if constexpr (P & 1) {  // the middle node of an odd P: its odd part vanishes
    T e = (Q & 1) ? m.B[HQ * P + HP] * y[HQ] : T(0);
#pragma unroll
    for (int i = 0; i < HQ; ++i) e += m.B[i * P + HP] * ye[i];
    out[HP] = e;
  }
}

// The interpolation matrix read from a shared-memory copy at every use (the
// volatile read keeps the compiler from holding all P*Q entries in registers
// for the whole tile, which at high order costs resident CTAs).  Same values
// and arithmetic order as reading Mat1D::B, so the same results to the bit.
template <class T>
struct SharedB {
  const volatile T* B;
  const volatile T* Ep = nullptr;  // shared copies of Mat1D::Ep / Em (the even-odd contractions)
  const volatile T* Em = nullptr;
};

// Shared-memory plane stride for a tile of 8 elements: an odd multiple of 8
// doubles, so two adjacent columns of a half-warp land 8 doubles (16 banks)
// apart.  Tiles of >= 16 elements need no padding (a half-warp is one column).
__host__ __device__ constexpr int plane_stride(int n, int E) {
  return (E >= 16 || (n / 8) % 2 == 1) ? n : n + 8;
}
__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }

// ---------------------------------------------------------------------------
// Tiled layouts owned by a mass plan (built once at create time)
//   offsets  [tile][i][e]           i = local node (x fastest)
//   qdata    [tile][qx][col][e]     col = q / Q  (the other axes), q = qx + Q*col
// Elements past num_elem are padding (offset 0, qdata 0) and never scattered.
// ---------------------------------------------------------------------------
static __global__ void tile_offsets_kernel(const int* __restrict__ offsets, int num_elem, int elem_size, int E,
                                    int64_t n_out, int* __restrict__ out) {
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n_out; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t el = t % E, rest = t / E;
    const int64_t i = rest % elem_size, tile = rest / elem_size;
    const int64_t e = tile * E + el;
    out[t] = e < num_elem ? offsets[e * elem_size + i] : 0;
  }
}

static __global__ void tile_qdata_kernel(const double* __restrict__ qdata, int num_elem, int Q, int nq, int E, int64_t n_out,
                                  double* __restrict__ out) {
  const int ncol = nq / Q;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n_out; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t el = t % E, rest = t / E;
    const int64_t col = rest % ncol, rest2 = rest / ncol;
    const int64_t qx = rest2 % Q, tile = rest2 / Q;
    const int64_t e = tile * E + el;
    const int64_t q = qx + Q * col;
    out[t] = e < num_elem ? qdata[q * num_elem + e] : 0.0;
  }
}

// ---------------------------------------------------------------------------
// dim = 3 fused apply.  E = 8 elements, 8*Q*Q threads.
//   phase A  (px,py):  gather z-column, contract z          -> S1
//   phase B  (px,qz):  contract y                            -> S2
//   phase C  (qy,qz):  contract x, times qdata, contract x^T -> S3
//   phase F  (px,qz):  contract y^T                          -> S4
//   phase G  (px,py):  contract z^T, scatter-add (or E-vector store)
// S1, S3 share buffer A and S2, S4 buffer B; each array is laid out so its
// reader's columns are contiguous, and its planes are padded (plane_stride).
// ---------------------------------------------------------------------------
template <int P, int Q>
struct Mass3D {
  static constexpr int E = 8;
  static constexpr int NT = E * Q * Q;
  static constexpr int PS1 = plane_stride(P * Q * E, E);  // S1[py][qz*P+px][e]
  static constexpr int PS2 = plane_stride(Q * Q * E, E);  // S2[px][qz*Q+qy][e]
  static constexpr int PS3 = plane_stride(P * Q * E, E);  // S3[qy][qz*P+px][e]
  static constexpr int PS4 = plane_stride(P * P * E, E);  // S4[qz][py*P+px][e]
  static constexpr int SA = cmax(P * PS1, Q * PS3);
  static constexpr int SB = cmax(P * PS2, Q * PS4);
  static constexpr int SMEM = (SA + SB) * 8;
  static constexpr int ES = P * P * P, NQ = Q * Q * Q;
  // resident CTAs per SM the register-capped variant asks for: 5, or what
  // shared memory (227 KB) and threads (2048) allow (8 at P = 4, with the
  // even-odd contractions, measured 1.096 ms against 0.973 ms at 5)
  static constexpr int MINB_OCC = cmax(1, (5 < 232448 / SMEM ? 5 : 232448 / SMEM) < 2048 / NT
                                              ? (5 < 232448 / SMEM ? 5 : 232448 / SMEM)
                                              : 2048 / NT);
};

// Bulk L2 prefetch (no multicast; cp.async.bulk.prefetch wants a 16-byte
// aligned start and a size that is a multiple of 16 bytes).
__device__ __forceinline__ void l2_prefetch_bulk(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// One thread's L2 prefetch of a tile's qdata and offsets blocks, laid out
// [tile][...][e] (NQ * E values and ES * E offsets a tile).  Each block
// starts at a multiple of its size from a 256-byte aligned allocation, and
// both sizes are multiples of 16 bytes (E = 8 or 32 elements a tile).
template <int ES, int NQ, int E, class S>
__device__ __forceinline__ void prefetch_tile_l2(const int* offs, const S* qd, int64_t tile) {
  static_assert((NQ * E * sizeof(S)) % 16 == 0 && (ES * E * 4) % 16 == 0, "bulk prefetch sizes");
  l2_prefetch_bulk(qd + tile * (int64_t(NQ) * E), unsigned(NQ * E * sizeof(S)));
  l2_prefetch_bulk(offs + tile * (int64_t(ES) * E), unsigned(ES * E * 4));
}

// One 8-element tile of the 3D fused apply (the body of mass3d_apply_kernel and
// of the batched kernels): sa / sb are the CTA's shared buffers A and B.
template <int P, int Q, class T, class Ext, int NCB, class S = T, class M = Mat1D<P, Q, T>, bool EO = false,
          bool GROUPED = false>
__device__ __forceinline__ void mass3d_tile(const M& m, T* __restrict__ sa, T* __restrict__ sb,
                                            const int* __restrict__ offs, const S* __restrict__ qd,
                                            const S* __restrict__ u, T* __restrict__ v, T* __restrict__ ev,
                                            int num_elem, int num_comp_run, int64_t comp_stride,
                                            const Ext& ext, const int64_t tile, double& dsum, int t_in = -1) {
  using L = Mass3D<P, Q>;
  constexpr int E = L::E;
  // GROUPED: t_in is the thread's index in a group of L::NT running this
  // tile (a block may run several tiles, or have threads to spare: t_in >=
  // L::NT only takes part in the barriers); otherwise the block is the tile
  const int t = GROUPED ? t_in : int(threadIdx.x), e = t % E, col = t / E;
  const bool live = GROUPED ? t < L::NT : true;
  const bool nodal = col < P * P;  // (px, py) = (col % P, col / P)
  const bool mixed = col < P * Q;  // (px, qz) = (col % P, col / P)
  const int64_t eg = tile * E + e;
  const bool valid = eg < num_elem;
  // Prefetch: this thread's qdata row (qy, qz) = (col % Q, col / Q), all qx.
  T qv[Q];
  if (live) {
    const S* qt = qd + tile * (int64_t(L::NQ) * E) + col * E + e;
#pragma unroll
    for (int qx = 0; qx < Q; ++qx) qv[qx] = load_as<T>(qt + qx * (Q * Q * E));
  }
  int off[P];
  if (nodal) {
    const int* ot = offs + tile * (int64_t(L::ES) * E) + col * E + e;
#pragma unroll
    for (int pz = 0; pz < P; ++pz) off[pz] = __ldg(ot + pz * (P * P * E));
  }

  for (int k0 = 0; k0 < num_comp_run; k0 += NCB) {
    if (nodal) {  // phase A
      T x[NCB][P];
#pragma unroll
      for (int pz = 0; pz < P; ++pz) {
        T sc = T(1);
        // the solver's diagonal is the same for every component of a node
        if constexpr (Ext::kScale) sc = __ldg(ext.scale + off[pz]);
#pragma unroll
        for (int c = 0; c < NCB; ++c) {
          x[c][pz] = load_as<T>(u + off[pz] + (k0 + c) * comp_stride);
          if constexpr (Ext::kScale) x[c][pz] *= sc;
        }
      }
      const int px = col % P, py = col / P;
#pragma unroll
      for (int c = 0; c < NCB; ++c) {
        if constexpr (EO) {
          T o[Q];
          eo_fwd<P, Q>(m, x[c], o);
#pragma unroll
          for (int qz = 0; qz < Q; ++qz) sa[c * L::SA + py * L::PS1 + (qz * P + px) * E + e] = o[qz];
        } else {
#pragma unroll
          for (int qz = 0; qz < Q; ++qz) {
            T s = T(0);
#pragma unroll
            for (int pz = 0; pz < P; ++pz) s += m.B[qz * P + pz] * x[c][pz];
            sa[c * L::SA + py * L::PS1 + (qz * P + px) * E + e] = s;
          }
        }
      }
    }
    __syncthreads();
    if (mixed) {  // phase B
      const int px = col % P, qz = col / P;
#pragma unroll
      for (int c = 0; c < NCB; ++c) {
        T y[P];
#pragma unroll
        for (int py = 0; py < P; ++py) y[py] = sa[c * L::SA + py * L::PS1 + col * E + e];
        if constexpr (EO) {
          T o[Q];
          eo_fwd<P, Q>(m, y, o);
#pragma unroll
          for (int qy = 0; qy < Q; ++qy) sb[c * L::SB + px * L::PS2 + (qz * Q + qy) * E + e] = o[qy];
        } else {
#pragma unroll
          for (int qy = 0; qy < Q; ++qy) {
            T s = T(0);
#pragma unroll
            for (int py = 0; py < P; ++py) s += m.B[qy * P + py] * y[py];
            sb[c * L::SB + px * L::PS2 + (qz * Q + qy) * E + e] = s;
          }
        }
      }
    }
    __syncthreads();
    if (live) {  // phase C: x, pointwise mass, x^T
      const int qy = col % Q, qz = col / Q;
#pragma unroll
      for (int c = 0; c < NCB; ++c) {
        T w[P];
#pragma unroll
        for (int px = 0; px < P; ++px) w[px] = sb[c * L::SB + px * L::PS2 + col * E + e];
        T r[Q];
        if constexpr (EO) {
          T t[Q];
          eo_fwd<P, Q>(m, w, t);
#pragma unroll
          for (int qx = 0; qx < Q; ++qx) {
            r[qx] = qv[qx] * t[qx];
            if constexpr (Ext::kDot) dsum += double(r[qx]) * double(t[qx]);
          }
          T o[P];
          eo_bwd<P, Q>(m, r, o);
#pragma unroll
          for (int px = 0; px < P; ++px) sa[c * L::SA + qy * L::PS3 + (qz * P + px) * E + e] = o[px];
        } else {
#pragma unroll
          for (int qx = 0; qx < Q; ++qx) {
            T s = T(0);
#pragma unroll
            for (int px = 0; px < P; ++px) s += m.B[qx * P + px] * w[px];
            r[qx] = qv[qx] * s;
            if constexpr (Ext::kDot) dsum += double(r[qx]) * double(s);
          }
#pragma unroll
          for (int px = 0; px < P; ++px) {
            T s = T(0);
#pragma unroll
            for (int qx = 0; qx < Q; ++qx) s += m.B[qx * P + px] * r[qx];
            sa[c * L::SA + qy * L::PS3 + (qz * P + px) * E + e] = s;
          }
        }
      }
    }
    __syncthreads();
    if (mixed) {  // phase F: y^T
      const int px = col % P, qz = col / P;
#pragma unroll
      for (int c = 0; c < NCB; ++c) {
        T y[Q];
#pragma unroll
        for (int qy = 0; qy < Q; ++qy) y[qy] = sa[c * L::SA + qy * L::PS3 + col * E + e];
        if constexpr (EO) {
          T o[P];
          eo_bwd<P, Q>(m, y, o);
#pragma unroll
          for (int py = 0; py < P; ++py) sb[c * L::SB + qz * L::PS4 + (py * P + px) * E + e] = o[py];
        } else {
#pragma unroll
          for (int py = 0; py < P; ++py) {
            T s = T(0);
#pragma unroll
            for (int qy = 0; qy < Q; ++qy) s += m.B[qy * P + py] * y[qy];
            sb[c * L::SB + qz * L::PS4 + (py * P + px) * E + e] = s;
          }
        }
      }
    }
    __syncthreads();
    if (nodal) {  // phase G: z^T and the scatter
#pragma unroll
      for (int c = 0; c < NCB; ++c) {
        T z[Q];
#pragma unroll
        for (int qz = 0; qz < Q; ++qz) z[qz] = sb[c * L::SB + qz * L::PS4 + col * E + e];
        const int64_t ks = (k0 + c) * comp_stride;
        T zo[P];
        if constexpr (EO) eo_bwd<P, Q>(m, z, zo);
#pragma unroll
        for (int pz = 0; pz < P; ++pz) {
          T s = T(0);
          if constexpr (EO) {
            s = zo[pz];
          } else {
#pragma unroll
            for (int qz = 0; qz < Q; ++qz) s += m.B[qz * P + pz] * z[qz];
          }
          if (valid) {
            if (ev)
              ev[(int64_t(k0 + c) * L::ES + pz * P * P + col) * num_elem + eg] = s;
            else
              atomicAdd(v + off[pz] + ks, s);
          }
        }
      }
    }
    // The next components' phase A writes buffer A, whose last readers
    // (phase F) finished before the barrier above; their phase B writes
    // buffer B only after the next barrier, which every phase-G reader has
    // passed.  The same holds between one tile and the next.
  }
}

// num_comp_run components are processed (1 for the reference apply_mass,
// which only touches component 0); component k reads/writes at + k*comp_stride.
// ev == nullptr: atomic scatter-add into v.  ev != nullptr: the element
// contributions are stored in the E-vector layout [k][i][e] (deterministic
// mode; a transpose-map reduction follows).
// MINB > 1 asks for MINB resident CTAs per SM (a register cap), trading a
// little spilling for more warps to hide memory latency; MINB = 0 leaves the
// register count to ptxas (fewer registers than MINB = 1 at P <= 7).  Ext adds the
// solver's scaled gather and u^T M u reduction (apply_ext.cuh); with it the
// kernel is persistent (tiles blockIdx.x, +gridDim.x, ...) so that each CTA
// reduces once.  NCB > 1 runs NCB components through each phase together
// (num_comp_run a multiple of NCB, shared memory NCB * (SA + SB)): more loads
// in flight and a third of the barriers for a 3-component field.  SB: the
// contractions read the interpolation matrix from a shared-memory copy
// (SharedB) instead of the kernel parameter.  l2_ahead > 0 (one CTA per tile):
// CTA b first has the qdata and offsets of tile b + l2_ahead prefetched into
// L2, so that the CTA which takes that tile about a wave later finds them
// there instead of waiting on DRAM (P = 5: 1.05x sustained); persistent (Ext
// with a reduction), l2_ahead != 0: each CTA prefetches its next tile.
template <int P, int Q, int MINB = 1, class T = double, class Ext = ApplyPlain, int NCB = 1, class S = T,
          bool SB = false, bool EO = false>
__global__ void __launch_bounds__(Mass3D<P, Q>::NT, MINB) mass3d_apply_kernel(
    const __grid_constant__ Mat1D<P, Q, T> m, const int* __restrict__ offs, const S* __restrict__ qd,
    const S* __restrict__ u, T* __restrict__ v, T* __restrict__ ev, int num_elem, int num_comp_run,
    int64_t comp_stride, const Ext ext, int64_t l2_ahead = 0) {
  using L = Mass3D<P, Q>;
  constexpr int E = L::E;
  extern __shared__ __align__(16) unsigned char smem_bytes[];
  T* sa = reinterpret_cast<T*>(smem_bytes);
  T* sb = sa + NCB * L::SA;
  if constexpr (Ext::kDot) {
    if (ext.st->done) return;  // uniform: the solve has stopped
  }
  if constexpr (!Ext::kDot) {
    const int64_t ahead = blockIdx.x + l2_ahead;
    if (l2_ahead > 0 && threadIdx.x == 0 && ahead < (int64_t(num_elem) + E - 1) / E)
      prefetch_tile_l2<L::ES, L::NQ, E, S>(offs, qd, ahead);
  }
  double dsum = 0.0;
  auto run = [&](const auto& mat) {
    if constexpr (Ext::kDot) {  // persistent: one reduction per CTA
      const int64_t n_tiles = (int64_t(num_elem) + E - 1) / E;
      for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        // l2_ahead != 0: this CTA's next tile (a wave ahead) into L2 first
        if (l2_ahead != 0 && threadIdx.x == 0 && tile + gridDim.x < n_tiles)
          prefetch_tile_l2<L::ES, L::NQ, E, S>(offs, qd, tile + gridDim.x);
        mass3d_tile<P, Q, T, Ext, NCB, S, std::decay_t<decltype(mat)>, EO>(mat, sa, sb, offs, qd, u, v, ev, num_elem,
                                                                           num_comp_run, comp_stride, ext, tile, dsum);
      }
      double dv[1] = {dsum};
      grid_sum<1>(dv, ext.part, &ext.st->ticket, [&](const double* tot) { cg_after_apply(ext.st, tot[0]); });
    } else {
      mass3d_tile<P, Q, T, Ext, NCB, S, std::decay_t<decltype(mat)>, EO>(mat, sa, sb, offs, qd, u, v, ev, num_elem,
                                                                         num_comp_run, comp_stride, ext, blockIdx.x,
                                                                         dsum);
    }
  };
  if constexpr (SB) {
    constexpr int NP = ((Q + 1) / 2) * (P / 2), NM = (Q / 2) * (P / 2);
    __shared__ T b_s[P * Q + (EO ? NP + NM : 0)];
    for (int i = threadIdx.x; i < P * Q; i += blockDim.x) b_s[i] = m.B[i];
    if constexpr (EO) {
      for (int i = threadIdx.x; i < NP; i += blockDim.x) b_s[P * Q + i] = m.Ep[i];
      for (int i = threadIdx.x; i < NM; i += blockDim.x) b_s[P * Q + NP + i] = m.Em[i];
    }
    __syncthreads();
    if constexpr (EO)
      run(SharedB<T>{b_s, b_s + P * Q, b_s + P * Q + NP});
    else
      run(SharedB<T>{b_s});
  } else {
    run(m);
  }
}

// ---------------------------------------------------------------------------
// dim = 3 geometric factors: qdata[q][e] = det(dx/dX) * w_q.
// Same thread roles; per coordinate component c the z pass makes B- and
// G-contracted columns, the y pass the three mixed products, the x pass the
// three derivatives d x_c / d X_d, kept in registers until the determinant.
// ---------------------------------------------------------------------------
template <int P, int Q>
struct Build3D {
  static constexpr int E = 8;
  static constexpr int NT = E * Q * Q;
  static constexpr int PS1 = plane_stride(P * Q * E, E);
  static constexpr int PS2 = plane_stride(Q * Q * E, E);
  static constexpr int S1 = P * PS1;  // one array [py][qz*P+px][e]
  static constexpr int S2 = P * PS2;  // one array [px][qz*Q+qy][e]
  static constexpr int SMEM = (2 * S1 + 3 * S2) * 8;
};

template <int P, int Q>
__global__ void __launch_bounds__(Build3D<P, Q>::NT, 1) mass3d_build_kernel(
    const __grid_constant__ Mat1D<P, Q> m, const int* __restrict__ offsets, const double* __restrict__ x,
    int64_t comp_stride, double* __restrict__ qdata, int num_elem) {
  using L = Build3D<P, Q>;
  constexpr int E = L::E;
  extern __shared__ double smem[];
  double* s1b = smem;
  double* s1g = smem + L::S1;
  double* sbb = smem + 2 * L::S1;
  double* sgb = sbb + L::S2;
  double* sbg = sgb + L::S2;
  const int t = threadIdx.x, e = t % E, col = t / E;
  const int64_t eg = int64_t(blockIdx.x) * E + e;
  const bool valid = eg < num_elem;
  const bool nodal = col < P * P, mixed = col < P * Q;
  double J[3][3][Q];  // J[d][c][qx] = d x_c / d X_d at (qx, qy, qz)

#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (nodal) {
      double xz[P];
      const int* orow = offsets + (valid ? eg : 0) * int64_t(P * P * P) + col;
#pragma unroll
      for (int pz = 0; pz < P; ++pz) xz[pz] = __ldg(x + __ldg(orow + pz * P * P) + c * comp_stride);
      const int px = col % P, py = col / P;
#pragma unroll
      for (int qz = 0; qz < Q; ++qz) {
        double sb = 0.0, sg = 0.0;
#pragma unroll
        for (int pz = 0; pz < P; ++pz) {
          sb += m.B[qz * P + pz] * xz[pz];
          sg += m.G[qz * P + pz] * xz[pz];
        }
        s1b[py * L::PS1 + (qz * P + px) * E + e] = sb;
        s1g[py * L::PS1 + (qz * P + px) * E + e] = sg;
      }
    }
    __syncthreads();
    if (mixed) {
      double yb[P], yg[P];
#pragma unroll
      for (int py = 0; py < P; ++py) {
        yb[py] = s1b[py * L::PS1 + col * E + e];
        yg[py] = s1g[py * L::PS1 + col * E + e];
      }
      const int px = col % P, qz = col / P;
#pragma unroll
      for (int qy = 0; qy < Q; ++qy) {
        double bb = 0.0, gb = 0.0, bg = 0.0;
#pragma unroll
        for (int py = 0; py < P; ++py) {
          bb += m.B[qy * P + py] * yb[py];
          gb += m.G[qy * P + py] * yb[py];
          bg += m.B[qy * P + py] * yg[py];
        }
        const int idx = px * L::PS2 + (qz * Q + qy) * E + e;
        sbb[idx] = bb;
        sgb[idx] = gb;
        sbg[idx] = bg;
      }
    }
    __syncthreads();
    {
      double wbb[P], wgb[P], wbg[P];
#pragma unroll
      for (int px = 0; px < P; ++px) {
        const int idx = px * L::PS2 + col * E + e;
        wbb[px] = sbb[idx];
        wgb[px] = sgb[idx];
        wbg[px] = sbg[idx];
      }
#pragma unroll
      for (int qx = 0; qx < Q; ++qx) {
        double d0 = 0.0, d1 = 0.0, d2 = 0.0;
#pragma unroll
        for (int px = 0; px < P; ++px) {
          d0 += m.G[qx * P + px] * wbb[px];
          d1 += m.B[qx * P + px] * wgb[px];
          d2 += m.B[qx * P + px] * wbg[px];
        }
        J[0][c][qx] = d0;
        J[1][c][qx] = d1;
        J[2][c][qx] = d2;
      }
    }
    __syncthreads();
  }
  if (!valid) return;
  const int qy = col % Q, qz = col / Q;
#pragma unroll
  for (int qx = 0; qx < Q; ++qx) {
    // include/qfunctions/mass.hpp:27-31, the same cofactor expansion
    const double det = J[0][0][qx] * (J[1][1][qx] * J[2][2][qx] - J[1][2][qx] * J[2][1][qx]) -
                       J[0][1][qx] * (J[1][0][qx] * J[2][2][qx] - J[1][2][qx] * J[2][0][qx]) +
                       J[0][2][qx] * (J[1][0][qx] * J[2][1][qx] - J[1][1][qx] * J[2][0][qx]);
    const double w = m.W[qz] * (m.W[qy] * m.W[qx]);  // src/tensor-contract.cpp:169-192 product order
    qdata[(int64_t((qz * Q + qy) * Q + qx)) * num_elem + eg] = det * w;
  }
}

// ---------------------------------------------------------------------------
// dim = 2 fused apply.  E = 32 elements, 32*Q threads; a thread owns a column
// along y.  phase A (px): gather, contract y -> S1[px][qy][e];
// phase C (qy): contract x, times qdata, contract x^T -> S3[qy][px][e];
// phase G (px): contract y^T, scatter.
// ---------------------------------------------------------------------------
template <int P, int Q>
struct Mass2D {
  static constexpr int E = 32;
  static constexpr int NT = E * Q;
  static constexpr int S1 = P * Q * E, S3 = Q * P * E;
  static constexpr int SMEM = (S1 + S3) * 8;
  static constexpr int ES = P * P, NQ = Q * Q;
};

// One 32-element tile of the 2D fused apply: s1 / s3 the CTA's shared buffers.
template <int P, int Q, class T, class Ext, class S = T, class M = Mat1D<P, Q, T>, bool EO = false,
          bool GROUPED = false>
__device__ __forceinline__ void mass2d_tile(const M& m, T* __restrict__ s1, T* __restrict__ s3,
                                            const int* __restrict__ offs, const S* __restrict__ qd,
                                            const S* __restrict__ u, T* __restrict__ v, T* __restrict__ ev,
                                            int num_elem, int num_comp_run, int64_t comp_stride,
                                            const Ext& ext, const int64_t tile, double& dsum, int t_in = -1) {
  using L = Mass2D<P, Q>;
  constexpr int E = L::E;
  // GROUPED, t_in: as mass3d_tile's (t_in >= L::NT: barriers only)
  const int t = GROUPED ? t_in : int(threadIdx.x), e = t % E, col = t / E;
  const bool live = GROUPED ? t < L::NT : true;
  const bool nodal = col < P;
  const int64_t eg = tile * E + e;
  const bool valid = eg < num_elem;
  T qv[Q];
  if (live) {
    const S* qt = qd + tile * (int64_t(L::NQ) * E) + col * E + e;
#pragma unroll
    for (int qx = 0; qx < Q; ++qx) qv[qx] = load_as<T>(qt + qx * (Q * E));
  }
  int off[P];
  if (nodal) {
    const int* ot = offs + tile * (int64_t(L::ES) * E) + col * E + e;
#pragma unroll
    for (int py = 0; py < P; ++py) off[py] = __ldg(ot + py * (P * E));
  }
  for (int k = 0; k < num_comp_run; ++k) {
    const int64_t ks = k * comp_stride;
    if (nodal) {
      T x[P];
#pragma unroll
      for (int py = 0; py < P; ++py) {
        x[py] = load_as<T>(u + off[py] + ks);
        if constexpr (Ext::kScale) x[py] *= __ldg(ext.scale + off[py]);
      }
      if constexpr (EO) {
        T o[Q];
        eo_fwd<P, Q>(m, x, o);
#pragma unroll
        for (int qy = 0; qy < Q; ++qy) s1[(col * Q + qy) * E + e] = o[qy];
      } else {
#pragma unroll
        for (int qy = 0; qy < Q; ++qy) {
          T s = T(0);
#pragma unroll
          for (int py = 0; py < P; ++py) s += m.B[qy * P + py] * x[py];
          s1[(col * Q + qy) * E + e] = s;
        }
      }
    }
    __syncthreads();
    if (live) {
      T w[P];
#pragma unroll
      for (int px = 0; px < P; ++px) w[px] = s1[(px * Q + col) * E + e];
      T r[Q];
      if constexpr (EO) {
        T t[Q];
        eo_fwd<P, Q>(m, w, t);
#pragma unroll
        for (int qx = 0; qx < Q; ++qx) {
          r[qx] = qv[qx] * t[qx];
          if constexpr (Ext::kDot) dsum += double(r[qx]) * double(t[qx]);
        }
        T o[P];
        eo_bwd<P, Q>(m, r, o);
#pragma unroll
        for (int px = 0; px < P; ++px) s3[(col * P + px) * E + e] = o[px];
      } else {
#pragma unroll
        for (int qx = 0; qx < Q; ++qx) {
          T s = T(0);
#pragma unroll
          for (int px = 0; px < P; ++px) s += m.B[qx * P + px] * w[px];
          r[qx] = qv[qx] * s;
          if constexpr (Ext::kDot) dsum += double(r[qx]) * double(s);
        }
#pragma unroll
        for (int px = 0; px < P; ++px) {
          T s = T(0);
#pragma unroll
          for (int qx = 0; qx < Q; ++qx) s += m.B[qx * P + px] * r[qx];
          s3[(col * P + px) * E + e] = s;
        }
      }
    }
    __syncthreads();
    if (nodal) {
      T z[Q];
#pragma unroll
      for (int qy = 0; qy < Q; ++qy) z[qy] = s3[(qy * P + col) * E + e];
      T zo[P];
      if constexpr (EO) eo_bwd<P, Q>(m, z, zo);
#pragma unroll
      for (int py = 0; py < P; ++py) {
        T s = T(0);
        if constexpr (EO) {
          s = zo[py];
        } else {
#pragma unroll
          for (int qy = 0; qy < Q; ++qy) s += m.B[qy * P + py] * z[qy];
        }
        if (valid) {
          if (ev)
            ev[(int64_t(k) * L::ES + py * P + col) * num_elem + eg] = s;
          else
            atomicAdd(v + off[py] + ks, s);
        }
      }
    }
    __syncthreads();
  }
}

// SB: the contractions read the interpolation matrix from a shared-memory
// copy (SharedB) instead of the kernel parameter.  l2_ahead > 0 (one CTA per
// tile): CTA b has tile b + l2_ahead's qdata and offsets prefetched into L2,
// as the 3D kernel.
template <int P, int Q, class T = double, class Ext = ApplyPlain, class S = T, int MINB = 0, bool SB = false,
          bool EO = false>
__global__ void __launch_bounds__(Mass2D<P, Q>::NT, MINB) mass2d_apply_kernel(
    const __grid_constant__ Mat1D<P, Q, T> m, const int* __restrict__ offs, const S* __restrict__ qd,
    const S* __restrict__ u, T* __restrict__ v, T* __restrict__ ev, int num_elem, int num_comp_run,
    int64_t comp_stride, const Ext ext, int64_t l2_ahead = 0) {
  using L = Mass2D<P, Q>;
  constexpr int E = L::E;
  extern __shared__ __align__(16) unsigned char smem_bytes[];
  T* s1 = reinterpret_cast<T*>(smem_bytes);
  T* s3 = s1 + L::S1;
  if constexpr (Ext::kDot) {
    if (ext.st->done) return;
  }
  if constexpr (!Ext::kDot) {
    const int64_t ahead = blockIdx.x + l2_ahead;
    if (l2_ahead > 0 && threadIdx.x == 0 && ahead < (int64_t(num_elem) + E - 1) / E)
      prefetch_tile_l2<L::ES, L::NQ, E, S>(offs, qd, ahead);
  }
  double dsum = 0.0;
  auto run = [&](const auto& mat) {
    if constexpr (Ext::kDot) {  // persistent, one reduction per CTA
      const int64_t n_tiles = (int64_t(num_elem) + E - 1) / E;
      for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x)
        mass2d_tile<P, Q, T, Ext, S, std::decay_t<decltype(mat)>, EO>(mat, s1, s3, offs, qd, u, v, ev, num_elem,
                                                                      num_comp_run, comp_stride, ext, tile, dsum);
      double dv[1] = {dsum};
      grid_sum<1>(dv, ext.part, &ext.st->ticket, [&](const double* tot) { cg_after_apply(ext.st, tot[0]); });
    } else {
      mass2d_tile<P, Q, T, Ext, S, std::decay_t<decltype(mat)>, EO>(mat, s1, s3, offs, qd, u, v, ev, num_elem,
                                                                    num_comp_run, comp_stride, ext, blockIdx.x, dsum);
    }
  };
  if constexpr (SB) {
    __shared__ T b_s[P * Q];
    for (int i = threadIdx.x; i < P * Q; i += blockDim.x) b_s[i] = m.B[i];
    __syncthreads();
    run(SharedB<T>{b_s});
  } else {
    run(m);
  }
}

template <int P, int Q>
__global__ void __launch_bounds__(32 * Q) mass2d_build_kernel(const __grid_constant__ Mat1D<P, Q> m,
                                                             const int* __restrict__ offsets,
                                                             const double* __restrict__ x, int64_t comp_stride,
                                                             double* __restrict__ qdata, int num_elem) {
  constexpr int E = 32;
  __shared__ double s1b[P * Q * E], s1g[P * Q * E];
  const int t = threadIdx.x, e = t % E, col = t / E;
  const int64_t eg = int64_t(blockIdx.x) * E + e;
  const bool valid = eg < num_elem;
  double J[2][2][Q];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    if (col < P) {
      double xy[P];
      const int* orow = offsets + (valid ? eg : 0) * int64_t(P * P) + col;
#pragma unroll
      for (int py = 0; py < P; ++py) xy[py] = __ldg(x + __ldg(orow + py * P) + c * comp_stride);
#pragma unroll
      for (int qy = 0; qy < Q; ++qy) {
        double sb = 0.0, sg = 0.0;
#pragma unroll
        for (int py = 0; py < P; ++py) {
          sb += m.B[qy * P + py] * xy[py];
          sg += m.G[qy * P + py] * xy[py];
        }
        s1b[(col * Q + qy) * E + e] = sb;
        s1g[(col * Q + qy) * E + e] = sg;
      }
    }
    __syncthreads();
    {
      double wb[P], wg[P];
#pragma unroll
      for (int px = 0; px < P; ++px) {
        wb[px] = s1b[(px * Q + col) * E + e];
        wg[px] = s1g[(px * Q + col) * E + e];
      }
#pragma unroll
      for (int qx = 0; qx < Q; ++qx) {
        double d0 = 0.0, d1 = 0.0;
#pragma unroll
        for (int px = 0; px < P; ++px) {
          d0 += m.G[qx * P + px] * wb[px];
          d1 += m.B[qx * P + px] * wg[px];
        }
        J[0][c][qx] = d0;
        J[1][c][qx] = d1;
      }
    }
    __syncthreads();
  }
  if (!valid) return;
  const int qy = col;
#pragma unroll
  for (int qx = 0; qx < Q; ++qx) {
    const double det = J[0][0][qx] * J[1][1][qx] - J[0][1][qx] * J[1][0][qx];
    const double w = m.W[qy] * m.W[qx];
    qdata[int64_t(qy * Q + qx) * num_elem + eg] = det * w;
  }
}

// ---------------------------------------------------------------------------
// dim = 1: one thread per element, everything in registers.
// ---------------------------------------------------------------------------
// One element of mass1d_apply_kernel (E = 128 elements per tile).
template <int P, int Q, class T, class Ext, class S = T>
__device__ __forceinline__ void mass1d_element(const Mat1D<P, Q, T>& m, const int* __restrict__ offs,
                                               const S* __restrict__ qd, const S* __restrict__ u,
                                               T* __restrict__ v, T* __restrict__ ev, int num_elem,
                                               int num_comp_run, int64_t comp_stride, const Ext& ext,
                                               int64_t tile, int e, int64_t eg, double& dsum) {
  constexpr int E = 128;
  int off[P];
  T qv[Q];
#pragma unroll
  for (int px = 0; px < P; ++px) off[px] = __ldg(offs + (tile * P + px) * E + e);
#pragma unroll
  for (int qx = 0; qx < Q; ++qx) qv[qx] = load_as<T>(qd + (tile * Q + qx) * E + e);
  for (int k = 0; k < num_comp_run; ++k) {
    const int64_t ks = k * comp_stride;
    T x[P], r[Q];
#pragma unroll
    for (int px = 0; px < P; ++px) {
      x[px] = load_as<T>(u + off[px] + ks);
      if constexpr (Ext::kScale) x[px] *= __ldg(ext.scale + off[px]);
    }
#pragma unroll
    for (int qx = 0; qx < Q; ++qx) {
      T s = T(0);
#pragma unroll
      for (int px = 0; px < P; ++px) s += m.B[qx * P + px] * x[px];
      r[qx] = qv[qx] * s;
      if constexpr (Ext::kDot) dsum += double(r[qx]) * double(s);
    }
#pragma unroll
    for (int px = 0; px < P; ++px) {
      T s = T(0);
#pragma unroll
      for (int qx = 0; qx < Q; ++qx) s += m.B[qx * P + px] * r[qx];
      if (ev)
        ev[(int64_t(k) * P + px) * num_elem + eg] = s;
      else
        atomicAdd(v + off[px] + ks, s);
    }
  }
}

template <int P, int Q, class T = double, class Ext = ApplyPlain, class S = T>
__global__ void __launch_bounds__(128) mass1d_apply_kernel(const __grid_constant__ Mat1D<P, Q, T> m,
                                                          const int* __restrict__ offs, const S* __restrict__ qd,
                                                          const S* __restrict__ u, T* __restrict__ v,
                                                          T* __restrict__ ev, int num_elem, int num_comp_run,
                                                          int64_t comp_stride, const Ext ext) {
  constexpr int E = 128;
  const int e = threadIdx.x;
  if constexpr (Ext::kDot) {
    if (ext.st->done) return;
  }
  double dsum = 0.0;
  if constexpr (!Ext::kDot) {
    const int64_t tile = blockIdx.x, eg = tile * E + e;
    if (eg < num_elem)
      mass1d_element<P, Q, T, Ext, S>(m, offs, qd, u, v, ev, num_elem, num_comp_run, comp_stride, ext, tile, e, eg,
                                   dsum);
  } else {  // persistent, one reduction per CTA
    const int64_t n_tiles = (int64_t(num_elem) + E - 1) / E;
    for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
      const int64_t eg = tile * E + e;
      if (eg < num_elem)
        mass1d_element<P, Q, T, Ext, S>(m, offs, qd, u, v, ev, num_elem, num_comp_run, comp_stride, ext, tile, e,
                                     eg, dsum);
    }
    double dv[1] = {dsum};
    grid_sum<1>(dv, ext.part, &ext.st->ticket, [&](const double* tot) { cg_after_apply(ext.st, tot[0]); });
  }
}

template <int P, int Q>
__global__ void __launch_bounds__(128) mass1d_build_kernel(const __grid_constant__ Mat1D<P, Q> m,
                                                          const int* __restrict__ offsets,
                                                          const double* __restrict__ x, int64_t comp_stride,
                                                          double* __restrict__ qdata, int num_elem) {
  const int64_t eg = int64_t(blockIdx.x) * 128 + threadIdx.x;
  if (eg >= num_elem) return;
  double xe[P];
#pragma unroll
  for (int px = 0; px < P; ++px) xe[px] = __ldg(x + __ldg(offsets + eg * P + px));
#pragma unroll
  for (int qx = 0; qx < Q; ++qx) {
    double d = 0.0;
#pragma unroll
    for (int px = 0; px < P; ++px) d += m.G[qx * P + px] * xe[px];
    qdata[int64_t(qx) * num_elem + eg] = d * m.W[qx];
  }
}

}  // namespace fem_b200
