// The mass apply in FP32 and in BF16 storage (sm_100a): the fused kernels of
// mass_kernels.cuh instantiated with FP32 arithmetic, reading u and qdata as
// FP32 or as BF16 (converted to FP32 at the load) and accumulating v in FP32.
// The plan converts its tiled FP64 qdata once per storage type.  The
// reference computes in FP64 only (src/operator.cpp:148-182); these are the
// reduced-storage forms of the same operator.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <type_traits>

#include "mass_tc.cuh"
#include "plan.hpp"
#include "transpose_scatter.cuh"

namespace fem_b200 {
namespace {

__global__ void qdata_to_f32_kernel(int64_t n, const double* __restrict__ in, float* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = float(in[i]);
}

__global__ void qdata_to_bf16_kernel(int64_t n, const double* __restrict__ in, __nv_bfloat16* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = __float2bfloat16_rn(float(in[i]));
}

template <int P, int Q>
Mat1D<P, Q, float> f32_mat(const BasisData& b) {
  Mat1D<P, Q, float> m;
  for (int i = 0; i < Q * P; ++i) m.B[i] = float(b.interp[i]), m.G[i] = float(b.grad[i]);
  for (int i = 0; i < Q; ++i) m.W[i] = float(b.q_weight[i]);
  fill_eo(m);
  return m;
}

// The register policy: as the FP64 plan's simple variant, except at P = 5,
// where single-precision arithmetic fits six resident CTAs a SM (32
// registers, 24 B of spills): 100^3 hexes, FP32 storage, 0.636 ms at 4 CTAs
// (56 registers), 0.562 ms at 5, 0.530 ms at 6-7 (sustained, interleaved).
template <int P>
constexpr int lowp_min_blocks() {
  return P >= 8 ? 1 : P == 6 ? 2 : P == 5 ? 6 : 0;
}

template <class S>
using LowpLauncher = void (*)(const MassPlan&, const S*, const S*, float*, float*, cudaStream_t);

// The even-odd contractions (centro-symmetric B) where they measured faster in
// single precision (interleaved A/B against the direct form, ~64M DoFs): 3D
// P = 5 (FP32 0.576 -> 0.522 ms, BF16 0.604 -> 0.555 one component; three
// components alike), P = 7 (FP32 1.21x, BF16 1.15x), P = 8 (1.04-1.07x) and
// BF16 at P = 4 (0.878 -> 0.839 ms; FP32 there 0.711 -> 0.765) and P = 6
// (1.10x; FP32 there 0.82x); 2D only P = 8 (1.06-1.28x).
template <int P, class S>
constexpr bool lowp_even_odd_3d() {
  return P == 5 || P >= 7 || ((P == 4 || P == 6) && std::is_same<S, __nv_bfloat16>::value);
}

template <int P, int Q, class S, bool EO = lowp_even_odd_3d<P, S>() || P == 8>
void launch_lowp(const MassPlan& p, const S* qd, const S* u, float* v, float* ev, cudaStream_t s) {
  if constexpr (EO) {
    if (!p.centro_symmetric) return launch_lowp<P, Q, S, false>(p, qd, u, v, ev, s);
  }
  constexpr bool eo3 = EO && lowp_even_odd_3d<P, S>(), eo2 = EO && P == 8;
  if (p.dim == 3) {
    using L = Mass3D<P, Q>;
    constexpr int smem = (L::SA + L::SB) * 4;
    const auto kern = mass3d_apply_kernel<P, Q, lowp_min_blocks<P>(), float, ApplyPlain, 1, S, false, eo3>;
    static std::atomic<uint64_t> smem_set{0};
    set_smem(kern, smem, smem_set);
    const int64_t wave = resident_ctas(reinterpret_cast<const void*>(kern), L::NT, smem);  // L2 prefetch distance
    kern<<<unsigned(p.n_tiles), L::NT, smem, s>>>(f32_mat<P, Q>(p.basis), p.offs_t.get(), qd, u, v, ev, p.num_elem,
                                                  p.comp_run, p.comp_stride, ApplyPlain{}, wave);
  } else if (p.dim == 2) {
    using L = Mass2D<P, Q>;
    constexpr int smem = (L::S1 + L::S3) * 4;
    const auto kern = mass2d_apply_kernel<P, Q, float, ApplyPlain, S, 0, false, eo2>;
    static std::atomic<uint64_t> smem_set{0};
    set_smem(kern, smem, smem_set);
    // no L2 prefetch in 2D reduced storage: measured mixed (BF16 at P = 2: 0.85-0.88x)
    kern<<<unsigned(p.n_tiles), L::NT, smem, s>>>(f32_mat<P, Q>(p.basis), p.offs_t.get(), qd, u, v, ev, p.num_elem,
                                                  p.comp_run, p.comp_stride, ApplyPlain{}, 0);
  } else {
    mass1d_apply_kernel<P, Q, float, ApplyPlain, S><<<unsigned(p.n_tiles), 128, 0, s>>>(
        f32_mat<P, Q>(p.basis), p.offs_t.get(), qd, u, v, ev, p.num_elem, p.comp_run, p.comp_stride, ApplyPlain{});
  }
  FEM_LAUNCH_CHECK();
}

constexpr int kMinP = 2, kMaxP = 8, kQSpan = 3;

struct LowpDispatch {
  LowpLauncher<float> f32[kMaxP + 1][kQSpan] = {};
  LowpLauncher<__nv_bfloat16> bf16[kMaxP + 1][kQSpan] = {};
};

template <int P, int DQ>
struct LowpTable {
  static void fill(LowpDispatch& d) {
    d.f32[P][DQ] = launch_lowp<P, P + DQ, float>;
    d.bf16[P][DQ] = launch_lowp<P, P + DQ, __nv_bfloat16>;
    if constexpr (DQ + 1 < kQSpan)
      LowpTable<P, DQ + 1>::fill(d);
    else if constexpr (P + 1 <= kMaxP)
      LowpTable<P + 1, 0>::fill(d);
  }
};

const LowpDispatch& lowp_dispatch() {
  static const LowpDispatch d = [] {
    LowpDispatch t;
    LowpTable<kMinP, 0>::fill(t);
    return t;
  }();
  return d;
}

// The plan's tiled qdata in storage S, converted from the FP64 copy on first use.
template <class S>
const S* lowp_qdata(MassPlan& p, cudaStream_t s) {
  const size_t nq = p.qd_t.size();
  if constexpr (std::is_same<S, float>::value) {
    if (p.qd_t32.size() != nq) {
      p.qd_t32.alloc(nq);
      qdata_to_f32_kernel<<<grid_for(int64_t(nq), 256), 256, 0, s>>>(int64_t(nq), p.qd_t.get(), p.qd_t32.get());
      FEM_LAUNCH_CHECK();
    }
    return p.qd_t32.get();
  } else {
    if (p.qd_t16.size() != nq) {
      p.qd_t16.alloc(nq);
      qdata_to_bf16_kernel<<<grid_for(int64_t(nq), 256), 256, 0, s>>>(int64_t(nq), p.qd_t.get(), p.qd_t16.get());
      FEM_LAUNCH_CHECK();
    }
    return p.qd_t16.get();
  }
}

// ---- tensor-core applies (mass_tc.cuh) --------------------------------------
// TF32 rounding on the host (nearest, ties away: cvt.rna's rule).
float host_tf32(float x) {
  uint32_t w;
  std::memcpy(&w, &x, 4);
  w = (w + 0x1000u) & 0xFFFFE000u;
  float y;
  std::memcpy(&y, &w, 4);
  return y;
}

// The B operands of the tensor-core kernel from the FP64 interpolation matrix:
// forward n = q, k = p (B[q][p]); backward n = p, k = q (B[q][p] too); rows
// 0-7 the TF32 part, rows 8-15 the TF32 part of the remainder (split) or 0.
TcMats tc_mats(const BasisData& b) {
  TcMats m;
  std::memset(&m, 0, sizeof(m));
  for (int n = 0; n < 8; ++n)
    for (int k = 0; k < 8; ++k) {
      for (int dir = 0; dir < 2; ++dir) {
        const int q = dir == 0 ? n : k, pp = dir == 0 ? k : n;
        if (q >= b.Q || pp >= b.P) continue;
        const double x = b.interp[size_t(q * b.P + pp)];
        const float hi = host_tf32(float(x));
        const float lo = host_tf32(float(x - double(hi)));
        m.op[2 * dir][tc::kmajor_index(n, k)] = hi;
        m.op[2 * dir][tc::kmajor_index(n + 8, k)] = lo;
        m.op[2 * dir + 1][tc::kmajor_index(n, k)] = hi;
      }
    }
  return m;
}

template <class S>
using TcLauncher = void (*)(const MassPlan&, const S*, const S*, float*, cudaStream_t);

template <int P, int Q, bool SPLIT, class S>
void launch_tc(const MassPlan& p, const S* qd, const S* u, float* v, cudaStream_t s) {
  using L = TcMass3D<P, Q>;
  constexpr int smem = L::smem(SPLIT);
  const auto kern = mass3d_apply_tc_kernel<P, Q, SPLIT, S>;
  static std::atomic<uint64_t> smem_set{0};
  set_smem(kern, smem, smem_set);
  // persistent CTAs: 8 a SM (the shared-memory padding of TcMass3D::smem keeps
  // at most as many resident as tensor memory holds), tiles from a ticket
  int sms = 0;
  FEM_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p.device));
  const int grid = int(std::min<int64_t>(p.n_tiles, int64_t(sms) * 8));
  MassPlan& mp = const_cast<MassPlan&>(p);
  if (!mp.tc_ticket.get()) mp.tc_ticket.alloc(1);
  FEM_CUDA_CHECK(cudaMemsetAsync(mp.tc_ticket.get(), 0, sizeof(int), s));
  kern<<<grid, L::NT, smem, s>>>(tc_mats(p.basis), p.offs_t.get(), qd, u, v, p.num_elem, p.comp_run, p.comp_stride,
                                 p.n_tiles, mp.tc_ticket.get(), p.status.get());
  FEM_LAUNCH_CHECK();
}

constexpr int kTcMinP = 6;

struct TcDispatch {
  TcLauncher<float> f32_split[kMaxP + 1][kQSpan] = {};
  TcLauncher<float> f32[kMaxP + 1][kQSpan] = {};
  TcLauncher<__nv_bfloat16> bf16[kMaxP + 1][kQSpan] = {};
  template <int P, int DQ>
  void fill() {
    constexpr int Q = P + DQ;
    if constexpr (Q <= 8) {
      f32_split[P][DQ] = launch_tc<P, Q, true, float>;
      f32[P][DQ] = launch_tc<P, Q, false, float>;
      bf16[P][DQ] = launch_tc<P, Q, false, __nv_bfloat16>;
    }
    if constexpr (DQ + 1 < kQSpan)
      fill<P, DQ + 1>();
    else if constexpr (P + 1 <= kMaxP)
      fill<P + 1, 0>();
  }
  TcDispatch() { fill<kTcMinP, 0>(); }
};

const TcDispatch& tc_dispatch() {
  static TcDispatch d;
  return d;
}

// v = M u on the tensor cores: u, qdata in S, v in FP32; split: the 3xTF32
// form (FP32 storage only).
template <class S>
void tc_apply(MassPlan& p, const S* u, float* v, bool split, cudaStream_t s) {
  if (p.dim != 3 || p.P < kTcMinP || p.P > kMaxP || p.Q < p.P || p.Q > 8)
    throw unsupported_error("tensor-core apply: no kernel for " + shape_str(p.dim, p.P, p.Q) +
                            " (dim 3, P = 6..8, Q = P..8)");
  if (p.scatter_mode != FEM_B200_SCATTER_ATOMIC)
    throw unsupported_error("tensor-core apply: atomic scatter only");
  TcLauncher<S> launch = nullptr;
  if constexpr (std::is_same<S, float>::value)
    launch = split ? tc_dispatch().f32_split[p.P][p.Q - p.P] : tc_dispatch().f32[p.P][p.Q - p.P];
  else
    launch = tc_dispatch().bf16[p.P][p.Q - p.P];
  const S* qd = lowp_qdata<S>(p, s);
  FEM_CUDA_CHECK(cudaMemsetAsync(v, 0, size_t(p.l_size) * sizeof(float), s));
  launch(p, qd, u, v, s);
}

// v = M u with u, qdata in S and v in FP32
template <class S>
void lowp_apply(MassPlan& p, const S* u, float* v, cudaStream_t s) {
  const S* qd = lowp_qdata<S>(p, s);
  FEM_CUDA_CHECK(cudaMemsetAsync(v, 0, size_t(p.l_size) * sizeof(float), s));
  const LowpDispatch& d = lowp_dispatch();
  LowpLauncher<S> launch = nullptr;
  if constexpr (std::is_same<S, float>::value)
    launch = d.f32[p.P][p.Q - p.P];
  else
    launch = d.bf16[p.P][p.Q - p.P];
  if (p.scatter_mode == FEM_B200_SCATTER_ATOMIC) {
    launch(p, qd, u, v, nullptr, s);
    return;
  }
  if (p.evec32.size() != p.evec.size()) p.evec32.alloc(p.evec.size());
  const RestrictionData& r = *p.r;
  launch(p, qd, u, nullptr, p.evec32.get(), s);
  launch_csr_scatter(r.num_nodes, p.num_elem, p.es, p.comp_run, p.comp_stride, r.l_vec_indices.get(),
                     r.t_offsets.get(), r.t_indices.get(), p.evec32.get(), v, s);
  FEM_LAUNCH_CHECK();
}

}  // namespace
}  // namespace fem_b200

using namespace fem_b200;

extern "C" {

int fem_b200_mass_apply_f32(fem_b200_mass op, const float* u, int64_t n_u, float* v, int64_t n_v, void* stream) {
  return guarded([&] {
    require(op && op->d, "operator_apply: NULL handle");
    MassPlan& p = *op->d;
    require(n_u == p.l_size && u, "operator_apply: input vector size does not match active_in_l_size");
    require(n_v == p.l_size && v, "operator_apply: output vector size does not match active_out_l_size");
    DeviceGuard g(p.device);
    lowp_apply<float>(p, u, v, as_stream(stream));
  });
}

int fem_b200_mass_apply_f32_tc(fem_b200_mass op, const float* u, int64_t n_u, float* v, int64_t n_v, int split,
                               void* stream) {
  return guarded([&] {
    require(op && op->d, "operator_apply: NULL handle");
    MassPlan& p = *op->d;
    require(n_u == p.l_size && u, "operator_apply: input vector size does not match active_in_l_size");
    require(n_v == p.l_size && v, "operator_apply: output vector size does not match active_out_l_size");
    require(split == 0 || split == 1, "tensor-core apply: split must be 0 or 1");
    DeviceGuard g(p.device);
    tc_apply<float>(p, u, v, split == 1, as_stream(stream));
  });
}

int fem_b200_mass_apply_bf16_tc(fem_b200_mass op, const void* u, int64_t n_u, float* v, int64_t n_v, void* stream) {
  return guarded([&] {
    require(op && op->d, "operator_apply: NULL handle");
    MassPlan& p = *op->d;
    require(n_u == p.l_size && u, "operator_apply: input vector size does not match active_in_l_size");
    require(n_v == p.l_size && v, "operator_apply: output vector size does not match active_out_l_size");
    DeviceGuard g(p.device);
    tc_apply<__nv_bfloat16>(p, static_cast<const __nv_bfloat16*>(u), v, false, as_stream(stream));
  });
}

int fem_b200_mass_apply_bf16(fem_b200_mass op, const void* u, int64_t n_u, float* v, int64_t n_v, void* stream) {
  return guarded([&] {
    require(op && op->d, "operator_apply: NULL handle");
    MassPlan& p = *op->d;
    require(n_u == p.l_size && u, "operator_apply: input vector size does not match active_in_l_size");
    require(n_v == p.l_size && v, "operator_apply: output vector size does not match active_out_l_size");
    DeviceGuard g(p.device);
    lowp_apply<__nv_bfloat16>(p, static_cast<const __nv_bfloat16*>(u), v, as_stream(stream));
  });
}

}  // extern "C"
