// Dispatch of the fused dim-3 basis kernels (basis_kernels.cuh) over the
// compiled (P, Q) set, for fem_b200_basis_apply.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>

#include "basis_kernels.cuh"
#include "plan.hpp"

namespace fem_b200 {
namespace {

using BasisLauncher = void (*)(const BasisData&, int, const double*, double*, cudaStream_t);

// Which kernels read the 1D matrices from a shared copy (SharedBG) instead of
// the parameter, where that beat the parameter on a B200: interp and interp^T
// from P = 6 (1.2-1.5x; at P = 8 interp 5.7x, the parameter form spilled 656
// B), grad from P = 5 (1.1-2.3x).  grad^T never gained (0.7-1.0x).
template <int P, int MODE>
constexpr bool basis_shared_matrix() {
  return MODE <= 1 ? P >= 6 : MODE == 2 ? P >= 5 : false;
}

// interp and interp^T with the even-odd contractions (centro-symmetric B),
// where they measured faster (interleaved A/B, ~64M-DoF sizes): interp from
// P = 5 (1.05x at 5, 1.10x at 6, 1.38x at 7, 1.31x at 8), interp^T from P = 6
// (1.42x, 1.26x, 1.42x); P = 4 and interp^T at P = 5 equal.
template <int P, int MODE>
constexpr bool basis_even_odd() {
  return MODE == 0 ? P >= 5 : MODE == 1 ? P >= 6 : false;
}

bool centro_symmetric(const BasisData& b) {
  double mx = 0.0, asym = 0.0;
  for (int q = 0; q < b.Q; ++q)
    for (int j = 0; j < b.P; ++j) {
      const double x = b.interp[size_t(q * b.P + j)], y = b.interp[size_t((b.Q - 1 - q) * b.P + (b.P - 1 - j))];
      mx = std::max(mx, std::fabs(x));
      asym = std::max(asym, std::fabs(x - y));
    }
  return asym <= 1e-14 * mx;
}

// MODE: 0 interp, 1 interp^T, 2 grad, 3 grad^T
template <int P, int Q, int MODE, bool EO = basis_even_odd<P, MODE>()>
void launch_basis3(const BasisData& b, int ne, const double* u, double* v, cudaStream_t s) {
  if constexpr (EO) {
    if (!centro_symmetric(b)) return launch_basis3<P, Q, MODE, false>(b, ne, u, v, s);
  }
  using L = Basis3D<P, Q>;
  constexpr int smem = 8 * (MODE <= 1 ? L::SMEM_INTERP : MODE == 2 ? L::SMEM_GRAD_N : L::SMEM_GRAD_T);
  constexpr bool SB = basis_shared_matrix<P, MODE>() && !EO;
  const auto kern = MODE == 0   ? basis3d_interp_kernel<P, Q, SB, EO>
                    : MODE == 1 ? basis3d_interp_t_kernel<P, Q, SB, EO>
                    : MODE == 2 ? basis3d_grad_kernel<P, Q, SB>
                                : basis3d_grad_t_kernel<P, Q, SB>;
  static std::atomic<uint64_t> smem_set{0};
  set_smem(kern, smem, smem_set);
  const unsigned grid = unsigned((int64_t(ne) + L::E - 1) / L::E);
  kern<<<grid, L::NT, smem, s>>>(make_mat<P, Q>(b), u, v, ne, b.num_comp);
  FEM_LAUNCH_CHECK();
}

constexpr int kMinP = 2, kMaxP = 8, kQSpan = 3;

struct BasisDispatch {
  BasisLauncher fn[kMaxP + 1][kQSpan][4] = {};
};

template <int P, int DQ, int MODE>
void fill_one(BasisDispatch& d) {
  constexpr int Q = P + DQ;
  using L = Basis3D<P, Q>;
  constexpr int smem = 8 * (MODE <= 1 ? L::SMEM_INTERP : MODE == 2 ? L::SMEM_GRAD_N : L::SMEM_GRAD_T) +
                       (basis_shared_matrix<P, MODE>() ? 16 * P * Q : 0);
  if constexpr (smem <= kMaxSmemPerCta && L::NT <= 1024) d.fn[P][DQ][MODE] = launch_basis3<P, Q, MODE>;
}

template <int P, int DQ>
struct BasisTable {
  static void fill(BasisDispatch& d) {
    fill_one<P, DQ, 0>(d);
    fill_one<P, DQ, 1>(d);
    fill_one<P, DQ, 2>(d);
    fill_one<P, DQ, 3>(d);
    if constexpr (DQ + 1 < kQSpan)
      BasisTable<P, DQ + 1>::fill(d);
    else if constexpr (P + 1 <= kMaxP)
      BasisTable<P + 1, 0>::fill(d);
  }
};

const BasisDispatch& basis_dispatch() {
  static const BasisDispatch d = [] {
    BasisDispatch t;
    BasisTable<kMinP, 0>::fill(t);
    return t;
  }();
  return d;
}

}  // namespace

bool basis3d_fused_apply(const BasisData& b, int num_elem, bool transpose, bool grad, const double* u, double* v,
                         cudaStream_t s) {
  if (b.dim != 3 || b.P < kMinP || b.P > kMaxP || b.Q < b.P || b.Q >= b.P + kQSpan) return false;
  const BasisLauncher f = basis_dispatch().fn[b.P][b.Q - b.P][(grad ? 2 : 0) + (transpose ? 1 : 0)];
  if (!f) return false;
  f(b, num_elem, u, v, s);
  return true;
}

}  // namespace fem_b200
