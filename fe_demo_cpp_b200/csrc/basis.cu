// Dispatch of the fused dim-3 basis kernels (basis_kernels.cuh) over the
// compiled (P, Q) set, for fem_b200_basis_apply.
#include <cuda_runtime.h>

#include <atomic>

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

// MODE: 0 interp, 1 interp^T, 2 grad, 3 grad^T
template <int P, int Q, int MODE>
void launch_basis3(const BasisData& b, int ne, const double* u, double* v, cudaStream_t s) {
  using L = Basis3D<P, Q>;
  constexpr int smem = 8 * (MODE <= 1 ? L::SMEM_INTERP : MODE == 2 ? L::SMEM_GRAD_N : L::SMEM_GRAD_T);
  constexpr bool SB = basis_shared_matrix<P, MODE>();
  const auto kern = MODE == 0   ? basis3d_interp_kernel<P, Q, SB>
                    : MODE == 1 ? basis3d_interp_t_kernel<P, Q, SB>
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
