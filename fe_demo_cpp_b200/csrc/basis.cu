// Dispatch of the fused dim-3 basis kernels (basis_kernels.cuh) over the
// compiled (P, Q) set, for fem_b200_basis_apply.
#include <cuda_runtime.h>

#include <atomic>

#include "basis_kernels.cuh"
#include "plan.hpp"

namespace fem_b200 {
namespace {

using BasisLauncher = void (*)(const BasisData&, int, const double*, double*, cudaStream_t);

// MODE: 0 interp, 1 interp^T, 2 grad, 3 grad^T
template <int P, int Q, int MODE>
void launch_basis3(const BasisData& b, int ne, const double* u, double* v, cudaStream_t s) {
  using L = Basis3D<P, Q>;
  constexpr int smem = 8 * (MODE <= 1 ? L::SMEM_INTERP : MODE == 2 ? L::SMEM_GRAD_N : L::SMEM_GRAD_T);
  const auto kern = MODE == 0   ? basis3d_interp_kernel<P, Q>
                    : MODE == 1 ? basis3d_interp_t_kernel<P, Q>
                    : MODE == 2 ? basis3d_grad_kernel<P, Q>
                                : basis3d_grad_t_kernel<P, Q>;
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
  constexpr int smem = 8 * (MODE <= 1 ? L::SMEM_INTERP : MODE == 2 ? L::SMEM_GRAD_N : L::SMEM_GRAD_T);
  // interp NoTranspose at Q >= 9 (648-thread CTAs) spills 1.2 KB a thread and
  // measures slower than the generic passes: those keep the generic path
  constexpr bool slow = MODE == 0 && Q >= 9;
  if constexpr (smem <= kMaxSmemPerCta && L::NT <= 1024 && !slow) d.fn[P][DQ][MODE] = launch_basis3<P, Q, MODE>;
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
