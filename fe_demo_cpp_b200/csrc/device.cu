// libfem_b200: device objects (restriction, basis, mass plan), kernel
// dispatch and the extern "C" entry points declared in include/fem_b200.h.
#include <cuda_runtime.h>

#include <cmath>

#include <algorithm>
#include <atomic>
#include <map>
#include <tuple>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "common.hpp"
#include "fem_b200.h"
#include "host_setup.hpp"
#include "mass_kernels.cuh"
#include "mass_pipe.cuh"
#include "mass_x2.cuh"
#include "mass_element.cuh"
#include "mass_narrow.cuh"
#include "mass_prefetch.cuh"
#include "plan.hpp"
#include "restriction_kernels.cuh"

namespace fem_b200 {

thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }


// The simple kernel's register policy: no minimum of resident CTAs (ptxas'
// own heuristic: 55 registers at P=5 where a minimum of 1 lets it take 72 and
// lose a resident CTA); at P = 6 two resident 392-thread CTAs (83 registers,
// 80 B of spills, against one CTA at 98 registers); at P = 7 two CTAs and at
// P = 8 one, with the interpolation matrix read from shared memory
// (plain_shared_matrix).
template <int P>
constexpr int plain_min_blocks() {
  return P >= 8 ? 1 : P >= 6 ? 2 : 0;
}

// At P >= 7 the compiler holds all P*Q matrix entries in registers for the
// whole tile; read from a shared copy at each use instead (SharedB), P = 8
// keeps 80 registers with 24 B of spills instead of 728 B, P = 7 fits two
// resident CTAs: 1.69x (P = 8) and 1.34x (P = 7) on 64M-DoF boxes.  Below
// P = 7 the extra loads cost more than the registers they free (P = 5: 2.3x
// slower).
template <int P>
constexpr bool plain_shared_matrix() {
  return P >= 7;
}

// Each CTA prefetches into L2 the qdata and offsets of the tile one wave of
// resident CTAs ahead (prefetch distances of 0.5-2 waves measured alike, 4
// waves began to evict): over 10-20 launches P = 4 1.09x, P = 5 1.10x,
// P = 6 1.06x; sustained (300 launches, interleaved with the kernel without
// it) P = 5 1.05x.
// The even-odd contractions (eo_fwd / eo_bwd) where they measured faster, for
// a centro-symmetric B: P = 4 1.10x, P = 6 1.53x (68 registers without spills
// instead of 72 with 84 B), P = 7 1.85x and P = 8 1.47x against the
// shared-matrix form (the folds are half of B, so holding them in registers
// no longer starves the CTA: P = 7 two CTAs at 64 registers, no spills).
// P = 5: equal in short bursts at full clock, but 1.026x over the bench's
// sustained 200-launch region, where the power cap sets the clock (fewer
// FP64 operations: 0.847 -> 0.825 ms at 1680-1810 MHz, two interleaved runs).
template <int P>
constexpr bool plain_even_odd() {
  return P >= 4;
}

template <int P, int Q, int MINB, bool SB, bool EO>
void launch_apply3_kernel(const MassPlan& p, const double* u, double* v, double* ev, cudaStream_t s);

// The simple variant: even-odd where it applies, else the direct form
// (shared-memory matrix at P >= 7).
template <int P, int Q>
void launch_apply3(const MassPlan& p, const double* u, double* v, double* ev, cudaStream_t s) {
  if constexpr (plain_even_odd<P>()) {
    if (p.centro_symmetric) return launch_apply3_kernel<P, Q, plain_min_blocks<P>(), false, true>(p, u, v, ev, s);
  }
  launch_apply3_kernel<P, Q, plain_min_blocks<P>(), plain_shared_matrix<P>(), false>(p, u, v, ev, s);
}

template <int P, int Q, int MINB, bool SB, bool EO>
void launch_apply3_kernel(const MassPlan& p, const double* u, double* v, double* ev, cudaStream_t s) {
  using L = Mass3D<P, Q>;
  const auto kern = mass3d_apply_kernel<P, Q, MINB, double, ApplyPlain, 1, double, SB, EO>;
  static std::atomic<uint64_t> smem_set{0};
  set_smem(kern, L::SMEM, smem_set);
  const int64_t wave = resident_ctas(reinterpret_cast<const void*>(kern), L::NT, L::SMEM);
  kern<<<unsigned(p.tiles()), L::NT, L::SMEM, s>>>(make_mat<P, Q>(p.basis), p.offs(), p.qd(), u, v, ev, p.elems(),
                                                   p.comp_run, p.comp_stride, ApplyPlain{}, wave);
  FEM_LAUNCH_CHECK();
}

// Persistent grid: SMs x resident CTAs (from the occupancy calculator), at
// most one CTA per tile.
template <class K>
int persistent_grid(K kernel, int threads, int smem, int64_t n_tiles) {
  return int(std::min<int64_t>(n_tiles, resident_ctas(reinterpret_cast<const void*>(kernel), threads, smem)));
}

// The pipelined variant, with the even-odd contractions where the one-tile
// kernel takes them (plain_even_odd, centro-symmetric B).
template <int P, int Q, bool EO = plain_even_odd<P>()>
void launch_apply3_pipe(const MassPlan& p, const double* u, double* v, double* ev, cudaStream_t s) {
  if constexpr (EO) {
    if (!p.centro_symmetric) return launch_apply3_pipe<P, Q, false>(p, u, v, ev, s);
  }
  using L = Pipe3D<P, Q>;
  const auto kern = mass3d_apply_pipe_kernel<P, Q, EO>;
  static std::atomic<uint64_t> smem_set{0};
  set_smem(kern, L::SMEM, smem_set);
  const int grid = persistent_grid(kern, L::NT, L::SMEM, p.tiles());
  kern<<<grid, L::NT, L::SMEM, s>>>(make_mat<P, Q>(p.basis), p.offs(), p.qd(), u, v, ev, p.elems(), p.comp_run,
                                    p.comp_stride, p.tiles(), p.status.get());
  FEM_LAUNCH_CHECK();
}

template <int P, int Q>
void launch_apply3_pf(const MassPlan& p, const double* u, double* v, double* ev, cudaStream_t s) {
  using L = Mass3D<P, Q>;
  constexpr int smem = Prefetch3D<P, Q>::SMEM;
  static std::atomic<uint64_t> smem_set{0};
  set_smem(mass3d_apply_prefetch_kernel<P, Q>, smem, smem_set);
  const int grid = persistent_grid(mass3d_apply_prefetch_kernel<P, Q>, L::NT, smem, p.tiles());
  mass3d_apply_prefetch_kernel<P, Q><<<grid, L::NT, smem, s>>>(make_mat<P, Q>(p.basis), p.offs(),
                                                                p.qd(), u, v, ev, p.elems(), p.comp_run,
                                                                p.comp_stride, int(p.tiles()), p.status.get());
  FEM_LAUNCH_CHECK();
}

template <int P, int Q>
void launch_apply3_x2(const MassPlan& p, const double* u, double* v, double* ev, cudaStream_t s) {
  using L = Mass3DX2<P, Q>;
  static std::atomic<uint64_t> smem_set{0};
  set_smem(mass3d_apply_x2_kernel<P, Q>, L::SMEM, smem_set);
  const unsigned grid = unsigned((p.tiles() + 1) / 2);  // the plan's tile arrays hold an even number of tiles
  mass3d_apply_x2_kernel<P, Q><<<grid, L::NT, L::SMEM, s>>>(make_mat<P, Q>(p.basis), p.offs(), p.qd(),
                                                             u, v, ev, p.elems(), p.comp_run, p.comp_stride);
  FEM_LAUNCH_CHECK();
}

// Half-tile CTAs (4 elements): at P = 8 no register cap (one CTA per SM,
// no spills: 1.5x the one-tile kernel there), below two resident CTAs
// (P = 7: 128 registers, P = 6: 96).
template <int P, int Q>
void launch_apply3_narrow(const MassPlan& p, const double* u, double* v, double* ev, cudaStream_t s) {
  using L = Narrow3D<P, Q>;
  constexpr int minb = P >= 8 ? 0 : 2;
  const auto kern = mass3d_apply_narrow_kernel<P, Q, minb>;
  static std::atomic<uint64_t> smem_set{0};
  set_smem(kern, L::SMEM, smem_set);
  kern<<<unsigned(2 * p.tiles()), L::NT, L::SMEM, s>>>(make_mat<P, Q>(p.basis), p.offs(), p.qd(), u,
                                                       v, ev, p.elems(), p.comp_run, p.comp_stride);
  FEM_LAUNCH_CHECK();
}

// Staged element kernel: one-warp CTAs (4 tiles).  ~64M-DoF boxes, one and
// three components, interleaved runs on one box each: P = 3 unstaged 1.32 /
// 0.94 ms, staged in 64-thread CTAs 1.24 / 0.77 ms; on another box staged
// in 32 / 64 / 128-thread CTAs 1.27 / 1.30 / 1.45 ms (one component), 0.755 /
// 0.77 / 0.91 ms (three), and P = 2 unstaged 2.99 / 1.48 ms, staged in
// 32-thread CTAs 2.62 / 1.42 ms.
constexpr int kElemStageCT = 32;

// One element per thread (P <= 3): the staged kernel (qdata and offsets
// bulk-copied into shared memory per CTA); for unaligned pointers
// 128-thread CTAs reading them from global memory.
template <int P, int Q>
void launch_apply3_element(const MassPlan& p, const double* u, double* v, double* ev, cudaStream_t s) {
  using LS = ElemStage<P, Q, kElemStageCT>;
  if (LS::SMEM <= kMaxSmemPerCta && (reinterpret_cast<uintptr_t>(p.offs()) & 15) == 0 &&
      (reinterpret_cast<uintptr_t>(p.qd()) & 15) == 0) {
    const auto kern = mass3d_apply_element_staged_kernel<P, Q, kElemStageCT>;
    static std::atomic<uint64_t> smem_set{0};
    set_smem(kern, LS::SMEM, smem_set);
    const int64_t wave = resident_ctas(reinterpret_cast<const void*>(kern), kElemStageCT, LS::SMEM);
    kern<<<unsigned((p.tiles() + LS::TILES - 1) / LS::TILES), kElemStageCT, LS::SMEM, s>>>(
        make_mat<P, Q>(p.basis), p.offs(), p.qd(), u, v, ev, p.elems(), p.comp_run, p.comp_stride, wave,
        p.status.get());
    FEM_LAUNCH_CHECK();
    return;
  }
  const unsigned grid = unsigned((p.tiles() * 8 + 127) / 128);
  const auto kern = mass3d_apply_element_kernel<P, Q>;
  // L2 prefetch a wave ahead at P = 3 (1.05-1.07x); at P = 2 it measured
  // slightly slower (0.98x) and stays off
  const int64_t wave = P == 3 ? resident_ctas(reinterpret_cast<const void*>(kern), 128, 0) : 0;
  kern<<<grid, 128, 0, s>>>(make_mat<P, Q>(p.basis), p.offs(), p.qd(), u, v, ev, p.elems(), p.comp_run,
                            p.comp_stride, wave);
  FEM_LAUNCH_CHECK();
}

// dim 2: the interpolation matrix from shared memory at P >= 7, where holding
// it in registers leaves one resident CTA (145-168 registers): 1.46x at
// P = 7, 1.15x at P = 8 (16M-node boxes); slower below.  EO: the even-odd
// contractions (centro-symmetric B), in place of it.
template <int P, int Q, bool SB, bool EO>
void launch_apply2_kernel(const MassPlan& p, const double* u, double* v, double* ev, cudaStream_t s) {
  using L = Mass2D<P, Q>;
  const auto kern = mass2d_apply_kernel<P, Q, double, ApplyPlain, double, 0, SB, EO>;
  static std::atomic<uint64_t> smem_set{0};
  set_smem(kern, L::SMEM, smem_set);
  // L2 prefetch a wave ahead at P <= 4 (P = 2, 3: 1.10-1.12x one component,
  // 1.03-1.04x three); neutral at P = 5, so off from there
  const int64_t wave = P <= 4 ? resident_ctas(reinterpret_cast<const void*>(kern), L::NT, L::SMEM) : 0;
  kern<<<unsigned(p.tiles()), L::NT, L::SMEM, s>>>(make_mat<P, Q>(p.basis), p.offs(), p.qd(), u, v, ev, p.elems(),
                                                   p.comp_run, p.comp_stride, ApplyPlain{}, wave);
  FEM_LAUNCH_CHECK();
}

// dim 2 even-odd where it measured faster (interleaved A/B, ~64M-DoF quad
// boxes): P = 6 1.52x, P = 7 1.82x, P = 8 1.51x (three components 1.32-1.76x);
// P = 4, 5 equal.
template <int P>
constexpr bool plain_even_odd_2d() {
  return P >= 6;
}

template <int P, int Q>
void launch_apply2(const MassPlan& p, const double* u, double* v, double* ev, cudaStream_t s) {
  if constexpr (plain_even_odd_2d<P>()) {
    if (p.centro_symmetric) return launch_apply2_kernel<P, Q, false, true>(p, u, v, ev, s);
  }
  launch_apply2_kernel<P, Q, (P >= 7), false>(p, u, v, ev, s);
}

template <int P, int Q>
void launch_apply1(const MassPlan& p, const double* u, double* v, double* ev, cudaStream_t s) {
  mass1d_apply_kernel<P, Q><<<unsigned(p.tiles()), 128, 0, s>>>(make_mat<P, Q>(p.basis), p.offs(),
                                                                 p.qd(), u, v, ev, p.elems(), p.comp_run,
                                                                 p.comp_stride, ApplyPlain{});
  FEM_LAUNCH_CHECK();
}

template <int P, int Q>
void launch_build3(const BasisData& b, const RestrictionData& r, const double* x, double* qdata, cudaStream_t s) {
  using L = Build3D<P, Q>;
  static std::atomic<uint64_t> smem_set{0};
  set_smem(mass3d_build_kernel<P, Q>, L::SMEM, smem_set);
  const unsigned grid = unsigned((int64_t(r.num_elem) + L::E - 1) / L::E);
  mass3d_build_kernel<P, Q><<<grid, L::NT, L::SMEM, s>>>(make_mat<P, Q>(b), r.offsets.get(), x, r.comp_stride, qdata,
                                                        r.num_elem);
  FEM_LAUNCH_CHECK();
}

template <int P, int Q>
void launch_build2(const BasisData& b, const RestrictionData& r, const double* x, double* qdata, cudaStream_t s) {
  const unsigned grid = unsigned((int64_t(r.num_elem) + 31) / 32);
  mass2d_build_kernel<P, Q><<<grid, 32 * Q, 0, s>>>(make_mat<P, Q>(b), r.offsets.get(), x, r.comp_stride, qdata,
                                                   r.num_elem);
  FEM_LAUNCH_CHECK();
}

template <int P, int Q>
void launch_build1(const BasisData& b, const RestrictionData& r, const double* x, double* qdata, cudaStream_t s) {
  const unsigned grid = unsigned((int64_t(r.num_elem) + 127) / 128);
  mass1d_build_kernel<P, Q><<<grid, 128, 0, s>>>(make_mat<P, Q>(b), r.offsets.get(), x, r.comp_stride, qdata,
                                                r.num_elem);
  FEM_LAUNCH_CHECK();
}

// Compiled (P, Q) set: P = 2..8, Q = P .. P+2 (Q = P + 1 is the Gauss rule
// of the benchmarks; Q = P the collocated GLL case).
constexpr int kMinP = 2, kMaxP = 8, kQSpan = 3;

template <int P, int DQ>
struct Table {
  static void fill(ApplyLauncher (*ap)[kMaxP + 1][kQSpan], BuildLauncher (*bd)[kMaxP + 1][kQSpan],
                   ApplyLauncher (*pp)[kQSpan], ApplyLauncher (*xx)[kQSpan], ApplyLauncher (*pf)[kQSpan],
                   ApplyLauncher (*oc)[kQSpan], ApplyLauncher (*nw)[kQSpan], ApplyLauncher (*el)[kQSpan]) {
    constexpr int Q = P + DQ;
    ap[0][P][DQ] = launch_apply1<P, Q>;
    ap[1][P][DQ] = launch_apply2<P, Q>;
    ap[2][P][DQ] = launch_apply3<P, Q>;
    if constexpr (Pipe3D<P, Q>::SMEM <= kMaxSmemPerCta) pp[P][DQ] = launch_apply3_pipe<P, Q>;
    if constexpr (Mass3DX2<P, Q>::SMEM <= kMaxSmemPerCta && Mass3DX2<P, Q>::NT <= 1024) xx[P][DQ] = launch_apply3_x2<P, Q>;
    if constexpr (Prefetch3D<P, Q>::SMEM <= kMaxSmemPerCta) pf[P][DQ] = launch_apply3_pf<P, Q>;
    if constexpr (Mass3D<P, Q>::MINB_OCC > 1) oc[P][DQ] = launch_apply3_kernel<P, Q, Mass3D<P, Q>::MINB_OCC, false, false>;
    if constexpr (Narrow3D<P, Q>::SMEM <= kMaxSmemPerCta) nw[P][DQ] = launch_apply3_narrow<P, Q>;
    if constexpr (P <= 3) el[P][DQ] = launch_apply3_element<P, Q>;  // staged: 67-92 registers (P=2), 156-164 (P=3)
    bd[0][P][DQ] = launch_build1<P, Q>;
    bd[1][P][DQ] = launch_build2<P, Q>;
    bd[2][P][DQ] = launch_build3<P, Q>;
    if constexpr (DQ + 1 < kQSpan)
      Table<P, DQ + 1>::fill(ap, bd, pp, xx, pf, oc, nw, el);
    else if constexpr (P + 1 <= kMaxP)
      Table<P + 1, 0>::fill(ap, bd, pp, xx, pf, oc, nw, el);
  }
};

struct Dispatch {
  ApplyLauncher apply[3][kMaxP + 1][kQSpan] = {};
  BuildLauncher build[3][kMaxP + 1][kQSpan] = {};
  ApplyLauncher apply3_pipe[kMaxP + 1][kQSpan] = {};
  ApplyLauncher apply3_x2[kMaxP + 1][kQSpan] = {};
  ApplyLauncher apply3_pf[kMaxP + 1][kQSpan] = {};
  ApplyLauncher apply3_occ[kMaxP + 1][kQSpan] = {};
  ApplyLauncher apply3_nw[kMaxP + 1][kQSpan] = {};
  ApplyLauncher apply3_el[kMaxP + 1][kQSpan] = {};
  Dispatch() {
    Table<kMinP, 0>::fill(apply, build, apply3_pipe, apply3_x2, apply3_pf, apply3_occ, apply3_nw, apply3_el);
  }
};

const Dispatch& dispatch() {
  static Dispatch d;
  return d;
}

// ---------------------------------------------------------------------------
// Autotuner: which variant ran fastest for a (device, dim, P, Q, components,
// scatter mode, size class).  Filled by fem_b200_mass_autotune; consulted by
// FEM_B200_KERNEL_AUTO when a plan is created or reset to AUTO.
// ---------------------------------------------------------------------------
struct TuneKey {
  int device, dim, P, Q, comp_run, scatter, size_class;
  bool operator<(const TuneKey& o) const {
    return std::tie(device, dim, P, Q, comp_run, scatter, size_class) <
           std::tie(o.device, o.dim, o.P, o.Q, o.comp_run, o.scatter, o.size_class);
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, int> g_tune;

TuneKey tune_key(const MassPlan& p) {
  int size_class = 0;
  for (int64_t n = p.num_elem; n > 1; n >>= 1) ++size_class;  // log2(num_elem)
  return {p.device, p.dim, p.P, p.Q, p.comp_run, p.scatter_mode, size_class};
}

ApplyLauncher variant_launcher(const MassPlan& p, int variant) {
  switch (variant) {
    case FEM_B200_KERNEL_SIMPLE: return p.launch_simple;
    case FEM_B200_KERNEL_PIPELINED: return p.launch_pipe;
    case FEM_B200_KERNEL_PAIRED: return p.launch_x2;
    case FEM_B200_KERNEL_PREFETCH: return p.launch_pf;
    case FEM_B200_KERNEL_OCCUPANCY: return p.launch_occ;
    case FEM_B200_KERNEL_NARROW: return p.launch_nw;
    case FEM_B200_KERNEL_ELEMENT: return p.launch_el;
    default: return nullptr;
  }
}

// The variant a plan runs until it is autotuned: where one variant beat the
// one-tile kernel on every B200 of the order sweep (64M-DoF box meshes,
// Q = P + 1, one and three components), that one; else the one-tile kernel.
// element at P <= 3 (P = 2: 2.5x, P = 3: 1.1-1.15x).  At P = 6 with a
// centro-symmetric B the pipelined kernel with the even-odd contractions
// (0.723 / 0.634 ms against the one-tile kernel's 0.778 / 0.675 ms, one /
// three components, two interleaved runs on one box; at P = 4 and 7 it
// trails: 1.054 vs 0.954, 0.752 vs 0.602 ms).  Elsewhere the one-tile kernel
// (with the even-odd contractions at P = 4 and P >= 6); the ranking of the
// others moves from box to box, which the autotuner settles.
int default_variant(const MassPlan& p) {
  if (p.dim == 3 && p.Q == p.P + 1 && p.P <= 3) return FEM_B200_KERNEL_ELEMENT;
  if (p.dim == 3 && p.P == 6 && p.Q == 7 && p.centro_symmetric) return FEM_B200_KERNEL_PIPELINED;
  return FEM_B200_KERNEL_SIMPLE;
}

// The variant FEM_B200_KERNEL_AUTO selects for a plan: the autotuned choice
// for its key if there is one, else default_variant.
ApplyLauncher auto_kernel(const MassPlan& p) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  auto it = g_tune.find(tune_key(p));
  if (it != g_tune.end()) {
    ApplyLauncher l = variant_launcher(p, it->second);
    if (l) return l;
  }
  ApplyLauncher l = variant_launcher(p, default_variant(p));
  return l ? l : p.launch_simple;
}

bool fused_supported(int dim, int P, int Q) {
  return dim >= 1 && dim <= 3 && P >= kMinP && P <= kMaxP && Q >= P && Q < P + kQSpan;
}

// Shared memory of the 3D build kernel (5 planes of partial contractions).
int build3d_smem(int P, int Q) {
  const int E = 8;
  return (2 * P * plane_stride(P * Q * E, E) + 3 * P * plane_stride(Q * Q * E, E)) * 8;
}

std::string shape_str(int dim, int P, int Q) {
  return "dim=" + std::to_string(dim) + ", P=" + std::to_string(P) + ", Q=" + std::to_string(Q);
}

bool device_path_supported(int dim, int P, int Q) {
  return fused_supported(dim, P, Q) && !(dim == 3 && build3d_smem(P, Q) > kMaxSmemPerCta);
}

}  // namespace fem_b200

using namespace fem_b200;


// ===========================================================================
// Scratch for fem_b200_basis_apply_static: the ping-pong pass buffers of the
// basis contractions, in a fixed device array instead of cudaMalloc'd memory.
// Every GPU that loads this library holds it (16 MiB) until the process exits.
// ===========================================================================
static constexpr int64_t kStaticScratchDoubles = int64_t(1) << 21;  // 2,097,152 doubles = 16 MiB
static __device__ __align__(256) double g_basis_static_scratch[kStaticScratchDoubles];

namespace {
std::mutex g_static_scratch_mu;
double* g_static_scratch_ptr[64] = {};

// Device address of g_basis_static_scratch on the current device `dev`.  In
// host code the symbol itself is only a host-side stand-in, never a device
// address, so the address is looked up once per device and cached.
double* static_scratch_on(int dev) {
  require(dev >= 0 && dev < 64, "basis apply (static scratch): device index out of range");
  std::lock_guard<std::mutex> lock(g_static_scratch_mu);
  if (!g_static_scratch_ptr[dev]) {
    void* p = nullptr;
    FEM_CUDA_CHECK(cudaGetSymbolAddress(&p, g_basis_static_scratch));
    g_static_scratch_ptr[dev] = static_cast<double*>(p);
  }
  return g_static_scratch_ptr[dev];
}
}  // namespace

// ===========================================================================
// extern "C" entry points
// ===========================================================================
extern "C" {

const char* fem_b200_last_error(void) { return g_last_error.c_str(); }

int fem_b200_version(void) { return 100; }

int fem_b200_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  return n;
}

// ---- host set-up ----------------------------------------------------------
int fem_b200_gauss_legendre(int Q, double* x, double* w) {
  return guarded([&] {
    require(x && w, "gauss_legendre_quadrature: NULL output");
    gauss_legendre(Q, x, w);
  });
}

int fem_b200_gauss_lobatto(int Q, double* x, double* w) {
  return guarded([&] {
    require(x != nullptr, "gauss_lobatto_points: NULL output");
    gauss_lobatto(Q, x, w);
  });
}

int fem_b200_lagrange_basis_matrix(int P, const double* nodes, int M, const double* pts, double* interp,
                                   double* grad) {
  return guarded([&] {
    require(P >= 1 && M >= 0 && nodes && (M == 0 || (pts && interp && grad)), "lagrange_basis_matrix: bad arguments");
    lagrange_matrices(P, nodes, M, pts, interp, grad);
  });
}

int fem_b200_tensor_h1_lagrange(int dim, int num_comp, int P, int Q, int quad_mode, double* q_ref, double* q_weight,
                                double* interp, double* grad) {
  return guarded([&] {
    BasisData b = make_basis(dim, num_comp, P, Q, quad_mode);
    if (q_ref) std::copy(b.q_ref.begin(), b.q_ref.end(), q_ref);
    if (q_weight) std::copy(b.q_weight.begin(), b.q_weight.end(), q_weight);
    if (interp) std::copy(b.interp.begin(), b.interp.end(), interp);
    if (grad) std::copy(b.grad.begin(), b.grad.end(), grad);
  });
}

int fem_b200_restriction_check_offset(int num_elem, int elem_size, int num_comp, int comp_stride, int l_size,
                                      const int* offsets, int64_t n_offsets) {
  return guarded([&] { check_offset(num_elem, elem_size, num_comp, comp_stride, l_size, offsets, n_offsets); });
}

int fem_b200_restriction_check_strided(int num_elem, int elem_size, int num_comp, int l_size, const int* strides) {
  return guarded([&] { check_strided(num_elem, elem_size, num_comp, l_size, strides); });
}

int fem_b200_transpose_map(int num_elem, int elem_size, int l_size, const int* offsets, int* l_vec_indices,
                           int* t_offsets, int* t_indices, int* num_nodes) {
  return guarded([&] {
    require(num_elem > 0 && elem_size > 0 && l_size > 0 && offsets && l_vec_indices && t_offsets && t_indices,
            "build_transpose_map: bad arguments");
    for (int64_t t = 0; t < int64_t(num_elem) * elem_size; ++t)
      require(offsets[t] >= 0 && offsets[t] < l_size, "build_transpose_map: offset out of range");
    const int n = transpose_map(num_elem, elem_size, l_size, offsets, l_vec_indices, t_offsets, t_indices);
    if (num_nodes) *num_nodes = n;
  });
}

// ---- restriction ------------------------------------------------------------
int fem_b200_restriction_create_offset(int num_elem, int elem_size, int num_comp, int comp_stride, int l_size,
                                       const int* offsets, int scatter_mode, fem_b200_restriction* out) {
  return guarded([&] {
    require(out != nullptr, "elem_restriction_create: NULL output handle");
    require(scatter_mode == FEM_B200_SCATTER_ATOMIC || scatter_mode == FEM_B200_SCATTER_DETERMINISTIC,
            "elem_restriction_create: unknown scatter mode");
    const int64_t n_t = int64_t(num_elem) * elem_size;
    check_offset(num_elem, elem_size, num_comp, comp_stride, l_size, offsets, n_t);
    *out = new fem_b200_restriction_s{
        make_offset_restriction(num_elem, elem_size, num_comp, comp_stride, l_size, offsets, offsets, scatter_mode, 0)};
  });
}

int fem_b200_restriction_create_strided(int num_elem, int elem_size, int num_comp, int l_size, const int* strides,
                                        fem_b200_restriction* out) {
  return guarded([&] {
    require(out != nullptr, "elem_restriction_create_strided: NULL output handle");
    check_strided(num_elem, elem_size, num_comp, l_size, strides);
    auto d = std::make_shared<RestrictionData>();
    d->device = current_device();
    d->strided = true;
    d->num_elem = num_elem, d->elem_size = elem_size, d->num_comp = num_comp, d->l_size = l_size;
    d->e_size = int64_t(num_comp) * elem_size * num_elem;
    if (strides) {
      for (int i = 0; i < 3; ++i) d->strides[i] = strides[i];
    } else {
      d->strides[0] = num_elem, d->strides[1] = int64_t(elem_size) * num_elem, d->strides[2] = 1;
    }
    *out = new fem_b200_restriction_s{std::move(d)};
  });
}

int fem_b200_restriction_destroy(fem_b200_restriction r) {
  return guarded([&] { delete r; });
}

int fem_b200_restriction_sizes(fem_b200_restriction r, int* num_elem, int* elem_size, int* num_comp, int* l_size,
                               int64_t* e_size) {
  return guarded([&] {
    require(r && r->d, "restriction: NULL handle");
    const RestrictionData& d = *r->d;
    if (num_elem) *num_elem = d.num_elem;
    if (elem_size) *elem_size = d.elem_size;
    if (num_comp) *num_comp = d.num_comp;
    if (l_size) *l_size = d.l_size;
    if (e_size) *e_size = d.e_size;
  });
}

int fem_b200_restriction_transpose_map(fem_b200_restriction r, int* l_vec_indices, int* t_offsets, int* t_indices,
                                       int* num_nodes) {
  return guarded([&] {
    require(r && r->d, "restriction: NULL handle");
    const RestrictionData& d = *r->d;
    require(!d.strided && d.scatter_mode == FEM_B200_SCATTER_DETERMINISTIC,
            "restriction has no transpose map (deterministic offset restrictions only)");
    DeviceGuard g(d.device);
    if (num_nodes) *num_nodes = d.num_nodes;
    const int64_t n_t = int64_t(d.num_elem) * d.elem_size;
    if (l_vec_indices)
      FEM_CUDA_CHECK(cudaMemcpy(l_vec_indices, d.l_vec_indices.get(), d.num_nodes * sizeof(int), cudaMemcpyDeviceToHost));
    if (t_offsets)
      FEM_CUDA_CHECK(cudaMemcpy(t_offsets, d.t_offsets.get(), (d.num_nodes + 1) * sizeof(int), cudaMemcpyDeviceToHost));
    if (t_indices) FEM_CUDA_CHECK(cudaMemcpy(t_indices, d.t_indices.get(), n_t * sizeof(int), cudaMemcpyDeviceToHost));
  });
}

int fem_b200_restriction_apply(fem_b200_restriction r, int t_mode, const double* in, int64_t n_in, double* out,
                               int64_t n_out, void* stream) {
  return guarded([&] {
    require(r && r->d, "elem_restriction_apply: NULL handle");
    const RestrictionData& d = *r->d;
    const bool tr = t_mode == FEM_B200_TRANSPOSE;
    require(t_mode == FEM_B200_NOTRANSPOSE || tr, "elem_restriction_apply: unknown t_mode");
    require(n_in == (tr ? d.e_size : d.l_size), "elem_restriction_apply: in has the wrong size");
    require(n_out == (tr ? int64_t(d.l_size) : d.e_size),
            tr ? "elem_restriction_apply: Transpose adds into out, which must already have l_size entries"
               : "elem_restriction_apply: out must have e_size entries");
    require(in && out, "elem_restriction_apply: NULL array");
    DeviceGuard g(d.device);
    cudaStream_t s = as_stream(stream);
    if (d.strided) {
      const int grid = grid_for(d.e_size, 256);
      if (!tr)
        strided_kernel<0><<<grid, 256, 0, s>>>(d.num_elem, d.elem_size, d.num_comp, d.strides[0], d.strides[1],
                                               d.strides[2], in, out);
      else
        strided_kernel<1><<<grid, 256, 0, s>>>(d.num_elem, d.elem_size, d.num_comp, d.strides[0], d.strides[1],
                                               d.strides[2], in, out);
    } else if (!tr || d.scatter_mode == FEM_B200_SCATTER_ATOMIC) {
      const dim3 grid(unsigned((d.elem_size + kTile - 1) / kTile), unsigned((d.num_elem + kTile - 1) / kTile));
      const dim3 block(kTile, 8);
      if (!tr)
        offset_tile_kernel<0><<<grid, block, 0, s>>>(d.offsets.get(), d.num_elem, d.elem_size, d.num_comp,
                                                     d.comp_stride, in, out);
      else
        offset_tile_kernel<1><<<grid, block, 0, s>>>(d.offsets.get(), d.num_elem, d.elem_size, d.num_comp,
                                                     d.comp_stride, in, out);
    } else {
      launch_csr_scatter(d.num_nodes, d.num_elem, d.elem_size, d.num_comp, d.comp_stride, d.l_vec_indices.get(),
                         d.t_offsets.get(), d.t_indices.get(), in, out, s);
    }
    FEM_LAUNCH_CHECK();
  });
}

int fem_b200_restriction_multiplicity(fem_b200_restriction r, double* mult, int64_t n, void* stream) {
  return guarded([&] {
    require(r && r->d, "elem_restriction_get_multiplicity: NULL handle");
    const RestrictionData& d = *r->d;
    require(n == d.l_size && mult, "elem_restriction_get_multiplicity: mult must have l_size entries");
    DeviceGuard g(d.device);
    cudaStream_t s = as_stream(stream);
    FEM_CUDA_CHECK(cudaMemsetAsync(mult, 0, n * sizeof(double), s));
    if (d.strided) {
      // every strided index is hit once: scatter a vector of ones
      DevBuf<double> ones(size_t(d.e_size));
      std::vector<double> h(size_t(d.e_size), 1.0);
      FEM_CUDA_CHECK(cudaMemcpyAsync(ones.get(), h.data(), d.e_size * sizeof(double), cudaMemcpyHostToDevice, s));
      strided_kernel<1><<<grid_for(d.e_size, 256), 256, 0, s>>>(d.num_elem, d.elem_size, d.num_comp, d.strides[0],
                                                                 d.strides[1], d.strides[2], ones.get(), mult);
      FEM_LAUNCH_CHECK();
      FEM_CUDA_CHECK(cudaStreamSynchronize(s));
      return;
    }
    const dim3 grid(unsigned((d.elem_size + kTile - 1) / kTile), unsigned((d.num_elem + kTile - 1) / kTile));
    offset_tile_kernel<2><<<grid, dim3(kTile, 8), 0, s>>>(d.offsets.get(), d.num_elem, d.elem_size, d.num_comp,
                                                          d.comp_stride, nullptr, mult);
    FEM_LAUNCH_CHECK();
  });
}

// ---- basis --------------------------------------------------------------------
int fem_b200_basis_create(int dim, int num_comp, int P, int Q, int quad_mode, fem_b200_basis* out) {
  return guarded([&] {
    require(out != nullptr, "create_tensor_H1_lagrange: NULL output handle");
    auto d = std::make_unique<BasisDev>();
    d->h = make_basis(dim, num_comp, P, Q, quad_mode);
    d->device = current_device();
    d->interp.alloc(d->h.interp.size());
    d->grad.alloc(d->h.grad.size());
    d->weight.alloc(d->h.q_weight.size());
    FEM_CUDA_CHECK(cudaMemcpy(d->interp.get(), d->h.interp.data(), d->interp.bytes(), cudaMemcpyHostToDevice));
    FEM_CUDA_CHECK(cudaMemcpy(d->grad.get(), d->h.grad.data(), d->grad.bytes(), cudaMemcpyHostToDevice));
    FEM_CUDA_CHECK(cudaMemcpy(d->weight.get(), d->h.q_weight.data(), d->weight.bytes(), cudaMemcpyHostToDevice));
    *out = new fem_b200_basis_s{std::move(d)};
  });
}

int fem_b200_basis_create_from(int dim, int num_comp, int P, int Q, const double* q_weight, const double* interp,
                               const double* grad, fem_b200_basis* out) {
  return guarded([&] {
    require(out != nullptr, "basis: NULL output handle");
    require(dim >= 1 && dim <= 3 && num_comp >= 1 && P >= 1 && Q >= 1, "basis: bad sizes");
    require(q_weight && interp && grad, "basis: NULL matrix");
    auto d = std::make_unique<BasisDev>();
    d->h.dim = dim, d->h.num_comp = num_comp, d->h.P = P, d->h.Q = Q, d->h.quad_mode = -1;
    d->h.q_ref.assign(size_t(Q), 0.0);
    d->h.q_weight.assign(q_weight, q_weight + Q);
    d->h.interp.assign(interp, interp + size_t(Q) * P);
    d->h.grad.assign(grad, grad + size_t(Q) * P);
    d->device = current_device();
    d->interp.alloc(d->h.interp.size());
    d->grad.alloc(d->h.grad.size());
    d->weight.alloc(d->h.q_weight.size());
    FEM_CUDA_CHECK(cudaMemcpy(d->interp.get(), d->h.interp.data(), d->interp.bytes(), cudaMemcpyHostToDevice));
    FEM_CUDA_CHECK(cudaMemcpy(d->grad.get(), d->h.grad.data(), d->grad.bytes(), cudaMemcpyHostToDevice));
    FEM_CUDA_CHECK(cudaMemcpy(d->weight.get(), d->h.q_weight.data(), d->weight.bytes(), cudaMemcpyHostToDevice));
    *out = new fem_b200_basis_s{std::move(d)};
  });
}

int fem_b200_basis_destroy(fem_b200_basis b) {
  return guarded([&] { delete b; });
}

int fem_b200_basis_apply(fem_b200_basis b, int num_elem, int t_mode, int eval_mode, const double* u, int64_t n_u,
                         double* v, int64_t n_v, void* stream) {
  return guarded([&] {
    require(b && b->d, "tensor_basis_apply: NULL handle");
    BasisDev& bd = *b->d;
    const BasisData& h = bd.h;
    const bool tr = t_mode == FEM_B200_TRANSPOSE;
    require(t_mode == FEM_B200_NOTRANSPOSE || tr, "tensor_basis_apply: unknown t_mode");
    require(num_elem > 0, "tensor_basis_apply: num_elem must be positive");
    const int64_t pn = ipow(h.P, h.dim) * h.num_comp * num_elem;  // nodal size
    const int64_t qn = ipow(h.Q, h.dim) * h.num_comp * num_elem;  // one block at the points
    DeviceGuard g(bd.device);
    cudaStream_t s = as_stream(stream);
    if (eval_mode == FEM_B200_EVAL_WEIGHT) {
      require(!tr, "EvalMode::Weight is incompatible with ContractMode::Transpose");
      require(n_v == ipow(h.Q, h.dim) * num_elem && v, "tensor_basis_apply: v has the wrong size");
      weight_kernel<<<grid_for(n_v, 256), 256, 0, s>>>(h.dim, h.Q, bd.weight.get(), num_elem, v);
      FEM_LAUNCH_CHECK();
      return;
    }
    require(eval_mode == FEM_B200_EVAL_INTERP || eval_mode == FEM_B200_EVAL_GRAD,
            "tensor_basis_apply: unknown eval_mode");
    const bool grad = eval_mode == FEM_B200_EVAL_GRAD;
    const int64_t in_n = tr ? (grad ? h.dim * qn : qn) : pn;
    const int64_t out_n = tr ? pn : (grad ? h.dim * qn : qn);
    require(n_u == in_n && u, "tensor_basis_apply: u has the wrong size");
    require(n_v == out_n && v, "tensor_basis_apply: v has the wrong size");
    // dim 3: one fused pass, no scratch
    if (basis3d_fused_apply(h, num_elem, tr, grad, u, v, s)) return;
    const int P = tr ? h.Q : h.P, Q = tr ? h.P : h.Q;  // contracted in / out sizes
    const int64_t big = h.num_comp * ipow(std::max(h.P, h.Q), h.dim) * num_elem;
    std::lock_guard<std::mutex> lock(bd.scratch_mu);
    if (h.dim > 1 && bd.scratch.size() < size_t(2 * big)) bd.scratch.alloc(size_t(2 * big));
    double* tmp[2] = {bd.scratch.get(), bd.scratch.get() + big};
    const int naxes = grad ? h.dim : 1;
    for (int ax = 0; ax < naxes; ++ax) {
      int64_t pre = h.num_comp * ipow(P, h.dim - 1), post = num_elem;
      for (int dd = 0; dd < h.dim; ++dd) {
        const double* mat = (grad && dd == ax) ? bd.grad.get() : bd.interp.get();
        const double* src = dd == 0 ? (tr && grad ? u + ax * qn : u) : tmp[dd % 2];
        const bool last = dd == h.dim - 1;
        double* dst = last ? (tr ? v : (grad ? v + ax * qn : v)) : tmp[(dd + 1) % 2];
        const int add = (last && tr && grad && ax > 0) ? 1 : 0;
        const int64_t n = pre * Q * post;
        contract_kernel<<<grid_for(n, 256), 256, 0, s>>>(pre, P, post, Q, mat, tr ? 1 : 0, add, src, dst);
        FEM_LAUNCH_CHECK();
        pre /= P;
        post *= Q;
      }
    }
  });
}

// Same contractions as fem_b200_basis_apply: dim 3 first through the fused
// one-pass kernels (no scratch at all, no size limit), otherwise the generic
// passes with their buffers in g_basis_static_scratch.  Nothing is allocated.
// Each pass overwrites the scratch it writes, so nothing has to be cleared
// between calls; the scratch address is looked up only when a call uses it.
int fem_b200_basis_apply_static(fem_b200_basis b, int num_elem, int t_mode, int eval_mode, const double* u,
                                int64_t n_u, double* v, int64_t n_v, void* stream) {
  return guarded([&] {
    require(b && b->d, "tensor_basis_apply: NULL handle");
    BasisDev& bd = *b->d;
    const BasisData& h = bd.h;
    const bool tr = t_mode == FEM_B200_TRANSPOSE;
    require(t_mode == FEM_B200_NOTRANSPOSE || tr, "tensor_basis_apply: unknown t_mode");
    require(num_elem > 0, "tensor_basis_apply: num_elem must be positive");
    const int64_t pn = ipow(h.P, h.dim) * h.num_comp * num_elem;
    const int64_t qn = ipow(h.Q, h.dim) * h.num_comp * num_elem;
    DeviceGuard g(bd.device);
    cudaStream_t s = as_stream(stream);
    if (eval_mode == FEM_B200_EVAL_WEIGHT) {
      require(!tr, "EvalMode::Weight is incompatible with ContractMode::Transpose");
      require(n_v == ipow(h.Q, h.dim) * num_elem && v, "tensor_basis_apply: v has the wrong size");
      weight_kernel<<<grid_for(n_v, 256), 256, 0, s>>>(h.dim, h.Q, bd.weight.get(), num_elem, v);
      FEM_LAUNCH_CHECK();
      return;
    }
    require(eval_mode == FEM_B200_EVAL_INTERP || eval_mode == FEM_B200_EVAL_GRAD,
            "tensor_basis_apply: unknown eval_mode");
    const bool grad = eval_mode == FEM_B200_EVAL_GRAD;
    const int64_t in_n = tr ? (grad ? h.dim * qn : qn) : pn;
    const int64_t out_n = tr ? pn : (grad ? h.dim * qn : qn);
    require(n_u == in_n && u, "tensor_basis_apply: u has the wrong size");
    require(n_v == out_n && v, "tensor_basis_apply: v has the wrong size");
    // dim 3: one fused pass, no scratch (the same kernels as fem_b200_basis_apply)
    if (basis3d_fused_apply(h, num_elem, tr, grad, u, v, s)) return;
    const int P = tr ? h.Q : h.P, Q = tr ? h.P : h.Q;
    const int64_t big = h.num_comp * ipow(std::max(h.P, h.Q), h.dim) * num_elem;
    const int64_t need = h.dim > 1 ? 2 * big : 0;
    if (need > kStaticScratchDoubles)
      throw arg_error("tensor_basis_apply (static scratch): this call needs " + std::to_string(need) +
                      " doubles of scratch (2 * num_comp * max(P,Q)^dim * num_elem) but the static scratch holds " +
                      std::to_string(kStaticScratchDoubles) + " (16 MiB); split the elements into smaller calls");
    double* scratch = need > 0 ? static_scratch_on(bd.device) : nullptr;  // dim 1 passes use no scratch
    double* tmp[2] = {scratch, scratch ? scratch + big : nullptr};
    const int naxes = grad ? h.dim : 1;
    for (int ax = 0; ax < naxes; ++ax) {
      int64_t pre = h.num_comp * ipow(P, h.dim - 1), post = num_elem;
      for (int dd = 0; dd < h.dim; ++dd) {
        const double* mat = (grad && dd == ax) ? bd.grad.get() : bd.interp.get();
        const double* src = dd == 0 ? (tr && grad ? u + ax * qn : u) : tmp[dd % 2];
        const bool last = dd == h.dim - 1;
        double* dst = last ? (tr ? v : (grad ? v + ax * qn : v)) : tmp[(dd + 1) % 2];
        const int add = (last && tr && grad && ax > 0) ? 1 : 0;
        const int64_t n = pre * Q * post;
        contract_kernel<<<grid_for(n, 256), 256, 0, s>>>(pre, P, post, Q, mat, tr ? 1 : 0, add, src, dst);
        FEM_LAUNCH_CHECK();
        pre /= P;
        post *= Q;
      }
    }
  });
}

// ---- device memory and raw launchers (the C++ drop-in's building blocks) ----
int fem_b200_malloc(void** ptr, size_t bytes) {
  return guarded([&] {
    require(ptr != nullptr, "fem_b200_malloc: NULL output");
    *ptr = nullptr;
    if (bytes) FEM_CUDA_CHECK(cudaMalloc(ptr, bytes));
  });
}

int fem_b200_free(void* ptr) {
  return guarded([&] {
    if (ptr) FEM_CUDA_CHECK(cudaFree(ptr));
  });
}

int fem_b200_memcpy(void* dst, const void* src, size_t bytes, int kind, void* stream) {
  return guarded([&] {
    require(kind >= 0 && kind <= 2, "fem_b200_memcpy: kind must be 0 (H2D), 1 (D2H) or 2 (D2D)");
    if (!bytes) return;
    require(dst && src, "fem_b200_memcpy: NULL pointer");
    const cudaMemcpyKind k[3] = {cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost, cudaMemcpyDeviceToDevice};
    cudaStream_t s = as_stream(stream);
    FEM_CUDA_CHECK(cudaMemcpyAsync(dst, src, bytes, k[kind], s));
    if (kind != 2) FEM_CUDA_CHECK(cudaStreamSynchronize(s));
  });
}

int fem_b200_memset_zero(void* ptr, size_t bytes, void* stream) {
  return guarded([&] {
    if (bytes) FEM_CUDA_CHECK(cudaMemsetAsync(ptr, 0, bytes, as_stream(stream)));
  });
}

int fem_b200_synchronize(void* stream) {
  return guarded([&] { FEM_CUDA_CHECK(cudaStreamSynchronize(as_stream(stream))); });
}

int fem_b200_device_info(int device, char* name, int name_len, int* ints, int64_t* sizes) {
  return guarded([&] {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
      (void)cudaGetLastError();
      n = 0;
    }
    require(device >= 0 && device < n, "device_info: no such CUDA device");
    cudaDeviceProp prop;
    FEM_CUDA_CHECK(cudaGetDeviceProperties(&prop, device));
    if (name && name_len > 0) {
      std::strncpy(name, prop.name, size_t(name_len) - 1);
      name[name_len - 1] = '\0';
    }
    if (ints) {
      ints[0] = prop.major, ints[1] = prop.minor, ints[2] = prop.multiProcessorCount, ints[3] = prop.warpSize;
      ints[4] = prop.maxThreadsPerBlock, ints[5] = prop.regsPerBlock;
    }
    if (sizes) {
      DeviceGuard g(device);
      size_t free_b = 0, total_b = 0;
      FEM_CUDA_CHECK(cudaMemGetInfo(&free_b, &total_b));
      sizes[0] = int64_t(prop.sharedMemPerBlock), sizes[1] = int64_t(prop.sharedMemPerBlockOptin);
      sizes[2] = int64_t(prop.sharedMemPerMultiprocessor), sizes[3] = int64_t(prop.totalGlobalMem);
      sizes[4] = int64_t(free_b);
    }
  });
}

int fem_b200_offset_gather(int num_elem, int elem_size, int num_comp, int comp_stride, const int* offsets,
                           const double* l_in, double* e_out, void* stream) {
  return guarded([&] {
    require(num_elem > 0 && elem_size > 0 && num_comp > 0 && offsets && l_in && e_out, "offset gather: bad arguments");
    const dim3 grid(unsigned((elem_size + kTile - 1) / kTile), unsigned((num_elem + kTile - 1) / kTile));
    offset_tile_kernel<0><<<grid, dim3(kTile, 8), 0, as_stream(stream)>>>(offsets, num_elem, elem_size, num_comp,
                                                                         comp_stride, l_in, e_out);
    FEM_LAUNCH_CHECK();
  });
}

int fem_b200_offset_scatter_add(int num_elem, int elem_size, int num_comp, int comp_stride, const int* offsets,
                                const double* e_in, double* l_out, void* stream) {
  return guarded([&] {
    require(num_elem > 0 && elem_size > 0 && num_comp > 0 && offsets && e_in && l_out, "offset scatter: bad arguments");
    const dim3 grid(unsigned((elem_size + kTile - 1) / kTile), unsigned((num_elem + kTile - 1) / kTile));
    offset_tile_kernel<1><<<grid, dim3(kTile, 8), 0, as_stream(stream)>>>(offsets, num_elem, elem_size, num_comp,
                                                                         comp_stride, e_in, l_out);
    FEM_LAUNCH_CHECK();
  });
}

int fem_b200_transpose_scatter_add(int num_nodes, int num_elem, int elem_size, int num_comp, int comp_stride,
                                   const int* l_vec_indices, const int* t_offsets, const int* t_indices,
                                   const double* e_in, double* l_out, void* stream) {
  return guarded([&] {
    require(num_nodes >= 0 && num_elem > 0 && elem_size > 0 && num_comp > 0, "transpose scatter: bad sizes");
    if (num_nodes == 0) return;
    require(l_vec_indices && t_offsets && t_indices && e_in && l_out, "transpose scatter: NULL array");
    launch_csr_scatter(num_nodes, num_elem, elem_size, num_comp, comp_stride, l_vec_indices, t_offsets, t_indices,
                       e_in, l_out, as_stream(stream));
    FEM_LAUNCH_CHECK();
  });
}

int fem_b200_strided_apply(int t_mode, int num_elem, int elem_size, int num_comp, const int* strides,
                           const double* in, double* out, void* stream) {
  return guarded([&] {
    require(num_elem > 0 && elem_size > 0 && num_comp > 0 && strides && in && out, "strided apply: bad arguments");
    const int64_t n = int64_t(num_elem) * elem_size * num_comp;
    if (t_mode == FEM_B200_NOTRANSPOSE)
      strided_kernel<0><<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(num_elem, elem_size, num_comp, strides[0],
                                                                         strides[1], strides[2], in, out);
    else
      strided_kernel<1><<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(num_elem, elem_size, num_comp, strides[0],
                                                                         strides[1], strides[2], in, out);
    FEM_LAUNCH_CHECK();
  });
}

int fem_b200_contract(int64_t A, int B, int64_t C, int J, const double* t, int t_mode, int add, const double* u,
                      double* v, void* stream) {
  return guarded([&] {
    require(A >= 0 && B >= 0 && C >= 0 && J >= 0, "tensor_contract_apply: negative size");
    const int64_t n = A * J * C;
    if (n == 0) return;
    require(t && u && v, "tensor_contract_apply: NULL array");
    contract_kernel<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(A, B, C, J, t, t_mode == FEM_B200_TRANSPOSE,
                                                                     add ? 1 : 0, u, v);
    FEM_LAUNCH_CHECK();
  });
}

int fem_b200_qfunction_apply_mass(int64_t Q, const double* u, const double* qdata, double* v, void* stream) {
  return guarded([&] {
    require(Q > 0 && u && qdata && v, "apply_mass: bad arguments");
    qf_apply_mass_kernel<<<grid_for(Q, 256), 256, 0, as_stream(stream)>>>(Q, u, qdata, v);
    FEM_LAUNCH_CHECK();
  });
}

int fem_b200_qfunction_build_mass(int dim, int64_t Q, const double* J, const double* w, double* qdata, void* stream) {
  return guarded([&] {
    require(dim >= 1 && dim <= 3, "build_mass: dim must be 1, 2 or 3");
    require(Q > 0 && J && w && qdata, "build_mass: bad arguments");
    qf_build_mass_kernel<<<grid_for(Q, 256), 256, 0, as_stream(stream)>>>(dim, Q, J, w, qdata);
    FEM_LAUNCH_CHECK();
  });
}

// ---- mass ---------------------------------------------------------------------
int fem_b200_mass_build(fem_b200_restriction rx, fem_b200_basis bx, const double* x, int64_t n_x, double* qdata,
                        int64_t n_qdata, void* stream) {
  return guarded([&] {
    require(rx && rx->d && bx && bx->d, "mass build: NULL handle");
    const RestrictionData& r = *rx->d;
    const BasisData& b = bx->d->h;
    require(!r.strided, "mass build: the coordinate restriction must be an offset restriction");
    require(b.num_comp == b.dim && r.num_comp == b.dim, "mass build: coordinates need num_comp == dim");
    require(r.elem_size == ipow(b.P, b.dim), "operator_set_field 'dx': restriction elem_size must equal basis P_1d^dim");
    require(n_x == r.l_size && x, "mass build: x must have l_size entries");
    require(n_qdata == ipow(b.Q, b.dim) * r.num_elem && qdata, "mass build: qdata must have Q^dim*num_elem entries");
    if (!fused_supported(b.dim, b.P, b.Q) || (b.dim == 3 && build3d_smem(b.P, b.Q) > kMaxSmemPerCta))
      throw unsupported_error("mass build: no device kernel for " + shape_str(b.dim, b.P, b.Q) +
                              " (P in 2..8, Q in P..P+2; dim 3 with P = 8 up to Q = 9)");
    DeviceGuard g(r.device);
    mass_build_impl(b, r, x, qdata, as_stream(stream));
  });
}

int fem_b200_mass_create(fem_b200_restriction ru, fem_b200_basis bu, const double* qdata, int64_t n_qdata, int qf,
                         fem_b200_mass* out) {
  return guarded([&] {
    require(out != nullptr, "operator_create: NULL output handle");
    require(ru && ru->d && bu && bu->d, "operator_set_field: NULL handle");
    const std::shared_ptr<RestrictionData>& r = ru->d;
    const BasisData& b = bu->d->h;
    require(qf == FEM_B200_QF_APPLY_MASS || qf == FEM_B200_QF_APPLY_MASS_VECTOR, "operator_create: unknown QFunction");
    require(!r->strided, "operator_set_field 'u': the active field needs an offset restriction");
    require(r->num_comp == b.num_comp, "operator_set_field 'u': restriction and basis num_comp differ");
    require(r->elem_size == ipow(b.P, b.dim), "operator_set_field 'u': restriction elem_size must equal basis P_1d^dim");
    const int64_t nq = ipow(b.Q, b.dim);
    require(n_qdata == nq * r->num_elem && qdata, "operator_set_field 'qdata': passive vector size must equal restriction l_size");
    if (!fused_supported(b.dim, b.P, b.Q))
      throw unsupported_error("operator_apply: no fused device kernel for " + shape_str(b.dim, b.P, b.Q) +
                              " (P in 2..8, Q in P..P+2)");
    DeviceGuard g(r->device);
    auto p = make_mass_plan(r, b, qdata, qf, 0);
    FEM_CUDA_CHECK(cudaDeviceSynchronize());
    *out = new fem_b200_mass_s{std::move(p)};
  });
}

int fem_b200_mass_destroy(fem_b200_mass op) {
  return guarded([&] { delete op; });
}

}  // extern "C"

namespace fem_b200 {
// Reads and clears the plan's device status word (the caller has synchronised).
void check_status(MassPlan& p, cudaStream_t s) {
  int st = 0;
  if (s) {  // pageable destination: returns once the copy is done
    FEM_CUDA_CHECK(cudaMemcpyAsync(&st, p.status.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  } else {
    FEM_CUDA_CHECK(cudaMemcpy(&st, p.status.get(), sizeof(int), cudaMemcpyDeviceToHost));
  }
  if (st) {
    FEM_CUDA_CHECK(cudaMemsetAsync(p.status.get(), 0, sizeof(int), s));
    throw cuda_error("operator_apply: a bounded wait in the mass kernel ran out (status " + std::to_string(st) +
                     "); the result is not valid");
  }
}

// ---- stream-ordered cores of the create / build entry points ---------------
std::shared_ptr<RestrictionData> make_offset_restriction(int num_elem, int elem_size, int num_comp, int comp_stride,
                                                         int l_size, const int* offs, const int* host_offsets,
                                                         int scatter_mode, cudaStream_t s) {
  const int64_t n_t = int64_t(num_elem) * elem_size;
  auto d = std::make_shared<RestrictionData>();
  d->device = current_device();
  d->num_elem = num_elem, d->elem_size = elem_size, d->num_comp = num_comp;
  d->comp_stride = comp_stride;
  d->l_size = l_size;
  d->e_size = int64_t(num_comp) * n_t;
  d->scatter_mode = scatter_mode;
  d->offsets.alloc(size_t(n_t));
  FEM_CUDA_CHECK(cudaMemcpyAsync(d->offsets.get(), offs, n_t * sizeof(int), cudaMemcpyDefault, s));
  std::vector<int> lvi, toff, tidx;
  if (scatter_mode == FEM_B200_SCATTER_DETERMINISTIC) {
    require(host_offsets != nullptr, "elem_restriction_create: the deterministic scatter needs host offsets");
    lvi.resize(size_t(l_size)), toff.resize(size_t(l_size) + 1), tidx.resize(size_t(n_t));
    const int n = transpose_map(num_elem, elem_size, l_size, host_offsets, lvi.data(), toff.data(), tidx.data());
    d->num_nodes = n;
    d->l_vec_indices.alloc(size_t(n));
    d->t_offsets.alloc(size_t(n) + 1);
    d->t_indices.alloc(size_t(n_t));
    FEM_CUDA_CHECK(cudaMemcpyAsync(d->l_vec_indices.get(), lvi.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
    FEM_CUDA_CHECK(cudaMemcpyAsync(d->t_offsets.get(), toff.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
    FEM_CUDA_CHECK(cudaMemcpyAsync(d->t_indices.get(), tidx.data(), n_t * sizeof(int), cudaMemcpyHostToDevice, s));
  }
  FEM_CUDA_CHECK(cudaStreamSynchronize(s));  // the host vectors go out of scope
  return d;
}

void mass_build_impl(const BasisData& b, const RestrictionData& r, const double* x, double* qdata, cudaStream_t s) {
  dispatch().build[b.dim - 1][b.P][b.Q - b.P](b, r, x, qdata, s);
}

std::unique_ptr<MassPlan> make_mass_plan(const std::shared_ptr<RestrictionData>& r, const BasisData& b,
                                         const double* qdata, int qf, cudaStream_t s) {
  const int64_t nq = ipow(b.Q, b.dim);
  auto p = std::make_unique<MassPlan>();
  p->device = r->device;
  p->dim = b.dim, p->P = b.P, p->Q = b.Q, p->num_comp = b.num_comp;
  p->qf = qf;
  p->comp_run = qf == FEM_B200_QF_APPLY_MASS ? 1 : b.num_comp;
  p->scatter_mode = r->scatter_mode;
  p->num_elem = r->num_elem, p->l_size = r->l_size, p->es = r->elem_size, p->nq = int(nq);
  p->comp_stride = r->comp_stride;
  p->basis = b;
  p->r = r;
  p->tile_e = b.dim == 3 ? 8 : (b.dim == 2 ? 32 : 128);
  {
    double mx = 0.0, asym = 0.0;
    for (int q = 0; q < b.Q; ++q)
      for (int j = 0; j < b.P; ++j) {
        const double x = b.interp[size_t(q * b.P + j)];
        const double y = b.interp[size_t((b.Q - 1 - q) * b.P + (b.P - 1 - j))];
        mx = std::max(mx, std::fabs(x));
        asym = std::max(asym, std::fabs(x - y));
      }
    p->centro_symmetric = asym <= 1e-14 * mx;
  }
  p->n_tiles = (int64_t(p->num_elem) + p->tile_e - 1) / p->tile_e;
  // an even number of tiles, so a kernel taking two tiles per CTA stays inside
  const int64_t ne_pad = ((p->n_tiles + 1) / 2) * 2 * p->tile_e;
  p->offs_t.alloc(size_t(ne_pad * p->es));
  p->qd_t.alloc(size_t(ne_pad * p->nq));
  tile_offsets_kernel<<<grid_for(ne_pad * p->es, 256), 256, 0, s>>>(r->offsets.get(), p->num_elem, p->es,
                                                                     p->tile_e, ne_pad * p->es, p->offs_t.get());
  FEM_LAUNCH_CHECK();
  tile_qdata_kernel<<<grid_for(ne_pad * p->nq, 256), 256, 0, s>>>(qdata, p->num_elem, p->Q, p->nq, p->tile_e,
                                                                   ne_pad * p->nq, p->qd_t.get());
  FEM_LAUNCH_CHECK();
  if (p->scatter_mode == FEM_B200_SCATTER_DETERMINISTIC)
    p->evec.alloc(size_t(int64_t(p->comp_run) * p->es * p->num_elem));
  p->status.alloc(1);
  FEM_CUDA_CHECK(cudaMemsetAsync(p->status.get(), 0, sizeof(int), s));
  p->launch_simple = dispatch().apply[b.dim - 1][b.P][b.Q - b.P];
  p->launch_pipe = b.dim == 3 ? dispatch().apply3_pipe[b.P][b.Q - b.P] : nullptr;
  p->launch_x2 = b.dim == 3 ? dispatch().apply3_x2[b.P][b.Q - b.P] : nullptr;
  p->launch_pf = b.dim == 3 ? dispatch().apply3_pf[b.P][b.Q - b.P] : nullptr;
  p->launch_occ = b.dim == 3 ? dispatch().apply3_occ[b.P][b.Q - b.P] : nullptr;
  p->launch_nw = b.dim == 3 ? dispatch().apply3_nw[b.P][b.Q - b.P] : nullptr;
  p->launch_el = b.dim == 3 ? dispatch().apply3_el[b.P][b.Q - b.P] : nullptr;
  p->launch = auto_kernel(*p);
  FEM_CUDA_CHECK(cudaStreamSynchronize(s));
  return p;
}

void mass_apply_impl(MassPlan& p, const double* u, double* v, bool zero, cudaStream_t s) {
  if (zero) FEM_CUDA_CHECK(cudaMemsetAsync(v, 0, size_t(p.l_size) * sizeof(double), s));
  if (p.scatter_mode == FEM_B200_SCATTER_ATOMIC) {
    p.launch(p, u, v, nullptr, s);
    return;
  }
  const RestrictionData& r = *p.r;
  p.launch(p, u, v, p.evec.get(), s);
  launch_csr_scatter(r.num_nodes, p.num_elem, p.es, p.comp_run, p.comp_stride, r.l_vec_indices.get(),
                     r.t_offsets.get(), r.t_indices.get(), p.evec.get(), v, s);
  FEM_LAUNCH_CHECK();
}
}  // namespace fem_b200

extern "C" {

int fem_b200_mass_apply(fem_b200_mass op, const double* u, int64_t n_u, double* v, int64_t n_v, void* stream) {
  return guarded([&] {
    require(op && op->d, "operator_apply: NULL handle");
    MassPlan& p = *op->d;
    require(n_u == p.l_size && u, "operator_apply: input vector size does not match active_in_l_size");
    require(n_v == p.l_size && v, "operator_apply: output vector size does not match active_out_l_size");
    DeviceGuard g(p.device);
    mass_apply_impl(p, u, v, true, as_stream(stream));
  });
}

int fem_b200_mass_apply_add(fem_b200_mass op, const double* u, int64_t n_u, double* v, int64_t n_v, void* stream) {
  return guarded([&] {
    require(op && op->d, "operator_apply: NULL handle");
    MassPlan& p = *op->d;
    require(n_u == p.l_size && u, "operator_apply: input vector size does not match active_in_l_size");
    require(n_v == p.l_size && v, "operator_apply: output vector size does not match active_out_l_size");
    DeviceGuard g(p.device);
    mass_apply_impl(p, u, v, false, as_stream(stream));
  });
}

int fem_b200_mass_apply_host(fem_b200_mass op, const double* u_host, int64_t n_u, double* v_host, int64_t n_v,
                             void* stream) {
  return guarded([&] {
    require(op && op->d, "operator_apply: NULL handle");
    MassPlan& p = *op->d;
    require(n_u == p.l_size && u_host, "operator_apply: input vector size does not match active_in_l_size");
    require(n_v == p.l_size && v_host, "operator_apply: output vector size does not match active_out_l_size");
    DeviceGuard g(p.device);
    cudaStream_t s = as_stream(stream);
    if (p.hu.size() != size_t(p.l_size)) p.hu.alloc(size_t(p.l_size));
    if (p.hv.size() != size_t(p.l_size)) p.hv.alloc(size_t(p.l_size));
    if (host_pipeline_applies(p)) {
      mass_apply_host_pipelined(p, u_host, v_host, s);
    } else {
      const size_t bytes = size_t(p.l_size) * sizeof(double);
      FEM_CUDA_CHECK(cudaMemcpyAsync(p.hu.get(), u_host, bytes, cudaMemcpyHostToDevice, s));
      mass_apply_impl(p, p.hu.get(), p.hv.get(), true, s);
      FEM_CUDA_CHECK(cudaMemcpyAsync(v_host, p.hv.get(), bytes, cudaMemcpyDeviceToHost, s));
      FEM_CUDA_CHECK(cudaStreamSynchronize(s));
    }
    check_status(p);
  });
}

int fem_b200_mass_set_host_chunks(fem_b200_mass op, int chunks) {
  return guarded([&] {
    require(op && op->d, "mass_set_host_chunks: NULL handle");
    require(chunks >= 0 && chunks <= 4096, "mass_set_host_chunks: chunks must be in 0..4096");
    op->d->host_chunks = chunks;
  });
}

int fem_b200_mass_autotune(fem_b200_mass op, const double* u, int64_t n_u, double* v, int64_t n_v, int reps,
                           int* chosen, float* best_ms, void* stream) {
  return guarded([&] {
    require(op && op->d, "operator autotune: NULL handle");
    MassPlan& p = *op->d;
    require(n_u == p.l_size && u, "operator autotune: u must have l_size entries");
    require(n_v == p.l_size && v, "operator autotune: v must have l_size entries");
    require(reps >= 1 && reps <= 1000, "operator autotune: reps must be in 1..1000");
    DeviceGuard g(p.device);
    cudaStream_t s = as_stream(stream);
    cudaEvent_t t0, t1;
    FEM_CUDA_CHECK(cudaEventCreate(&t0));
    FEM_CUDA_CHECK(cudaEventCreate(&t1));
    int best = FEM_B200_KERNEL_SIMPLE;
    float best_t = -1.0f;
    try {
      for (int variant = FEM_B200_KERNEL_SIMPLE; variant <= FEM_B200_KERNEL_ELEMENT; ++variant) {
        ApplyLauncher l = variant_launcher(p, variant);
        if (!l) continue;
        p.launch = l;
        for (int i = 0; i < 2; ++i) mass_apply_impl(p, u, v, false, s);  // warm-up (v is scratch)
        FEM_CUDA_CHECK(cudaEventRecord(t0, s));
        for (int i = 0; i < reps; ++i) mass_apply_impl(p, u, v, false, s);
        FEM_CUDA_CHECK(cudaEventRecord(t1, s));
        FEM_CUDA_CHECK(cudaEventSynchronize(t1));
        check_status(p);
        float ms = 0.0f;
        FEM_CUDA_CHECK(cudaEventElapsedTime(&ms, t0, t1));
        ms /= float(reps);
        if (best_t < 0.0f || ms < best_t) best_t = ms, best = variant;
      }
    } catch (...) {
      (void)cudaEventDestroy(t0);
      (void)cudaEventDestroy(t1);
      p.launch = variant_launcher(p, p.variant) ? variant_launcher(p, p.variant) : auto_kernel(p);
      throw;
    }
    (void)cudaEventDestroy(t0);
    (void)cudaEventDestroy(t1);
    {
      std::lock_guard<std::mutex> lock(g_tune_mu);
      g_tune[tune_key(p)] = best;
    }
    p.variant = FEM_B200_KERNEL_AUTO;
    p.launch = variant_launcher(p, best);
    if (chosen) *chosen = best;
    if (best_ms) *best_ms = best_t;
  });
}

int fem_b200_mass_check(fem_b200_mass op, void* stream) {
  return guarded([&] {
    require(op && op->d, "operator check: NULL handle");
    MassPlan& p = *op->d;
    DeviceGuard g(p.device);
    FEM_CUDA_CHECK(cudaStreamSynchronize(as_stream(stream)));
    check_status(p);
  });
}

int fem_b200_mass_set_kernel(fem_b200_mass op, int variant) {
  return guarded([&] {
    require(op && op->d, "operator kernel: NULL handle");
    MassPlan& p = *op->d;
    require(variant >= FEM_B200_KERNEL_AUTO && variant <= FEM_B200_KERNEL_ELEMENT, "operator kernel: unknown variant");
    if (variant == FEM_B200_KERNEL_ELEMENT && !p.launch_el)
      throw unsupported_error("operator kernel: no element-per-thread kernel for " + shape_str(p.dim, p.P, p.Q));
    if (variant == FEM_B200_KERNEL_NARROW && !p.launch_nw)
      throw unsupported_error("operator kernel: no half-tile kernel for " + shape_str(p.dim, p.P, p.Q));
    if (variant == FEM_B200_KERNEL_OCCUPANCY && !p.launch_occ)
      throw unsupported_error("operator kernel: no register-capped kernel for " + shape_str(p.dim, p.P, p.Q));
    if (variant == FEM_B200_KERNEL_PREFETCH && !p.launch_pf)
      throw unsupported_error("operator kernel: no prefetching kernel for " + shape_str(p.dim, p.P, p.Q));
    if (variant == FEM_B200_KERNEL_PIPELINED && !p.launch_pipe)
      throw unsupported_error("operator kernel: no pipelined kernel for " + shape_str(p.dim, p.P, p.Q));
    if (variant == FEM_B200_KERNEL_PAIRED && !p.launch_x2)
      throw unsupported_error("operator kernel: no paired kernel for " + shape_str(p.dim, p.P, p.Q));
    p.variant = variant;
    switch (variant) {
      case FEM_B200_KERNEL_SIMPLE: p.launch = p.launch_simple; break;
      case FEM_B200_KERNEL_PIPELINED: p.launch = p.launch_pipe; break;
      case FEM_B200_KERNEL_PAIRED: p.launch = p.launch_x2; break;
      case FEM_B200_KERNEL_PREFETCH: p.launch = p.launch_pf; break;
      case FEM_B200_KERNEL_OCCUPANCY: p.launch = p.launch_occ; break;
      case FEM_B200_KERNEL_NARROW: p.launch = p.launch_nw; break;
      case FEM_B200_KERNEL_ELEMENT: p.launch = p.launch_el; break;
      default: p.launch = auto_kernel(p);
    }
  });
}

int fem_b200_mass_info(fem_b200_mass op, int* launches_per_apply, int* tile_elems, int64_t* device_bytes,
                       int* kernel_variant) {
  return guarded([&] {
    require(op && op->d, "mass info: NULL handle");
    const MassPlan& p = *op->d;
    if (launches_per_apply) *launches_per_apply = p.scatter_mode == FEM_B200_SCATTER_ATOMIC ? 1 : 2;
    if (kernel_variant)
      *kernel_variant = p.launch == p.launch_x2     ? FEM_B200_KERNEL_PAIRED
                        : p.launch == p.launch_pipe ? FEM_B200_KERNEL_PIPELINED
                        : p.launch == p.launch_pf   ? FEM_B200_KERNEL_PREFETCH
                        : p.launch == p.launch_occ  ? FEM_B200_KERNEL_OCCUPANCY
                        : p.launch == p.launch_nw   ? FEM_B200_KERNEL_NARROW
                        : p.launch == p.launch_el   ? FEM_B200_KERNEL_ELEMENT
                                                    : FEM_B200_KERNEL_SIMPLE;
    if (tile_elems) *tile_elems = p.tile_e;
    if (device_bytes)
      *device_bytes = int64_t(p.offs_t.bytes() + p.qd_t.bytes() + p.evec.bytes() + p.hu.bytes() + p.hv.bytes());
  });
}

}  // extern "C"
