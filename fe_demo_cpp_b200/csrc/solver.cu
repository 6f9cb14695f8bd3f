// Jacobi-preconditioned CG mass solves on the device (sm_100a):
//   * the assembled diagonal of the mass operator, one fused kernel;
//   * the FP32 instantiation of the fused apply (inner solves);
//   * FP64 PCG, and FP32 PCG inside FP64 iterative refinement.
// CG dot products accumulate in FP64 in every precision; the outer residual
// of the refinement is an FP64 apply.  The reference has no solver; this is
// the growth direction its survey names (Jacobi diagonal + CG + mixed-
// precision refinement), tested against a host FP64 CG around the oracle.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "mass_kernels.cuh"
#include "plan.hpp"

namespace fem_b200 {

// ---------------------------------------------------------------------------
// Assembled diagonal: diag_i = sum_e sum_q qdata_q * prod_d B[q_d][i_d]^2,
// i.e. the transposed sum-factorised contractions with B squared entrywise
// applied to qdata, then the scatter-add.  Same thread roles and layouts as
// mass3d_apply_kernel's phases C (x^T), F (y^T) and G (z^T); m.B holds B^2.
// ---------------------------------------------------------------------------
template <int P, int Q>
__global__ void __launch_bounds__(Mass3D<P, Q>::NT) mass3d_diag_kernel(const __grid_constant__ Mat1D<P, Q> m,
                                                                      const int* __restrict__ offs,
                                                                      const double* __restrict__ qd,
                                                                      double* __restrict__ diag, int num_elem,
                                                                      int num_comp, int64_t comp_stride) {
  using L = Mass3D<P, Q>;
  constexpr int E = L::E;
  extern __shared__ __align__(16) unsigned char smem_bytes[];
  double* sa = reinterpret_cast<double*>(smem_bytes);
  double* sb = sa + L::SA;
  const int t = threadIdx.x, e = t % E, col = t / E;
  const int64_t tile = blockIdx.x, eg = tile * E + e;
  const bool valid = eg < num_elem;
  {  // x^T of the thread's qdata row (qy, qz)
    double qv[Q];
    const double* qt = qd + tile * (int64_t(L::NQ) * E) + col * E + e;
#pragma unroll
    for (int qx = 0; qx < Q; ++qx) qv[qx] = qt[qx * (Q * Q * E)];
    const int qy = col % Q, qz = col / Q;
#pragma unroll
    for (int px = 0; px < P; ++px) {
      double s = 0.0;
#pragma unroll
      for (int qx = 0; qx < Q; ++qx) s += m.B[qx * P + px] * qv[qx];
      sa[qy * L::PS3 + (qz * P + px) * E + e] = s;
    }
  }
  __syncthreads();
  if (col < P * Q) {  // y^T
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
  if (col < P * P && valid) {  // z^T and the scatter-add, every component
    double z[Q];
#pragma unroll
    for (int qz = 0; qz < Q; ++qz) z[qz] = sb[qz * L::PS4 + col * E + e];
    const int* ot = offs + tile * (int64_t(L::ES) * E) + col * E + e;
#pragma unroll
    for (int pz = 0; pz < P; ++pz) {
      double s = 0.0;
#pragma unroll
      for (int qz = 0; qz < Q; ++qz) s += m.B[qz * P + pz] * z[qz];
      const int64_t off = ot[pz * (P * P * E)];
      for (int k = 0; k < num_comp; ++k) atomicAdd(diag + off + k * comp_stride, s);
    }
  }
}

template <int P, int Q>
__global__ void __launch_bounds__(Mass2D<P, Q>::NT) mass2d_diag_kernel(const __grid_constant__ Mat1D<P, Q> m,
                                                                      const int* __restrict__ offs,
                                                                      const double* __restrict__ qd,
                                                                      double* __restrict__ diag, int num_elem,
                                                                      int num_comp, int64_t comp_stride) {
  using L = Mass2D<P, Q>;
  constexpr int E = L::E;
  __shared__ double s3[Q * P * E];
  const int t = threadIdx.x, e = t % E, col = t / E;  // col = qy
  const int64_t tile = blockIdx.x, eg = tile * E + e;
  {
    double qv[Q];
    const double* qt = qd + tile * (int64_t(L::NQ) * E) + col * E + e;
#pragma unroll
    for (int qx = 0; qx < Q; ++qx) qv[qx] = qt[qx * (Q * E)];
#pragma unroll
    for (int px = 0; px < P; ++px) {
      double s = 0.0;
#pragma unroll
      for (int qx = 0; qx < Q; ++qx) s += m.B[qx * P + px] * qv[qx];
      s3[(col * P + px) * E + e] = s;
    }
  }
  __syncthreads();
  if (col < P && eg < num_elem) {  // col = px
    double z[Q];
#pragma unroll
    for (int qy = 0; qy < Q; ++qy) z[qy] = s3[(qy * P + col) * E + e];
    const int* ot = offs + tile * (int64_t(L::ES) * E) + col * E + e;
#pragma unroll
    for (int py = 0; py < P; ++py) {
      double s = 0.0;
#pragma unroll
      for (int qy = 0; qy < Q; ++qy) s += m.B[qy * P + py] * z[qy];
      const int64_t off = ot[py * (P * E)];
      for (int k = 0; k < num_comp; ++k) atomicAdd(diag + off + k * comp_stride, s);
    }
  }
}

template <int P, int Q>
__global__ void __launch_bounds__(128) mass1d_diag_kernel(const __grid_constant__ Mat1D<P, Q> m,
                                                         const int* __restrict__ offs, const double* __restrict__ qd,
                                                         double* __restrict__ diag, int num_elem, int num_comp,
                                                         int64_t comp_stride) {
  const int e = threadIdx.x;
  const int64_t tile = blockIdx.x, eg = tile * 128 + e;
  if (eg >= num_elem) return;
#pragma unroll
  for (int px = 0; px < P; ++px) {
    double s = 0.0;
#pragma unroll
    for (int qx = 0; qx < Q; ++qx) s += m.B[qx * P + px] * qd[(tile * Q + qx) * 128 + e];
    const int64_t off = offs[(tile * P + px) * 128 + e];
    for (int k = 0; k < num_comp; ++k) atomicAdd(diag + off + k * comp_stride, s);
  }
}

// ---------------------------------------------------------------------------
// CG vector kernels.  Reductions accumulate in FP64 (warp shuffles, then one
// atomicAdd per block into a device scalar).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

template <int N>
__device__ __forceinline__ void block_sums(double (&v)[N], double* out) {
  __shared__ double part[N][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    v[i] = warp_sum(v[i]);
    if (lane == 0) part[i][w] = v[i];
  }
  __syncthreads();
  if (w == 0) {
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      double s = lane < nw ? part[i][lane] : 0.0;
      s = warp_sum(s);
      if (lane == 0) atomicAdd(out + i, s);
    }
  }
}

template <class T>
__global__ void dot_kernel(int64_t n, const T* __restrict__ x, const T* __restrict__ y, double* __restrict__ out) {
  double v[1] = {0.0};
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    v[0] += double(x[i]) * double(y[i]);
  block_sums<1>(v, out);
}

// x += a p; r -= a Ap; z = dinv r; out[0] += r.z, out[1] += r.r
template <class T>
__global__ void cg_update_kernel(int64_t n, double alpha, const T* __restrict__ p, const T* __restrict__ ap,
                                 const T* __restrict__ dinv, T* __restrict__ x, T* __restrict__ r, T* __restrict__ z,
                                 double* __restrict__ out) {
  double v[2] = {0.0, 0.0};
  const T a = T(alpha);
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    x[i] += a * p[i];
    const T ri = r[i] - a * ap[i];
    r[i] = ri;
    const T zi = dinv[i] * ri;
    z[i] = zi;
    v[0] += double(ri) * double(zi);
    v[1] += double(ri) * double(ri);
  }
  block_sums<2>(v, out);
}

// p = z + beta p
template <class T>
__global__ void cg_direction_kernel(int64_t n, double beta, const T* __restrict__ z, T* __restrict__ p) {
  const T b = T(beta);
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    p[i] = z[i] + b * p[i];
}

// start: x = 0, r = b * scale (converted), z = dinv r, p = z; out[0] += r.z, out[1] += r.r
template <class T>
__global__ void cg_start_kernel(int64_t n, const double* __restrict__ b, double scale, const T* __restrict__ dinv,
                                T* __restrict__ x, T* __restrict__ r, T* __restrict__ z, T* __restrict__ p,
                                double* __restrict__ out) {
  double v[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const T ri = T(b[i] * scale);
    const T zi = dinv[i] * ri;
    x[i] = T(0);
    r[i] = ri;
    z[i] = zi;
    p[i] = zi;
    v[0] += double(ri) * double(zi);
    v[1] += double(ri) * double(ri);
  }
  block_sums<2>(v, out);
}

template <class T>
__global__ void invert_kernel(int64_t n, const double* __restrict__ d, T* __restrict__ dinv) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    dinv[i] = d[i] != 0.0 ? T(1.0 / d[i]) : T(0);
}

// u += s * d (FP64 += FP32 correction)
__global__ void add_scaled_kernel(int64_t n, double s, const float* __restrict__ d, double* __restrict__ u) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    u[i] += s * double(d[i]);
}

// r = f - Mu; out[0] += r.r
__global__ void residual_kernel(int64_t n, const double* __restrict__ f, const double* __restrict__ mu,
                                double* __restrict__ r, double* __restrict__ out) {
  double v[1] = {0.0};
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const double ri = f[i] - mu[i];
    r[i] = ri;
    v[0] += ri * ri;
  }
  block_sums<1>(v, out);
}

__global__ void to_float_kernel(int64_t n, const double* __restrict__ in, float* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = float(in[i]);
}

// ---------------------------------------------------------------------------
// dispatch of the diagonal and FP32 apply kernels over the compiled (P, Q) set
// ---------------------------------------------------------------------------
using DiagLauncher = void (*)(const MassPlan&, double*, cudaStream_t);
using Apply32Launcher = void (*)(const MassPlan&, const float*, float*, cudaStream_t);

template <int P, int Q>
Mat1D<P, Q> squared_mat(const BasisData& b) {
  Mat1D<P, Q> m;
  for (int i = 0; i < Q * P; ++i) m.B[i] = b.interp[i] * b.interp[i];
  std::memset(m.G, 0, sizeof(m.G));
  std::memcpy(m.W, b.q_weight.data(), sizeof(m.W));
  return m;
}

template <int P, int Q>
Mat1D<P, Q, float> float_mat(const BasisData& b) {
  Mat1D<P, Q, float> m;
  for (int i = 0; i < Q * P; ++i) m.B[i] = float(b.interp[i]), m.G[i] = float(b.grad[i]);
  for (int i = 0; i < Q; ++i) m.W[i] = float(b.q_weight[i]);
  return m;
}

template <int P, int Q>
void launch_diag(const MassPlan& p, double* diag, cudaStream_t s) {
  const int nc = p.comp_run;
  if (p.dim == 3) {
    using L = Mass3D<P, Q>;
    static std::atomic<uint64_t> smem_set{0};
    set_smem(mass3d_diag_kernel<P, Q>, L::SMEM, smem_set);
    mass3d_diag_kernel<P, Q><<<unsigned(p.n_tiles), L::NT, L::SMEM, s>>>(
        squared_mat<P, Q>(p.basis), p.offs_t.get(), p.qd_t.get(), diag, p.num_elem, nc, p.comp_stride);
  } else if (p.dim == 2) {
    mass2d_diag_kernel<P, Q><<<unsigned(p.n_tiles), Mass2D<P, Q>::NT, 0, s>>>(
        squared_mat<P, Q>(p.basis), p.offs_t.get(), p.qd_t.get(), diag, p.num_elem, nc, p.comp_stride);
  } else {
    mass1d_diag_kernel<P, Q><<<unsigned(p.n_tiles), 128, 0, s>>>(squared_mat<P, Q>(p.basis), p.offs_t.get(),
                                                                  p.qd_t.get(), diag, p.num_elem, nc, p.comp_stride);
  }
  FEM_CUDA_CHECK(cudaGetLastError());
}

template <int P, int Q>
void launch_apply32(const MassPlan& p, const float* u, float* v, cudaStream_t s) {
  if (p.dim == 3) {
    using L = Mass3D<P, Q>;
    constexpr int smem = (L::SA + L::SB) * 4;
    static std::atomic<uint64_t> smem_set{0};
    set_smem(mass3d_apply_kernel<P, Q, 1, float>, smem, smem_set);
    mass3d_apply_kernel<P, Q, 1, float><<<unsigned(p.n_tiles), L::NT, smem, s>>>(
        float_mat<P, Q>(p.basis), p.offs_t.get(), p.qd_t32.get(), u, v, nullptr, p.num_elem, p.comp_run,
        p.comp_stride);
  } else if (p.dim == 2) {
    using L = Mass2D<P, Q>;
    constexpr int smem = (L::S1 + L::S3) * 4;
    mass2d_apply_kernel<P, Q, float><<<unsigned(p.n_tiles), L::NT, smem, s>>>(
        float_mat<P, Q>(p.basis), p.offs_t.get(), p.qd_t32.get(), u, v, nullptr, p.num_elem, p.comp_run,
        p.comp_stride);
  } else {
    mass1d_apply_kernel<P, Q, float><<<unsigned(p.n_tiles), 128, 0, s>>>(
        float_mat<P, Q>(p.basis), p.offs_t.get(), p.qd_t32.get(), u, v, nullptr, p.num_elem, p.comp_run,
        p.comp_stride);
  }
  FEM_CUDA_CHECK(cudaGetLastError());
}

constexpr int kSolveMinP = 2, kSolveMaxP = 8, kSolveQSpan = 3;

template <int P, int DQ>
struct SolveTable {
  static void fill(DiagLauncher (*dg)[kSolveQSpan], Apply32Launcher (*ap)[kSolveQSpan]) {
    dg[P][DQ] = launch_diag<P, P + DQ>;
    ap[P][DQ] = launch_apply32<P, P + DQ>;
    if constexpr (DQ + 1 < kSolveQSpan)
      SolveTable<P, DQ + 1>::fill(dg, ap);
    else if constexpr (P + 1 <= kSolveMaxP)
      SolveTable<P + 1, 0>::fill(dg, ap);
  }
};

struct SolveDispatch {
  DiagLauncher diag[kSolveMaxP + 1][kSolveQSpan] = {};
  Apply32Launcher apply32[kSolveMaxP + 1][kSolveQSpan] = {};
  SolveDispatch() { SolveTable<kSolveMinP, 0>::fill(diag, apply32); }
};

const SolveDispatch& solve_dispatch() {
  static SolveDispatch d;
  return d;
}

inline int red_grid(int64_t n) { return int(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8))); }

// The plan's solver state: diagonal, its inverse in both precisions, the FP32
// copy of qdata, CG vectors, and the device scalars of the reductions.
void ensure_solver_state(MassPlan& p, bool fp32, cudaStream_t s) {
  const size_t n = size_t(p.l_size);
  if (p.diag.size() != n) {
    p.diag.alloc(n);
    FEM_CUDA_CHECK(cudaMemsetAsync(p.diag.get(), 0, n * sizeof(double), s));
    solve_dispatch().diag[p.P][p.Q - p.P](p, p.diag.get(), s);
    p.dinv.alloc(n);
    invert_kernel<double><<<red_grid(int64_t(n)), 256, 0, s>>>(int64_t(n), p.diag.get(), p.dinv.get());
    FEM_CUDA_CHECK(cudaGetLastError());
    p.cg_r.alloc(n), p.cg_z.alloc(n), p.cg_p.alloc(n), p.cg_ap.alloc(n);
    p.red.alloc(4);
  }
  if (fp32 && p.qd_t32.size() != p.qd_t.size()) {
    p.qd_t32.alloc(p.qd_t.size());
    to_float_kernel<<<red_grid(int64_t(p.qd_t.size())), 256, 0, s>>>(int64_t(p.qd_t.size()), p.qd_t.get(),
                                                                    p.qd_t32.get());
    FEM_CUDA_CHECK(cudaGetLastError());
    p.dinv32.alloc(n);
    invert_kernel<float><<<red_grid(int64_t(n)), 256, 0, s>>>(int64_t(n), p.diag.get(), p.dinv32.get());
    FEM_CUDA_CHECK(cudaGetLastError());
    p.f_r.alloc(n), p.f_z.alloc(n), p.f_p.alloc(n), p.f_ap.alloc(n), p.f_x.alloc(n);
  }
}

// Reads the first k reduction scalars (synchronises the stream) and clears them.
void read_reductions(MassPlan& p, double* out, int k, cudaStream_t s) {
  FEM_CUDA_CHECK(cudaMemcpyAsync(out, p.red.get(), k * sizeof(double), cudaMemcpyDeviceToHost, s));
  FEM_CUDA_CHECK(cudaMemsetAsync(p.red.get(), 0, 4 * sizeof(double), s));
  FEM_CUDA_CHECK(cudaStreamSynchronize(s));
}

struct CgResult {
  int iterations = 0;
  double rel = 0.0;  // final recursive residual / initial
};

// Jacobi PCG on `apply` for A x = b*scale, x starting at 0, until
// ||r|| <= rtol ||r0|| or max_it.  T = double (FP64) or float (FP32 vectors).
template <class T, class ApplyFn>
CgResult pcg(MassPlan& p, ApplyFn apply, const double* b, double scale, const T* dinv, T* x, T* r, T* z, T* pv, T* ap,
             double rtol, int max_it, cudaStream_t s) {
  const int64_t n = p.l_size;
  const int g = red_grid(n);
  double red[2];
  FEM_CUDA_CHECK(cudaMemsetAsync(p.red.get(), 0, 4 * sizeof(double), s));
  cg_start_kernel<T><<<g, 256, 0, s>>>(n, b, scale, dinv, x, r, z, pv, p.red.get());
  FEM_CUDA_CHECK(cudaGetLastError());
  read_reductions(p, red, 2, s);
  double rz = red[0];
  const double r0 = std::sqrt(red[1]);
  CgResult res;
  if (r0 == 0.0) return res;
  double rnorm = r0;
  for (int it = 0; it < max_it && rnorm > rtol * r0; ++it) {
    apply(pv, ap);
    dot_kernel<T><<<g, 256, 0, s>>>(n, pv, ap, p.red.get());
    FEM_CUDA_CHECK(cudaGetLastError());
    read_reductions(p, red, 1, s);
    if (!(red[0] > 0.0)) throw cuda_error("mass solve: the operator is not positive definite on this vector");
    const double alpha = rz / red[0];
    cg_update_kernel<T><<<g, 256, 0, s>>>(n, alpha, pv, ap, dinv, x, r, z, p.red.get());
    FEM_CUDA_CHECK(cudaGetLastError());
    read_reductions(p, red, 2, s);
    const double beta = red[0] / rz;
    rz = red[0];
    rnorm = std::sqrt(red[1]);
    cg_direction_kernel<T><<<g, 256, 0, s>>>(n, beta, z, pv);
    FEM_CUDA_CHECK(cudaGetLastError());
    res.iterations = it + 1;
  }
  res.rel = rnorm / r0;
  return res;
}

}  // namespace fem_b200

using namespace fem_b200;

extern "C" {

int fem_b200_mass_diagonal(fem_b200_mass op, double* diag, int64_t n, void* stream) {
  return guarded([&] {
    require(op && op->d, "mass diagonal: NULL handle");
    MassPlan& p = *op->d;
    require(n == p.l_size && diag, "mass diagonal: diag must have l_size entries");
    DeviceGuard g(p.device);
    cudaStream_t s = as_stream(stream);
    FEM_CUDA_CHECK(cudaMemsetAsync(diag, 0, size_t(n) * sizeof(double), s));
    solve_dispatch().diag[p.P][p.Q - p.P](p, diag, s);
  });
}

int fem_b200_mass_solve(fem_b200_mass op, const double* f, int64_t n_f, double* u, int64_t n_u, double rtol,
                        int max_iter, int precision, int* iterations, int* refinements, double* rel_residual,
                        void* stream) {
  return guarded([&] {
    require(op && op->d, "mass solve: NULL handle");
    MassPlan& p = *op->d;
    require(n_f == p.l_size && f && n_u == p.l_size && u, "mass solve: f and u must have l_size entries");
    require(rtol > 0.0 && rtol < 1.0, "mass solve: rtol must be in (0, 1)");
    require(max_iter >= 1, "mass solve: max_iter must be positive");
    require(precision == FEM_B200_SOLVE_FP64 || precision == FEM_B200_SOLVE_FP32_IR,
            "mass solve: unknown precision");
    if (p.comp_run != p.num_comp)
      throw unsupported_error(
          "mass solve: the reference apply_mass leaves components 1.. out (a singular operator); use "
          "FEM_B200_QF_APPLY_MASS_VECTOR for a multi-component solve");
    DeviceGuard g(p.device);
    cudaStream_t s = as_stream(stream);
    const int64_t n = p.l_size;
    const int grid = red_grid(n);
    ensure_solver_state(p, precision == FEM_B200_SOLVE_FP32_IR, s);
    int total_it = 0, outer = 0;
    double red[2];
    // ||f||
    FEM_CUDA_CHECK(cudaMemsetAsync(p.red.get(), 0, 4 * sizeof(double), s));
    dot_kernel<double><<<grid, 256, 0, s>>>(n, f, f, p.red.get());
    FEM_CUDA_CHECK(cudaGetLastError());
    read_reductions(p, red, 1, s);
    const double nf = std::sqrt(red[0]);
    if (nf == 0.0) {
      FEM_CUDA_CHECK(cudaMemsetAsync(u, 0, size_t(n) * sizeof(double), s));
      if (iterations) *iterations = 0;
      if (refinements) *refinements = 0;
      if (rel_residual) *rel_residual = 0.0;
      FEM_CUDA_CHECK(cudaStreamSynchronize(s));
      return;
    }
    auto apply64 = [&](const double* x, double* y) { mass_apply_impl(p, x, y, true, s); };
    if (precision == FEM_B200_SOLVE_FP64) {
      CgResult r = pcg<double>(p, apply64, f, 1.0, p.dinv.get(), u, p.cg_r.get(), p.cg_z.get(), p.cg_p.get(),
                               p.cg_ap.get(), rtol, max_iter, s);
      total_it = r.iterations;
    } else {
      // FP64 outer loop: r = f - M u (FP64), correction from FP32 PCG on r/||r||
      auto apply32 = [&](const float* x, float* y) {
        FEM_CUDA_CHECK(cudaMemsetAsync(y, 0, size_t(n) * sizeof(float), s));
        solve_dispatch().apply32[p.P][p.Q - p.P](p, x, y, s);
      };
      FEM_CUDA_CHECK(cudaMemsetAsync(u, 0, size_t(n) * sizeof(double), s));
      FEM_CUDA_CHECK(cudaMemcpyAsync(p.cg_r.get(), f, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, s));
      double nr = nf;
      const double inner_rtol = 1e-5;
      for (outer = 0; outer < 50 && nr > rtol * nf && total_it < max_iter; ++outer) {
        CgResult r = pcg<float>(p, apply32, p.cg_r.get(), 1.0 / nr, p.dinv32.get(), p.f_x.get(), p.f_r.get(),
                                p.f_z.get(), p.f_p.get(), p.f_ap.get(), inner_rtol, max_iter - total_it, s);
        total_it += r.iterations;
        add_scaled_kernel<<<grid, 256, 0, s>>>(n, nr, p.f_x.get(), u);
        FEM_CUDA_CHECK(cudaGetLastError());
        apply64(u, p.cg_ap.get());
        residual_kernel<<<grid, 256, 0, s>>>(n, f, p.cg_ap.get(), p.cg_r.get(), p.red.get());
        FEM_CUDA_CHECK(cudaGetLastError());
        read_reductions(p, red, 1, s);
        nr = std::sqrt(red[0]);
      }
    }
    // the true FP64 residual ||f - M u|| / ||f||
    apply64(u, p.cg_ap.get());
    residual_kernel<<<grid, 256, 0, s>>>(n, f, p.cg_ap.get(), p.cg_r.get(), p.red.get());
    FEM_CUDA_CHECK(cudaGetLastError());
    read_reductions(p, red, 1, s);
    check_status(p);
    if (iterations) *iterations = total_it;
    if (refinements) *refinements = outer;
    if (rel_residual) *rel_residual = std::sqrt(red[0]) / nf;
  });
}

}  // extern "C"
