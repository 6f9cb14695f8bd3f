// Jacobi-preconditioned CG mass solves on the device (sm_100a):
//   * the assembled diagonal of the mass operator, one fused kernel;
//   * Chronopoulos-Gear PCG (one reduction point per iteration) whose scalars
//     stay on the device, so the host queues iterations without waiting;
//     the Jacobi scaling is folded into the apply's gather and (u, M u) into
//     its quadrature-point pass (apply_ext.cuh);
//   * FP64 PCG, and FP32 PCG or BF16-storage PCG (FP32 arithmetic) inside
//     FP64 iterative refinement.
// Reductions accumulate in FP64 in every precision, in a fixed order; the
// outer residual of the refinement is an FP64 apply.  The reference has no
// solver: these solve M u = f with its mass operator and are tested against
// the oracle's apply (f = M u* for a known u*).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "mass_kernels.cuh"
#include "plan.hpp"
#include "transpose_scatter.cuh"

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
                                                                      double* __restrict__ diag, double* __restrict__ ev,
                                                                      int num_elem, int num_comp, int64_t comp_stride) {
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
      for (int k = 0; k < num_comp; ++k) {
        if (ev)
          ev[(int64_t(k) * L::ES + pz * P * P + col) * num_elem + eg] = s;
        else
          atomicAdd(diag + off + k * comp_stride, s);
      }
    }
  }
}

template <int P, int Q>
__global__ void __launch_bounds__(Mass2D<P, Q>::NT) mass2d_diag_kernel(const __grid_constant__ Mat1D<P, Q> m,
                                                                      const int* __restrict__ offs,
                                                                      const double* __restrict__ qd,
                                                                      double* __restrict__ diag, double* __restrict__ ev,
                                                                      int num_elem, int num_comp, int64_t comp_stride) {
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
      for (int k = 0; k < num_comp; ++k) {
        if (ev)
          ev[(int64_t(k) * L::ES + py * P + col) * num_elem + eg] = s;
        else
          atomicAdd(diag + off + k * comp_stride, s);
      }
    }
  }
}

template <int P, int Q>
__global__ void __launch_bounds__(128) mass1d_diag_kernel(const __grid_constant__ Mat1D<P, Q> m,
                                                         const int* __restrict__ offs, const double* __restrict__ qd,
                                                         double* __restrict__ diag, double* __restrict__ ev,
                                                         int num_elem, int num_comp, int64_t comp_stride) {
  const int e = threadIdx.x;
  const int64_t tile = blockIdx.x, eg = tile * 128 + e;
  if (eg >= num_elem) return;
#pragma unroll
  for (int px = 0; px < P; ++px) {
    double s = 0.0;
#pragma unroll
    for (int qx = 0; qx < Q; ++qx) s += m.B[qx * P + px] * qd[(tile * Q + qx) * 128 + e];
    const int64_t off = offs[(tile * P + px) * 128 + e];
    for (int k = 0; k < num_comp; ++k) {
      if (ev)
        ev[(int64_t(k) * P + px) * num_elem + eg] = s;
      else
        atomicAdd(diag + off + k * comp_stride, s);
    }
  }
}


// ---------------------------------------------------------------------------
// Chronopoulos-Gear PCG vector kernels.  With u = D^-1 r and w = M u:
//   p = u + beta p;  s = w + beta s;  x += alpha p;  r -= alpha s;
//   gamma = (r, D^-1 r), rr = (r, r)  -> this kernel's grid reduction;
//   w = M (D^-1 r), delta = (u, M u)  -> the apply's grid reduction, which
//   sets beta = gamma / gamma_old and alpha = gamma / (delta - beta gamma / alpha).
// Every kernel returns at once when the solve has stopped (st->done), so the
// host can queue several iterations between convergence checks.
// ---------------------------------------------------------------------------
template <class T>
__global__ void cg_init_kernel(int64_t n, const double* __restrict__ b, double scale, const T* __restrict__ dinv,
                               T* __restrict__ x, T* __restrict__ r, T* __restrict__ p, T* __restrict__ sv,
                               T* __restrict__ w, CgScalars* st, double* part, double rtol, int max_iters) {
  double v[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const T ri = T(b[i] * scale);
    x[i] = T(0), p[i] = T(0), sv[i] = T(0), w[i] = T(0);
    r[i] = ri;
    v[0] += double(ri) * double(dinv[i] * ri);
    v[1] += double(ri) * double(ri);
  }
  grid_sum<2>(v, part, &st->ticket, [&](const double* tot) {
    st->gamma = tot[0], st->gamma_old = tot[0];
    st->rr = tot[1], st->rr0 = tot[1];
    st->tol2 = rtol * rtol * tot[1];
    st->alpha = 0.0, st->beta = 0.0, st->delta = 0.0;
    st->iters = 0, st->max_iters = max_iters;
    st->done = tot[1] > 0.0 ? 0 : 1;
  });
}

// 16 bytes of T: the unit of the vectorised update.
template <class T>
struct alignas(16) Pack {
  static constexpr int K = 16 / int(sizeof(T));
  T a[K];
};

template <class T, bool VEC>
__global__ void cg_update_kernel(int64_t n, const T* __restrict__ dinv, T* __restrict__ x, T* __restrict__ r,
                                 T* __restrict__ p, T* __restrict__ sv, T* __restrict__ w, CgScalars* st,
                                 double* part) {
  if (st->done) return;
  const T a = T(st->alpha), bt = T(st->beta);
  double v[2] = {0.0, 0.0};
  auto step = [&](T di, T& ri, T& pi, T& si, T& wi, T& xi) {
    pi = di * ri + bt * pi;
    si = wi + bt * si;
    wi = T(0);
    xi += a * pi;
    ri = ri - a * si;
    v[0] += double(ri) * double(di * ri);
    v[1] += double(ri) * double(ri);
  };
  const int64_t tid = blockIdx.x * int64_t(blockDim.x) + threadIdx.x, stride = int64_t(gridDim.x) * blockDim.x;
  int64_t head = 0;
  if constexpr (VEC) {  // every vector 16-byte aligned (checked by the host)
    using PK = Pack<T>;
    constexpr int K = PK::K;
    const int64_t nv = n / K;
    for (int64_t j = tid; j < nv; j += stride) {
      const PK D = reinterpret_cast<const PK*>(dinv)[j];
      PK R = reinterpret_cast<const PK*>(r)[j], Pv = reinterpret_cast<const PK*>(p)[j];
      PK S = reinterpret_cast<const PK*>(sv)[j], W = reinterpret_cast<const PK*>(w)[j];
      PK X = reinterpret_cast<const PK*>(x)[j];
#pragma unroll
      for (int k = 0; k < K; ++k) step(D.a[k], R.a[k], Pv.a[k], S.a[k], W.a[k], X.a[k]);
      reinterpret_cast<PK*>(r)[j] = R, reinterpret_cast<PK*>(p)[j] = Pv;
      reinterpret_cast<PK*>(sv)[j] = S, reinterpret_cast<PK*>(w)[j] = W;
      reinterpret_cast<PK*>(x)[j] = X;
    }
    head = nv * K;
  }
  for (int64_t i = head + tid; i < n; i += stride) {
    T ri = r[i], pi = p[i], si = sv[i], wi = w[i], xi = x[i];
    step(dinv[i], ri, pi, si, wi, xi);
    r[i] = ri, p[i] = pi, sv[i] = si, w[i] = wi, x[i] = xi;
  }
  grid_sum<2>(v, part, &st->ticket, [&](const double* tot) {
    st->gamma_old = st->gamma, st->gamma = tot[0];
    st->rr = tot[1];
    st->iters += 1;
    if (tot[1] <= st->tol2)
      st->done = 1;
    else if (st->iters >= st->max_iters)
      st->done = 2;
  });
}

// ---- BF16-storage inner PCG (FEM_B200_SOLVE_BF16_IR) -----------------------
// r, p, s stored in BF16 (2 bytes an entry); x (the correction, whose
// rounding would stay in the refined solution), w (the apply's atomic target)
// and dinv in FP32; FP32 arithmetic, FP64 reductions: the same recurrences as
// cg_init_kernel / cg_update_kernel.
using bf16 = __nv_bfloat16;

__global__ void cg_init_bf16_kernel(int64_t n, const double* __restrict__ b, double scale,
                                    const float* __restrict__ dinv, float* __restrict__ x, bf16* __restrict__ r,
                                    bf16* __restrict__ p, bf16* __restrict__ sv, float* __restrict__ w,
                                    CgScalars* st, double* part, double rtol, int max_iters) {
  double v[2] = {0.0, 0.0};
  const bf16 zero = __float2bfloat16_rn(0.0f);
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const bf16 rb = __float2bfloat16_rn(float(b[i] * scale));
    const float ri = __bfloat162float(rb);
    x[i] = 0.0f, p[i] = zero, sv[i] = zero, w[i] = 0.0f;
    r[i] = rb;
    v[0] += double(ri) * double(dinv[i] * ri);
    v[1] += double(ri) * double(ri);
  }
  grid_sum<2>(v, part, &st->ticket, [&](const double* tot) {
    st->gamma = tot[0], st->gamma_old = tot[0];
    st->rr = tot[1], st->rr0 = tot[1];
    st->tol2 = rtol * rtol * tot[1];
    st->alpha = 0.0, st->beta = 0.0, st->delta = 0.0;
    st->iters = 0, st->max_iters = max_iters;
    st->done = tot[1] > 0.0 ? 0 : 1;
  });
}

// Eight entries a thread: one 16-byte access to each BF16 vector, two to each
// FP32 one (vec: every vector 16-byte aligned, checked by the host; the
// scalar loop takes the entries past the last multiple of 8).
__global__ void cg_update_bf16_kernel(int64_t n, const float* __restrict__ dinv, float* __restrict__ x,
                                      bf16* __restrict__ r, bf16* __restrict__ p, bf16* __restrict__ sv,
                                      float* __restrict__ w, CgScalars* st, double* part, bool vec) {
  if (st->done) return;
  const float a = float(st->alpha), bt = float(st->beta);
  double v[2] = {0.0, 0.0};
  auto step = [&](float di, float& ri, float& pi, float& si, float& wi, float& xi) {
    pi = di * ri + bt * pi;
    si = wi + bt * si;
    wi = 0.0f;
    xi += a * pi;
    ri = ri - a * si;
  };
  const int64_t tid = blockIdx.x * int64_t(blockDim.x) + threadIdx.x, stride = int64_t(gridDim.x) * blockDim.x;
  int64_t head = 0;
  if (vec) {
    const int64_t nv = n / 8;
    for (int64_t j = tid; j < nv; j += stride) {
      uint4 R = reinterpret_cast<const uint4*>(r)[j], Pv = reinterpret_cast<const uint4*>(p)[j];
      uint4 S = reinterpret_cast<const uint4*>(sv)[j];
      float4 X0 = reinterpret_cast<const float4*>(x)[2 * j], X1 = reinterpret_cast<const float4*>(x)[2 * j + 1];
      float4 D0 = reinterpret_cast<const float4*>(dinv)[2 * j], D1 = reinterpret_cast<const float4*>(dinv)[2 * j + 1];
      float4 W0 = reinterpret_cast<const float4*>(w)[2 * j], W1 = reinterpret_cast<const float4*>(w)[2 * j + 1];
      bf16* rb = reinterpret_cast<bf16*>(&R);
      bf16* pb = reinterpret_cast<bf16*>(&Pv);
      bf16* sb = reinterpret_cast<bf16*>(&S);
      float xx[8] = {X0.x, X0.y, X0.z, X0.w, X1.x, X1.y, X1.z, X1.w};
      const float dd[8] = {D0.x, D0.y, D0.z, D0.w, D1.x, D1.y, D1.z, D1.w};
      float ww[8] = {W0.x, W0.y, W0.z, W0.w, W1.x, W1.y, W1.z, W1.w};
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        float ri = __bfloat162float(rb[k]), pi = __bfloat162float(pb[k]), si = __bfloat162float(sb[k]);
        step(dd[k], ri, pi, si, ww[k], xx[k]);
        rb[k] = __float2bfloat16_rn(ri), pb[k] = __float2bfloat16_rn(pi), sb[k] = __float2bfloat16_rn(si);
        const float rr = __bfloat162float(rb[k]);
        v[0] += double(rr) * double(dd[k] * rr);
        v[1] += double(rr) * double(rr);
      }
      reinterpret_cast<uint4*>(r)[j] = R, reinterpret_cast<uint4*>(p)[j] = Pv;
      reinterpret_cast<uint4*>(sv)[j] = S;
      reinterpret_cast<float4*>(x)[2 * j] = make_float4(xx[0], xx[1], xx[2], xx[3]);
      reinterpret_cast<float4*>(x)[2 * j + 1] = make_float4(xx[4], xx[5], xx[6], xx[7]);
      reinterpret_cast<float4*>(w)[2 * j] = make_float4(0.f, 0.f, 0.f, 0.f);
      reinterpret_cast<float4*>(w)[2 * j + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    head = nv * 8;
  }
  for (int64_t i = head + tid; i < n; i += stride) {
    float ri = __bfloat162float(r[i]), pi = __bfloat162float(p[i]), si = __bfloat162float(sv[i]);
    float wi = w[i], xi = x[i];
    step(dinv[i], ri, pi, si, wi, xi);
    r[i] = __float2bfloat16_rn(ri), p[i] = __float2bfloat16_rn(pi), sv[i] = __float2bfloat16_rn(si);
    w[i] = wi, x[i] = xi;
    const float rr = __bfloat162float(r[i]);
    v[0] += double(rr) * double(dinv[i] * rr);
    v[1] += double(rr) * double(rr);
  }
  grid_sum<2>(v, part, &st->ticket, [&](const double* tot) {
    st->gamma_old = st->gamma, st->gamma = tot[0];
    st->rr = tot[1];
    st->iters += 1;
    if (tot[1] <= st->tol2)
      st->done = 1;
    else if (st->iters >= st->max_iters)
      st->done = 2;
  });
}

__global__ void to_bf16_kernel(int64_t n, const double* __restrict__ in, bf16* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = __float2bfloat16_rn(float(in[i]));
}

// diag[off + k*comp_stride] = diag[off] for the components k >= 1 of every
// element node: the mass diagonal is the same for every component.
__global__ void broadcast_comp_kernel(int64_t n, const int* __restrict__ offsets, int num_comp, int64_t comp_stride,
                                      double* __restrict__ diag) {
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t off = offsets[t];
    const double d = diag[off];
    for (int k = 1; k < num_comp; ++k) diag[off + k * comp_stride] = d;
  }
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

// r = f - mu (mu == nullptr: r = f); st->res = (r, r)
__global__ void residual_kernel(int64_t n, const double* __restrict__ f, const double* __restrict__ mu,
                                double* __restrict__ r, CgScalars* st, double* part) {
  double v[1] = {0.0};
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const double ri = mu ? f[i] - mu[i] : f[i];
    r[i] = ri;
    v[0] += ri * ri;
  }
  grid_sum<1>(v, part, &st->ticket, [&](const double* tot) { st->res = tot[0]; });
}

__global__ void to_float_kernel(int64_t n, const double* __restrict__ in, float* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = float(in[i]);
}

// ---------------------------------------------------------------------------
// dispatch of the diagonal and CG apply kernels over the compiled (P, Q) set
// ---------------------------------------------------------------------------
using DiagLauncher = void (*)(const MassPlan&, double*, double*, cudaStream_t);
template <class T, class S = T>
using CgApplyLauncher = void (*)(const MassPlan&, const S*, T*, T*, const S*, const ApplyCg<T>&, cudaStream_t);

template <int P, int Q>
Mat1D<P, Q> squared_mat(const BasisData& b) {
  Mat1D<P, Q> m;
  for (int i = 0; i < Q * P; ++i) m.B[i] = b.interp[i] * b.interp[i];
  std::memset(m.G, 0, sizeof(m.G));
  std::memcpy(m.W, b.q_weight.data(), sizeof(m.W));
  return m;
}

template <int P, int Q, class T>
Mat1D<P, Q, T> typed_mat(const BasisData& b) {
  Mat1D<P, Q, T> m;
  for (int i = 0; i < Q * P; ++i) m.B[i] = T(b.interp[i]), m.G[i] = T(b.grad[i]);
  for (int i = 0; i < Q; ++i) m.W[i] = T(b.q_weight[i]);
  fill_eo(m);
  return m;
}

template <int P, int Q>
void launch_diag(const MassPlan& p, double* diag, double* ev, cudaStream_t s) {
  const int nc = 1;  // component 0; broadcast_comp_kernel copies it to the others
  if (p.dim == 3) {
    using L = Mass3D<P, Q>;
    static std::atomic<uint64_t> smem_set{0};
    set_smem(mass3d_diag_kernel<P, Q>, L::SMEM, smem_set);
    mass3d_diag_kernel<P, Q><<<unsigned(p.n_tiles), L::NT, L::SMEM, s>>>(
        squared_mat<P, Q>(p.basis), p.offs_t.get(), p.qd_t.get(), diag, ev, p.num_elem, nc, p.comp_stride);
  } else if (p.dim == 2) {
    mass2d_diag_kernel<P, Q><<<unsigned(p.n_tiles), Mass2D<P, Q>::NT, 0, s>>>(
        squared_mat<P, Q>(p.basis), p.offs_t.get(), p.qd_t.get(), diag, ev, p.num_elem, nc, p.comp_stride);
  } else {
    mass1d_diag_kernel<P, Q><<<unsigned(p.n_tiles), 128, 0, s>>>(
        squared_mat<P, Q>(p.basis), p.offs_t.get(), p.qd_t.get(), diag, ev, p.num_elem, nc, p.comp_stride);
  }
  FEM_LAUNCH_CHECK();
}

// Resident CTAs per SM the persistent CG apply asks for: the most, up to
// kCgMaxBlocks, that leave a thread kCgMinRegs registers (P <= 5); higher
// orders leave registers to ptxas (0), P = 8 asks for one CTA (see
// plain_min_blocks in device.cu).
constexpr int kCgMaxBlocks = 4, kCgMinRegs = 56;
constexpr int cg_min_blocks(int threads, int P, bool shared_matrix = false) {
  if (P > 5) return P >= 8 ? 1 : P == 7 && shared_matrix ? 2 : 0;
  for (int b = kCgMaxBlocks; b > 1; --b)
    if (65536 / (b * threads) >= kCgMinRegs && b * threads <= 2048) return b;
  return 1;
}

// CTAs of a persistent launch: SMs x resident CTAs per SM, at most n_tiles.
template <class K>
unsigned resident_grid(K kernel, int threads, int smem, int64_t n_tiles) {
  return unsigned(std::min<int64_t>(resident_ctas(reinterpret_cast<const void*>(kernel), threads, smem), n_tiles));
}

// w (+)= M (dinv . r) with delta = (dinv . r)^T M (dinv . r) reduced into the
// solver scalars.  ev != nullptr: element contributions to the E-vector.
// Where the Krylov apply takes the even-odd contractions (centro-symmetric B).
// 64^3 hexes, 3 components, one box, direct -> even-odd ms a solve:
//   FP32 storage  P = 4 17.4 -> 16.8, P = 5 32.0 -> 31.1, P = 6 58.0 -> 58.7,
//                 P = 7 92.1 -> 89.9;
//   BF16 storage  P = 4 27.6 -> 19.5, P = 5 41.4 -> 31.3, P = 6 75.4 -> 57.4,
//                 P = 7 124.0 -> 91.6 (the direct-form BF16 apply stalled 4x
//                 longer on its loads: 12 against 2.8 long-scoreboard stalls
//                 per issue at P = 5).
// FP64 (one component at a time) as the one-tile apply: P >= 4 (P = 5 51.6
// -> 50.7 ms a solve).
template <int P, class T, class S, int NCB>
constexpr bool cg_even_odd() {
  if constexpr (sizeof(T) == 8) return P >= 4 && NCB == 1;
  if constexpr (std::is_same<S, __nv_bfloat16>::value) return P >= 4;
  return P >= 4 && P != 6;
}

template <int P, int Q, class T, int NCB, class S = T, bool EO = cg_even_odd<P, T, S, NCB>()>
void launch_cg_apply3(const MassPlan& p, const S* r, T* w, T* ev, const S* qd, const ApplyCg<T>& ext,
                      cudaStream_t s) {
  using L = Mass3D<P, Q>;
  constexpr int smem = NCB * (L::SA + L::SB) * int(sizeof(T));
  static std::atomic<uint64_t> smem_set{0};
  // FP64, one component at a time: the even-odd contractions at P = 4 and
  // P >= 6 for a centro-symmetric B (as the one-tile apply), else at P >= 7
  // the direct form from a shared copy of the matrix (cg_even_odd).  Last argument: each CTA
  // prefetches its next tile into L2 (FP64 solve 57.2 -> 56.5 ms at 64^3,
  // P = 5, 3 components; FP32 unchanged).
  if constexpr (EO) {
    if (!p.centro_symmetric) return launch_cg_apply3<P, Q, T, NCB, S, false>(p, r, w, ev, qd, ext, s);
  }
  constexpr bool sb = P >= 7 && sizeof(T) == 8 && !EO;
  const auto kern = mass3d_apply_kernel<P, Q, cg_min_blocks(L::NT, P, sb || (EO && P == 7)), T, ApplyCg<T>, NCB, S,
                                        sb, EO>;
  set_smem(kern, smem, smem_set);
  kern<<<resident_grid(kern, L::NT, smem, p.n_tiles), L::NT, smem, s>>>(
      typed_mat<P, Q, T>(p.basis), p.offs_t.get(), qd, r, w, ev, p.num_elem, p.comp_run, p.comp_stride, ext, 1);
  FEM_LAUNCH_CHECK();
}

template <int P, int Q, class T, class S = T>
void launch_cg_apply(const MassPlan& p, const S* r, T* w, T* ev, const S* qd, const ApplyCg<T>& ext,
                     cudaStream_t s) {
  if (p.dim == 3) {
    // FP32: components batched through the phases where shared memory allows;
    // FP64: one at a time.  64^3 hexes, P = 5, 3 components: FP32 solve 32.1
    // ms batched vs 34.7 ms one at a time; FP64 56.2 ms batched (3 resident
    // CTAs, shared memory bound) vs 52.1 ms one at a time (4 CTAs); BF16
    // storage 41.6 ms batched vs 43.7 ms one at a time.
    constexpr int smem1 = (Mass3D<P, Q>::SA + Mass3D<P, Q>::SB) * int(sizeof(T));
    if constexpr (sizeof(T) == 4 && 3 * smem1 <= kMaxSmemPerCta) {
      if (p.comp_run == 3) return launch_cg_apply3<P, Q, T, 3, S>(p, r, w, ev, qd, ext, s);
    }
    if constexpr (sizeof(T) == 4 && 2 * smem1 <= kMaxSmemPerCta) {
      if (p.comp_run == 2) return launch_cg_apply3<P, Q, T, 2, S>(p, r, w, ev, qd, ext, s);
    }
    return launch_cg_apply3<P, Q, T, 1, S>(p, r, w, ev, qd, ext, s);
  }
  if (p.dim == 2) {
    using L = Mass2D<P, Q>;
    constexpr int smem = (L::S1 + L::S3) * int(sizeof(T));
    static std::atomic<uint64_t> smem_set{0};
    const auto kern = mass2d_apply_kernel<P, Q, T, ApplyCg<T>, S>;
    set_smem(kern, smem, smem_set);
    kern<<<resident_grid(kern, L::NT, smem, p.n_tiles), L::NT, smem, s>>>(
        typed_mat<P, Q, T>(p.basis), p.offs_t.get(), qd, r, w, ev, p.num_elem, p.comp_run, p.comp_stride, ext, 0);
  } else {
    const auto kern = mass1d_apply_kernel<P, Q, T, ApplyCg<T>, S>;
    kern<<<resident_grid(kern, 128, 0, p.n_tiles), 128, 0, s>>>(
        typed_mat<P, Q, T>(p.basis), p.offs_t.get(), qd, r, w, ev, p.num_elem, p.comp_run, p.comp_stride, ext);
  }
  FEM_LAUNCH_CHECK();
}

constexpr int kSolveMinP = 2, kSolveMaxP = 8, kSolveQSpan = 3;

struct SolveDispatch {
  DiagLauncher diag[kSolveMaxP + 1][kSolveQSpan] = {};
  CgApplyLauncher<double> cg64[kSolveMaxP + 1][kSolveQSpan] = {};
  CgApplyLauncher<float> cg32[kSolveMaxP + 1][kSolveQSpan] = {};
  CgApplyLauncher<float, __nv_bfloat16> cg16[kSolveMaxP + 1][kSolveQSpan] = {};
};

template <int P, int DQ>
struct SolveTable {
  static void fill(SolveDispatch& d) {
    d.diag[P][DQ] = launch_diag<P, P + DQ>;
    d.cg64[P][DQ] = launch_cg_apply<P, P + DQ, double>;
    d.cg32[P][DQ] = launch_cg_apply<P, P + DQ, float>;
    d.cg16[P][DQ] = launch_cg_apply<P, P + DQ, float, __nv_bfloat16>;
    if constexpr (DQ + 1 < kSolveQSpan)
      SolveTable<P, DQ + 1>::fill(d);
    else if constexpr (P + 1 <= kSolveMaxP)
      SolveTable<P + 1, 0>::fill(d);
  }
};

const SolveDispatch& solve_dispatch() {
  static const SolveDispatch d = [] {
    SolveDispatch t;
    SolveTable<kSolveMinP, 0>::fill(t);
    return t;
  }();
  return d;
}

inline int red_grid(int64_t n) { return int(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8))); }

bool deterministic(const MassPlan& p) { return p.scatter_mode != FEM_B200_SCATTER_ATOMIC; }

// diag = the assembled diagonal (zeroed first); transpose-map order in
// deterministic plans, atomics otherwise.  Component 0 is assembled and
// copied to the others, so every component of a node holds the same bits
// (the CG apply reads one scale per node).
void assemble_diagonal(MassPlan& p, double* diag, cudaStream_t s) {
  FEM_CUDA_CHECK(cudaMemsetAsync(diag, 0, size_t(p.l_size) * sizeof(double), s));
  const DiagLauncher launch = solve_dispatch().diag[p.P][p.Q - p.P];
  const RestrictionData& r = *p.r;
  if (!deterministic(p)) {
    launch(p, diag, nullptr, s);
  } else {
    launch(p, diag, p.evec.get(), s);
    launch_csr_scatter(r.num_nodes, p.num_elem, p.es, 1, p.comp_stride, r.l_vec_indices.get(), r.t_offsets.get(),
                       r.t_indices.get(), p.evec.get(), diag, s);
    FEM_LAUNCH_CHECK();
  }
  if (p.comp_run > 1) {
    const int64_t n = int64_t(p.num_elem) * p.es;
    broadcast_comp_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, r.offsets.get(), p.comp_run, p.comp_stride, diag);
    FEM_LAUNCH_CHECK();
  }
}

// The plan's solver state: diagonal and its inverse, FP32 dinv and the
// reduced-precision qdata and Krylov vectors of the inner solves, reduction
// partials and the device scalars.  Each part is keyed on its own buffer: an
// FP32 or BF16 apply may have made the FP32 / BF16 qdata copy already.
void ensure_solver_state(MassPlan& p, int precision, cudaStream_t s) {
  const size_t n = size_t(p.l_size), nq = p.qd_t.size();
  if (p.diag.size() != n) {
    p.diag.alloc(n);
    assemble_diagonal(p, p.diag.get(), s);
    p.dinv.alloc(n);
    invert_kernel<double><<<red_grid(int64_t(n)), 256, 0, s>>>(int64_t(n), p.diag.get(), p.dinv.get());
    FEM_LAUNCH_CHECK();
    p.cg_r.alloc(n), p.cg_p.alloc(n), p.cg_s.alloc(n), p.cg_w.alloc(n);
    p.part.alloc(2 * size_t(std::max<int64_t>(p.n_tiles, 148 * 8)));
    p.cg_st.alloc(1);
    FEM_CUDA_CHECK(cudaMemsetAsync(p.cg_st.get(), 0, sizeof(CgScalars), s));
    if (!p.cg_host_ext) p.cg_host.alloc(1);
  }
  if (precision == FEM_B200_SOLVE_FP64) return;
  if (p.dinv32.size() != n) {
    p.dinv32.alloc(n);
    invert_kernel<float><<<red_grid(int64_t(n)), 256, 0, s>>>(int64_t(n), p.diag.get(), p.dinv32.get());
    FEM_LAUNCH_CHECK();
    p.f_w.alloc(n), p.f_x.alloc(n);
  }
  if (deterministic(p) && p.evec32.size() != p.evec.size()) p.evec32.alloc(p.evec.size());
  if (precision == FEM_B200_SOLVE_FP32_IR) {
    if (p.qd_t32.size() != nq) {
      p.qd_t32.alloc(nq);
      to_float_kernel<<<red_grid(int64_t(nq)), 256, 0, s>>>(int64_t(nq), p.qd_t.get(), p.qd_t32.get());
      FEM_LAUNCH_CHECK();
    }
    if (p.f_r.size() != n) p.f_r.alloc(n), p.f_p.alloc(n), p.f_s.alloc(n);
  } else {
    if (p.qd_t16.size() != nq) {
      p.qd_t16.alloc(nq);
      to_bf16_kernel<<<red_grid(int64_t(nq)), 256, 0, s>>>(int64_t(nq), p.qd_t.get(), p.qd_t16.get());
      FEM_LAUNCH_CHECK();
    }
    if (p.h_r.size() != n) p.h_r.alloc(n), p.h_p.alloc(n), p.h_s.alloc(n);
  }
}

// The host's copy of the device scalars (synchronises the stream).
CgScalars* host_scalars(MassPlan& p) { return p.cg_host_ext ? p.cg_host_ext : p.cg_host.get(); }

const CgScalars& read_scalars(MassPlan& p, cudaStream_t s) {
  FEM_CUDA_CHECK(cudaMemcpyAsync(host_scalars(p), p.cg_st.get(), sizeof(CgScalars), cudaMemcpyDeviceToHost, s));
  FEM_CUDA_CHECK(cudaStreamSynchronize(s));
  return *host_scalars(p);
}

inline bool aligned16(const void* ptr) { return (reinterpret_cast<uintptr_t>(ptr) & 15) == 0; }

// Krylov vectors r, p, s in storage S; x, w (the apply's target), the
// E-vector and dinv in the arithmetic type T.
template <class T, class S = T>
struct Krylov {
  T* x;
  S *r, *p, *s;
  T *w, *ev;
  const T* dinv;
  const S* qd;
  CgApplyLauncher<T, S> apply;
};

template <class T, class S>
void cg_apply(MassPlan& p, const Krylov<T, S>& k, cudaStream_t s) {
  const ApplyCg<T> ext{k.dinv, p.part.get(), p.cg_st.get()};
  if (!deterministic(p)) {
    k.apply(p, k.r, k.w, nullptr, k.qd, ext, s);
    return;
  }
  const RestrictionData& r = *p.r;
  k.apply(p, k.r, nullptr, k.ev, k.qd, ext, s);
  launch_csr_scatter(r.num_nodes, p.num_elem, p.es, p.comp_run, p.comp_stride, r.l_vec_indices.get(),
                     r.t_offsets.get(), r.t_indices.get(), k.ev, k.w, s, &p.cg_st.get()->done);
  FEM_LAUNCH_CHECK();
}

// Jacobi PCG on M x = b * scale from x = 0 until ||r|| <= rtol ||r0|| or
// max_it residual updates.  The host queues iterations in growing batches and
// reads the scalars between batches; kernels queued after the stop return at
// once.  Returns the final scalars.
template <class T, class S = T>
CgScalars krylov_solve(MassPlan& p, const Krylov<T, S>& k, const double* b, double scale, double rtol, int max_it,
                       cudaStream_t s) {
  constexpr bool mixed = !std::is_same<T, S>::value;
  const int64_t n = p.l_size;
  const int g = red_grid(n);
  if constexpr (mixed)
    cg_init_bf16_kernel<<<g, 256, 0, s>>>(n, b, scale, k.dinv, k.x, k.r, k.p, k.s, k.w, p.cg_st.get(), p.part.get(),
                                          rtol, max_it);
  else
    cg_init_kernel<T><<<g, 256, 0, s>>>(n, b, scale, k.dinv, k.x, k.r, k.p, k.s, k.w, p.cg_st.get(), p.part.get(),
                                        rtol, max_it);
  FEM_LAUNCH_CHECK();
  cg_apply(p, k, s);
  const bool vec = aligned16(k.dinv) && aligned16(k.x) && aligned16(k.r) && aligned16(k.p) && aligned16(k.s) &&
                   aligned16(k.w);
  int batch = 4;
  for (int queued = 0;; queued += batch, batch = std::min(batch * 2, 32)) {
    for (int j = 0; j < batch; ++j) {
      if constexpr (mixed)
        cg_update_bf16_kernel<<<g, 256, 0, s>>>(n, k.dinv, k.x, k.r, k.p, k.s, k.w, p.cg_st.get(), p.part.get(), vec);
      else if (vec)
        cg_update_kernel<T, true><<<g, 256, 0, s>>>(n, k.dinv, k.x, k.r, k.p, k.s, k.w, p.cg_st.get(), p.part.get());
      else
        cg_update_kernel<T, false><<<g, 256, 0, s>>>(n, k.dinv, k.x, k.r, k.p, k.s, k.w, p.cg_st.get(),
                                                     p.part.get());
      FEM_LAUNCH_CHECK();
      cg_apply(p, k, s);
    }
    const CgScalars& st = read_scalars(p, s);
    if (st.done) break;
    if (queued > max_it + 64) throw cuda_error("mass solve: the device iteration count did not advance");
  }
  const CgScalars st = *host_scalars(p);
  if (st.done == 3 && st.iters == 0)
    throw cuda_error("mass solve: breakdown, (u, M u) <= 0: the operator is not positive definite on this "
                     "right-hand side");
  return st;
}

// r = f - M u (cg_w: scratch for M u; u == nullptr: r = f); returns ||r||.
double outer_residual(MassPlan& p, const double* f, const double* u, cudaStream_t s) {
  const int64_t n = p.l_size;
  if (u) mass_apply_impl(p, u, p.cg_w.get(), true, s);
  residual_kernel<<<red_grid(n), 256, 0, s>>>(n, f, u ? p.cg_w.get() : nullptr, p.cg_r.get(), p.cg_st.get(),
                                               p.part.get());
  FEM_LAUNCH_CHECK();
  return std::sqrt(read_scalars(p, s).res);
}

// The inner solves' relative tolerance: what the last cycle still needs (with
// a factor 2 margin), but not below what the Krylov vectors' storage attains:
// FP32 (unit roundoff 6e-8) reaches 5e-6; BF16 (unit roundoff 3.9e-3) stalls
// near its rounding level, so each BF16 cycle asks for 2 decimal digits.
constexpr double kInnerFloor = 5e-6, kInnerFloorBf16 = 1e-2;

// FP64 outer loop: r = f - M u in FP64, correction d from the inner PCG on
// r / ||r|| (storage S), u += ||r|| d.
template <class T, class S>
void refine(MassPlan& p, const Krylov<T, S>& k, const double* f, double* u, double rtol, int max_iter, double floor,
            int& total_it, int& outer, double& nf, double& nr, cudaStream_t s) {
  nf = outer_residual(p, f, nullptr, s);
  FEM_CUDA_CHECK(cudaMemsetAsync(u, 0, size_t(p.l_size) * sizeof(double), s));
  nr = nf;
  while (nr > rtol * nf && total_it < max_iter && outer < 100) {
    const double inner = std::min(0.5, std::max(floor, 0.5 * rtol * nf / nr));
    const CgScalars st = krylov_solve<T, S>(p, k, p.cg_r.get(), 1.0 / nr, inner, max_iter - total_it, s);
    total_it += st.iters;
    ++outer;
    add_scaled_kernel<<<red_grid(p.l_size), 256, 0, s>>>(p.l_size, nr, k.x, u);
    FEM_LAUNCH_CHECK();
    const double prev = nr;
    nr = outer_residual(p, f, u, s);
    if (!(nr < prev)) break;  // no progress: the inner solve has stalled
  }
}

SolveStats mass_solve_impl(MassPlan& p, const double* f, double* u, double rtol, int max_iter, int precision,
                           cudaStream_t s) {
  ensure_solver_state(p, precision, s);
  const SolveDispatch& d = solve_dispatch();
  const int di = p.Q - p.P;
  int total_it = 0, outer = 0;
  double nf = 0.0, nr = 0.0;
  if (precision == FEM_B200_SOLVE_FP64) {
    const Krylov<double> k{u, p.cg_r.get(), p.cg_p.get(), p.cg_s.get(), p.cg_w.get(), p.evec.get(),
                           p.dinv.get(), p.qd_t.get(), d.cg64[p.P][di]};
    const CgScalars st = krylov_solve<double>(p, k, f, 1.0, rtol, max_iter, s);
    total_it = st.iters;
    nf = std::sqrt(st.rr0);
    nr = outer_residual(p, f, u, s);  // the true FP64 residual
  } else if (precision == FEM_B200_SOLVE_FP32_IR) {
    const Krylov<float> k{p.f_x.get(), p.f_r.get(), p.f_p.get(), p.f_s.get(), p.f_w.get(), p.evec32.get(),
                          p.dinv32.get(), p.qd_t32.get(), d.cg32[p.P][di]};
    refine(p, k, f, u, rtol, max_iter, kInnerFloor, total_it, outer, nf, nr, s);
  } else {
    const Krylov<float, __nv_bfloat16> k{p.f_x.get(),  p.h_r.get(),    p.h_p.get(),    p.h_s.get(),
                                         p.f_w.get(),  p.evec32.get(), p.dinv32.get(), p.qd_t16.get(),
                                         d.cg16[p.P][di]};
    refine(p, k, f, u, rtol, max_iter, kInnerFloorBf16, total_it, outer, nf, nr, s);
  }
  check_status(p, s);
  SolveStats out;
  out.iterations = total_it;
  out.refinements = outer;
  out.rel_residual = nf > 0.0 ? nr / nf : 0.0;
  return out;
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
    assemble_diagonal(p, diag, as_stream(stream));
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
    require(precision == FEM_B200_SOLVE_FP64 || precision == FEM_B200_SOLVE_FP32_IR ||
                precision == FEM_B200_SOLVE_BF16_IR,
            "mass solve: unknown precision");
    if (p.comp_run != p.num_comp)
      throw unsupported_error(
          "mass solve: the reference apply_mass leaves components 1.. out (a singular operator); use "
          "FEM_B200_QF_APPLY_MASS_VECTOR for a multi-component solve");
    DeviceGuard g(p.device);
    const SolveStats st = mass_solve_impl(p, f, u, rtol, max_iter, precision, as_stream(stream));
    if (iterations) *iterations = st.iterations;
    if (refinements) *refinements = st.refinements;
    if (rel_residual) *rel_residual = st.rel_residual;
  });
}

}  // extern "C"
