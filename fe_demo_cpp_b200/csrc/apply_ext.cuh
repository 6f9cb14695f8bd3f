// Optional extras of the fused mass apply kernels, used by the device solver:
//   * a scaled gather, u_i = dinv_i * r_i at each gathered node (the Jacobi
//     preconditioner applied on the fly, so z = D^-1 r is never stored);
//   * delta = u^T M u, reduced from the quadrature points of the same pass
//     (u^T M u = sum_e sum_q qdata_q |(B E_e u)_q|^2, the pointwise mass
//     form), so CG needs no separate dot-product pass over M u;
//   * a deterministic grid reduction: every CTA writes its partial sum, the
//     last CTA to finish adds the partials in a fixed order and updates the
//     solver's device-resident scalars.  Results are bitwise reproducible.
// ApplyPlain switches all of it off (the operator apply).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace fem_b200 {

// Device-resident state of one Krylov solve (Chronopoulos-Gear PCG).
struct CgScalars {
  double gamma;      // (r, D^-1 r) of the current residual
  double gamma_old;  // the previous one
  double delta;      // (u, M u), u = D^-1 r
  double alpha, beta;
  double rr;    // (r, r)
  double rr0;   // (r0, r0)
  double tol2;  // stop when rr <= tol2 (rtol^2 rr0)
  double res;   // (r, r) of the last FP64 residual (outer loop)
  int iters;    // residual updates done
  int max_iters;
  int done;             // 0 running, 1 converged, 2 iteration limit, 3 breakdown
  unsigned int ticket;  // CTAs finished in the current kernel (reset by the last)
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block sum of N values in a fixed order; the result is valid in thread 0.
template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N]) {
  __shared__ double part[N][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();  // part may be in use by a previous call
#pragma unroll
  for (int i = 0; i < N; ++i) {
    v[i] = warp_sum(v[i]);
    if (lane == 0) part[i][w] = v[i];
  }
  __syncthreads();
  if (w == 0) {
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = warp_sum(lane < nw ? part[i][lane] : 0.0);
  }
}

// Grid sum of N values per thread.  part holds N * gridDim.x doubles.  The
// last CTA calls fin(sums) in thread 0 and re-arms the ticket.  Every thread
// of every CTA must call this.
template <int N, class Fin>
__device__ __forceinline__ void grid_sum(double (&v)[N], double* part, unsigned int* ticket, Fin fin) {
  __shared__ bool last;
  block_sum<N>(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < N; ++i) part[int64_t(i) * gridDim.x + blockIdx.x] = v[i];
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double s[N];
#pragma unroll
  for (int i = 0; i < N; ++i) s[i] = 0.0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
#pragma unroll
    for (int i = 0; i < N; ++i) s[i] += __ldcg(part + int64_t(i) * gridDim.x + b);
  }
  block_sum<N>(s);
  if (threadIdx.x == 0) {
    fin(s);
    *ticket = 0;
  }
}

struct ApplyPlain {
  static constexpr bool kScale = false, kDot = false;
};

template <class T>
struct ApplyCg {
  static constexpr bool kScale = true, kDot = true;
  const T* scale;  // dinv, l_size entries, the same for every component of a node
  double* part;    // >= number of CTAs
  CgScalars* st;
};

// After w = M u: the step length and direction weight of the next update
// (Chronopoulos-Gear: alpha = gamma / (delta - beta gamma / alpha_old)).
__device__ __forceinline__ void cg_after_apply(CgScalars* st, double delta) {
  st->delta = delta;
  double alpha, beta;
  if (st->iters == 0) {
    beta = 0.0;
    alpha = st->gamma / delta;
  } else {
    beta = st->gamma / st->gamma_old;
    alpha = st->gamma / (delta - beta * st->gamma / st->alpha);
  }
  if (!(delta > 0.0) || !(alpha > 0.0) || !(alpha < 1e300)) st->done = 3;
  st->alpha = alpha;
  st->beta = beta;
}

}  // namespace fem_b200
