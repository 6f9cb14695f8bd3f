// The transpose-map (deterministic) scatter v += E^T ev, shared by the
// element restriction, the mass operator, the Krylov solver and the FP32
// storage path (sm_100a).  The map is the reference's
// (src/cuda/cuda-elem-restriction.cu:148-176): for each used L-vector node,
// in increasing L order, its E-vector entries t_indices[t_offsets[n] ..
// t_offsets[n+1]) as t = e*elem_size + i, increasing.  Summing them in that
// order is the order of the reference's CPU scatter
// (src/elem-restriction.cpp:73-82) and of its CUDA deterministic kernel
// (src/cuda/cuda-elem-restriction.cu:75-95); each node then makes one add
// into v.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

namespace fem_b200 {

// v += E^T ev through the transpose map (the reference's deterministic
// scatter: one thread per L-vector node, its contributions summed in the
// map's order).  T is the value type.  I is the index type of the E-vector
// arithmetic in the inner loop: int where every E-vector index fits (fewer
// instructions in a latency-bound loop), int64_t otherwise; the L-vector
// index is always 64-bit.  A non-null stop makes the kernel return when
// *stop is non-zero (a converged Krylov solve whose kernels are still queued).
template <class T, class I>
__global__ void csr_scatter_kernel(int num_nodes, int num_elem, int elem_size, int num_comp, int64_t comp_stride,
                                   const int* __restrict__ l_vec_indices, const int* __restrict__ t_offsets,
                                   const int* __restrict__ t_indices, const T* __restrict__ ev, T* __restrict__ v,
                                   const int* stop) {
  if (stop && *stop) return;
  const I ne = I(num_elem), es = I(elem_size);
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < num_nodes; n += gridDim.x * blockDim.x) {
    const int64_t l = l_vec_indices[n];
    const int t0 = t_offsets[n], t1 = t_offsets[n + 1];
    for (int k = 0; k < num_comp; ++k) {
      T sum = T(0);
      for (int t = t0; t < t1; ++t) {
        const int ti = t_indices[t];
        const int e = ti / elem_size, i = ti - e * elem_size;
        sum += ev[(I(k) * es + i) * ne + e];
      }
      v[l + k * comp_stride] += sum;
    }
  }
}

// The transpose-map reduction with the narrowest index type that fits.
template <class T>
void launch_csr_scatter(int num_nodes, int num_elem, int elem_size, int num_comp, int64_t comp_stride,
                        const int* l_vec_indices, const int* t_offsets, const int* t_indices, const T* ev, T* v,
                        cudaStream_t s, const int* stop = nullptr) {
  const int64_t e_size = int64_t(num_comp) * elem_size * num_elem;
  const unsigned grid = unsigned(std::max<int64_t>(1, std::min<int64_t>((num_nodes + 255) / 256, 148LL * 64)));
  if (e_size < (int64_t(1) << 31))
    csr_scatter_kernel<T, int><<<grid, 256, 0, s>>>(num_nodes, num_elem, elem_size, num_comp, comp_stride,
                                                    l_vec_indices, t_offsets, t_indices, ev, v, stop);
  else
    csr_scatter_kernel<T, int64_t><<<grid, 256, 0, s>>>(num_nodes, num_elem, elem_size, num_comp, comp_stride,
                                                        l_vec_indices, t_offsets, t_indices, ev, v, stop);
}

}  // namespace fem_b200
