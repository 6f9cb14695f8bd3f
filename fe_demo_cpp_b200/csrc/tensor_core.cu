// Self-test of the tensor-core layer (tc_ptx.cuh) that the tensor-core mass
// apply (mass_tc.cuh) is built on: descriptors, tensor memory, the MMA and
// its completion, checked on one product before any apply relies on them.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "common.hpp"
#include "plan.hpp"
#include "tc_ptx.cuh"

namespace fem_b200 {
namespace {

// One CTA, 128 threads: D = A B^T, M = 128, N = 16, K = 8, TF32, A and B
// staged K-major exactly as the mass apply stages them, D read back from
// tensor memory (thread t: row t).  A [128][8], B [16][8], D [128][16].
__global__ void __launch_bounds__(128) tc_selftest_kernel(const float* __restrict__ A, const float* __restrict__ B,
                                                          float* __restrict__ D, int* __restrict__ status) {
  __shared__ __align__(1024) float a_k[tc::kTcBlockFloats];
  __shared__ __align__(1024) float b_k[2 * tc::kTcSboBytes / 4];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t taddr_s;
  const int t = threadIdx.x, warp = t >> 5;
  for (int k = 0; k < 8; ++k) a_k[tc::kmajor_index(t, k)] = tc::to_tf32(A[t * 8 + k]);
  if (t < 16)
    for (int k = 0; k < 8; ++k) b_k[tc::kmajor_index(t, k)] = tc::to_tf32(B[t * 8 + k]);
  if (t == 0) tc::mbar_init(&bar, 1);
  if (warp == 0) tc::tmem_alloc(&taddr_s, 32);
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t taddr = taddr_s;
  if (t == 0) {
    tc::mma_tf32(taddr, tc::kmajor_desc(tc::smem_u32(a_k)), tc::kmajor_desc(tc::smem_u32(b_k)), tc::idesc_tf32(128, 16),
                 0);
    tc::mma_commit(&bar);
  }
  if (!tc::mbar_wait(&bar, 0, 1 << 20)) atomicOr(status, 1);
  tc::fence_after_sync();
  float r[16];
  tc::tmem_ld16(taddr + (uint32_t(32 * warp) << 16), r);
  tc::tmem_wait_ld();
  for (int n = 0; n < 16; ++n) D[t * 16 + n] = r[n];
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(taddr, 32);
}

float round_tf32(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  u = (u + 0x1000u) & 0xFFFFE000u;
  float y;
  std::memcpy(&y, &u, 4);
  return y;
}

}  // namespace
}  // namespace fem_b200

using namespace fem_b200;

extern "C" {

int fem_b200_tc_selftest(double* max_rel_err) {
  return guarded([&] {
    require(max_rel_err != nullptr, "tc self-test: NULL output");
    std::vector<float> A(128 * 8), B(16 * 8);
    for (int i = 0; i < 128 * 8; ++i) A[size_t(i)] = float(std::sin(0.37 * i + 0.1) * (1.0 + (i % 7)));
    for (int i = 0; i < 16 * 8; ++i) B[size_t(i)] = float(std::cos(0.53 * i + 0.2));
    DevBuf<float> dA(A.size()), dB(B.size()), dD(128 * 16);
    DevBuf<int> st(1);
    FEM_CUDA_CHECK(cudaMemcpy(dA.get(), A.data(), A.size() * 4, cudaMemcpyHostToDevice));
    FEM_CUDA_CHECK(cudaMemcpy(dB.get(), B.data(), B.size() * 4, cudaMemcpyHostToDevice));
    FEM_CUDA_CHECK(cudaMemset(st.get(), 0, 4));
    tc_selftest_kernel<<<1, 128>>>(dA.get(), dB.get(), dD.get(), st.get());
    FEM_LAUNCH_CHECK();
    std::vector<float> h(128 * 16);
    int hs = 0;
    FEM_CUDA_CHECK(cudaMemcpy(h.data(), dD.get(), h.size() * 4, cudaMemcpyDeviceToHost));
    FEM_CUDA_CHECK(cudaMemcpy(&hs, st.get(), 4, cudaMemcpyDeviceToHost));
    if (hs) throw cuda_error("tc self-test: the MMA completion wait ran out");
    double err = 0.0, scale = 0.0;
    for (int m = 0; m < 128; ++m)
      for (int n = 0; n < 16; ++n) {
        double want = 0.0;
        for (int k = 0; k < 8; ++k)
          want += double(round_tf32(A[size_t(m * 8 + k)])) * double(round_tf32(B[size_t(n * 8 + k)]));
        err = std::fmax(err, std::fabs(h[size_t(m * 16 + n)] - want));
        scale = std::fmax(scale, std::fabs(want));
      }
    *max_rel_err = err / scale;
  });
}

}  // extern "C"
