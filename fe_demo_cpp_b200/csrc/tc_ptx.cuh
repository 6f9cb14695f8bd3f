// Thin inline-PTX layer over the 5th-generation tensor cores (sm_100a):
// tensor memory allocation, tcgen05.mma (kind::tf32, one CTA), commits to an
// mbarrier, tensor-memory loads, the shared-memory matrix descriptor of the
// canonical K-major no-swizzle layout, and the instruction descriptor.  Field
// layouts follow the PTX ISA's tcgen05 descriptor tables (the bit positions
// CUTLASS names in UMMA::SmemDescriptor / InstrDescriptor).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace fem_b200 {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- tensor memory -----------------------------------------------------------
// One warp allocates `cols` columns (a power of 2, >= 32) and writes the base
// address to *dst (shared memory); the permit is released at once, so other
// CTAs on the SM can allocate.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 lanes x 16 consecutive 32-bit columns: thread t of the warp gets lane
// (lane base of taddr) + t, columns col .. col + 15.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&r)[16]) {
  uint32_t u[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7]), "=r"(u[8]),
        "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]), "=r"(u[13]), "=r"(u[14]), "=r"(u[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) r[i] = __uint_as_float(u[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---- mbarrier ------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// Waits for the phase with parity `parity` to complete; gives up after
// `limit` polls and returns false (the caller records the failure).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit) {
  const uint32_t a = smem_u32(bar);
  for (int i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// ---- MMA -------------------------------------------------------------------------
// Generic-proxy shared-memory writes made visible to the tensor cores.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[tmem] (+)= A[smem desc] * B[smem desc]^T, kind::tf32 (FP32 accumulate);
// accumulate = 0 overwrites D.  Issued by one thread.
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}
// The MMAs issued so far by this thread arrive on `bar` once complete.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// Canonical K-major layout without swizzle, for 32-bit elements: an operand
// of R rows x 8 columns (one K = 8 MMA step) in 8-row x 16-byte core
// matrices, element (r, k) at byte
//   (r % 8) * 16 + (r / 8) * 288 + (k / 4) * 144 + (k % 4) * 4,
// i.e. the two K halves 144 bytes apart (leading byte offset) and row groups
// 288 bytes apart (stride byte offset).  The strides are padded past the
// dense 128 / 256 so that the column-wise (transposing) stores of a warp --
// 8 lanes a row group, 4 row groups -- fall in 32 distinct banks.
constexpr int kTcLboBytes = 144, kTcSboBytes = 288;
constexpr int kTcBlockFloats = 16 * kTcSboBytes / 4;  // 128 rows
__host__ __device__ constexpr int kmajor_index(int r, int k) {
  return (r % 8) * 4 + (r / 8) * (kTcSboBytes / 4) + (k / 4) * (kTcLboBytes / 4) + k % 4;
}

// Shared-memory matrix descriptor of that layout: start address, leading and
// stride byte offsets (multiples of 16 bytes), version 1, no swizzle.
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= uint64_t((addr >> 4) & 0x3FFF);
  d |= uint64_t((uint32_t(kTcLboBytes) >> 4) & 0x3FFF) << 16;
  d |= uint64_t((uint32_t(kTcSboBytes) >> 4) & 0x3FFF) << 32;
  d |= uint64_t(1) << 46;  // version (sm_100); base offset 0, layout type 0 (no swizzle)
  return d;
}

// Instruction descriptor of kind::tf32: FP32 accumulator, A and B K-major,
// M x N.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4)                  // D format F32
         | (2u << 7) | (2u << 10)    // A, B format TF32
         | (uint32_t(N >> 3) << 17)  // N
         | (uint32_t(M >> 4) << 24); // M
}

// FP32 -> TF32 (round to nearest, ties away), as a 32-bit container.
__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

}  // namespace tc
}  // namespace fem_b200
