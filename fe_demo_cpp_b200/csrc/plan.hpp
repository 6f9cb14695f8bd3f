// Shared host-side types of libfem_b200: device buffers, restriction /
// basis / mass-plan state, launch helpers.  Used by device.cu (the operator
// entry points) and solver.cu (diagonal, mixed-precision solves).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "common.hpp"
#include "copy_pool.hpp"
#include "fem_b200.h"
#include "host_setup.hpp"
#include "mass_kernels.cuh"

namespace fem_b200 {

// ---------------------------------------------------------------------------
// Stream-ordered allocation.  Inside an AllocScope, the DevBufs a thread
// allocates come from `pool` in `stream` order (cudaMallocFromPoolAsync) and
// are returned in that stream's order when released (cudaFreeAsync), so a
// request that builds and frees its buffers does not synchronise the device
// under the other requests' kernels (cudaFree would).
// ---------------------------------------------------------------------------
struct AllocCtx {
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;
};
inline AllocCtx*& alloc_ctx() {
  static thread_local AllocCtx* ctx = nullptr;
  return ctx;
}
struct AllocScope {
  AllocCtx ctx;
  AllocCtx* prev;
  AllocScope(cudaStream_t s, cudaMemPool_t pool) : ctx{s, pool}, prev(alloc_ctx()) { alloc_ctx() = &ctx; }
  ~AllocScope() { alloc_ctx() = prev; }
  AllocScope(const AllocScope&) = delete;
  AllocScope& operator=(const AllocScope&) = delete;
};

// ---------------------------------------------------------------------------
// RAII device buffer (move-only), the reference's DeviceArray semantics
// (include/cuda/device-array.hpp:18-95) without the synchronous copies.
// ---------------------------------------------------------------------------
template <class T>
class DevBuf {
 public:
  DevBuf() = default;
  explicit DevBuf(size_t n) { alloc(n); }
  ~DevBuf() { release(); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_), s_(o.s_), async_(o.async_) { o.p_ = nullptr, o.n_ = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p_ = o.p_, n_ = o.n_, s_ = o.s_, async_ = o.async_;
      o.p_ = nullptr, o.n_ = 0;
    }
    return *this;
  }
  void alloc(size_t n) {
    release();
    if (n == 0) return;
    if (AllocCtx* c = alloc_ctx()) {
      FEM_CUDA_CHECK(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p_), n * sizeof(T), c->pool, c->stream));
      s_ = c->stream, async_ = true;
    } else {
      FEM_CUDA_CHECK(cudaMalloc(&p_, n * sizeof(T)));
      s_ = nullptr, async_ = false;
    }
    n_ = n;
  }
  T* get() const { return p_; }
  size_t size() const { return n_; }
  size_t bytes() const { return n_ * sizeof(T); }

 private:
  void release() noexcept {
    if (p_) {
      if (async_)
        (void)cudaFreeAsync(p_, s_);
      else
        (void)cudaFree(p_);
    }
    p_ = nullptr, n_ = 0;
  }
  T* p_ = nullptr;
  size_t n_ = 0;
  cudaStream_t s_ = nullptr;
  bool async_ = false;
};

// RAII page-locked host buffer.
template <class T>
class PinnedBuf {
 public:
  PinnedBuf() = default;
  ~PinnedBuf() {
    if (p_) (void)cudaFreeHost(p_);
  }
  PinnedBuf(const PinnedBuf&) = delete;
  PinnedBuf& operator=(const PinnedBuf&) = delete;
  void alloc(size_t n) {
    if (p_) (void)cudaFreeHost(p_);
    p_ = nullptr;
    FEM_CUDA_CHECK(cudaMallocHost(&p_, n * sizeof(T)));
  }
  T* get() const { return p_; }

 private:
  T* p_ = nullptr;
};

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    FEM_CUDA_CHECK(cudaGetDevice(&prev));
    if (prev != dev) FEM_CUDA_CHECK(cudaSetDevice(dev));
  }
  ~DeviceGuard() {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != prev && prev >= 0) (void)cudaSetDevice(prev);
  }
};

inline int current_device() {
  int d = 0;
  FEM_CUDA_CHECK(cudaGetDevice(&d));
  return d;
}

inline cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

inline int grid_for(int64_t n, int threads) {
  const int64_t b = (n + threads - 1) / threads;
  return int(std::max<int64_t>(1, std::min<int64_t>(b, 148LL * 64)));
}

#define FEM_LAUNCH_CHECK() FEM_CUDA_CHECK(cudaGetLastError())

// ---------------------------------------------------------------------------
// Restriction
// ---------------------------------------------------------------------------
struct RestrictionData {
  int device = 0;
  bool strided = false;
  int num_elem = 0, elem_size = 0, num_comp = 0, comp_stride = 0, l_size = 0;
  int64_t e_size = 0;
  int64_t strides[3] = {0, 0, 0};
  int scatter_mode = FEM_B200_SCATTER_ATOMIC;
  DevBuf<int> offsets;  // [num_elem][elem_size]
  int num_nodes = 0;    // transpose map (deterministic offset restrictions)
  DevBuf<int> l_vec_indices, t_offsets, t_indices;
};

// ---------------------------------------------------------------------------
// Basis: host data plus device copies for the generic contraction kernels
// ---------------------------------------------------------------------------
struct BasisDev {
  int device = 0;
  BasisData h;
  DevBuf<double> interp, grad, weight;
  DevBuf<double> scratch;  // ping-pong pass buffers, grown on demand
  std::mutex scratch_mu;
};

// ---------------------------------------------------------------------------
// Mass plan
// ---------------------------------------------------------------------------
// The host-memory apply's pipeline state (host_apply.cu): copy streams,
// events and the element chunks with the L-vector node span each touches.
struct HostPipeline {
  cudaStream_t h2d = nullptr, d2h = nullptr;
  std::vector<cudaEvent_t> ev;  // 2 + 2 per chunk: start, v zeroed, then (u span in, chunk applied)
  int64_t tiles_per_chunk = 0;
  int target = 0;               // the chunk count it was built for
  std::vector<int64_t> lo, hi;  // per chunk: smallest and largest offset of its elements
  // staging for pageable host vectors, made by the first such apply: a ring
  // of page-locked slots per direction and an event per slot (the memcpy
  // threads are one pool for the process, host_apply.cu)
  PinnedBuf<double> ring_in, ring_out;
  std::vector<cudaEvent_t> slot_ev;  // kSlots for the copies in, then kSlots for the copies out
  HostPipeline() = default;
  HostPipeline(const HostPipeline&) = delete;
  HostPipeline& operator=(const HostPipeline&) = delete;
  ~HostPipeline() {
    for (cudaEvent_t e : slot_ev)
      if (e) (void)cudaEventDestroy(e);
    for (cudaEvent_t e : ev)
      if (e) (void)cudaEventDestroy(e);
    if (h2d) (void)cudaStreamDestroy(h2d);
    if (d2h) (void)cudaStreamDestroy(d2h);
  }
};

struct MassPlan;
using ApplyLauncher = void (*)(const MassPlan&, const double*, double*, double*, cudaStream_t);
using BuildLauncher = void (*)(const BasisData&, const RestrictionData&, const double*, double*, cudaStream_t);

struct MassPlan {
  int device = 0;
  int dim = 0, P = 0, Q = 0, num_comp = 0, comp_run = 0, qf = 0, scatter_mode = 0;
  int num_elem = 0, l_size = 0, es = 0, nq = 0;
  int64_t comp_stride = 0;
  int tile_e = 0;
  int64_t n_tiles = 0;
  // B[Q-1-q][P-1-p] = B[q][p] to rounding (symmetric nodes and points): the
  // even-odd contractions (eo_fwd / eo_bwd) apply
  bool centro_symmetric = false;
  BasisData basis;
  std::shared_ptr<RestrictionData> r;
  DevBuf<int> offs_t;
  DevBuf<double> qd_t;
  DevBuf<double> evec;    // deterministic mode: element contributions
  DevBuf<double> hu, hv;  // staging for the host-memory apply
  std::unique_ptr<HostPipeline> pipe;
  int host_chunks = 0;  // host-memory apply: 0 default, 1 unpipelined, n >= 2 about n chunks
  // The tile range the apply launchers cover: every tile, or span_tiles
  // tiles from span_first (an element chunk of the host-memory apply; atomic
  // scatter only, where the element index serves only the bounds check).
  int64_t span_first = 0, span_tiles = -1;
  const int* offs() const { return offs_t.get() + span_first * es * tile_e; }
  const double* qd() const { return qd_t.get() + span_first * int64_t(nq) * tile_e; }
  int64_t tiles() const { return span_tiles < 0 ? n_tiles : span_tiles; }
  int elems() const {
    return span_tiles < 0 ? num_elem : int(std::min<int64_t>(span_tiles * tile_e, num_elem - span_first * tile_e));
  }
  DevBuf<int> status;     // device status word (bit 0: a bounded wait ran out)
  ApplyLauncher launch = nullptr;       // the kernel in use
  ApplyLauncher launch_simple = nullptr;
  ApplyLauncher launch_pipe = nullptr;  // nullptr where the pipelined kernel does not apply
  ApplyLauncher launch_x2 = nullptr;    // two elements per thread (dim 3)
  ApplyLauncher launch_pf = nullptr;    // persistent, prefetching (dim 3)
  ApplyLauncher launch_occ = nullptr;   // one-tile CTAs, register-capped for occupancy (dim 3)
  ApplyLauncher launch_nw = nullptr;    // half-tile CTAs (4 elements), for high order (dim 3)
  ApplyLauncher launch_el = nullptr;    // one element per thread, no shared memory (dim 3, P = 2)
  int variant = FEM_B200_KERNEL_AUTO;
  // solver state (solver.cu), allocated by the first solve
  DevBuf<double> diag, dinv;              // assembled diagonal and its inverse
  DevBuf<double> cg_r, cg_p, cg_s, cg_w;  // FP64 Krylov vectors (cg_r, cg_w: outer residual, M u)
  DevBuf<double> part;                    // per-CTA partial sums of the grid reductions
  DevBuf<CgScalars> cg_st;                // device-resident solver scalars
  PinnedBuf<CgScalars> cg_host;           // their host copy
  CgScalars* cg_host_ext = nullptr;       // or a page-locked copy owned by the caller (a server slot)
  DevBuf<float> qd_t32, dinv32, evec32;   // FP32 copies (inner solves, FP32 applies)
  DevBuf<__nv_bfloat16> qd_t16;           // BF16 qdata (BF16-storage applies)
  DevBuf<float> f_r, f_p, f_s, f_w, f_x;  // FP32 Krylov vectors (f_w, f_x: also the BF16 solve's)
  DevBuf<__nv_bfloat16> h_r, h_p, h_s;    // BF16 Krylov vectors
  DevBuf<int> tc_ticket;                  // tile counter of the tensor-core apply (zeroed before each launch)
};

template <int P, int Q>
Mat1D<P, Q> make_mat(const BasisData& b) {
  Mat1D<P, Q> m;
  std::memcpy(m.B, b.interp.data(), sizeof(m.B));
  std::memcpy(m.G, b.grad.data(), sizeof(m.G));
  std::memcpy(m.W, b.q_weight.data(), sizeof(m.W));
  fill_eo(m);
  return m;
}

constexpr int kMaxSmemPerCta = 227 * 1024;

// SMs x resident CTAs per SM of `kernel` on the current device (occupancy
// calculator), cached per (kernel, device, threads, shared memory).
inline int resident_ctas(const void* kernel, int threads, int smem) {
  struct Key {
    const void* k;
    int dev, threads, smem;
    bool operator<(const Key& o) const {
      return std::tie(k, dev, threads, smem) < std::tie(o.k, o.dev, o.threads, o.smem);
    }
  };
  static std::mutex mu;
  static std::map<Key, int> cache;
  const Key key{kernel, current_device(), threads, smem};
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  int sms = 0, blocks = 0;
  FEM_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, key.dev));
  FEM_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, threads, smem));
  const int g = sms * std::max(blocks, 1);
  std::lock_guard<std::mutex> lock(mu);
  cache[key] = g;
  return g;
}

// Opt a kernel into more than 48 KB of dynamic shared memory, once per device
// (the attribute belongs to the device context).
template <class K>
void set_smem(K kernel, int bytes, std::atomic<uint64_t>& done) {
  if (bytes <= 48 * 1024) return;
  const int dev = current_device();
  const uint64_t bit = uint64_t(1) << (dev & 63);
  if (done.load() & bit) return;
  FEM_CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  done.fetch_or(bit);
}

// Defined in device.cu.
void check_status(MassPlan& p, cudaStream_t s = nullptr);
void mass_apply_impl(MassPlan& p, const double* u, double* v, bool zero, cudaStream_t s);
// The host-memory apply with its copies pipelined against the element chunks
// (host_apply.cu); host_pipeline_applies says whether the plan qualifies
// (atomic scatter, at least two chunks, not set to unpipelined).
// Synchronous: returns with v_host written.
bool host_pipeline_applies(const MassPlan& p);
void mass_apply_host_pipelined(MassPlan& p, const double* u_host, double* v_host, cudaStream_t s);
std::string shape_str(int dim, int P, int Q);
// A fused apply and build kernel exist for (dim, P, Q).
bool device_path_supported(int dim, int P, int Q);
// An offset restriction over device offsets `offs` (its copy is taken);
// host_offsets (the same values) are needed for the deterministic scatter's
// transpose map, else may be null.  Work in `s`, synchronised before return.
std::shared_ptr<RestrictionData> make_offset_restriction(int num_elem, int elem_size, int num_comp, int comp_stride,
                                                         int l_size, const int* offs, const int* host_offsets,
                                                         int scatter_mode, cudaStream_t s);
// qdata = det(J) w from coordinates x (the fused build kernel), in `s`.
void mass_build_impl(const BasisData& b, const RestrictionData& r, const double* x, double* qdata, cudaStream_t s);
// A mass plan (tiled offsets and qdata) in `s`, synchronised before return.
std::unique_ptr<MassPlan> make_mass_plan(const std::shared_ptr<RestrictionData>& r, const BasisData& b,
                                         const double* qdata, int qf, cudaStream_t s);

// Defined in basis.cu: the fused dim-3 interp / grad applies (E-vector <->
// Q-vector, no scratch); false where no fused kernel exists for the shape.
bool basis3d_fused_apply(const BasisData& b, int num_elem, bool transpose, bool grad, const double* u, double* v,
                         cudaStream_t s);

// Defined in solver.cu.
struct SolveStats {
  int iterations = 0, refinements = 0;
  double rel_residual = 0.0;
};
SolveStats mass_solve_impl(MassPlan& p, const double* f, double* u, double rtol, int max_iter, int precision,
                           cudaStream_t s);

}  // namespace fem_b200

// The C ABI's opaque handles.
struct fem_b200_restriction_s {
  std::shared_ptr<fem_b200::RestrictionData> d;
};
struct fem_b200_basis_s {
  std::unique_ptr<fem_b200::BasisDev> d;
};
struct fem_b200_mass_s {
  std::unique_ptr<fem_b200::MassPlan> d;
};
