// Batched mass apply over many independent meshes of uneven size and order
// (sm_100a): v_i = M_i u_i for every operator of the batch, replayed as ONE
// captured CUDA graph.
//
// The meshes are grouped into classes of equal (dim, P, Q, components, basis);
// each class is one kernel over a device table of (mesh, tile) pairs, with
// the per-mesh pointers and sizes in a device descriptor table, so the
// per-tile work is the single-mesh kernels' tile functions (mass3d_tile,
// mass2d_tile, mass1d_element) unchanged.  The graph holds one kernel that
// zeroes every v_i, then the class kernels on parallel branches (classes
// write disjoint outputs).  Rebinding the u_i / v_i pointers rewrites the
// descriptor table and keeps the graph.  Each class's schedule -- one CTA
// per tile, or a persistent grid of resident CTAs -- is chosen by timing
// both (fem_b200_batch_autotune).
//
// The reference applies one operator at a time (src/operator.cpp:148-182);
// the batch is the same operator over many meshes with no counterpart there.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>
#include <type_traits>

#include "plan.hpp"

namespace fem_b200 {

// One mesh of a batch, read by the device.
template <class T>
struct BatchMesh {
  const int* offs;  // the plan's tiled offsets
  const T* qd;      // its tiled qdata in T
  const T* u;
  T* v;
  int64_t l_size;
  int64_t comp_stride;
  int num_elem, comp_run;
};

template <class T>
__global__ void batch_zero_kernel(const BatchMesh<T>* __restrict__ meshes) {
  const BatchMesh<T> mm = meshes[blockIdx.y];
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < mm.l_size; i += int64_t(gridDim.x) * blockDim.x)
    mm.v[i] = T(0);
}

__global__ void batch_to_float_kernel(int64_t n, const double* __restrict__ in, float* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = float(in[i]);
}

// Tiles g = blockIdx.x, +gridDim.x, ... of a class; tiles[g] = (mesh, tile).
// FP64 classes of P >= 7 read the 1D matrix from a shared copy (SharedB), as
// the single-mesh one-tile kernels do: the parameter form holds all P*Q
// entries in registers and keeps one resident CTA.
template <int P, class T>
constexpr bool batch_shared_matrix() {
  return P >= 7 && sizeof(T) == 8;
}

// Runs body(m) with m the matrix parameter or (SB) a CTA-wide shared copy.
template <bool SB, int P, int Q, class T, class F>
__device__ __forceinline__ void with_interp(const Mat1D<P, Q, T>& mp, F&& body) {
  if constexpr (SB) {
    __shared__ T b_s[P * Q];
    for (int i = threadIdx.x; i < P * Q; i += blockDim.x) b_s[i] = mp.B[i];
    __syncthreads();
    body(SharedB<T>{b_s});
  } else {
    body(mp);
  }
}

// EO: the even-odd contractions (eo_fwd / eo_bwd; centro-symmetric B); SB:
// the 1D matrix from a shared copy (the high-order fallback without EO).
template <int P, int Q, int MINB, class T, int NCB, bool EO = false, bool SB = batch_shared_matrix<P, T>() && !EO>
__global__ void __launch_bounds__(Mass3D<P, Q>::NT, MINB)
    mass3d_batch_kernel(const __grid_constant__ Mat1D<P, Q, T> m, const BatchMesh<T>* __restrict__ meshes,
                        const int2* __restrict__ tiles, int64_t n_tiles) {
  using L = Mass3D<P, Q>;
  extern __shared__ __align__(16) unsigned char smem_bytes[];
  T* sa = reinterpret_cast<T*>(smem_bytes);
  T* sb = sa + NCB * L::SA;
  double dsum = 0.0;
  with_interp<SB>(m, [&](const auto& mat) {
    for (int64_t g = blockIdx.x; g < n_tiles; g += gridDim.x) {
      const int2 tm = tiles[g];
      const BatchMesh<T> mm = meshes[tm.x];
      mass3d_tile<P, Q, T, ApplyPlain, NCB, T, std::decay_t<decltype(mat)>, EO>(
          mat, sa, sb, mm.offs, mm.qd, mm.u, mm.v, nullptr, mm.num_elem, mm.comp_run, mm.comp_stride, ApplyPlain{},
          tm.y, dsum);
    }
  });
}

template <int P, int Q, class T>
__global__ void __launch_bounds__(Mass2D<P, Q>::NT)
    mass2d_batch_kernel(const __grid_constant__ Mat1D<P, Q, T> m, const BatchMesh<T>* __restrict__ meshes,
                        const int2* __restrict__ tiles, int64_t n_tiles) {
  using L = Mass2D<P, Q>;
  extern __shared__ __align__(16) unsigned char smem_bytes[];
  T* s1 = reinterpret_cast<T*>(smem_bytes);
  T* s3 = s1 + L::S1;
  double dsum = 0.0;
  with_interp<batch_shared_matrix<P, T>()>(m, [&](const auto& mat) {
    for (int64_t g = blockIdx.x; g < n_tiles; g += gridDim.x) {
      const int2 tm = tiles[g];
      const BatchMesh<T> mm = meshes[tm.x];
      mass2d_tile<P, Q, T, ApplyPlain>(mat, s1, s3, mm.offs, mm.qd, mm.u, mm.v, nullptr, mm.num_elem, mm.comp_run,
                                       mm.comp_stride, ApplyPlain{}, tm.y, dsum);
    }
  });
}

template <int P, int Q, class T>
__global__ void __launch_bounds__(128)
    mass1d_batch_kernel(const __grid_constant__ Mat1D<P, Q, T> m, const BatchMesh<T>* __restrict__ meshes,
                        const int2* __restrict__ tiles, int64_t n_tiles) {
  double dsum = 0.0;
  for (int64_t g = blockIdx.x; g < n_tiles; g += gridDim.x) {
    const int2 tm = tiles[g];
    const BatchMesh<T> mm = meshes[tm.x];
    const int64_t eg = int64_t(tm.y) * 128 + threadIdx.x;
    if (eg < mm.num_elem)
      mass1d_element<P, Q, T, ApplyPlain>(m, mm.offs, mm.qd, mm.u, mm.v, nullptr, mm.num_elem, mm.comp_run,
                                          mm.comp_stride, ApplyPlain{}, tm.y, int(threadIdx.x), eg, dsum);
  }
}

// ---------------------------------------------------------------------------
// One persistent launch for the whole batch.  Work items come from a ticket:
// first the zeroing of every v_i in chunks, then, class by class (heaviest
// first), groups of tiles of one mesh.  The block has kPersistBD threads and
// runs K = kPersistBD / NT tiles of a class at once in thread groups of the
// class's tile width NT (a P = 2 3D tile needs 72 threads, a P = 6 one 392),
// each group with its own slice of shared memory; threads beyond K * NT only
// join the barriers.  The shapes compiled in are those of uneven mesh
// batches: dim 2 and 3, P = 2..6, Q = P + 1, one basis a P (the Lagrange
// basis on GLL nodes at Gauss points; the 1D matrices travel in the kernel
// parameter).  Compute items wait (bounded) until every zeroing item is
// done -- once a block, the counter is then known complete; zeroing items
// come first in ticket order and wait on nothing, so the wait ends.
// ---------------------------------------------------------------------------
constexpr int kPersistBD = 416;          // 13 warps: the 3D P = 6 tile (392 threads), rounded up
constexpr int kPersistZeroChunk = 1 << 16;  // entries of v a zeroing item

template <class T>
struct PersistMats {
  Mat1D<2, 3, T> p2;
  Mat1D<3, 4, T> p3;
  Mat1D<4, 5, T> p4;
  Mat1D<5, 6, T> p5;
  Mat1D<6, 7, T> p6;
};

template <int P, class T>
__device__ __forceinline__ const Mat1D<P, P + 1, T>& persist_mat(const PersistMats<T>& m) {
  if constexpr (P == 2) return m.p2;
  else if constexpr (P == 3) return m.p3;
  else if constexpr (P == 4) return m.p4;
  else if constexpr (P == 5) return m.p5;
  else return m.p6;
}

// the even-odd contractions where the class kernels use them (centro-symmetric
// bases only: the plan checks)
template <int P, class T>
constexpr bool persist_even_odd() {
  return sizeof(T) == 8 ? (P == 4 || P == 6) : P == 6;
}

template <int D, int P>
struct PersistShape {
  static constexpr int Q = P + 1;
  static constexpr int NT = D == 3 ? Mass3D<P, Q>::NT : Mass2D<P, Q>::NT;
  static constexpr int K = kPersistBD / NT;  // tiles a block runs at once
  template <class T>
  static constexpr int smem() {
    return D == 3 ? (Mass3D<P, Q>::SA + Mass3D<P, Q>::SB) * int(sizeof(T)) : (Mass2D<P, Q>::S1 + Mass2D<P, Q>::S3) * int(sizeof(T));
  }
  static constexpr int slot = (D - 2) * 5 + (P - 2);  // the class id in the work items
};

template <class T>
constexpr int persist_smem() {
  int m = 0;
#define FEM_PERSIST_MAX(D, P) m = cmax(m, PersistShape<D, P>::K * PersistShape<D, P>::template smem<T>());
  FEM_PERSIST_MAX(2, 2) FEM_PERSIST_MAX(2, 3) FEM_PERSIST_MAX(2, 4) FEM_PERSIST_MAX(2, 5) FEM_PERSIST_MAX(2, 6)
  FEM_PERSIST_MAX(3, 2) FEM_PERSIST_MAX(3, 3) FEM_PERSIST_MAX(3, 4) FEM_PERSIST_MAX(3, 5) FEM_PERSIST_MAX(3, 6)
#undef FEM_PERSIST_MAX
  return m;
}

// Up to K tiles (tile0 ..) of one mesh, one a thread group.
template <int D, int P, class T>
__device__ __forceinline__ void persist_tiles(const PersistMats<T>& mats, const BatchMesh<T>& mm, int tile0,
                                              int count, unsigned char* smem) {
  using S = PersistShape<D, P>;
  constexpr int Q = S::Q;
  const int g = int(threadIdx.x) / S::NT;
  const bool in_group = g < min(S::K, count);
  const int t = in_group ? int(threadIdx.x) % S::NT : S::NT;
  T* base = reinterpret_cast<T*>(smem + (in_group ? g : 0) * S::template smem<T>());
  double dsum = 0.0;
  const int64_t tile = tile0 + (in_group ? g : 0);
  if constexpr (D == 3) {
    using L = Mass3D<P, Q>;
    mass3d_tile<P, Q, T, ApplyPlain, 1, T, Mat1D<P, Q, T>, persist_even_odd<P, T>(), true>(
        persist_mat<P>(mats), base, base + L::SA, mm.offs, mm.qd, mm.u, mm.v, nullptr, mm.num_elem, mm.comp_run,
        mm.comp_stride, ApplyPlain{}, tile, dsum, t);
  } else {
    using L = Mass2D<P, Q>;
    mass2d_tile<P, Q, T, ApplyPlain, T, Mat1D<P, Q, T>, false, true>(persist_mat<P>(mats), base, base + L::S1, mm.offs,
                                                               mm.qd, mm.u, mm.v, nullptr, mm.num_elem, mm.comp_run,
                                                               mm.comp_stride, ApplyPlain{}, tile, dsum, t);
  }
}

// items[i] = {class slot (-1: zero a chunk of v), mesh, first tile (or chunk), tile count};
// ctl[0] the ticket, ctl[1] zeroing items done (both zeroed before the launch)
template <class T, int MINB>
__global__ void __launch_bounds__(kPersistBD, MINB)
    batch_persistent_kernel(const __grid_constant__ PersistMats<T> mats, const BatchMesh<T>* __restrict__ meshes,
                            const int4* __restrict__ items, int n_items, int n_zero_items, int* __restrict__ ctl,
                            int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_bytes[];
  __shared__ int s_item;
  bool ready = false;  // every thread alike: the zeroing is known complete
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(ctl, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n_items) break;
    const int4 w = items[it];
    const BatchMesh<T> mm = meshes[w.y];
    if (w.x < 0) {
      const int64_t a = int64_t(w.z) * kPersistZeroChunk;
      const int64_t b = min(mm.l_size, a + kPersistZeroChunk);
      for (int64_t i = a + threadIdx.x; i < b; i += blockDim.x) mm.v[i] = T(0);
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(ctl + 1, 1);
      }
      continue;
    }
    if (!ready) {
      if (threadIdx.x == 0) {
        int spins = 0;
        while (true) {
          int done;
          asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(done) : "l"(ctl + 1) : "memory");
          if (done >= n_zero_items) break;
          if (++spins > (1 << 22)) {
            atomicOr(status, 8);
            break;
          }
          __nanosleep(100);
        }
      }
      __syncthreads();
      ready = true;
    }
    switch (w.x) {
      case PersistShape<2, 2>::slot: persist_tiles<2, 2, T>(mats, mm, w.z, w.w, smem_bytes); break;
      case PersistShape<2, 3>::slot: persist_tiles<2, 3, T>(mats, mm, w.z, w.w, smem_bytes); break;
      case PersistShape<2, 4>::slot: persist_tiles<2, 4, T>(mats, mm, w.z, w.w, smem_bytes); break;
      case PersistShape<2, 5>::slot: persist_tiles<2, 5, T>(mats, mm, w.z, w.w, smem_bytes); break;
      case PersistShape<2, 6>::slot: persist_tiles<2, 6, T>(mats, mm, w.z, w.w, smem_bytes); break;
      case PersistShape<3, 2>::slot: persist_tiles<3, 2, T>(mats, mm, w.z, w.w, smem_bytes); break;
      case PersistShape<3, 3>::slot: persist_tiles<3, 3, T>(mats, mm, w.z, w.w, smem_bytes); break;
      case PersistShape<3, 4>::slot: persist_tiles<3, 4, T>(mats, mm, w.z, w.w, smem_bytes); break;
      case PersistShape<3, 5>::slot: persist_tiles<3, 5, T>(mats, mm, w.z, w.w, smem_bytes); break;
      default: persist_tiles<3, 6, T>(mats, mm, w.z, w.w, smem_bytes); break;
    }
    __syncthreads();  // the groups' shared memory and s_item are reused by the next item
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
template <int P, int Q, class T>
Mat1D<P, Q, T> batch_mat(const BasisData& b) {
  Mat1D<P, Q, T> m;
  for (int i = 0; i < Q * P; ++i) m.B[i] = T(b.interp[i]), m.G[i] = T(b.grad[i]);
  for (int i = 0; i < Q; ++i) m.W[i] = T(b.q_weight[i]);
  fill_eo(m);
  return m;
}

struct BatchClass;
// Launch a class's kernel with `grid` CTAs (0: the occupancy-limited
// persistent grid); returns the grid used.
using ClassLauncher = unsigned (*)(const BatchClass&, const void* meshes, unsigned grid, cudaStream_t);

struct BatchClass {
  int dim = 0, P = 0, Q = 0, comp_run = 0, ncb = 1;
  bool centro_symmetric = false;  // the members' B (one per class): even-odd contractions apply
  BasisData basis;
  std::vector<int> members;  // indices into the batch
  DevBuf<int2> tiles;
  int64_t n_tiles = 0;
  int64_t dofs = 0;        // sum of l_size (all components)
  int schedule = 0;        // 0: one CTA per tile, 1: persistent
  ClassLauncher launch = nullptr;
};

constexpr int kBatchMaxStreams = 4;

// Resident CTAs per SM a 3D batch kernel asks for (a register cap): up to 4
// for P <= 5 (3 with three components batched), 2 for P = 6, 1 above, and
// no more than leave 56 registers a thread (72 with three components, 80 at
// P = 6).
constexpr int batch_min_blocks(int P, int threads, int ncb, bool shared_matrix = false) {
  const int cap = P > 7 ? 1 : P == 7 ? (shared_matrix ? 2 : 1) : P == 6 ? 2 : ncb == 3 ? 3 : 4;
  const int regs = P == 7 ? 64 : P == 6 ? 80 : ncb == 3 ? 72 : 56;
  for (int b = cap; b > 1; --b)
    if (b * threads <= 2048 && 65536 / (b * threads) >= regs) return b;
  return P >= 8 ? 1 : 0;  // as the single-mesh kernel (plain_min_blocks)
}

// FP64 classes from P = 4 (512 uneven meshes: P = 5 added 69.6 -> 70.5
// GDoF/s), FP32 classes from P = 6 with one component at a time (FP32: 113.0
// -> 116.4 GDoF/s) and at P = 4, 5 also with components batched (116.4 ->
// 119.0 GDoF/s), use the even-odd contractions when their B is
// centro-symmetric (as the single-mesh one-tile kernel at those orders; P = 7
// with two resident CTAs); otherwise the direct form, from a shared copy of
// the matrix at P >= 7.
template <int P, int Q, class T, int NCB,
          bool EO = sizeof(T) == 8 ? P >= 4 && NCB == 1 : (P == 4 || P == 5 || (P >= 6 && NCB == 1))>
unsigned launch_batch3(const BatchClass& c, const void* meshes, unsigned grid, cudaStream_t s) {
  if constexpr (EO) {
    if (!c.centro_symmetric) return launch_batch3<P, Q, T, NCB, false>(c, meshes, grid, s);
  }
  using L = Mass3D<P, Q>;
  constexpr int smem = NCB * (L::SA + L::SB) * int(sizeof(T));
  constexpr bool sb = batch_shared_matrix<P, T>() && !EO;
  constexpr int minb = batch_min_blocks(P, L::NT, NCB, sb || (EO && P == 7));
  const auto kern = mass3d_batch_kernel<P, Q, minb, T, NCB, EO, sb>;
  static std::atomic<uint64_t> smem_set{0};
  set_smem(kern, smem, smem_set);
  if (grid == 0) grid = unsigned(std::min<int64_t>(resident_ctas(reinterpret_cast<const void*>(kern), L::NT, smem),
                                                   c.n_tiles));
  kern<<<grid, L::NT, smem, s>>>(batch_mat<P, Q, T>(c.basis), static_cast<const BatchMesh<T>*>(meshes),
                                 c.tiles.get(), c.n_tiles);
  FEM_LAUNCH_CHECK();
  return grid;
}

template <int P, int Q, class T>
unsigned launch_batch2(const BatchClass& c, const void* meshes, unsigned grid, cudaStream_t s) {
  using L = Mass2D<P, Q>;
  constexpr int smem = (L::S1 + L::S3) * int(sizeof(T));
  const auto kern = mass2d_batch_kernel<P, Q, T>;
  static std::atomic<uint64_t> smem_set{0};
  set_smem(kern, smem, smem_set);
  if (grid == 0) grid = unsigned(std::min<int64_t>(resident_ctas(reinterpret_cast<const void*>(kern), L::NT, smem),
                                                   c.n_tiles));
  kern<<<grid, L::NT, smem, s>>>(batch_mat<P, Q, T>(c.basis), static_cast<const BatchMesh<T>*>(meshes),
                                 c.tiles.get(), c.n_tiles);
  FEM_LAUNCH_CHECK();
  return grid;
}

template <int P, int Q, class T>
unsigned launch_batch1(const BatchClass& c, const void* meshes, unsigned grid, cudaStream_t s) {
  const auto kern = mass1d_batch_kernel<P, Q, T>;
  if (grid == 0)
    grid = unsigned(std::min<int64_t>(resident_ctas(reinterpret_cast<const void*>(kern), 128, 0), c.n_tiles));
  kern<<<grid, 128, 0, s>>>(batch_mat<P, Q, T>(c.basis), static_cast<const BatchMesh<T>*>(meshes), c.tiles.get(),
                            c.n_tiles);
  FEM_LAUNCH_CHECK();
  return grid;
}

constexpr int kBatchMinP = 2, kBatchMaxP = 8, kBatchQSpan = 3;

// [dim-1][P][Q-P][ncb 1 or 3][T: 0 double, 1 float]
struct BatchDispatch {
  ClassLauncher fn[3][kBatchMaxP + 1][kBatchQSpan][2][2] = {};
};

template <int P, int DQ>
struct BatchTable {
  static void fill(BatchDispatch& d) {
    constexpr int Q = P + DQ;
    d.fn[0][P][DQ][0][0] = launch_batch1<P, Q, double>;
    d.fn[0][P][DQ][0][1] = launch_batch1<P, Q, float>;
    d.fn[1][P][DQ][0][0] = launch_batch2<P, Q, double>;
    d.fn[1][P][DQ][0][1] = launch_batch2<P, Q, float>;
    d.fn[2][P][DQ][0][0] = launch_batch3<P, Q, double, 1>;
    d.fn[2][P][DQ][0][1] = launch_batch3<P, Q, float, 1>;
    constexpr int smem8 = (Mass3D<P, Q>::SA + Mass3D<P, Q>::SB) * 8;
    if constexpr (P <= 5 && 3 * smem8 <= kMaxSmemPerCta) d.fn[2][P][DQ][1][0] = launch_batch3<P, Q, double, 3>;
    if constexpr (P <= 5 && 3 * smem8 / 2 <= kMaxSmemPerCta) d.fn[2][P][DQ][1][1] = launch_batch3<P, Q, float, 3>;
    if constexpr (DQ + 1 < kBatchQSpan)
      BatchTable<P, DQ + 1>::fill(d);
    else if constexpr (P + 1 <= kBatchMaxP)
      BatchTable<P + 1, 0>::fill(d);
  }
};

const BatchDispatch& batch_dispatch() {
  static const BatchDispatch d = [] {
    BatchDispatch t;
    BatchTable<kBatchMinP, 0>::fill(t);
    return t;
  }();
  return d;
}

struct BatchPlan {
  int device = 0;
  int precision = 0;  // FEM_B200_PRECISION_FP64 / _FP32
  std::vector<MassPlan*> ops;
  std::vector<BatchClass> classes;
  DevBuf<unsigned char> meshes;  // BatchMesh<T>[ops.size()]
  std::vector<unsigned char> meshes_host;
  bool bound = false;
  int64_t max_l_size = 0;
  cudaStream_t streams[kBatchMaxStreams] = {};
  cudaEvent_t fork = nullptr, join[kBatchMaxStreams] = {};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_kernels = 0;
  int branches = 1;  // parallel graph branches (classes run concurrently), autotuned
  // the one-launch form (batch_persistent_kernel): eligible when every class
  // is one of its compiled shapes; mode FEM_B200_BATCH_AUTO runs it unless
  // the autotuner found the per-class graph faster
  bool persist_ok = false;
  int mode = FEM_B200_BATCH_AUTO;
  bool persist_chosen = true;  // AUTO's choice
  DevBuf<int4> items;
  int n_items = 0, n_zero_items = 0;
  DevBuf<int> ctl;     // ticket, zeroing items done
  DevBuf<int> status;  // bit 3: the wait for the zeroing ran out
  std::vector<unsigned char> persist_mats;  // PersistMats<T>, the kernel parameter
  bool persistent() const {
    return persist_ok && (mode == FEM_B200_BATCH_PERSISTENT || (mode == FEM_B200_BATCH_AUTO && persist_chosen));
  }

  ~BatchPlan() {
    int prev = -1;
    (void)cudaGetDevice(&prev);
    (void)cudaSetDevice(device);
    if (exec) (void)cudaGraphExecDestroy(exec);
    if (graph) (void)cudaGraphDestroy(graph);
    for (auto& st : streams)
      if (st) (void)cudaStreamDestroy(st);
    for (auto& ev : join)
      if (ev) (void)cudaEventDestroy(ev);
    if (fork) (void)cudaEventDestroy(fork);
    if (prev >= 0) (void)cudaSetDevice(prev);
  }
  size_t mesh_bytes() const { return precision == FEM_B200_PRECISION_FP32 ? sizeof(BatchMesh<float>) : sizeof(BatchMesh<double>); }
  void drop_graph() {
    if (exec) (void)cudaGraphExecDestroy(exec);
    if (graph) (void)cudaGraphDestroy(graph);
    exec = nullptr, graph = nullptr;
  }
};

template <class T, int MINB>
void launch_persistent(BatchPlan& b, cudaStream_t s) {
  constexpr int smem = persist_smem<T>();
  const auto kern = batch_persistent_kernel<T, MINB>;
  static std::atomic<uint64_t> smem_set{0};
  set_smem(kern, smem, smem_set);
  const int grid = int(std::min<int64_t>(b.n_items, resident_ctas(reinterpret_cast<const void*>(kern), kPersistBD, smem)));
  FEM_CUDA_CHECK(cudaMemsetAsync(b.ctl.get(), 0, 2 * sizeof(int), s));
  PersistMats<T> m;
  std::memcpy(&m, b.persist_mats.data(), sizeof(m));
  kern<<<grid, kPersistBD, smem, s>>>(m, reinterpret_cast<const BatchMesh<T>*>(b.meshes.get()), b.items.get(),
                                      b.n_items, b.n_zero_items, b.ctl.get(), b.status.get());
  FEM_LAUNCH_CHECK();
}

template <class T>
void fill_persist_mats(BatchPlan& b) {
  PersistMats<T> m;
  std::memset(&m, 0, sizeof(m));
  for (const BatchClass& c : b.classes) {
    switch (c.P) {
      case 2: m.p2 = batch_mat<2, 3, T>(c.basis); break;
      case 3: m.p3 = batch_mat<3, 4, T>(c.basis); break;
      case 4: m.p4 = batch_mat<4, 5, T>(c.basis); break;
      case 5: m.p5 = batch_mat<5, 6, T>(c.basis); break;
      default: m.p6 = batch_mat<6, 7, T>(c.basis); break;
    }
  }
  b.persist_mats.resize(sizeof(m));
  std::memcpy(b.persist_mats.data(), &m, sizeof(m));
}

// The work items of the one-launch form, when every class fits it: dim 2 or
// 3, P = 2..6, Q = P + 1, one 1D matrix a P, centro-symmetric where the
// kernel takes the even-odd contractions.
void plan_persistent(BatchPlan& b) {
  const bool fp32 = b.precision == FEM_B200_PRECISION_FP32;
  std::map<int, std::vector<double>> interp_of_p;
  for (const BatchClass& c : b.classes) {
    if (c.dim < 2 || c.P < 2 || c.P > 6 || c.Q != c.P + 1) return;
    const bool eo = fp32 ? c.P == 6 : (c.P == 4 || c.P == 6);
    if (eo && !c.centro_symmetric) return;
    auto it = interp_of_p.find(c.P);
    if (it != interp_of_p.end() && it->second != c.basis.interp) return;
    interp_of_p[c.P] = c.basis.interp;
  }
  std::vector<int4> items;
  for (size_t i = 0; i < b.ops.size(); ++i) {
    const int64_t chunks = (b.ops[i]->l_size + kPersistZeroChunk - 1) / kPersistZeroChunk;
    for (int64_t k = 0; k < chunks; ++k) items.push_back(make_int4(-1, int(i), int(k), 0));
  }
  const int n_zero = int(items.size());
  for (const BatchClass& c : b.classes) {  // heaviest first (the classes' order)
    const int slot = (c.dim - 2) * 5 + (c.P - 2);
    const int nt = c.dim == 3 ? 8 * c.Q * c.Q : 32 * c.Q;
    const int k = kPersistBD / nt;
    for (int i : c.members)
      for (int64_t t = 0; t < b.ops[size_t(i)]->n_tiles; t += k)
        items.push_back(make_int4(slot, i, int(t), int(std::min<int64_t>(k, b.ops[size_t(i)]->n_tiles - t))));
  }
  if (items.size() >= size_t(INT32_MAX)) return;
  b.items.alloc(items.size());
  FEM_CUDA_CHECK(cudaMemcpy(b.items.get(), items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice));
  b.n_items = int(items.size());
  b.n_zero_items = n_zero;
  b.ctl.alloc(2);
  b.status.alloc(1);
  FEM_CUDA_CHECK(cudaMemset(b.status.get(), 0, sizeof(int)));
  if (fp32)
    fill_persist_mats<float>(b);
  else
    fill_persist_mats<double>(b);
  b.persist_ok = true;
}

// Every v_i zeroed, then every class (the heaviest first, round-robin over
// `branches` streams, which fork from and join into s0); or the one launch.
void enqueue_batch(BatchPlan& b, cudaStream_t s0, int branches) {
  if (b.persistent()) {
    if (b.precision == FEM_B200_PRECISION_FP32)
      launch_persistent<float, 3>(b, s0);
    else
      launch_persistent<double, 2>(b, s0);
    return;
  }
  const unsigned ops = unsigned(b.ops.size());
  const unsigned zx = unsigned(std::max<int64_t>(1, std::min<int64_t>(64, (b.max_l_size + 2047) / 2048)));
  if (b.precision == FEM_B200_PRECISION_FP32)
    batch_zero_kernel<float><<<dim3(zx, ops), 256, 0, s0>>>(reinterpret_cast<const BatchMesh<float>*>(b.meshes.get()));
  else
    batch_zero_kernel<double><<<dim3(zx, ops), 256, 0, s0>>>(
        reinterpret_cast<const BatchMesh<double>*>(b.meshes.get()));
  FEM_LAUNCH_CHECK();
  const int ns = int(std::min<size_t>(size_t(std::max(branches, 1)),
                                       std::min<size_t>(kBatchMaxStreams, b.classes.size())));
  if (ns > 1) {
    FEM_CUDA_CHECK(cudaEventRecord(b.fork, s0));
    for (int i = 1; i < ns; ++i) FEM_CUDA_CHECK(cudaStreamWaitEvent(b.streams[i], b.fork, 0));
  }
  for (size_t c = 0; c < b.classes.size(); ++c) {
    const BatchClass& cl = b.classes[c];
    cudaStream_t s = (ns > 1 && c % ns) ? b.streams[c % ns] : s0;
    cl.launch(cl, b.meshes.get(), cl.schedule == 0 ? unsigned(cl.n_tiles) : 0u, s);
  }
  if (ns > 1) {
    for (int i = 1; i < ns; ++i) {
      FEM_CUDA_CHECK(cudaEventRecord(b.join[i], b.streams[i]));
      FEM_CUDA_CHECK(cudaStreamWaitEvent(s0, b.join[i], 0));
    }
  }
}

void capture_batch(BatchPlan& b) {
  b.drop_graph();
  cudaStream_t s0 = b.streams[0];
  FEM_CUDA_CHECK(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
  try {
    enqueue_batch(b, s0, b.branches);
  } catch (...) {
    cudaGraph_t g = nullptr;
    (void)cudaStreamEndCapture(s0, &g);
    if (g) (void)cudaGraphDestroy(g);
    throw;
  }
  FEM_CUDA_CHECK(cudaStreamEndCapture(s0, &b.graph));
  FEM_CUDA_CHECK(cudaGraphInstantiate(&b.exec, b.graph, 0));
  b.graph_kernels = b.persistent() ? 1 : 1 + int(b.classes.size());
}

// Two timing events (RAII); time(s, f) = device ms of what f enqueues in s.
struct EventPair {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  EventPair() {
    FEM_CUDA_CHECK(cudaEventCreate(&e0));
    FEM_CUDA_CHECK(cudaEventCreate(&e1));
  }
  ~EventPair() {
    (void)cudaEventDestroy(e0);
    (void)cudaEventDestroy(e1);
  }
  template <class F>
  float time(cudaStream_t s, F&& f) {
    FEM_CUDA_CHECK(cudaEventRecord(e0, s));
    f();
    FEM_CUDA_CHECK(cudaEventRecord(e1, s));
    FEM_CUDA_CHECK(cudaEventSynchronize(e1));
    float ms = 0.0f;
    FEM_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
    return ms;
  }
};

template <class T>
void write_descriptors(BatchPlan& b, const void* const* u, void* const* v) {
  b.meshes_host.resize(b.ops.size() * sizeof(BatchMesh<T>));
  auto* d = reinterpret_cast<BatchMesh<T>*>(b.meshes_host.data());
  for (size_t i = 0; i < b.ops.size(); ++i) {
    const MassPlan& p = *b.ops[i];
    d[i].offs = p.offs_t.get();
    d[i].qd = std::is_same<T, float>::value ? reinterpret_cast<const T*>(p.qd_t32.get())
                                             : reinterpret_cast<const T*>(p.qd_t.get());
    d[i].u = static_cast<const T*>(u[i]);
    d[i].v = static_cast<T*>(v[i]);
    d[i].l_size = p.l_size;
    d[i].comp_stride = p.comp_stride;
    d[i].num_elem = p.num_elem;
    d[i].comp_run = p.comp_run;
  }
}

}  // namespace fem_b200

struct fem_b200_batch_s {
  std::unique_ptr<fem_b200::BatchPlan> d;
};

using namespace fem_b200;

extern "C" {

int fem_b200_batch_create(const fem_b200_mass* ops, int num_ops, int precision, fem_b200_batch* out) {
  return guarded([&] {
    require(out != nullptr, "batch create: NULL output handle");
    require(ops != nullptr && num_ops >= 1 && num_ops <= 65535, "batch create: 1..65535 operators");
    require(precision == FEM_B200_PRECISION_FP64 || precision == FEM_B200_PRECISION_FP32,
            "batch create: unknown precision");
    auto b = std::make_unique<BatchPlan>();
    b->precision = precision;
    for (int i = 0; i < num_ops; ++i) {
      require(ops[i] && ops[i]->d, "batch create: NULL operator");
      b->ops.push_back(ops[i]->d.get());
    }
    b->device = b->ops[0]->device;
    DeviceGuard g(b->device);
    const BatchDispatch& disp = batch_dispatch();
    const int ti = precision == FEM_B200_PRECISION_FP32 ? 1 : 0;
    std::map<std::tuple<int, int, int, int, std::vector<double>>, int> index;
    for (int i = 0; i < num_ops; ++i) {
      MassPlan& p = *b->ops[i];
      require(p.device == b->device, "batch create: every operator must be on the same device");
      if (p.scatter_mode != FEM_B200_SCATTER_ATOMIC)
        throw unsupported_error("batch create: operators with the deterministic scatter are not batched");
      b->max_l_size = std::max<int64_t>(b->max_l_size, p.l_size);
      if (ti == 1 && p.qd_t32.size() != p.qd_t.size()) {
        p.qd_t32.alloc(p.qd_t.size());
        batch_to_float_kernel<<<grid_for(int64_t(p.qd_t.size()), 256), 256>>>(int64_t(p.qd_t.size()), p.qd_t.get(),
                                                                             p.qd_t32.get());
        FEM_LAUNCH_CHECK();
      }
      const auto key = std::make_tuple(p.dim, p.P, p.Q, p.comp_run, p.basis.interp);
      auto it = index.find(key);
      if (it == index.end()) {
        BatchClass c;
        c.dim = p.dim, c.P = p.P, c.Q = p.Q, c.comp_run = p.comp_run;
        c.basis = p.basis;
        c.centro_symmetric = p.centro_symmetric;
        // three components through each phase together in FP32 only: for FP64
        // classes one at a time measured faster (512 uneven meshes, one graph:
        // 58.0 -> 62.1 GDoF/s), as for the FP64 Krylov apply
        c.ncb = (ti == 1 && p.dim == 3 && p.comp_run == 3 && p.P <= 5 && disp.fn[2][p.P][p.Q - p.P][1][ti]) ? 3 : 1;
        c.launch = disp.fn[p.dim - 1][p.P][p.Q - p.P][c.ncb == 3 ? 1 : 0][ti];
        require(c.launch != nullptr, "batch create: no batched kernel for this shape");
        it = index.emplace(key, int(b->classes.size())).first;
        b->classes.push_back(std::move(c));
      }
      BatchClass& c = b->classes[it->second];
      c.members.push_back(i);
      c.n_tiles += p.n_tiles;
      c.dofs += p.l_size;
    }
    for (BatchClass& c : b->classes) {
      require(c.n_tiles < (int64_t(1) << 31), "batch create: a class has more than 2^31 tiles");
      std::vector<int2> t;
      t.reserve(size_t(c.n_tiles));
      for (int i : c.members)
        for (int64_t k = 0; k < b->ops[i]->n_tiles; ++k) t.push_back(make_int2(i, int(k)));
      c.tiles.alloc(t.size());
      FEM_CUDA_CHECK(cudaMemcpy(c.tiles.get(), t.data(), t.size() * sizeof(int2), cudaMemcpyHostToDevice));
    }
    // heaviest classes first, so the parallel branches start with the long kernels
    std::stable_sort(b->classes.begin(), b->classes.end(),
                     [](const BatchClass& x, const BatchClass& y) { return x.n_tiles > y.n_tiles; });
    plan_persistent(*b);
    b->meshes.alloc(b->ops.size() * b->mesh_bytes());
    for (auto& st : b->streams) FEM_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    FEM_CUDA_CHECK(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    for (auto& ev : b->join) FEM_CUDA_CHECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    FEM_CUDA_CHECK(cudaDeviceSynchronize());
    *out = new fem_b200_batch_s{std::move(b)};
  });
}

int fem_b200_batch_bind(fem_b200_batch batch, const void* const* u, void* const* v, void* stream) {
  return guarded([&] {
    require(batch && batch->d, "batch bind: NULL handle");
    BatchPlan& b = *batch->d;
    require(u && v, "batch bind: NULL pointer arrays");
    for (size_t i = 0; i < b.ops.size(); ++i) require(u[i] && v[i], "batch bind: NULL vector pointer");
    DeviceGuard g(b.device);
    if (b.precision == FEM_B200_PRECISION_FP32)
      write_descriptors<float>(b, u, v);
    else
      write_descriptors<double>(b, u, v);
    // pageable source: the copy is staged before the call returns
    FEM_CUDA_CHECK(cudaMemcpyAsync(b.meshes.get(), b.meshes_host.data(), b.meshes_host.size(), cudaMemcpyHostToDevice,
                                   as_stream(stream)));
    b.bound = true;
  });
}

int fem_b200_batch_apply(fem_b200_batch batch, int use_graph, void* stream) {
  return guarded([&] {
    require(batch && batch->d, "batch apply: NULL handle");
    BatchPlan& b = *batch->d;
    require(b.bound, "batch apply: bind the vectors first (fem_b200_batch_bind)");
    DeviceGuard g(b.device);
    cudaStream_t s = as_stream(stream);
    if (!use_graph) {
      enqueue_batch(b, s, 1);
      return;
    }
    if (!b.exec) {
      // the kernels' attributes are set by one direct pass before the capture
      enqueue_batch(b, s, 1);
      FEM_CUDA_CHECK(cudaStreamSynchronize(s));
      capture_batch(b);
    }
    FEM_CUDA_CHECK(cudaGraphLaunch(b.exec, s));
  });
}

int fem_b200_batch_autotune(fem_b200_batch batch, int reps, void* stream) {
  return guarded([&] {
    require(batch && batch->d, "batch autotune: NULL handle");
    BatchPlan& b = *batch->d;
    require(b.bound, "batch autotune: bind the vectors first (fem_b200_batch_bind)");
    require(reps >= 1, "batch autotune: reps must be positive");
    DeviceGuard g(b.device);
    cudaStream_t s = as_stream(stream);
    enqueue_batch(b, s, 1);  // v zeroed; attributes set
    EventPair ev;
    // each class: one CTA per tile, or the persistent grid
    for (BatchClass& c : b.classes) {
      float best = 0.0f;
      for (int sched = 0; sched < 2; ++sched) {
        const unsigned grid = sched == 0 ? unsigned(c.n_tiles) : 0u;
        c.launch(c, b.meshes.get(), grid, s);  // warm-up
        const float ms = ev.time(s, [&] {
          for (int r = 0; r < reps; ++r) c.launch(c, b.meshes.get(), grid, s);
        });
        if (sched == 0 || ms < best) best = ms, c.schedule = sched;
      }
    }
    // then the graph's parallel branches: classes that run concurrently
    // contend for HBM, which pays off in some precisions only
    float best = 0.0f;
    int best_branches = 1;
    b.persist_chosen = false;  // the per-class graph first
    for (int nb : {1, 2, 4}) {
      b.branches = nb;
      capture_batch(b);
      FEM_CUDA_CHECK(cudaGraphLaunch(b.exec, s));  // warm-up
      const float ms = ev.time(s, [&] {
        for (int r = 0; r < reps; ++r) FEM_CUDA_CHECK(cudaGraphLaunch(b.exec, s));
      });
      if (nb == 1 || ms < best) best = ms, best_branches = nb;
    }
    b.branches = best_branches;
    // then the one persistent launch against that graph of class kernels
    if (b.persist_ok && b.mode == FEM_B200_BATCH_AUTO) {
      b.persist_chosen = true;
      capture_batch(b);
      FEM_CUDA_CHECK(cudaGraphLaunch(b.exec, s));  // warm-up
      const float ms = ev.time(s, [&] {
        for (int r = 0; r < reps; ++r) FEM_CUDA_CHECK(cudaGraphLaunch(b.exec, s));
      });
      b.persist_chosen = ms <= best;
    }
    capture_batch(b);
    FEM_CUDA_CHECK(cudaGraphLaunch(b.exec, s));  // leaves v_i = M_i u_i
    FEM_CUDA_CHECK(cudaStreamSynchronize(s));
  });
}

int fem_b200_batch_set_mode(fem_b200_batch batch, int mode) {
  return guarded([&] {
    require(batch && batch->d, "batch mode: NULL handle");
    BatchPlan& b = *batch->d;
    require(mode == FEM_B200_BATCH_AUTO || mode == FEM_B200_BATCH_CLASSES || mode == FEM_B200_BATCH_PERSISTENT,
            "batch mode: unknown mode");
    if (mode == FEM_B200_BATCH_PERSISTENT && !b.persist_ok)
      throw unsupported_error("batch mode: the one-launch kernel covers dim 2 and 3, P = 2..6, Q = P + 1 with one "
                              "basis a P; this batch has other classes");
    DeviceGuard g(b.device);
    b.mode = mode;
    b.drop_graph();
  });
}

int fem_b200_batch_check(fem_b200_batch batch, void* stream) {
  return guarded([&] {
    require(batch && batch->d, "batch check: NULL handle");
    BatchPlan& b = *batch->d;
    DeviceGuard g(b.device);
    FEM_CUDA_CHECK(cudaStreamSynchronize(as_stream(stream)));
    if (!b.status.get()) return;
    int st = 0;
    FEM_CUDA_CHECK(cudaMemcpy(&st, b.status.get(), sizeof(int), cudaMemcpyDeviceToHost));
    if (st) {
      FEM_CUDA_CHECK(cudaMemset(b.status.get(), 0, sizeof(int)));
      throw cuda_error("batch apply: a bounded wait in the persistent kernel ran out (status " + std::to_string(st) +
                       "); the result is not valid");
    }
  });
}

int fem_b200_batch_info(fem_b200_batch batch, int* num_classes, int64_t* total_tiles, int64_t* total_dofs,
                        int* graph_kernels, int* persistent_classes, int* graph_branches) {
  return guarded([&] {
    require(batch && batch->d, "batch info: NULL handle");
    const BatchPlan& b = *batch->d;
    int64_t tiles = 0, dofs = 0;
    int pers = 0;
    for (const BatchClass& c : b.classes) tiles += c.n_tiles, dofs += c.dofs, pers += c.schedule;
    if (num_classes) *num_classes = int(b.classes.size());
    if (total_tiles) *total_tiles = tiles;
    if (total_dofs) *total_dofs = dofs;
    if (graph_kernels) *graph_kernels = b.persistent() ? 1 : 1 + int(b.classes.size());
    if (persistent_classes) *persistent_classes = pers;
    if (graph_branches) *graph_branches = b.branches;
  });
}

int fem_b200_batch_destroy(fem_b200_batch batch) {
  return guarded([&] { delete batch; });
}

}  // extern "C"
