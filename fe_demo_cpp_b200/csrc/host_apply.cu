// The host-memory mass apply (operator_apply on host vectors,
// src/operator.cpp:148-182), with its PCIe copies overlapped with the
// kernels and with each other.
//
// The plan's tiles are cut into element chunks.  For each chunk the node
// span [lo, hi] of its offsets is found once, on the device.  Then, per apply:
//   - a copy stream brings u in by increasing L-index, each chunk's span
//     as soon as the previous spans are in;
//   - the compute stream zeroes v, then applies each chunk (the operator's
//     own kernel over the chunk's tiles) once its span of u has arrived;
//   - a second copy stream takes v out: after chunk c, every L-index below
//     the smallest lo of the chunks still to come is final.
// On a mesh numbered so that later elements use later nodes (a box mesh, or
// any bandwidth-reducing order) the three overlap and the apply costs about
// one PCIe direction instead of both plus the kernel; on any other order it
// degenerates to copy-in, apply, copy-out.  Only the atomic scatter is
// pipelined (the deterministic one reduces over all elements at the end).
//
// Pageable host vectors: the DMA engines reach pageable memory only through
// the driver's own staging (about 13 GB/s a direction), and page-locking the
// caller's vectors per call costs more than the copy (42 ms to register a
// touched 0.5 GB).  So each pageable direction goes through a plan-owned
// ring of page-locked slots, filled or drained by a pool of host memcpy
// threads while the DMA engines move the other slots: u by this thread ahead
// of each chunk, v by a second thread behind each chunk.
//
// Components: with the blocked layout (comp_stride past the node span) each
// component's window is pipelined on its own; otherwise one window covers
// [lo, hi + (components - 1) * comp_stride].  L entries outside every window
// are read by no element: u there is not copied, and v there is zero.
#include <cuda_runtime.h>

#include <climits>
#include <condition_variable>
#include <cstdint>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "plan.hpp"

namespace fem_b200 {
namespace {

// Blocks (c, j): the smallest and largest offset of the elements in slice j
// of chunk c (tiled layout [tile][i][e], padding elements excluded), folded
// into lo[c] / hi[c] (set beforehand to INT_MAX-like 0x7f7f7f7f and -1).
constexpr int kSpanSlices = 64;

__global__ void chunk_span_kernel(const int* __restrict__ offs, int es, int tile_e, int num_elem, int64_t n_tiles,
                                  int64_t tiles_per_chunk, int* __restrict__ lo, int* __restrict__ hi) {
  __shared__ int s_lo, s_hi;
  if (threadIdx.x == 0) s_lo = INT_MAX, s_hi = -1;
  __syncthreads();
  const int64_t per_tile = int64_t(es) * tile_e;
  const int64_t c0 = int64_t(blockIdx.x) * tiles_per_chunk;
  const int64_t c1 = c0 + tiles_per_chunk < n_tiles ? c0 + tiles_per_chunk : n_tiles;
  const int64_t step = (c1 - c0 + gridDim.y - 1) / gridDim.y;
  const int64_t t0 = c0 + blockIdx.y * step;
  const int64_t t1 = t0 + step < c1 ? t0 + step : c1;
  int mn = INT_MAX, mx = -1;
  for (int64_t pos = t0 * per_tile + threadIdx.x; pos < t1 * per_tile; pos += blockDim.x) {
    const int64_t tile = pos / per_tile;
    const int el = int(pos % tile_e);
    if (tile * tile_e + el < num_elem) {
      const int o = offs[pos];
      mn = o < mn ? o : mn;
      mx = o > mx ? o : mx;
    }
  }
  atomicMin(&s_lo, mn);
  atomicMax(&s_hi, mx);
  __syncthreads();
  if (threadIdx.x == 0 && s_hi >= 0) {
    atomicMin(lo + blockIdx.x, s_lo);
    atomicMax(hi + blockIdx.x, s_hi);
  }
}

// Chunks: about 24, each at least 512 tiles (a wave of the apply kernel), an
// even number of tiles (the two-tiles-per-CTA variant reads whole pairs).
// On a B200 over PCIe 5 x16 the two directions run at 55 GB/s alone and
// 46.5 GB/s each together, and the kernels take under a tenth of the copy
// time.  The copy in of the first chunk and the copies out of the last run
// alone, while every chunk adds a fixed cost to both copy streams: a 0.5 GB
// u and v took 18.8 ms unchunked, 14.1 ms in 8 chunks, 13.0-13.2 ms in 16 to
// 32, 14.1 ms in 64 and 15.3 ms in 128 (chunks tapered towards both ends:
// within 2% of uniform).
constexpr int64_t kTargetChunks = 24, kMinChunkTiles = 512;

int target_chunks(const MassPlan& p) { return p.host_chunks > 1 ? p.host_chunks : int(kTargetChunks); }

HostPipeline& pipeline(MassPlan& p, cudaStream_t s) {
  const int target = target_chunks(p);
  if (p.pipe && p.pipe->target == target) return *p.pipe;
  p.pipe.reset();
  auto hp = std::make_unique<HostPipeline>();
  hp->target = target;
  int64_t tpc = std::max<int64_t>(kMinChunkTiles, (p.n_tiles + target - 1) / target);
  tpc += tpc & 1;
  const int64_t n_chunks = (p.n_tiles + tpc - 1) / tpc;
  hp->tiles_per_chunk = tpc;
  DevBuf<int> span(size_t(2 * n_chunks));
  FEM_CUDA_CHECK(cudaMemsetAsync(span.get(), 0x7f, size_t(n_chunks) * sizeof(int), s));              // lo
  FEM_CUDA_CHECK(cudaMemsetAsync(span.get() + n_chunks, 0xff, size_t(n_chunks) * sizeof(int), s));  // hi = -1
  chunk_span_kernel<<<dim3(unsigned(n_chunks), kSpanSlices), 256, 0, s>>>(
      p.offs_t.get(), p.es, p.tile_e, p.num_elem, p.n_tiles, tpc, span.get(), span.get() + n_chunks);
  FEM_LAUNCH_CHECK();
  std::vector<int> h(size_t(2 * n_chunks));
  FEM_CUDA_CHECK(cudaMemcpyAsync(h.data(), span.get(), h.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
  FEM_CUDA_CHECK(cudaStreamSynchronize(s));
  hp->lo.assign(h.begin(), h.begin() + n_chunks);
  hp->hi.assign(h.begin() + n_chunks, h.end());
  FEM_CUDA_CHECK(cudaStreamCreateWithFlags(&hp->h2d, cudaStreamNonBlocking));
  FEM_CUDA_CHECK(cudaStreamCreateWithFlags(&hp->d2h, cudaStreamNonBlocking));
  hp->ev.assign(size_t(2 + 2 * n_chunks), nullptr);
  for (cudaEvent_t& e : hp->ev) FEM_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  p.pipe = std::move(hp);
  return *p.pipe;
}

bool page_locked(const void* ptr) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Staging of pageable host vectors: a page-locked ring of kSlots slots of
// kSlotElems doubles (8 MB) per direction.  A slot is filled (or drained) by
// the memcpy pool while the DMA engines move the others.
constexpr int kSlots = 6;
constexpr int64_t kSlotElems = int64_t(1) << 20;

// The memcpy threads, one pool for the process (half the hardware threads,
// 2 to 8), shared by every plan's staging; made on first use.
CopyPool& copy_pool() {
  static CopyPool pool(int(std::min(8u, std::max(2u, std::thread::hardware_concurrency() / 2))));
  return pool;
}

void ensure_staging(HostPipeline& hp) {
  if (!hp.slot_ev.empty()) return;
  hp.ring_in.alloc(size_t(kSlots * kSlotElems));
  hp.ring_out.alloc(size_t(kSlots * kSlotElems));
  std::vector<cudaEvent_t> ev(size_t(2 * kSlots), nullptr);
  for (cudaEvent_t& e : ev) {
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      for (cudaEvent_t made : ev)
        if (made) (void)cudaEventDestroy(made);
      FEM_CUDA_CHECK(cudaGetLastError());
    }
  }
  hp.slot_ev = std::move(ev);
}

struct Copy {
  int chunk;  // -1: after v is zeroed, else after this chunk's apply
  int64_t first, count;
};

// The thread that copies v out into pageable memory, and its handshake: the
// highest chunk whose apply event is recorded (-1: v zeroed).  An apply that
// fails part-way aborts it, and it is joined however the apply ends.
struct Writer {
  std::mutex mu;
  std::condition_variable cv;
  int recorded = -2;
  bool abort = false;
  std::string error;
  std::thread th;
  ~Writer() {
    if (!th.joinable()) return;
    {
      std::lock_guard<std::mutex> lock(mu);
      abort = true;
    }
    cv.notify_one();
    th.join();
  }
};

// Resets the plan's tile span however the apply ends.
struct SpanReset {
  MassPlan& p;
  ~SpanReset() { p.span_first = 0, p.span_tiles = -1; }
};

}  // namespace

bool host_pipeline_applies(const MassPlan& p) {
  return p.scatter_mode == FEM_B200_SCATTER_ATOMIC && p.host_chunks != 1 && p.n_tiles >= 2 * kMinChunkTiles;
}

void mass_apply_host_pipelined(MassPlan& p, const double* u_host, double* v_host, cudaStream_t s) {
  HostPipeline& hp = pipeline(p, s);
  const int n_chunks = int(hp.lo.size());
  const int64_t l_size = p.l_size, cs = p.comp_stride;
  int64_t w_lo = INT64_MAX, w_hi = -1;
  for (int c = 0; c < n_chunks; ++c) w_lo = std::min(w_lo, hp.lo[c]), w_hi = std::max(w_hi, hp.hi[c]);
  // windows: per component (blocked layout) or one covering every component
  const bool blocked = p.comp_run > 1 && cs > w_hi - w_lo;
  const int n_win = blocked ? p.comp_run : 1;
  const int64_t w_step = blocked ? cs : 0;
  const int64_t ext = blocked ? 0 : int64_t(p.comp_run - 1) * cs;

  double* hu = p.hu.get();
  double* hv = p.hv.get();
  cudaEvent_t ev_start = hp.ev[0], ev_zero = hp.ev[1];
  FEM_CUDA_CHECK(cudaEventRecord(ev_start, s));
  FEM_CUDA_CHECK(cudaStreamWaitEvent(hp.h2d, ev_start, 0));
  FEM_CUDA_CHECK(cudaStreamWaitEvent(hp.d2h, ev_start, 0));
  FEM_CUDA_CHECK(cudaMemsetAsync(hv, 0, size_t(l_size) * sizeof(double), s));
  FEM_CUDA_CHECK(cudaEventRecord(ev_zero, s));

  // the copies out, in issue order: the L entries outside every window
  // (zero once v is zeroed), then per chunk the entries it finalises
  std::vector<Copy> out;
  {
    int64_t at = 0;
    for (int k = 0; k < n_win; ++k) {
      const int64_t a = w_lo + k * w_step, b = std::min(l_size, w_hi + ext + 1 + k * w_step);
      if (a > at) out.push_back({-1, at, a - at});
      at = std::max(at, b);
    }
    if (at < l_size) out.push_back({-1, at, l_size - at});
  }
  std::vector<int64_t> suffix_lo(size_t(n_chunks) + 1, w_hi + ext + 1);
  for (int c = n_chunks - 1; c >= 0; --c) suffix_lo[c] = std::min(suffix_lo[c + 1], hp.lo[c]);
  {
    std::vector<int64_t> done(size_t(n_win), w_lo);
    for (int c = 0; c < n_chunks; ++c)
      for (int k = 0; k < n_win; ++k) {
        const int64_t final_end = suffix_lo[c + 1];
        if (final_end > done[k]) {
          out.push_back({c, done[k] + k * w_step, final_end - done[k]});
          done[k] = final_end;
        }
      }
  }

  // Page-locked v: the copies out are issued from this thread, each after its
  // chunk's apply.  Pageable v: a second thread drains them through the
  // staging ring, each copy issued once this thread has recorded the event it
  // waits on (a wait on an event not yet recorded would not wait).
  // Pageable u: this thread fills the input ring ahead of each chunk.
  const bool u_locked = page_locked(u_host), v_locked = page_locked(v_host);
  if (!u_locked || !v_locked) ensure_staging(hp);
  if (!v_locked) {  // ring-sized pieces
    std::vector<Copy> split;
    for (const Copy& o : out)
      for (int64_t off = 0; off < o.count; off += kSlotElems)
        split.push_back({o.chunk, o.first + off, std::min(kSlotElems, o.count - off)});
    out.swap(split);
  }
  auto chunk_event = [&](int chunk) { return chunk < 0 ? ev_zero : hp.ev[size_t(3 + 2 * chunk)]; };
  size_t next_out = 0;
  Writer w;
  auto publish = [&](int c) {
    if (v_locked) {
      for (; next_out < out.size() && out[next_out].chunk <= c; ++next_out) {
        const Copy& o = out[next_out];
        FEM_CUDA_CHECK(cudaStreamWaitEvent(hp.d2h, chunk_event(o.chunk), 0));
        FEM_CUDA_CHECK(cudaMemcpyAsync(v_host + o.first, hv + o.first, size_t(o.count) * sizeof(double),
                                       cudaMemcpyDeviceToHost, hp.d2h));
      }
    } else {
      {
        std::lock_guard<std::mutex> lock(w.mu);
        w.recorded = c;
      }
      w.cv.notify_one();
    }
  };
  if (!v_locked) {
    const int dev = p.device;
    w.th = std::thread([&, dev] {
      try {
        FEM_CUDA_CHECK(cudaSetDevice(dev));
        auto recorded = [&](int chunk, bool block) {  // false: not yet (block = false) or aborted
          std::unique_lock<std::mutex> lock(w.mu);
          if (block) w.cv.wait(lock, [&] { return w.abort || w.recorded >= chunk; });
          return w.recorded >= chunk;
        };
        auto issue = [&](size_t k) {
          const Copy& o = out[k];
          double* slot = hp.ring_out.get() + int64_t(k % kSlots) * kSlotElems;
          FEM_CUDA_CHECK(cudaStreamWaitEvent(hp.d2h, chunk_event(o.chunk), 0));
          FEM_CUDA_CHECK(cudaMemcpyAsync(slot, hv + o.first, size_t(o.count) * sizeof(double),
                                         cudaMemcpyDeviceToHost, hp.d2h));
          FEM_CUDA_CHECK(cudaEventRecord(hp.slot_ev[size_t(kSlots) + k % kSlots], hp.d2h));
        };
        size_t issued = 0;
        for (size_t j = 0; j < out.size(); ++j) {
          for (; issued <= j; ++issued) {
            if (!recorded(out[issued].chunk, true)) return;  // aborted
            issue(issued);
          }
          // keep the ring's other slots in flight: piece k reuses the slot of
          // piece k - kSlots, whose copy to v_host is done (k < j + kSlots)
          for (; issued < out.size() && issued < j + kSlots && recorded(out[issued].chunk, false); ++issued)
            issue(issued);
          FEM_CUDA_CHECK(cudaEventSynchronize(hp.slot_ev[size_t(kSlots) + j % kSlots]));
          copy_pool().copy(v_host + out[j].first, hp.ring_out.get() + int64_t(j % kSlots) * kSlotElems,
                        size_t(out[j].count) * sizeof(double));
        }
      } catch (const std::exception& e) {
        w.error = e.what();
      }
    });
  }
  publish(-1);

  int64_t k_in = 0;  // ring pieces copied in so far (pageable u)
  auto copy_in = [&](int64_t first, int64_t count) {
    if (u_locked) {
      FEM_CUDA_CHECK(cudaMemcpyAsync(hu + first, u_host + first, size_t(count) * sizeof(double),
                                     cudaMemcpyHostToDevice, hp.h2d));
      return;
    }
    for (int64_t off = 0; off < count; off += kSlotElems, ++k_in) {
      const int64_t n = std::min(kSlotElems, count - off);
      const int slot = int(k_in % kSlots);
      cudaEvent_t e = hp.slot_ev[size_t(slot)];
      FEM_CUDA_CHECK(cudaEventSynchronize(e));  // the slot's previous copy is done (never recorded: at once)
      double* st = hp.ring_in.get() + int64_t(slot) * kSlotElems;
      copy_pool().copy(st, u_host + first + off, size_t(n) * sizeof(double));
      FEM_CUDA_CHECK(cudaMemcpyAsync(hu + first + off, st, size_t(n) * sizeof(double), cudaMemcpyHostToDevice,
                                     hp.h2d));
      FEM_CUDA_CHECK(cudaEventRecord(e, hp.h2d));
    }
  };

  SpanReset reset{p};
  std::vector<int64_t> in_done(size_t(n_win), w_lo);
  for (int c = 0; c < n_chunks; ++c) {
    for (int k = 0; k < n_win; ++k) {
      const int64_t end = hp.hi[c] + ext + 1;
      if (end > in_done[k]) {
        copy_in(in_done[k] + k * w_step, end - in_done[k]);
        in_done[k] = end;
      }
    }
    cudaEvent_t ev_in = hp.ev[size_t(2 + 2 * c)], ev_done = hp.ev[size_t(3 + 2 * c)];
    FEM_CUDA_CHECK(cudaEventRecord(ev_in, hp.h2d));
    FEM_CUDA_CHECK(cudaStreamWaitEvent(s, ev_in, 0));
    p.span_first = int64_t(c) * hp.tiles_per_chunk;
    p.span_tiles = std::min<int64_t>(hp.tiles_per_chunk, p.n_tiles - p.span_first);
    p.launch(p, hu, hv, nullptr, s);
    FEM_CUDA_CHECK(cudaEventRecord(ev_done, s));
    publish(c);
  }
  if (w.th.joinable()) w.th.join();
  FEM_CUDA_CHECK(cudaStreamSynchronize(hp.d2h));
  FEM_CUDA_CHECK(cudaStreamSynchronize(hp.h2d));
  FEM_CUDA_CHECK(cudaStreamSynchronize(s));
  if (!w.error.empty()) throw std::runtime_error(w.error);
}

}  // namespace fem_b200
