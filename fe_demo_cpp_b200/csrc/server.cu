// Served mass solves (sm_100a): a request loop over a fixed device-memory
// budget.
//
// A request is one mass solve M u = f with its own mesh: a box generated on
// the device (the benchmark stream), or offsets / coordinates / f from the
// host.  The server admits requests in arrival order as soon as a slot is
// free AND the request's device-memory estimate fits the budget.  An admitted
// request keeps its mesh, qdata and Krylov vectors resident until it
// finishes.  Every slot has its own worker thread and CUDA stream, and its
// set-up (mesh, qdata build, plan), its solve (mass_solve_impl: FP32 PCG in
// FP64 refinement, or FP64 PCG) and its teardown are stream-ordered, with
// buffers from a stream-ordered memory pool.  So requests that arrive while
// others run are admitted as slots and memory free up, and their kernels
// overlap on the device.  A request's result does not depend on what else
// runs: with the deterministic scatter it is the same to the last bit alone
// and in any mix.
//
// The reference has no server; this is the serving loop around its
// operator_apply (src/operator.cpp:148-182) that the solver wraps.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "plan.hpp"

namespace fem_b200 {

// ---------------------------------------------------------------------------
// device box meshes: lexicographic elements and local nodes, interior
// vertices moved by U[-f h, f h] per coordinate, nodes at the GLL points of
// the trilinear (bilinear) map of the moved corners -- the construction of
// the benchmark meshes, with a counter-based random stream
// ---------------------------------------------------------------------------
// splitmix64 (Steele, Lea, Flood 2014) of (seed, i) -> [0, 1)
__device__ __forceinline__ double hash_uniform(uint64_t seed, uint64_t i) {
  uint64_t z = seed * 0x9E3779B97F4A7C15ull + i * 0xD1B54A32D192ED03ull + 0x632BE59BD9B4E019ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return double(z >> 11) * (1.0 / 9007199254740992.0);
}

struct BoxSpec {
  int dim, P;
  int n[3];        // elements per direction
  int64_t nn[3];   // nodes per direction
  double perturb;
  uint64_t seed;
  double s[8];     // GLL points mapped to [0, 1]
};

__global__ void box_offsets_kernel(BoxSpec b, int64_t total, int* __restrict__ offs) {
  const int P = b.P, es = b.dim == 3 ? P * P * P : P * P;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t e = t / es;
    const int i = int(t - e * es);
    const int64_t ex = e % b.n[0], ey = (e / b.n[0]) % b.n[1], ez = b.dim == 3 ? e / (int64_t(b.n[0]) * b.n[1]) : 0;
    const int ix = i % P, iy = (i / P) % P, iz = b.dim == 3 ? i / (P * P) : 0;
    const int64_t gx = ex * (P - 1) + ix, gy = ey * (P - 1) + iy, gz = ez * (P - 1) + iz;
    offs[t] = int(gx + b.nn[0] * (gy + b.nn[1] * gz));
  }
}

// Coordinate c of vertex (vx, vy, vz).
__device__ __forceinline__ double box_vertex(const BoxSpec& b, int64_t v[3], int c) {
  const double h = 1.0 / b.n[c];
  bool interior = true;
  for (int d = 0; d < b.dim; ++d) interior = interior && v[d] > 0 && v[d] < b.n[d];
  double x = v[c] * h;
  if (interior) {
    const int64_t vid = v[0] + (b.n[0] + 1) * (v[1] + int64_t(b.n[1] + 1) * v[2]);
    x += (2.0 * hash_uniform(b.seed, uint64_t(vid) * 3 + c) - 1.0) * (b.perturb * h);
  }
  return x;
}

// x[c * num_nodes + node], c < dim
__global__ void box_coords_kernel(BoxSpec b, int64_t num_nodes, double* __restrict__ x) {
  const int P = b.P;
  for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < num_nodes;
       g += int64_t(gridDim.x) * blockDim.x) {
    int64_t gi[3] = {g % b.nn[0], (g / b.nn[0]) % b.nn[1], b.dim == 3 ? g / (b.nn[0] * b.nn[1]) : 0};
    int64_t el[3];
    double s[3];
    for (int d = 0; d < 3; ++d) {
      if (d < b.dim) {
        el[d] = min(gi[d] / (P - 1), int64_t(b.n[d] - 1));
        s[d] = b.s[gi[d] - el[d] * (P - 1)];
      } else {
        el[d] = 0, s[d] = 0.0;
      }
    }
    const int corners = 1 << b.dim;
    for (int c = 0; c < b.dim; ++c) {
      double acc = 0.0;
      for (int k = 0; k < corners; ++k) {
        int64_t v[3];
        double w = 1.0;
        for (int d = 0; d < 3; ++d) {
          const int bit = d < b.dim ? (k >> d) & 1 : 0;
          v[d] = el[d] + bit;
          if (d < b.dim) w *= bit ? s[d] : 1.0 - s[d];
        }
        acc += w * box_vertex(b, v, c);
      }
      x[c * num_nodes + g] = acc;
    }
  }
}

// f = U[-1, 1] from (seed, i)
__global__ void uniform_rhs_kernel(int64_t n, uint64_t seed, double* __restrict__ f) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    f[i] = 2.0 * hash_uniform(seed ^ 0x5DEECE66Dull, uint64_t(i)) - 1.0;
}

// ---------------------------------------------------------------------------
// the server
// ---------------------------------------------------------------------------
struct ServerReq {
  int64_t id = 0;
  fem_b200_request r{};
  int num_elem = 0;
  int64_t num_nodes = 0;
  int64_t need = 0;  // device bytes reserved from the budget
  double t_submit = 0, t_start = 0, t_end = 0;
  bool done = false;
  int status = FEM_B200_SUCCESS;
  std::string message;
  SolveStats stats;
};

// Device bytes a request holds at most (its set-up temporaries included).
int64_t request_bytes(int dim, int P, int Q, int nc, int64_t ne, int64_t N, int scatter_mode) {
  const int64_t es = ipow(P, dim), nq = ipow(Q, dim), n = nc * N;
  const int64_t tile_e = dim == 3 ? 8 : 32;
  const int64_t ne_pad = ((ne + 2 * tile_e - 1) / (2 * tile_e)) * 2 * tile_e;
  int64_t b = 0;
  b += 4 * ne * es * 3 + 4 * ne_pad * es;          // generated, coordinate, field and tiled offsets
  b += 8 * dim * N;                                // coordinates
  b += 8 * ne * nq + 8 * ne_pad * nq + 4 * ne_pad * nq;  // built, tiled and FP32 qdata
  b += 16 * n;                                     // f, u
  b += 48 * n + 24 * n;                            // FP64 and FP32 Krylov vectors and diagonals
  b += 16 * std::max<int64_t>(ne_pad / tile_e, 148 * 8) + 4096;
  if (scatter_mode == FEM_B200_SCATTER_DETERMINISTIC) b += 12 * nc * es * ne + 4 * (2 * n + ne * es);
  return b + b / 32 + (4 << 20);                   // pool granularity
}

class SolveServer {
 public:
  SolveServer(int slots, int64_t budget) : budget_(budget), t0_(std::chrono::steady_clock::now()) {
    device_ = current_device();
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device_;
    FEM_CUDA_CHECK(cudaMemPoolCreate(&pool_, &props));
    uint64_t keep = UINT64_MAX;  // freed blocks stay in the pool for the next request
    FEM_CUDA_CHECK(cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep));
    // A block freed on one slot's stream is not handed to another slot before
    // that free has executed: with the pool's default, the allocator may reuse
    // it by making the new request's stream wait for the other request's
    // pending work, which serialises the slots (FP64 stream at 2000 req/s,
    // after 200 requests: 36-94 solves/s and 220 ms mean service, against 157
    // solves/s and 50 ms on a fresh pool).
    int no = 0;
    FEM_CUDA_CHECK(cudaMemPoolSetAttribute(pool_, cudaMemPoolReuseAllowInternalDependencies, &no));
    streams_.resize(slots), host_st_.resize(slots);
    for (int i = 0; i < slots; ++i) {
      FEM_CUDA_CHECK(cudaStreamCreateWithFlags(&streams_[i], cudaStreamNonBlocking));
      FEM_CUDA_CHECK(cudaMallocHost(&host_st_[i], sizeof(CgScalars)));
    }
    for (int i = 0; i < slots; ++i) threads_.emplace_back([this, i] { worker(i); });
  }

  ~SolveServer() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_work_.notify_all();
    for (auto& t : threads_) t.join();
    int prev = -1;
    (void)cudaGetDevice(&prev);
    (void)cudaSetDevice(device_);
    for (auto s : streams_) (void)cudaStreamDestroy(s);
    for (auto h : host_st_) (void)cudaFreeHost(h);
    (void)cudaMemPoolDestroy(pool_);
    if (prev >= 0) (void)cudaSetDevice(prev);
  }

  int64_t submit(const fem_b200_request& r) {
    auto q = std::make_shared<ServerReq>();
    q->r = r;
    validate(*q);
    q->need = request_bytes(r.dim, r.P, r.Q, r.num_comp, q->num_elem, q->num_nodes, r.scatter_mode);
    if (q->need > budget_)
      throw arg_error("server submit: the request needs " + std::to_string(q->need) +
                      " device bytes, more than the whole budget of " + std::to_string(budget_));
    {
      std::lock_guard<std::mutex> lk(mu_);
      require(!stop_, "server submit: the server is shutting down");
      q->id = next_id_++;
      q->t_submit = now();
      pending_.push_back(q);
      all_[q->id] = q;
      ++submitted_;
    }
    cv_work_.notify_all();
    return q->id;
  }

  // true when done (result filled, request forgotten); false on timeout
  bool wait(int64_t id, double timeout_s, fem_b200_result* out) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = all_.find(id);
    require(it != all_.end(), "server wait: unknown request id (or already collected)");
    std::shared_ptr<ServerReq> q = it->second;
    auto ready = [&] { return q->done; };
    if (timeout_s < 0)
      cv_done_.wait(lk, ready);
    else if (!cv_done_.wait_for(lk, std::chrono::duration<double>(timeout_s), ready))
      return false;
    fill(*q, out);
    all_.erase(id);
    return true;
  }

  void stats(int64_t* submitted, int64_t* completed, int* running, int64_t* pending, int64_t* in_use,
             int64_t* peak) {
    std::lock_guard<std::mutex> lk(mu_);
    if (submitted) *submitted = submitted_;
    if (completed) *completed = completed_;
    if (running) *running = running_;
    if (pending) *pending = int64_t(pending_.size());
    if (in_use) *in_use = used_;
    if (peak) *peak = peak_;
  }

 private:
  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
  }

  void validate(ServerReq& q) {
    const fem_b200_request& r = q.r;
    require(r.kind == FEM_B200_REQUEST_BOX || r.kind == FEM_B200_REQUEST_MESH, "server submit: unknown request kind");
    require(r.dim == 2 || r.dim == 3, "server submit: dim must be 2 or 3");
    require(r.num_comp >= 1 && r.num_comp <= 3, "server submit: num_comp must be 1..3");
    require(r.rtol > 0.0 && r.rtol < 1.0, "server submit: rtol must be in (0, 1)");
    require(r.max_iter >= 1, "server submit: max_iter must be positive");
    require(r.precision == FEM_B200_SOLVE_FP64 || r.precision == FEM_B200_SOLVE_FP32_IR ||
                r.precision == FEM_B200_SOLVE_BF16_IR,
            "server submit: unknown precision");
    require(r.scatter_mode == FEM_B200_SCATTER_ATOMIC || r.scatter_mode == FEM_B200_SCATTER_DETERMINISTIC,
            "server submit: unknown scatter mode");
    if (!device_path_supported(r.dim, r.P, r.Q))
      throw unsupported_error("server submit: no device kernels for " + shape_str(r.dim, r.P, r.Q));
    if (r.kind == FEM_B200_REQUEST_BOX) {
      int64_t ne = 1, nn = 1;
      for (int d = 0; d < r.dim; ++d) {
        require(r.shape[d] >= 1, "server submit: box shape must be positive");
        ne *= r.shape[d];
        nn *= int64_t(r.shape[d]) * (r.P - 1) + 1;
      }
      require(ne * ipow(r.P, r.dim) < (int64_t(1) << 31) && nn * std::max(r.num_comp, r.dim) < (int64_t(1) << 31),
              "server submit: box too large for int32 offsets");
      require(r.perturb >= 0.0 && r.perturb < 0.5, "server submit: perturb must be in [0, 0.5)");
      q.num_elem = int(ne), q.num_nodes = nn;
    } else {
      require(r.num_elem >= 1 && r.num_nodes >= 1 && r.offsets && r.coords && r.f,
              "server submit: a mesh request needs offsets, coords and f");
      require(int64_t(r.num_nodes) * std::max(r.num_comp, r.dim) < (int64_t(1) << 31),
              "server submit: mesh too large for int32 offsets");
      check_offset(r.num_elem, int(ipow(r.P, r.dim)), 1, r.num_nodes, r.num_nodes, r.offsets,
                   int64_t(r.num_elem) * ipow(r.P, r.dim));
      q.num_elem = r.num_elem, q.num_nodes = r.num_nodes;
    }
  }

  void fill(const ServerReq& q, fem_b200_result* out) const {
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    out->status = q.status;
    out->iterations = q.stats.iterations;
    out->refinements = q.stats.refinements;
    out->rel_residual = q.stats.rel_residual;
    out->t_submit = q.t_submit, out->t_start = q.t_start, out->t_end = q.t_end;
    out->dofs = q.r.num_comp * q.num_nodes;
    out->device_bytes = q.need;
    std::strncpy(out->message, q.message.c_str(), sizeof(out->message) - 1);
  }

  void worker(int slot) {
    for (;;) {
      std::shared_ptr<ServerReq> q;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_work_.wait(lk, [&] {
          return (stop_ && pending_.empty()) || (!pending_.empty() && used_ + pending_.front()->need <= budget_);
        });
        if (pending_.empty()) return;  // stopping, nothing left
        q = pending_.front();
        pending_.pop_front();
        used_ += q->need;
        peak_ = std::max(peak_, used_);
        ++running_;
        q->t_start = now();
      }
      try {
        run(*q, slot);
      } catch (const arg_error& e) {
        q->status = FEM_B200_ERROR_ARGUMENT, q->message = e.what();
      } catch (const unsupported_error& e) {
        q->status = FEM_B200_ERROR_UNSUPPORTED, q->message = e.what();
      } catch (const std::exception& e) {
        q->status = FEM_B200_ERROR_CUDA, q->message = e.what();
      }
      {
        std::lock_guard<std::mutex> lk(mu_);
        used_ -= q->need;
        --running_;
        ++completed_;
        q->t_end = now();
        q->done = true;
      }
      cv_done_.notify_all();
      cv_work_.notify_all();
    }
  }

  void run(ServerReq& q, int slot) {
    const fem_b200_request& r = q.r;
    DeviceGuard g(device_);
    cudaStream_t s = streams_[slot];
    const int dim = r.dim, P = r.P, Q = r.Q, nc = r.num_comp;
    const int es = int(ipow(P, dim));
    const int64_t ne = q.num_elem, N = q.num_nodes, n = nc * N, n_t = ne * es;
    {
      AllocScope scope(s, pool_);
      DevBuf<int> offs(static_cast<size_t>(n_t));
      DevBuf<double> x(static_cast<size_t>(dim * N)), f(static_cast<size_t>(n)), u(static_cast<size_t>(n));
      std::vector<int> host_offs;
      const int* host_offs_ptr = nullptr;
      if (r.kind == FEM_B200_REQUEST_BOX) {
        BoxSpec b{};
        b.dim = dim, b.P = P, b.perturb = r.perturb, b.seed = r.seed;
        for (int d = 0; d < 3; ++d) {
          b.n[d] = d < dim ? r.shape[d] : 1;
          b.nn[d] = d < dim ? int64_t(r.shape[d]) * (P - 1) + 1 : 1;
        }
        std::vector<double> xg(static_cast<size_t>(P)), wg(static_cast<size_t>(P));
        gauss_lobatto(P, xg.data(), wg.data());
        for (int i = 0; i < P; ++i) b.s[i] = 0.5 * (xg[i] + 1.0);
        box_offsets_kernel<<<grid_for(n_t, 256), 256, 0, s>>>(b, n_t, offs.get());
        FEM_LAUNCH_CHECK();
        box_coords_kernel<<<grid_for(N, 256), 256, 0, s>>>(b, N, x.get());
        FEM_LAUNCH_CHECK();
        uniform_rhs_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, r.seed, f.get());
        FEM_LAUNCH_CHECK();
        if (r.scatter_mode == FEM_B200_SCATTER_DETERMINISTIC) {
          host_offs.resize(size_t(n_t));
          FEM_CUDA_CHECK(cudaMemcpyAsync(host_offs.data(), offs.get(), n_t * sizeof(int), cudaMemcpyDeviceToHost, s));
          FEM_CUDA_CHECK(cudaStreamSynchronize(s));
          host_offs_ptr = host_offs.data();
        }
      } else {
        FEM_CUDA_CHECK(cudaMemcpyAsync(offs.get(), r.offsets, n_t * sizeof(int), cudaMemcpyHostToDevice, s));
        FEM_CUDA_CHECK(cudaMemcpyAsync(x.get(), r.coords, dim * N * sizeof(double), cudaMemcpyHostToDevice, s));
        FEM_CUDA_CHECK(cudaMemcpyAsync(f.get(), r.f, n * sizeof(double), cudaMemcpyHostToDevice, s));
        host_offs_ptr = r.offsets;
      }
      if (r.f_out)
        FEM_CUDA_CHECK(cudaMemcpyAsync(r.f_out, f.get(), n * sizeof(double), cudaMemcpyDeviceToHost, s));
      // qdata = det(J) w, then the plan (its own tiled copies)
      std::unique_ptr<MassPlan> plan;
      {
        auto rx = make_offset_restriction(int(ne), es, dim, int(N), int(dim * N), offs.get(), nullptr,
                                          FEM_B200_SCATTER_ATOMIC, s);
        auto ru = make_offset_restriction(int(ne), es, nc, int(N), int(n), offs.get(), host_offs_ptr,
                                          r.scatter_mode, s);
        DevBuf<double> qd(static_cast<size_t>(ne * ipow(Q, dim)));
        mass_build_impl(make_basis(dim, dim, P, Q, 0), *rx, x.get(), qd.get(), s);
        plan = make_mass_plan(ru, make_basis(dim, nc, P, Q, 0), qd.get(), FEM_B200_QF_APPLY_MASS_VECTOR, s);
      }
      offs = DevBuf<int>();
      x = DevBuf<double>();
      plan->cg_host_ext = host_st_[slot];
      q.stats = mass_solve_impl(*plan, f.get(), u.get(), r.rtol, r.max_iter, r.precision, s);
      if (r.u_out)
        FEM_CUDA_CHECK(cudaMemcpyAsync(r.u_out, u.get(), n * sizeof(double), cudaMemcpyDeviceToHost, s));
      plan.reset();
    }
    // the frees were queued in s: after this the memory is back in the pool
    FEM_CUDA_CHECK(cudaStreamSynchronize(s));
  }

  int device_ = 0;
  int64_t budget_;
  cudaMemPool_t pool_ = nullptr;
  std::vector<cudaStream_t> streams_;
  std::vector<CgScalars*> host_st_;
  std::vector<std::thread> threads_;
  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_;
  std::deque<std::shared_ptr<ServerReq>> pending_;
  std::unordered_map<int64_t, std::shared_ptr<ServerReq>> all_;
  int64_t used_ = 0, peak_ = 0, submitted_ = 0, completed_ = 0, next_id_ = 1;
  int running_ = 0;
  bool stop_ = false;
  std::chrono::steady_clock::time_point t0_;
};

}  // namespace fem_b200

struct fem_b200_server_s {
  std::unique_ptr<fem_b200::SolveServer> d;
};

using namespace fem_b200;

extern "C" {

int fem_b200_server_create(int slots, int64_t hbm_budget_bytes, fem_b200_server* out) {
  return guarded([&] {
    require(out != nullptr, "server create: NULL output handle");
    require(slots >= 1 && slots <= 64, "server create: slots must be 1..64");
    require(hbm_budget_bytes > 0, "server create: the budget must be positive");
    *out = new fem_b200_server_s{std::make_unique<SolveServer>(slots, hbm_budget_bytes)};
  });
}

int fem_b200_server_submit(fem_b200_server server, const fem_b200_request* req, int64_t* id) {
  return guarded([&] {
    require(server && server->d && req && id, "server submit: NULL argument");
    *id = server->d->submit(*req);
  });
}

int fem_b200_server_wait(fem_b200_server server, int64_t id, double timeout_s, fem_b200_result* result) {
  bool ready = false;
  const int rc = guarded([&] {
    require(server && server->d, "server wait: NULL handle");
    ready = server->d->wait(id, timeout_s, result);
  });
  if (rc != FEM_B200_SUCCESS) return rc;
  return ready ? FEM_B200_SUCCESS : FEM_B200_NOT_READY;
}

int fem_b200_server_stats(fem_b200_server server, int64_t* submitted, int64_t* completed, int* running,
                          int64_t* pending, int64_t* bytes_in_use, int64_t* bytes_peak) {
  return guarded([&] {
    require(server && server->d, "server stats: NULL handle");
    server->d->stats(submitted, completed, running, pending, bytes_in_use, bytes_peak);
  });
}

int fem_b200_server_destroy(fem_b200_server server) {
  return guarded([&] { delete server; });
}

}  // extern "C"
