// One mesh over several ranks through the C ABI (fem_b200_shard_*): the
// set-up of a rank's part of a mesh partitioned in contiguous element ranges
// (the element-range partition of fe_demo_cpp_b200/shard.py), and the device
// halves of the interface exchange -- pack the values shared with each peer
// into one send buffer, and after the caller's transport (NCCL, MPI, a copy)
// add the peers' values into v in rank order, so that a shared value gets
// the same bits on every rank.  The reference is single-process
// (src/operator.cpp:148-182); this partitions its operator.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "common.hpp"
#include "plan.hpp"

namespace fem_b200 {

struct ShardPlan {
  int device = 0;
  int world = 1, rank = 0, elem_size = 0;
  int e0 = 0, e1 = 0;
  std::vector<int> local_offsets;  // [(e1 - e0) * elem_size]
  std::vector<int64_t> l2g;        // global node id of each local node, ascending
  std::vector<unsigned char> owned;
  std::vector<int> peers;                    // ascending
  std::vector<std::vector<int64_t>> shared;  // local node indices shared with each peer, ascending
  int64_t shared_total = 0;                  // sum of the peers' counts (one component)
  // the send slots (the concatenated peer lists: {local node, segment start,
  // segment count, position}) and, per shared node, its terms in rank order
  // ({segment start, count, position} of a peer's value, or seg = -1 for the
  // local one): on the host from the set-up, on the device from the first
  // pack or unpack (the set-up needs no GPU)
  std::vector<int4> pack_h, terms_h;
  std::vector<int> node_h, ptr_h;
  int n_sum = 0;
  bool uploaded = false;
  DevBuf<int4> pack_slots, sum_terms;
  DevBuf<int> sum_node, sum_ptr;
  void upload() {
    if (uploaded) return;
    device = current_device();
    if (!pack_h.empty()) {
      pack_slots.alloc(pack_h.size());
      sum_node.alloc(node_h.size());
      sum_ptr.alloc(ptr_h.size());
      sum_terms.alloc(terms_h.size());
      FEM_CUDA_CHECK(cudaMemcpy(pack_slots.get(), pack_h.data(), pack_h.size() * sizeof(int4), cudaMemcpyHostToDevice));
      FEM_CUDA_CHECK(cudaMemcpy(sum_node.get(), node_h.data(), node_h.size() * sizeof(int), cudaMemcpyHostToDevice));
      FEM_CUDA_CHECK(cudaMemcpy(sum_ptr.get(), ptr_h.data(), ptr_h.size() * sizeof(int), cudaMemcpyHostToDevice));
      FEM_CUDA_CHECK(cudaMemcpy(sum_terms.get(), terms_h.data(), terms_h.size() * sizeof(int4), cudaMemcpyHostToDevice));
    }
    uploaded = true;
  }
};

namespace {

void element_range(int num_elem, int world, int rank, int& e0, int& e1) {
  const int base = num_elem / world, rem = num_elem % world;
  e0 = rank * base + std::min(rank, rem);
  e1 = e0 + base + (rank < rem ? 1 : 0);
}

// Slot j = {local node, segment start, segment count, position} of the
// concatenated peer lists; peer i's segment of the send buffer is contiguous,
// [comp][pos] from seg * num_comp.
__global__ void shard_pack_kernel(int64_t total, int num_comp, int64_t num_nodes, const int4* __restrict__ slots,
                                  const double* __restrict__ v, double* __restrict__ send) {
  const int64_t n = total * num_comp;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t k = t / total, j = t % total;
    const int4 sl = slots[j];
    send[int64_t(sl.y) * num_comp + k * sl.z + sl.w] = v[sl.x + k * num_nodes];
  }
}

// v[node] = sum of its terms in rank order, from 0 (the same expression on
// every rank that holds the node); the receive buffer holds each peer's
// segment [comp][pos] at seg * num_comp.
__global__ void shard_sum_kernel(int n_sum, int num_comp, int64_t num_nodes, const int* __restrict__ node,
                                 const int* __restrict__ ptr, const int4* __restrict__ terms,
                                 const double* __restrict__ recv, double* __restrict__ v) {
  const int64_t n = int64_t(n_sum) * num_comp;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n; t += int64_t(gridDim.x) * blockDim.x) {
    const int k = int(t / n_sum), i = int(t % n_sum);
    const int64_t at = node[i] + k * num_nodes;
    const double mine = v[at];
    double acc = 0.0;
    for (int j = ptr[i]; j < ptr[i + 1]; ++j) {
      const int4 tm = terms[j];
      acc += tm.x < 0 ? mine : recv[int64_t(tm.x) * num_comp + int64_t(k) * tm.y + tm.z];
    }
    v[at] = acc;
  }
}

}  // namespace
}  // namespace fem_b200

struct fem_b200_shard_s {
  std::unique_ptr<fem_b200::ShardPlan> d;
};

using namespace fem_b200;

extern "C" {

int fem_b200_shard_create(int num_elem, int elem_size, const int* offsets, int world, int rank, fem_b200_shard* out) {
  return guarded([&] {
    require(out != nullptr, "shard create: NULL output handle");
    require(num_elem > 0 && elem_size > 0 && offsets != nullptr, "shard create: empty mesh");
    require(world >= 1 && world <= 65536 && rank >= 0 && rank < world, "shard create: rank must be in [0, world)");
    require(world <= num_elem, "shard create: more ranks than elements");
    auto p = std::make_unique<ShardPlan>();
    p->world = world, p->rank = rank, p->elem_size = elem_size;
    element_range(num_elem, world, rank, p->e0, p->e1);
    const int64_t n_all = int64_t(num_elem) * elem_size;
    int max_node = 0;
    for (int64_t i = 0; i < n_all; ++i) {
      require(offsets[i] >= 0, "shard create: negative offset");
      max_node = std::max(max_node, offsets[i]);
    }
    // this rank's nodes, ascending global id, and their local numbers
    std::vector<int> local_of(size_t(max_node) + 1, -1);
    for (int64_t i = int64_t(p->e0) * elem_size; i < int64_t(p->e1) * elem_size; ++i) local_of[size_t(offsets[i])] = 0;
    for (int g = 0; g <= max_node; ++g)
      if (local_of[size_t(g)] == 0) local_of[size_t(g)] = int(p->l2g.size()), p->l2g.push_back(g);
      else local_of[size_t(g)] = -1;
    p->local_offsets.resize(size_t(int64_t(p->e1 - p->e0) * elem_size));
    for (int64_t i = 0; i < int64_t(p->local_offsets.size()); ++i)
      p->local_offsets[size_t(i)] = local_of[size_t(offsets[int64_t(p->e0) * elem_size + i])];
    // the peers touching each local node
    const int nl = int(p->l2g.size());
    p->owned.assign(size_t(nl), 1);
    std::vector<int> seen(size_t(nl), -1);
    for (int q = 0; q < world; ++q) {
      if (q == rank) continue;
      int q0 = 0, q1 = 0;
      element_range(num_elem, world, q, q0, q1);
      std::vector<int64_t> idx;
      for (int64_t i = int64_t(q0) * elem_size; i < int64_t(q1) * elem_size; ++i) {
        const int j = local_of[size_t(offsets[i])];
        if (j >= 0 && seen[size_t(j)] != q) seen[size_t(j)] = q, idx.push_back(j);
      }
      if (idx.empty()) continue;
      std::sort(idx.begin(), idx.end());
      if (q < rank)
        for (int64_t j : idx) p->owned[size_t(j)] = 0;
      p->peers.push_back(q);
      p->shared.push_back(std::move(idx));
    }
    // the send slots, and per shared node its terms in rank order
    std::vector<int4> pack;
    std::vector<std::vector<int4>> terms(static_cast<size_t>(nl));
    int64_t seg = 0;
    for (size_t i = 0; i < p->peers.size(); ++i) {
      const int count = int(p->shared[i].size());
      for (int pos = 0; pos < count; ++pos) {
        const int64_t j = p->shared[i][size_t(pos)];
        pack.push_back(make_int4(int(j), int(seg), count, pos));
        terms[size_t(j)].push_back(make_int4(int(seg), count, pos, p->peers[i]));
      }
      seg += count;
    }
    p->shared_total = seg;
    std::vector<int> node, ptr(1, 0);
    std::vector<int4> flat;
    for (int j = 0; j < nl; ++j) {
      if (terms[size_t(j)].empty()) continue;
      auto& tl = terms[size_t(j)];
      tl.push_back(make_int4(-1, 0, 0, rank));  // the local value
      std::sort(tl.begin(), tl.end(), [](const int4& a, const int4& b) { return a.w < b.w; });
      node.push_back(j);
      for (const int4& t : tl) flat.push_back(make_int4(t.x, t.y, t.z, 0));
      ptr.push_back(int(flat.size()));
    }
    p->n_sum = int(node.size());
    p->pack_h = std::move(pack);
    p->node_h = std::move(node);
    p->ptr_h = std::move(ptr);
    p->terms_h = std::move(flat);
    *out = new fem_b200_shard_s{std::move(p)};
  });
}

int fem_b200_shard_sizes(fem_b200_shard s, int* e0, int* e1, int* num_nodes, int* num_peers, int64_t* shared_total) {
  return guarded([&] {
    require(s && s->d, "shard sizes: NULL handle");
    const ShardPlan& p = *s->d;
    if (e0) *e0 = p.e0;
    if (e1) *e1 = p.e1;
    if (num_nodes) *num_nodes = int(p.l2g.size());
    if (num_peers) *num_peers = int(p.peers.size());
    if (shared_total) *shared_total = p.shared_total;
  });
}

int fem_b200_shard_local(fem_b200_shard s, int* local_offsets, int64_t* l2g, unsigned char* owned) {
  return guarded([&] {
    require(s && s->d, "shard local: NULL handle");
    const ShardPlan& p = *s->d;
    if (local_offsets) std::copy(p.local_offsets.begin(), p.local_offsets.end(), local_offsets);
    if (l2g) std::copy(p.l2g.begin(), p.l2g.end(), l2g);
    if (owned) std::copy(p.owned.begin(), p.owned.end(), owned);
  });
}

int fem_b200_shard_peer(fem_b200_shard s, int i, int* peer, int64_t* count, int64_t* local_idx) {
  return guarded([&] {
    require(s && s->d, "shard peer: NULL handle");
    const ShardPlan& p = *s->d;
    require(i >= 0 && i < int(p.peers.size()), "shard peer: index out of range");
    if (peer) *peer = p.peers[size_t(i)];
    if (count) *count = int64_t(p.shared[size_t(i)].size());
    if (local_idx) std::copy(p.shared[size_t(i)].begin(), p.shared[size_t(i)].end(), local_idx);
  });
}

int fem_b200_shard_pack(fem_b200_shard s, const double* v, int64_t n_v, int num_comp, double* send, int64_t n_send,
                        void* stream) {
  return guarded([&] {
    require(s && s->d, "shard pack: NULL handle");
    ShardPlan& p = *s->d;
    const int64_t nn = int64_t(p.l2g.size());
    require(num_comp >= 1 && n_v == nn * num_comp && v, "shard pack: v must hold num_comp x num_nodes values");
    require(n_send == p.shared_total * num_comp, "shard pack: send must hold num_comp x shared_total values");
    if (p.shared_total == 0) return;
    require(send != nullptr, "shard pack: NULL send buffer");
    p.upload();
    DeviceGuard g(p.device);
    const int64_t n = p.shared_total * num_comp;
    shard_pack_kernel<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(p.shared_total, num_comp, nn,
                                                                      p.pack_slots.get(), v, send);
    FEM_LAUNCH_CHECK();
  });
}

int fem_b200_shard_unpack_add(fem_b200_shard s, const double* recv, int64_t n_recv, int num_comp, double* v,
                              int64_t n_v, void* stream) {
  return guarded([&] {
    require(s && s->d, "shard unpack: NULL handle");
    ShardPlan& p = *s->d;
    const int64_t nn = int64_t(p.l2g.size());
    require(num_comp >= 1 && n_v == nn * num_comp && v, "shard unpack: v must hold num_comp x num_nodes values");
    require(n_recv == p.shared_total * num_comp, "shard unpack: recv must hold num_comp x shared_total values");
    if (p.n_sum == 0) return;
    require(recv != nullptr, "shard unpack: NULL receive buffer");
    p.upload();
    DeviceGuard g(p.device);
    const int64_t n = int64_t(p.n_sum) * num_comp;
    shard_sum_kernel<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(p.n_sum, num_comp, nn, p.sum_node.get(),
                                                                     p.sum_ptr.get(), p.sum_terms.get(), recv, v);
    FEM_LAUNCH_CHECK();
  });
}

int fem_b200_shard_destroy(fem_b200_shard s) {
  return guarded([&] { delete s; });
}

}  // extern "C"
