"""One mesh over several ranks (one process per GPU): elements partitioned in
contiguous ranges, each rank applying the mass operator to its elements on
its own device, then ONE interface exchange per apply that sums the L-DoFs
shared with other ranks.

* ``Shard``: this rank's elements, its compact node numbering (``l2g``,
  global ids ascending), the shared nodes per peer and the owned-node mask
  (a node belongs to the lowest rank that touches it).
* ``Shard.exchange(v)``: v_i = sum over the ranks touching node i, added in
  rank order on every rank, so a shared value has the same bits everywhere.
  Point-to-point sends of the shared values only (``batch_isend_irecv``: NCCL
  over NVLink for device tensors, gloo for host tensors).
* ``DistributedMass``: local apply + exchange; global dot products over owned
  nodes with one all-reduce.
* ``distributed_pcg``: Jacobi PCG on it (one fused scalar all-reduce of two
  dots per iteration).

The reference is single-process (src/operator.cpp:148-182); this is the
partition of its operator over ranks, with nothing on the data path but the
interface exchange and the scalar reductions.
"""
from __future__ import annotations

import numpy as np


def element_range(num_elem: int, world: int, rank: int):
    """Contiguous elements [e0, e1) of `rank` (sizes differ by at most one)."""
    base, rem = divmod(int(num_elem), int(world))
    e0 = rank * base + min(rank, rem)
    return e0, e0 + base + (1 if rank < rem else 0)


class Shard:
    """This rank's part of a mesh partitioned by element ranges.  Every rank
    holds the global offsets (the set-up reads the whole mesh)."""

    def __init__(self, offsets, elem_size: int, world: int, rank: int):
        offsets = np.asarray(offsets)
        num_elem = offsets.size // elem_size
        self.world, self.rank = int(world), int(rank)
        self.e0, self.e1 = element_range(num_elem, world, rank)
        mine = offsets[self.e0 * elem_size:self.e1 * elem_size].astype(np.int64)
        self.l2g, local = np.unique(mine, return_inverse=True)
        self.offsets = local.astype(np.int32)
        self.num_elem = self.e1 - self.e0
        self.num_nodes = int(self.l2g.size)
        # (node, rank) pairs of the whole mesh -> the ranks touching each node
        bounds = [element_range(num_elem, world, r) for r in range(world)]
        elem_rank = np.repeat(np.arange(world, dtype=np.int64), [b[1] - b[0] for b in bounds])
        pairs = np.unique(offsets.astype(np.int64) * world + np.repeat(elem_rank, elem_size))
        node_of, rank_of = pairs // world, pairs % world
        self.peers = []  # (peer, local indices of the shared nodes, ascending global id)
        for q in range(world):
            if q == self.rank:
                continue
            _, idx, _ = np.intersect1d(self.l2g, node_of[rank_of == q], assume_unique=True, return_indices=True)
            if idx.size:
                self.peers.append((q, idx.astype(np.int64)))
        self.owned = np.ones(self.num_nodes, dtype=bool)
        for q, idx in self.peers:
            if q < self.rank:
                self.owned[idx] = False
        self._dev_cache = {}

    def local_coords(self, coords, dim: int):
        """The rank's node coordinates, blocked [dim][num_nodes] like the global ones."""
        coords = np.asarray(coords).reshape(dim, -1)
        return np.ascontiguousarray(coords[:, self.l2g]).reshape(-1)

    def _indices(self, device, num_comp):
        key = (str(device), num_comp)
        if key not in self._dev_cache:
            import torch
            n = self.num_nodes
            per = []
            for q, idx in self.peers:
                full = np.concatenate([idx + k * n for k in range(num_comp)])
                per.append((q, torch.from_numpy(full).to(device)))
            self._dev_cache[key] = per
        return self._dev_cache[key]

    def exchange(self, v, num_comp: int = 1, group=None):
        """v (torch, blocked [num_comp][num_nodes]) := the global sum at every
        local node, contributions added in rank order."""
        import torch
        import torch.distributed as dist
        per = self._indices(v.device, num_comp)
        if not per:
            return v
        # gloo moves host memory: device values go through the host there
        host = v.is_cuda and dist.get_backend(group) == "gloo"
        sends = [v.index_select(0, idx).contiguous() for _, idx in per]
        if host:
            sends = [s.cpu() for s in sends]
        recvs = [torch.empty_like(s) for s in sends]
        ops = []
        for (q, _), s, r in zip(per, sends, recvs):
            ops.append(dist.P2POp(dist.isend, s, q, group))
            ops.append(dist.P2POp(dist.irecv, r, q, group))
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        if host:
            recvs = [r.to(v.device) for r in recvs]
        mine = v.clone()
        v.zero_()
        below = [(q, idx, r) for (q, idx), r in zip(per, recvs) if q < self.rank]
        above = [(q, idx, r) for (q, idx), r in zip(per, recvs) if q > self.rank]
        for _, idx, r in below:
            v.index_add_(0, idx, r)
        v.add_(mine)
        for _, idx, r in above:
            v.index_add_(0, idx, r)
        return v

    def owned_mask(self, device, num_comp: int = 1):
        import torch
        key = ("owned", str(device), num_comp)
        if key not in self._dev_cache:
            self._dev_cache[key] = torch.from_numpy(np.tile(self.owned, num_comp)).to(device)
        return self._dev_cache[key]


class DistributedMass:
    """The mass operator of one partitioned mesh: `local_apply(u, v)` applies
    this rank's elements (v overwritten), `local_diagonal(d)` assembles their
    diagonal; both on local L-vectors blocked [num_comp][num_nodes]."""

    def __init__(self, shard: Shard, local_apply, local_diagonal=None, num_comp: int = 1, group=None):
        self.shard, self.local_apply, self.local_diagonal = shard, local_apply, local_diagonal
        self.num_comp, self.group = num_comp, group

    def apply(self, u, v):
        self.local_apply(u, v)
        return self.shard.exchange(v, self.num_comp, self.group)

    def diagonal(self, d):
        self.local_diagonal(d)
        return self.shard.exchange(d, self.num_comp, self.group)

    def dots(self, pairs):
        """[(a, b), ...] -> global dot products over owned nodes, one all-reduce."""
        import torch
        import torch.distributed as dist
        m = self.shard.owned_mask(pairs[0][0].device, self.num_comp)
        t = torch.stack([torch.sum(torch.where(m, a * b, torch.zeros_like(a))) for a, b in pairs]).to(torch.float64)
        if t.is_cuda and dist.get_backend(self.group) == "gloo":
            t = t.cpu()
        dist.all_reduce(t, group=self.group)
        return t.tolist()

    @classmethod
    def on_device(cls, fem, shard: Shard, coords, dim: int, P: int, Q: int, num_comp: int, device, group=None):
        """The local operator through the device path (fused build and apply)."""
        import torch
        n = shard.num_nodes
        rx = fem.Restriction(shard.num_elem, P**dim, dim, n, dim * n, shard.offsets)
        qd = torch.empty(Q**dim * shard.num_elem, dtype=torch.float64, device=device)
        fem.mass_build(rx, fem.Basis(dim, dim, P, Q), torch.from_numpy(shard.local_coords(coords, dim)).to(device),
                       qd)
        op = fem.MassOperator(fem.Restriction(shard.num_elem, P**dim, num_comp, n, num_comp * n, shard.offsets),
                              fem.Basis(dim, num_comp, P, Q), qd, fem.QF.apply_mass_vector)
        d = cls(shard, op.apply, op.diagonal, num_comp, group)
        d.op = op
        return d


def distributed_pcg(A: DistributedMass, f, u, rtol=1e-10, max_iter=1000):
    """Jacobi PCG for A u = f from u = 0 (torch vectors on every rank); the
    preconditioner is the exchanged assembled diagonal.  Returns
    (iterations, ||r|| / ||f||) by the recursive residual."""
    import torch
    d = torch.empty_like(f)
    A.diagonal(d)
    dinv = torch.where(d != 0, 1.0 / d, torch.zeros_like(d))
    u.zero_()
    r = f.clone()
    z = dinv * r
    p = z.clone()
    q = torch.empty_like(f)
    rz, rr = A.dots([(r, z), (r, r)])
    r0 = rr ** 0.5
    it = 0
    while it < max_iter and rr ** 0.5 > rtol * r0 and r0 > 0:
        A.apply(p, q)
        (pq,) = A.dots([(p, q)])
        alpha = rz / pq
        u.add_(alpha * p)
        r.sub_(alpha * q)
        torch.mul(dinv, r, out=z)
        rz_new, rr = A.dots([(r, z), (r, r)])
        p.mul_(rz_new / rz).add_(z)
        rz = rz_new
        it += 1
    return it, (rr ** 0.5 / r0) if r0 > 0 else 0.0
