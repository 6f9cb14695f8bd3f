"""The C-ABI shard plan (fem_b200_shard_*, fe_demo_cpp_b200.ShardPlan).

CPU: the plan equals the Python partition (fe_demo_cpp_b200/shard.py) --
element ranges, compact numbering, owners, the nodes shared with each peer --
and, on gloo ranks (world 2 and 3), its send-buffer layout and rank-ordered
sums give the global operator (the oracle's apply on each rank's elements,
1e-14) with the same bits for a shared node on every rank.
GPU: the device pack / unpack-add of three ranks emulated in one process
(each rank's segments copied to its peers) against the host restatement of
the same layout and order, bitwise, and against the global operator.
"""
import socket

import numpy as np
import pytest

from fe_demo_cpp_b200.mesh import box_mesh
from fe_demo_cpp_b200.shard import Shard


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,shape,P", [(2, (3, 3, 4), 3), (3, (3, 2, 5), 3), (4, (2, 2, 5), 4)])
def test_abi_plan_matches_python_partition(fem, world, shape, P):
    m = box_mesh(shape, P, seed=2)
    for r in range(world):
        a = fem.ShardPlan(m.offsets, P**3, world, r)
        b = Shard(m.offsets, P**3, world, r)
        assert (a.e0, a.e1, a.num_nodes) == (b.e0, b.e1, b.num_nodes)
        assert np.array_equal(a.l2g, b.l2g) and np.array_equal(a.offsets, b.offsets)
        assert np.array_equal(a.owned, b.owned)
        assert [q for q, _ in a.peers] == [q for q, _ in b.peers]
        for (_, x), (_, y) in zip(a.peers, b.peers):
            assert np.array_equal(x, y)
        assert a.shared_total == sum(len(x) for _, x in a.peers)


def test_abi_plan_rejects_bad_arguments(fem):
    m = box_mesh((2, 2, 1), 2, seed=1)
    with pytest.raises(ValueError):
        fem.ShardPlan(m.offsets, 8, 5, 0)  # more ranks than elements
    with pytest.raises(ValueError):
        fem.ShardPlan(m.offsets, 8, 2, 2)  # rank out of range


@pytest.mark.parametrize("world,nc,shape,P", [(2, 1, (3, 3, 4), 3), (3, 2, (3, 2, 5), 3)])
def test_abi_plan_on_gloo_ranks(fem, world, nc, shape, P):
    import torch.multiprocessing as mp
    import shard_worker
    mp.spawn(shard_worker.run_abi, args=(world, free_port(), nc, shape, P), nprocs=world, join=True)


@pytest.mark.gpu
@pytest.mark.parametrize("nc", [1, 3])
def test_device_pack_unpack_three_ranks(fem, cuda, orc, nc):
    import torch
    import shard_worker
    from fe_demo_cpp_b200.mesh import random_vector
    world, P, Q = 3, 4, 5
    m = box_mesh((3, 3, 4), P, seed=9)
    N = m.num_nodes
    plans = [fem.ShardPlan(m.offsets, P**3, world, r) for r in range(world)]
    u_g = random_vector(nc * N, 8)
    v_loc, sends = [], []
    for pl in plans:
        n = pl.num_nodes
        qd = orc.mass_build(3, pl.num_elem, P, Q, n, pl.offsets, np.concatenate([m.coords[k * N + pl.l2g]
                                                                                 for k in range(3)]))
        u_l = np.concatenate([u_g[pl.l2g + k * N] for k in range(nc)])
        v = orc.mass_apply(3, pl.num_elem, P, Q, nc, n, nc * n, pl.offsets, qd, u_l, vector=True)
        v_loc.append(v)
        send = torch.full((nc * pl.shared_total,), float("nan"), dtype=torch.float64, device=cuda)
        pl.pack(torch.from_numpy(v).to(cuda), send, nc)
        assert np.array_equal(send.cpu().numpy(), shard_worker.host_pack(pl, v, nc))
        sends.append(send)
    qd_g = orc.mass_build(3, m.num_elem, P, Q, N, m.offsets, m.coords)
    v_g = orc.mass_apply(3, m.num_elem, P, Q, nc, N, nc * N, m.offsets, qd_g, u_g, vector=True)
    shared = {}
    for r, pl in enumerate(plans):
        recv = torch.empty_like(sends[r])
        seg = 0
        for q, idx in pl.peers:  # the transport: q's segment for r into r's receive buffer
            back = plans[q]
            s0 = 0
            for qq, idx2 in back.peers:
                if qq == r:
                    break
                s0 += len(idx2)
            recv[seg * nc:(seg + len(idx)) * nc] = sends[q][s0 * nc:(s0 + len(idx)) * nc]
            seg += len(idx)
        v = torch.from_numpy(v_loc[r]).to(cuda)
        pl.unpack_add(recv, v, nc)
        got = v.cpu().numpy()
        assert np.array_equal(got, shard_worker.host_unpack_add(pl, recv.cpu().numpy(), v_loc[r], nc, r))
        want = np.concatenate([v_g[pl.l2g + k * N] for k in range(nc)])
        assert np.abs(got - want).max() <= 1e-14 * np.abs(want).max()
        for j, g in enumerate(pl.l2g):
            x = got[j]
            if g in shared:
                assert shared[g] == x
            shared[g] = x
