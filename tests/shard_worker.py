"""Rank body of tests/test_shard.py (a module of its own, so that spawned
ranks can import it): the partitioned operator's host logic -- partition,
interface exchange, owned-node dots, distributed PCG -- on gloo, with the
oracle's apply standing in for each rank's device apply (the checker)."""
import datetime
import os

import numpy as np


def diag_by_formula(orc, dim, ne, P, Q, offsets, qd, n):
    """diag_i = sum_e sum_q qdata_q B_qi^2 (B the tensor interpolation), the
    scatter-added squared-interpolation form of e_i^T M e_i."""
    _, _, B, _ = orc.basis(1, 1, P, Q)
    B = B.reshape(Q, P)
    B2 = B * B
    if dim == 3:
        T = np.einsum("zc,yb,xa->zyxcba", B2, B2, B2).reshape(Q**3, P**3)
    else:
        T = np.einsum("yb,xa->yxba", B2, B2).reshape(Q**2, P**2)
    contrib = (qd.reshape(-1, ne).T @ T)  # [e][i]
    d = np.zeros(n)
    np.add.at(d, offsets.reshape(ne, -1), contrib)
    return d


def run(rank, world, port, nc, shape, P):
    import torch
    import torch.distributed as dist
    import oracle
    from fe_demo_cpp_b200.mesh import box_mesh, random_vector
    from fe_demo_cpp_b200.shard import DistributedMass, Shard, distributed_pcg

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        orc = oracle.orc()
        Q = P + 1
        m = box_mesh(shape, P, seed=4)
        N = m.num_nodes
        sh = Shard(m.offsets, P**3, world, rank)
        n_l = sh.num_nodes
        qd = orc.mass_build(3, sh.num_elem, P, Q, n_l, sh.offsets, sh.local_coords(m.coords, 3))
        gidx = np.concatenate([sh.l2g + k * N for k in range(nc)])

        def local_apply(u, v):
            v.copy_(torch.from_numpy(orc.mass_apply(3, sh.num_elem, P, Q, nc, n_l, nc * n_l, sh.offsets, qd,
                                                    u.numpy(), vector=True)))

        def local_diag(d):
            d.copy_(torch.from_numpy(np.tile(diag_by_formula(orc, 3, sh.num_elem, P, Q, sh.offsets, qd, n_l), nc)))

        A = DistributedMass(sh, local_apply, local_diag, nc)
        # the global operator, for checking
        qd_g = orc.mass_build(3, m.num_elem, P, Q, N, m.offsets, m.coords)
        offs_g = m.offsets
        u_g = random_vector(nc * N, 3)
        v_g = orc.mass_apply(3, m.num_elem, P, Q, nc, N, nc * N, offs_g, qd_g, u_g, vector=True)
        v_l = torch.empty(nc * n_l, dtype=torch.float64)
        A.apply(torch.from_numpy(u_g[gidx].copy()), v_l)
        err = np.abs(v_l.numpy() - v_g[gidx]).max() / np.abs(v_g).max()
        assert err <= 1e-14, ("apply", rank, err)
        # a shared node holds the same bits on every rank
        vals = [None] * world
        dist.all_gather_object(vals, (gidx, v_l.numpy()))
        ref = {}
        for g, v in vals:
            for gi, vi in zip(g.tolist(), v.tolist()):
                assert ref.setdefault(gi, vi) == vi, ("shared value differs", gi)
        # global dots count every DoF once
        (uu,) = A.dots([(torch.from_numpy(u_g[gidx].copy()), torch.from_numpy(u_g[gidx].copy()))])
        assert abs(uu - float(u_g @ u_g)) <= 1e-12 * float(u_g @ u_g), ("dot", uu)
        # assembled diagonal against e_i^T M e_i of the global operator (a sample)
        d_l = torch.empty(nc * n_l, dtype=torch.float64)
        A.diagonal(d_l)
        for j in range(0, nc * n_l, max(1, nc * n_l // 12)):
            e = np.zeros(nc * N)
            e[gidx[j]] = 1.0
            want = orc.mass_apply(3, m.num_elem, P, Q, nc, N, nc * N, offs_g, qd_g, e, vector=True)[gidx[j]]
            assert abs(float(d_l[j]) - want) <= 1e-13 * abs(want), ("diag", j)
        # distributed PCG recovers u* from f = M u*
        x_l = torch.empty(nc * n_l, dtype=torch.float64)
        its, rel = distributed_pcg(A, torch.from_numpy(v_g[gidx].copy()), x_l, rtol=1e-12, max_iter=500)
        err = np.linalg.norm(x_l.numpy() - u_g[gidx]) / np.linalg.norm(u_g[gidx])
        assert its > 0 and rel <= 1e-12 and err <= 1e-9, ("pcg", its, rel, err)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def run_device(rank, world, port, nc, shape, P):
    """The device path: each rank builds and applies its elements with the
    fused kernels on cuda:0 (ranks share the GPU; their kernels never wait on
    one another, the exchange goes through gloo on the host)."""
    import torch
    import torch.distributed as dist
    import oracle
    import fe_demo_cpp_b200 as fem
    from fe_demo_cpp_b200.mesh import box_mesh, random_vector
    from fe_demo_cpp_b200.shard import DistributedMass, Shard, distributed_pcg

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        fem.load()
        dev = torch.device("cuda", 0)
        orc = oracle.orc()
        Q = P + 1
        m = box_mesh(shape, P, seed=6)
        N = m.num_nodes
        sh = Shard(m.offsets, P**3, world, rank)
        A = DistributedMass.on_device(fem, sh, m.coords, 3, P, Q, nc, dev)
        gidx = np.concatenate([sh.l2g + k * N for k in range(nc)])
        qd_g = orc.mass_build(3, m.num_elem, P, Q, N, m.offsets, m.coords)
        u_g = random_vector(nc * N, 8)
        v_g = orc.mass_apply(3, m.num_elem, P, Q, nc, N, nc * N, m.offsets, qd_g, u_g, vector=True)
        v = torch.empty(nc * sh.num_nodes, dtype=torch.float64, device=dev)
        A.apply(torch.from_numpy(u_g[gidx].copy()).to(dev), v)
        err = np.abs(v.cpu().numpy() - v_g[gidx]).max() / np.abs(v_g).max()
        assert err <= 1e-13, ("apply", rank, err)
        x = torch.empty_like(v)
        its, rel = distributed_pcg(A, torch.from_numpy(v_g[gidx].copy()).to(dev), x, rtol=1e-12, max_iter=500)
        err = np.linalg.norm(x.cpu().numpy() - u_g[gidx]) / np.linalg.norm(u_g[gidx])
        assert rel <= 1e-12 and err <= 1e-9, ("pcg", its, rel, err)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def host_pack(plan, v, nc):
    """The send buffer of fem_b200_shard_pack, on the host: peer i's segment
    [comp][pos] from num_comp x (counts before i)."""
    n = plan.num_nodes
    return np.concatenate([np.concatenate([v[idx + k * n] for k in range(nc)]) for _, idx in plan.peers]) \
        if plan.peers else np.zeros(0)


def host_unpack_add(plan, recv, v, nc, rank):
    """fem_b200_shard_unpack_add on the host: every shared value := the sum of
    all ranks' values in rank order, from 0."""
    n = plan.num_nodes
    terms = {}
    seg = 0
    for q, idx in plan.peers:
        for pos, j in enumerate(idx):
            terms.setdefault(int(j), []).append((q, seg, len(idx), pos))
        seg += len(idx)
    out = v.copy()
    for j, tl in terms.items():
        tl = sorted(tl + [(rank, -1, 0, 0)])
        for k in range(nc):
            acc = 0.0
            for q, s0, cnt, pos in tl:
                acc += v[j + k * n] if s0 < 0 else recv[s0 * nc + k * cnt + pos]
            out[j + k * n] = acc
    return out


def run_abi(rank, world, port, nc, shape, P):
    """The C-ABI shard plan (fem_b200_shard_*) on gloo ranks: each rank builds
    its plan, applies the oracle to its elements, moves the packed segments to
    its peers over gloo and adds them in rank order; the result must equal the
    global operator at the rank's nodes, and shared values must have the same
    bits on every rank."""
    import torch
    import torch.distributed as dist
    import oracle
    import fe_demo_cpp_b200 as fem
    from fe_demo_cpp_b200.mesh import box_mesh, random_vector

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        orc = oracle.orc()
        Q = P + 1
        m = box_mesh(shape, P, seed=6)
        N = m.num_nodes
        plan = fem.ShardPlan(m.offsets, P**3, world, rank)
        n_l = plan.num_nodes
        qd = orc.mass_build(3, plan.num_elem, P, Q, n_l, plan.offsets,
                            np.concatenate([m.coords[k * N + plan.l2g] for k in range(3)]))
        u_g = random_vector(nc * N, 5)
        u_l = np.concatenate([u_g[plan.l2g + k * N] for k in range(nc)])
        v_l = orc.mass_apply(3, plan.num_elem, P, Q, nc, n_l, nc * n_l, plan.offsets, qd, u_l, vector=True)
        send = host_pack(plan, v_l, nc)
        recv = np.zeros_like(send)
        ops, seg = [], 0
        for q, idx in plan.peers:
            cnt = len(idx) * nc
            s = torch.from_numpy(send[seg:seg + cnt].copy())
            r = torch.empty(cnt, dtype=torch.float64)
            ops += [dist.P2POp(dist.isend, s, q), dist.P2POp(dist.irecv, r, q)]
            ops_r = (r, seg, cnt)
            ops[-1].recv_slot = ops_r
            seg += cnt
        for req in dist.batch_isend_irecv(ops) if ops else []:
            req.wait()
        for op in ops:
            if hasattr(op, "recv_slot"):
                r, s0, cnt = op.recv_slot
                recv[s0:s0 + cnt] = r.numpy()
        v_l = host_unpack_add(plan, recv, v_l, nc, rank)
        qd_g = orc.mass_build(3, m.num_elem, P, Q, N, m.offsets, m.coords)
        v_g = orc.mass_apply(3, m.num_elem, P, Q, nc, N, nc * N, m.offsets, qd_g, u_g, vector=True)
        want = np.concatenate([v_g[plan.l2g + k * N] for k in range(nc)])
        assert np.abs(v_l - want).max() <= 1e-14 * np.abs(want).max()
        # shared values: the same bits on every rank (gather every rank's values by global id)
        sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(sizes, torch.tensor([n_l]))
        width = int(max(s.item() for s in sizes))  # gloo gathers equal sizes: pad with id -1
        mine = torch.full((2, width), -1.0, dtype=torch.float64)
        mine[0, :n_l] = torch.from_numpy(plan.l2g.astype(np.float64))
        mine[1, :n_l] = torch.from_numpy(v_l[:n_l])
        allv = [torch.zeros(2, width, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(allv, mine)
        seen = {}
        for t in allv:
            for g, x in zip(t[0].numpy().astype(np.int64), t[1].numpy()):
                if g < 0:
                    continue
                if g in seen:
                    assert seen[g] == x, "a shared value differs between ranks"
                seen[g] = x
    finally:
        dist.destroy_process_group()
