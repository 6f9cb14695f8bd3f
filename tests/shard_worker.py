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
