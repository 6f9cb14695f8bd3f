"""Batched apply over many meshes (GPU): one captured graph applying
v_i = M_i u_i for operators of uneven dim, order, size and component count,
checked against each operator's own apply (normwise 1e-13, FP64; the same
tile arithmetic, only the order of the atomic adds differs), against the
oracle on a few members, and in FP32 against the FP64 result (normwise 1e-5,
FP32 storage of u, v and qdata)."""
import numpy as np
import pytest

from fe_demo_cpp_b200.mesh import box_mesh, component_layout, gll_nodes, random_vector

pytestmark = pytest.mark.gpu
TOL = 1e-13


def dev(a, cuda, dtype=None):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).to(cuda)
    return t.to(dtype) if dtype is not None else t


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.double().cpu().numpy()


def close(got, want, tol):
    scale = max(np.abs(want).max(), 1e-300)
    err = np.abs(got - want).max() / scale
    assert err <= tol, f"normwise relative error {err:.3e} > {tol:.0e}"


class _Line:
    pass


def line_mesh(n, P, seed):
    rng = np.random.default_rng([seed, 17])
    xv = np.linspace(0, 1, n + 1)
    xv[1:-1] += rng.uniform(-0.1 / n, 0.1 / n, n - 1)
    s = (gll_nodes(P) + 1) / 2
    m = _Line()
    m.dim, m.P, m.num_elem, m.num_nodes = 1, P, n, n * (P - 1) + 1
    m.coords = np.concatenate([xv[e] + (xv[e + 1] - xv[e]) * s[(0 if e == 0 else 1):] for e in range(n)])
    m.offsets = np.array([e * (P - 1) + i for e in range(n) for i in range(P)], dtype=np.int32)
    return m


def make_op(fem, cuda, dim, shape, P, Q, nc, qf, seed, interleaved=False):
    import torch
    m = line_mesh(shape[0], P, seed) if dim == 1 else box_mesh(shape, P, seed=seed)
    rx = fem.Restriction(m.num_elem, P**dim, dim, m.num_nodes, dim * m.num_nodes, m.offsets)
    qd = torch.empty(Q**dim * m.num_elem, dtype=torch.float64, device=cuda)
    fem.mass_build(rx, fem.Basis(dim, dim, P, Q), dev(m.coords, cuda), qd)
    if nc == 1:
        offs, cs, l_size = m.offsets, m.num_nodes, m.num_nodes
    else:
        offs, cs, l_size = component_layout(m, nc, interleaved)
    op = fem.MassOperator(fem.Restriction(m.num_elem, P**dim, nc, cs, l_size, offs), fem.Basis(dim, nc, P, Q), qd, qf)
    return op, dict(dim=dim, ne=m.num_elem, P=P, Q=Q, nc=nc, cs=cs, l_size=l_size, offs=offs, qd=host(qd),
                    vector=qf == fem.QF.apply_mass_vector)


def mixed_batch(fem, cuda):
    """Uneven members: 1D/2D/3D, P 2..8, Q = P..P+2, 1-3 components, both
    QFunctions, blocked and interleaved layouts, repeated shapes (so classes
    have several members) and single-element meshes (tail tiles)."""
    V, S = fem.QF.apply_mass_vector, fem.QF.apply_mass
    spec = [(3, (3, 2, 2), 4, 5, 1, S), (3, (5, 4, 3), 4, 5, 1, S), (3, (1, 1, 1), 4, 5, 1, S),
            (3, (4, 3, 3), 5, 6, 3, V), (3, (2, 2, 3), 5, 6, 3, V), (3, (3, 3, 2), 3, 4, 2, V),
            (3, (2, 2, 2), 6, 7, 1, S), (3, (2, 1, 2), 7, 9, 1, S), (3, (3, 2, 2), 2, 3, 3, S),
            (2, (7, 5), 3, 4, 1, S), (2, (9, 9), 5, 6, 2, V), (2, (1, 1), 2, 2, 1, S), (2, (12, 7), 3, 4, 1, S),
            (1, (300,), 4, 5, 1, S), (1, (9,), 3, 5, 2, V),
            # high order: the FP64 classes read the 1D matrix from shared memory
            (3, (2, 2, 1), 8, 9, 1, S), (2, (5, 4), 7, 8, 1, S), (2, (3, 3), 8, 9, 2, V)]
    ops, metas = [], []
    for i, (dim, shape, P, Q, nc, qf) in enumerate(spec):
        op, meta = make_op(fem, cuda, dim, shape, P, Q, nc, qf, seed=i, interleaved=(i % 2 == 1 and nc > 1))
        ops.append(op)
        metas.append(meta)
    return ops, metas


@pytest.mark.parametrize("graph", [True, False], ids=["graph", "direct"])
def test_batch_matches_each_operator_and_the_oracle(fem, cuda, orc, graph):
    import torch
    ops, metas = mixed_batch(fem, cuda)
    us = [dev(random_vector(mt["l_size"], 50 + i), cuda) for i, mt in enumerate(metas)]
    vs = [torch.full_like(u, 7.0) for u in us]  # garbage: the batch zeroes v
    b = fem.Batch(ops, "fp64")
    b.bind(us, vs)
    info = b.info()
    assert info["graph_kernels"] == info["classes"] + 1 and info["classes"] < len(ops)
    assert info["dofs"] == sum(mt["l_size"] for mt in metas)
    b.apply(graph=graph)
    for i, (op, mt) in enumerate(zip(ops, metas)):
        want = torch.empty_like(us[i])
        op.apply(us[i], want)
        close(host(vs[i]), host(want), TOL)
    for i in (0, 3, 10, 13, 14):  # the oracle on members of every dim
        mt = metas[i]
        want = orc.mass_apply(mt["dim"], mt["ne"], mt["P"], mt["Q"], mt["nc"], mt["cs"], mt["l_size"], mt["offs"],
                              mt["qd"], host(us[i]), vector=mt["vector"])
        close(host(vs[i]), want, TOL)


def test_graph_replay_rebind_and_autotune(fem, cuda):
    import torch
    ops, metas = mixed_batch(fem, cuda)
    us = [dev(random_vector(mt["l_size"], 70 + i), cuda) for i, mt in enumerate(metas)]
    vs = [torch.empty_like(u) for u in us]
    b = fem.Batch(ops, "fp64")
    b.bind(us, vs)
    b.apply()
    first = [host(v) for v in vs]
    for _ in range(3):  # replays of the same graph
        b.apply()
    for f, v in zip(first, vs):
        close(host(v), f, 1e-15 * 4)
    # new vectors bound into the same graph
    us2 = [2.0 * u - 1.0 for u in us]
    vs2 = [torch.empty_like(u) for u in us]
    b.bind(us2, vs2)
    b.apply()
    for i, op in enumerate(ops):
        want = torch.empty_like(us2[i])
        op.apply(us2[i], want)
        close(host(vs2[i]), host(want), TOL)
    b.autotune(reps=2)
    assert 0 <= b.info()["persistent_classes"] <= b.info()["classes"]
    assert b.info()["graph_branches"] in (1, 2, 4)
    for v in vs2:
        v.fill_(3.0)
    b.apply()
    for i, op in enumerate(ops):
        want = torch.empty_like(us2[i])
        op.apply(us2[i], want)
        close(host(vs2[i]), host(want), TOL)


def test_fp32_batch_within_fp32_rounding(fem, cuda):
    import torch
    ops, metas = mixed_batch(fem, cuda)
    us = [dev(random_vector(mt["l_size"], 90 + i), cuda) for i, mt in enumerate(metas)]
    us32 = [u.float() for u in us]
    vs32 = [torch.empty_like(u) for u in us32]
    b = fem.Batch(ops, "fp32")
    b.bind(us32, vs32)
    b.autotune(reps=2)
    b.apply()
    for i, op in enumerate(ops):
        want = torch.empty_like(us[i])
        op.apply(us32[i].double(), want)  # the same rounded input in FP64
        close(host(vs32[i]), host(want), 1e-5)


def test_batch_argument_errors(fem, cuda):
    import torch
    ops, metas = mixed_batch(fem, cuda)
    b = fem.Batch(ops[:3], "fp64")
    with pytest.raises(ValueError):
        b.apply()  # nothing bound
    us = [torch.zeros(mt["l_size"], dtype=torch.float64, device=cuda) for mt in metas[:3]]
    with pytest.raises(ValueError):
        b.bind(us, [torch.zeros(5, dtype=torch.float64, device=cuda)] * 3)
    with pytest.raises(ValueError):
        fem.Batch(ops[:3], "fp16")
    m = box_mesh((2, 2, 2), 3, seed=0)
    qd = torch.zeros(64 * 8, dtype=torch.float64, device=cuda)
    det = fem.MassOperator(fem.Restriction(8, 27, 1, m.num_nodes, m.num_nodes, m.offsets, 1), fem.Basis(3, 1, 3, 4),
                           qd)
    with pytest.raises(fem.FemUnsupported):
        fem.Batch([ops[0], det], "fp64")


def uneven_batch(fem, cuda, n=24, seed=3):
    """Members of the uneven-mesh workload's family: 2D and 3D boxes, P 2..6,
    Q = P + 1, 1-3 components (vector mass and the component-0-only
    apply_mass), blocked and interleaved layouts, sizes from one element up."""
    V, S = fem.QF.apply_mass_vector, fem.QF.apply_mass
    rng = np.random.default_rng(seed)
    ops, metas = [], []
    for i in range(n):
        dim = 2 + i % 2
        P = 2 + (i // 2) % 5
        nc = 1 + (i // 3) % 3
        shape = tuple(int(x) for x in rng.integers(1, 6 if dim == 3 else 12, size=dim))
        op, meta = make_op(fem, cuda, dim, shape, P, P + 1, nc, V if i % 4 else S, seed=100 + i,
                           interleaved=(i % 5 == 1 and nc > 1))
        ops.append(op)
        metas.append(meta)
    return ops, metas


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_persistent_batch_one_launch(fem, cuda, orc, precision):
    """The whole batch in ONE persistent kernel launch: against each operator's
    own apply (FP64: 1e-13; FP32: against the FP64 apply of the FP32-rounded
    input, 1e-5), against the oracle on members of both dims, in both forms,
    over repeated launches (the ticket is re-armed every time)."""
    import torch
    ops, metas = uneven_batch(fem, cuda)
    dt = torch.float64 if precision == "fp64" else torch.float32
    us = [dev(random_vector(mt["l_size"], 200 + i), cuda, dt) for i, mt in enumerate(metas)]
    vs = [torch.full_like(u, float("nan")) for u in us]
    b = fem.Batch(ops, precision)
    b.bind(us, vs)
    b.set_mode("persistent")
    assert b.info()["graph_kernels"] == 1
    tol = TOL if precision == "fp64" else 1e-5
    for graph in (True, False, True):
        for v in vs:
            v.fill_(float("nan"))
        b.apply(graph=graph)
        b.check()
        for i, op in enumerate(ops):
            want = torch.empty(metas[i]["l_size"], dtype=torch.float64, device=cuda)
            op.apply(us[i].double(), want)
            close(host(vs[i]), host(want), tol)
    for i in (0, 1, 7, 10):
        mt = metas[i]
        want = orc.mass_apply(mt["dim"], mt["ne"], mt["P"], mt["Q"], mt["nc"], mt["cs"], mt["l_size"], mt["offs"],
                              mt["qd"], host(us[i]), vector=mt["vector"])
        close(host(vs[i]), want, tol)
    # the per-class form gives the same results; auto picks one after autotuning
    first = [host(v) for v in vs]
    b.set_mode("classes")
    assert b.info()["graph_kernels"] == b.info()["classes"] + 1
    b.apply()
    for f, v in zip(first, vs):
        close(host(v), f, tol)
    b.set_mode("auto")
    b.autotune(reps=2)
    b.apply()
    b.check()
    for f, v in zip(first, vs):
        close(host(v), f, tol)


def test_persistent_batch_refuses_other_shapes(fem, cuda):
    ops, metas = mixed_batch(fem, cuda)  # 1D members, Q != P + 1, P = 7, 8
    b = fem.Batch(ops, "fp64")
    with pytest.raises(fem.FemUnsupported):
        b.set_mode("persistent")
