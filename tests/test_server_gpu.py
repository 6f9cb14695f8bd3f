"""Served mass solves (GPU): the request loop of fem_b200_server_*.

* a device-generated box request, solved and checked on the host with the
  oracle (undistorted boxes, whose mesh the host generator reproduces):
  ||f - M u|| / ||f|| <= 1e-10 with M from the oracle's build and apply;
* a host-mesh request equals the direct solve through MassOperator.solve to
  the last bit (deterministic scatter: same kernels, fixed-order reductions);
* a request's result is the same alone and in a mix of concurrent requests
  (bitwise with the deterministic scatter; within 1e-8 with atomics, where
  the rounding of the scatter order differs);
* admission by the device-memory budget: requests that do not fit together
  never run together, and the peak stays under the budget.
"""
import numpy as np
import pytest

from fe_demo_cpp_b200.mesh import box_mesh, component_layout, random_vector

pytestmark = pytest.mark.gpu


def oracle_residual(orc, m, P, Q, nc, u, f):
    dim = m.dim
    qd = orc.mass_build(dim, m.num_elem, P, Q, m.num_nodes, m.offsets, m.coords)
    offs, cs, l_size = component_layout(m, nc, False)
    Mu = orc.mass_apply(dim, m.num_elem, P, Q, nc, cs, l_size, offs, qd, u, vector=True)
    return np.linalg.norm(f - Mu) / np.linalg.norm(f)


@pytest.mark.parametrize("dim,shape,P,nc,precision", [(3, (3, 3, 2), 3, 2, "fp32_ir"), (3, (2, 2, 2), 5, 3, "fp64"),
                                                      (2, (6, 5), 4, 1, "fp32_ir"), (2, (4, 4), 2, 3, "fp64")])
def test_box_request_against_the_oracle(fem, orc, cuda, dim, shape, P, nc, precision):
    m = box_mesh(shape, P, seed=0, perturb=0.0)
    n = nc * m.num_nodes
    u, f = np.empty(n), np.empty(n)
    with fem.Server(slots=2, hbm_budget=8 << 30) as srv:
        rid = srv.submit_box(dim, shape, P, num_comp=nc, seed=5, perturb=0.0, rtol=1e-11, precision=precision,
                             u_out=u, f_out=f)
        res = srv.wait(rid)
    assert res["status"] == 0, res["message"]
    assert res["dofs"] == n and res["iterations"] > 0
    assert np.abs(f).max() <= 1.0 and np.abs(f).min() < 0.5  # U[-1, 1]
    rel = oracle_residual(orc, m, P, P + 1, nc, u, f)
    assert rel <= 1e-10, rel
    assert abs(rel - res["rel_residual"]) <= 1e-12


def test_mesh_request_equals_direct_solve(fem, cuda):
    import torch
    P, Q, nc = 4, 5, 2
    m = box_mesh((5, 4, 3), P, seed=3)
    offs, cs, l_size = component_layout(m, nc, False)
    f = random_vector(l_size, 17)
    u_srv = np.empty(l_size)
    with fem.Server(slots=2, hbm_budget=8 << 30) as srv:
        res = srv.wait(srv.submit_mesh(3, P, m.offsets, m.coords, f, num_comp=nc, rtol=1e-11, deterministic=True,
                                       u_out=u_srv))
    assert res["status"] == 0, res["message"]
    rx = fem.Restriction(m.num_elem, P**3, 3, m.num_nodes, 3 * m.num_nodes, m.offsets)
    qd = torch.empty(Q**3 * m.num_elem, dtype=torch.float64, device=cuda)
    fem.mass_build(rx, fem.Basis(3, 3, P, Q), torch.from_numpy(m.coords).to(cuda), qd)
    op = fem.MassOperator(fem.Restriction(m.num_elem, P**3, nc, cs, l_size, offs, 1), fem.Basis(3, nc, P, Q), qd,
                          fem.QF.apply_mass_vector)
    u = torch.empty(l_size, dtype=torch.float64, device=cuda)
    info = op.solve(torch.from_numpy(f).to(cuda), u, rtol=1e-11, max_iter=2000, precision="fp32_ir")
    assert np.array_equal(u.cpu().numpy(), u_srv)
    assert info["iterations"] == res["iterations"] and info["refinements"] == res["refinements"]


MIX = [(3, (6, 5, 4), 3, 1), (2, (40, 30), 4, 3), (3, (4, 4, 4), 5, 3), (3, (8, 8, 6), 2, 1), (2, (12, 12), 6, 2),
       (3, (3, 3, 3), 6, 1), (3, (10, 8, 8), 4, 3), (2, (25, 25), 3, 1), (3, (5, 5, 5), 4, 2)]


@pytest.mark.parametrize("deterministic", [True, False], ids=["deterministic", "atomic"])
def test_result_same_alone_and_in_the_mix(fem, cuda, deterministic):
    shape, P, nc = (5, 4, 4), 4, 3
    n = nc * ((shape[0] * 3 + 1) * (shape[1] * 3 + 1) * (shape[2] * 3 + 1))
    alone = np.empty(n)
    with fem.Server(slots=4, hbm_budget=16 << 30) as srv:
        res_alone = srv.wait(srv.submit_box(3, shape, P, num_comp=nc, seed=11, deterministic=deterministic,
                                            u_out=alone))
        mixed = np.empty(n)
        ids = [srv.submit_box(d, sh, p, num_comp=c, seed=100 + i, deterministic=deterministic,
                              precision="fp32_ir" if i % 2 else "fp64") for i, (d, sh, p, c) in enumerate(MIX[:4])]
        ids.append(srv.submit_box(3, shape, P, num_comp=nc, seed=11, deterministic=deterministic, u_out=mixed))
        ids += [srv.submit_box(d, sh, p, num_comp=c, seed=200 + i, deterministic=deterministic)
                for i, (d, sh, p, c) in enumerate(MIX[4:])]
        results = [srv.wait(i) for i in ids]
        stats = srv.stats()
    assert res_alone["status"] == 0
    for r in results:
        assert r["status"] == 0, r["message"]
        assert r["rel_residual"] <= 1e-10
    if deterministic:
        assert np.array_equal(alone, mixed)
    else:
        assert np.linalg.norm(alone - mixed) / np.linalg.norm(alone) <= 1e-8
    # several requests were on the device at once
    spans = sorted((r["t_start"], r["t_end"]) for r in results)
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))
    assert stats["completed"] == len(ids) + 1 and stats["pending"] == 0 and stats["bytes_in_use"] == 0


def test_budget_admission(fem, cuda):
    shape, P = (8, 8, 8), 4
    with fem.Server(slots=1, hbm_budget=8 << 30) as srv:
        need = srv.wait(srv.submit_box(3, shape, P, seed=1))["device_bytes"]
    budget = int(1.5 * need)  # one request at a time, although there are 4 slots
    with fem.Server(slots=4, hbm_budget=budget) as srv:
        ids = [srv.submit_box(3, shape, P, seed=1 + i) for i in range(4)]
        results = [srv.wait(i) for i in ids]
        stats = srv.stats()
        with pytest.raises(ValueError):
            srv.submit_box(3, (16, 16, 16), P)  # alone above the budget
    spans = sorted((r["t_start"], r["t_end"]) for r in results)
    assert all(spans[i + 1][0] >= spans[i][1] for i in range(len(spans) - 1))
    assert stats["bytes_peak"] <= budget and stats["bytes_peak"] == need


def test_request_errors_and_timeout(fem, cuda):
    with fem.Server(slots=2, hbm_budget=8 << 30) as srv:
        with pytest.raises(fem.FemUnsupported):
            srv.submit_box(3, (2, 2, 2), 9)
        with pytest.raises(ValueError):
            srv.submit_box(4, (2, 2, 2), 3)
        with pytest.raises(ValueError):
            srv.wait(12345)
        rid = srv.submit_box(3, (24, 24, 24), 5, num_comp=3, seed=2)
        try:
            srv.wait(rid, timeout=0.0)
            finished = True
        except TimeoutError:
            finished = False
        if not finished:
            assert srv.wait(rid)["status"] == 0
