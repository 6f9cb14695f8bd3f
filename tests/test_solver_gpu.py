"""Device mass solves (GPU): the assembled Jacobi diagonal and the PCG solves
(FP64, and FP32 or BF16-storage inner PCG in FP64 iterative refinement)
through the C-ABI.

The reference has no solver; these operations sit on top of its mass
operator (include/operator.hpp:137-166 apply, include/qfunctions/mass.hpp
apply_mass).  The checks are against the oracle's mass apply:
  * diagonal: diag_i == e_i^T M e_i from the oracle, normwise 1e-13;
  * solves: f = M u* from the oracle for a random u*, then ||u - u*|| / ||u*||
    <= 1e-9 for rtol 1e-12 (Jacobi-preconditioned mass matrices have
    condition numbers of order 10-100), and the returned FP64 residual
    ||f - M u|| / ||f|| recomputed with the oracle.
"""
import numpy as np
import pytest

from fe_demo_cpp_b200.mesh import box_mesh, component_layout, gll_nodes, random_vector

pytestmark = pytest.mark.gpu
TOL = 1e-13


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


class _Line:
    pass


def line_mesh(n, P, seed):
    """n perturbed cells on [0, 1], P Gauss-Lobatto nodes per cell."""
    rng = np.random.default_rng([seed, 17])
    xv = np.linspace(0, 1, n + 1)
    xv[1:-1] += rng.uniform(-0.1 / n, 0.1 / n, n - 1)
    s = (gll_nodes(P) + 1) / 2
    m = _Line()
    m.dim, m.P, m.num_elem, m.num_nodes = 1, P, n, n * (P - 1) + 1
    m.coords = np.concatenate([xv[e] + (xv[e + 1] - xv[e]) * s[(0 if e == 0 else 1):] for e in range(n)])
    m.offsets = np.array([e * (P - 1) + i for e in range(n) for i in range(P)], dtype=np.int32)
    return m


def mesh(dim, shape, P, seed):
    return line_mesh(shape[0], P, seed) if dim == 1 else box_mesh(shape, P, seed=seed)


def qdata(fem, cuda, m, Q):
    import torch
    rx = fem.Restriction(m.num_elem, m.P**m.dim, m.dim, m.num_nodes, m.dim * m.num_nodes, m.offsets)
    qd = torch.empty(Q**m.dim * m.num_elem, dtype=torch.float64, device=cuda)
    fem.mass_build(rx, fem.Basis(m.dim, m.dim, m.P, Q), dev(m.coords, cuda), qd)
    return qd


def operator(fem, cuda, m, Q, nc=1, interleaved=False, scatter=0):
    qd = qdata(fem, cuda, m, Q)
    if nc == 1:
        offs, cs, l_size = m.offsets, m.num_nodes, m.num_nodes
    else:
        offs, cs, l_size = component_layout(m, nc, interleaved)
    ru = fem.Restriction(m.num_elem, m.P**m.dim, nc, cs, l_size, offs, scatter)
    op = fem.MassOperator(ru, fem.Basis(m.dim, nc, m.P, Q), qd, fem.QF.apply_mass_vector)
    return op, host(qd), offs, cs, l_size


CASES = [(1, (9,), 4, 5, 1), (2, (4, 3), 3, 4, 1), (2, (3, 3), 5, 6, 2), (3, (2, 2, 2), 3, 4, 1),
         (3, (3, 2, 2), 4, 5, 3), (3, (2, 2, 1), 6, 7, 1), (3, (2, 1, 1), 7, 8, 1), (3, (1, 1, 1), 8, 9, 1)]


@pytest.mark.parametrize("dim,shape,P,Q,nc", CASES)
def test_diagonal_matches_oracle_unit_vectors(fem, cuda, orc, dim, shape, P, Q, nc):
    import torch
    m = mesh(dim, shape, P, seed=2)
    op, qd_h, offs, cs, l_size = operator(fem, cuda, m, Q, nc, interleaved=(nc == 3))
    d = torch.full((l_size,), 5.0, dtype=torch.float64, device=cuda)  # overwritten
    op.diagonal(d)
    want = np.empty(l_size)
    for i in range(l_size):
        e = np.zeros(l_size)
        e[i] = 1.0
        want[i] = orc.mass_apply(dim, m.num_elem, P, Q, nc, cs, l_size, offs, qd_h, e, vector=True)[i]
    got = host(d)
    assert np.all(want > 0)
    assert np.abs(got - want).max() <= TOL * want.max()


def _solve_check(fem, cuda, orc, op, m, Q, nc, qd_h, offs, cs, l_size, precision, seed):
    import torch
    u_star = random_vector(l_size, seed)
    f = orc.mass_apply(m.dim, m.num_elem, m.P, Q, nc, cs, l_size, offs, qd_h, u_star, vector=True)
    u = torch.full((l_size,), 3.0, dtype=torch.float64, device=cuda)  # initial contents ignored
    info = op.solve(dev(f, cuda), u, rtol=1e-12, max_iter=2000, precision=precision)
    u_h = host(u)
    err = np.linalg.norm(u_h - u_star) / np.linalg.norm(u_star)
    assert err <= 1e-9, (precision, err, info)
    res = f - orc.mass_apply(m.dim, m.num_elem, m.P, Q, nc, cs, l_size, offs, qd_h, u_h, vector=True)
    rel = np.linalg.norm(res) / np.linalg.norm(f)
    assert rel <= 1e-11, (precision, rel, info)
    assert abs(info["rel_residual"] - rel) <= 1e-13 + 0.05 * rel
    assert 0 < info["iterations"] <= 2000
    return info, u_h


@pytest.mark.parametrize("dim,shape,P,Q,nc", CASES)
def test_fp64_solve_recovers_solution(fem, cuda, orc, dim, shape, P, Q, nc):
    m = mesh(dim, shape, P, seed=4)
    op, qd_h, offs, cs, l_size = operator(fem, cuda, m, Q, nc)
    info, _ = _solve_check(fem, cuda, orc, op, m, Q, nc, qd_h, offs, cs, l_size, "fp64", 11)
    assert info["refinements"] == 0


@pytest.mark.parametrize("dim,shape,P,Q,nc", CASES)
def test_fp32_refinement_reaches_fp64_accuracy(fem, cuda, orc, dim, shape, P, Q, nc):
    m = mesh(dim, shape, P, seed=6)
    op, qd_h, offs, cs, l_size = operator(fem, cuda, m, Q, nc)
    info, u32 = _solve_check(fem, cuda, orc, op, m, Q, nc, qd_h, offs, cs, l_size, "fp32_ir", 12)
    assert info["refinements"] >= 2  # 1e-12 is out of reach of one FP32 inner solve
    _, u64 = _solve_check(fem, cuda, orc, op, m, Q, nc, qd_h, offs, cs, l_size, "fp64", 12)
    assert np.linalg.norm(u32 - u64) / np.linalg.norm(u64) <= 1e-9


@pytest.mark.parametrize("dim,shape,P,Q,nc", CASES)
def test_bf16_refinement_reaches_fp64_accuracy(fem, cuda, orc, dim, shape, P, Q, nc):
    """BF16 r, p, s and qdata in the inner PCG: each inner solve gains about
    two digits, the FP64 refinement still reaches rtol 1e-12, and the result
    agrees with the FP64 solve to 1e-9 (within 1e-10 of it at rtol 1e-12)."""
    m = mesh(dim, shape, P, seed=8)
    op, qd_h, offs, cs, l_size = operator(fem, cuda, m, Q, nc)
    info, u16 = _solve_check(fem, cuda, orc, op, m, Q, nc, qd_h, offs, cs, l_size, "bf16_ir", 13)
    assert info["refinements"] >= 4  # 1e-12 is many BF16 inner solves away
    _, u64 = _solve_check(fem, cuda, orc, op, m, Q, nc, qd_h, offs, cs, l_size, "fp64", 13)
    assert np.linalg.norm(u16 - u64) / np.linalg.norm(u64) <= 1e-9


@pytest.mark.parametrize("precision,apply", [("fp32_ir", "apply_f32"), ("bf16_ir", "apply_bf16")])
def test_solve_after_reduced_precision_apply(fem, cuda, orc, precision, apply):
    """An FP32 / BF16 apply first makes the plan's reduced-precision qdata;
    the solve then still sets up the rest of its state."""
    import torch
    m = box_mesh((3, 2, 2), 4, seed=5)
    op, qd_h, offs, cs, l_size = operator(fem, cuda, m, 5)
    dt = torch.float32 if apply == "apply_f32" else torch.bfloat16
    getattr(op, apply)(torch.ones(l_size, dtype=dt, device=cuda), torch.empty(l_size, dtype=torch.float32,
                                                                                device=cuda))
    _solve_check(fem, cuda, orc, op, m, 5, 1, qd_h, offs, cs, l_size, precision, 41)


@pytest.mark.parametrize("scatter", [0, 1], ids=["atomic", "deterministic"])
@pytest.mark.parametrize("variant", [1, 2, 3, 4, 5, 6])
def test_solve_with_every_kernel_variant(fem, cuda, orc, scatter, variant):
    """The FP64 solve runs the plan's selected apply kernel; the FP32 inner
    apply is the simple kernel in every variant."""
    m = box_mesh((5, 4, 3), 4, seed=3)
    op, qd_h, offs, cs, l_size = operator(fem, cuda, m, 5, scatter=scatter)
    op.set_kernel(variant)
    for prec in ("fp64", "fp32_ir", "bf16_ir"):
        _solve_check(fem, cuda, orc, op, m, 5, 1, qd_h, offs, cs, l_size, prec, 20 + variant)


def test_solve_larger_mesh_iteration_counts(fem, cuda):
    """40x30x20 hexes, P=5: Jacobi-PCG iteration counts on the mass matrix are
    mesh-independent (tens of iterations), and every precision meets rtol."""
    import torch
    m = box_mesh((40, 30, 20), 5, seed=1)
    op, _, _, _, l_size = operator(fem, cuda, m, 6)
    g = torch.Generator(device=cuda).manual_seed(3)
    u_star = torch.rand(l_size, dtype=torch.float64, device=cuda, generator=g) - 0.5
    f = torch.empty_like(u_star)
    op.apply(u_star, f)
    for prec in ("fp64", "fp32_ir", "bf16_ir"):
        u = torch.empty_like(u_star)
        info = op.solve(f, u, rtol=1e-11, max_iter=1000, precision=prec)
        assert info["rel_residual"] <= 1e-10, (prec, info)
        assert info["iterations"] <= (200 if prec != "bf16_ir" else 400), (prec, info)
        err = float((u - u_star).norm() / u_star.norm())
        assert err <= 1e-8, (prec, err)


def test_zero_rhs_and_argument_errors(fem, cuda):
    import torch
    m = box_mesh((2, 2, 2), 3, seed=0)
    op, _, _, _, l_size = operator(fem, cuda, m, 4)
    f = torch.zeros(l_size, dtype=torch.float64, device=cuda)
    u = torch.full((l_size,), 9.0, dtype=torch.float64, device=cuda)
    info = op.solve(f, u)
    assert info == {"iterations": 0, "refinements": 0, "rel_residual": 0.0}
    assert float(u.abs().max()) == 0.0
    with pytest.raises(ValueError):
        op.solve(f, u, rtol=0.0)
    with pytest.raises(ValueError):
        op.solve(f, u, max_iter=0)
    with pytest.raises(ValueError):
        op.solve(f[:-1], u)
    with pytest.raises(ValueError):
        op.diagonal(torch.empty(l_size + 1, dtype=torch.float64, device=cuda))


def test_component0_apply_mass_is_not_solvable(fem, cuda):
    """The reference apply_mass leaves components 1.. at zero (a singular
    operator for num_comp > 1): the solve refuses it."""
    import torch
    m = box_mesh((2, 2, 2), 3, seed=0)
    qd = qdata(fem, cuda, m, 4)
    offs, cs, l_size = component_layout(m, 3, False)
    op = fem.MassOperator(fem.Restriction(m.num_elem, 27, 3, cs, l_size, offs), fem.Basis(3, 3, 3, 4), qd,
                          fem.QF.apply_mass)
    f = torch.ones(l_size, dtype=torch.float64, device=cuda)
    with pytest.raises(fem.FemUnsupported):
        op.solve(f, torch.empty_like(f))


@pytest.mark.parametrize("precision", ["fp64", "fp32_ir", "bf16_ir"])
def test_deterministic_solve_is_bitwise_reproducible(fem, cuda, precision):
    """Deterministic plans: transpose-map scatter and fixed-order grid
    reductions, so a repeated solve reproduces every bit."""
    import torch
    m = box_mesh((7, 6, 5), 4, seed=2)
    op, _, _, _, l_size = operator(fem, cuda, m, 5, nc=2, scatter=1)
    f = dev(random_vector(l_size, 31), cuda)
    out = []
    for _ in range(3):
        u = torch.empty_like(f)
        info = op.solve(f, u, rtol=1e-11, precision=precision)
        out.append((host(u), info))
    for u_h, info in out[1:]:
        assert np.array_equal(u_h, out[0][0])
        assert info == out[0][1]


def _oracle_apply_chunked(orc, m, qd_h, u_h, P, Q, slabs=8):
    """The scalar mass apply of the whole mesh through the oracle, in chunks
    of z-slabs (each a self-contained mesh, nodes renumbered compactly) run in
    parallel threads and added into the global vector in chunk order."""
    import concurrent.futures as cf
    import os
    nx, ny, nz = m.shape
    ne_slab, es, nq = nx * ny, P**3, Q**3
    bounds = [(z0 * ne_slab, min(nz, z0 + slabs) * ne_slab) for z0 in range(0, nz, slabs)]
    qd2 = qd_h.reshape(nq, m.num_elem)

    def chunk(lo_hi):
        lo, hi = lo_hi
        nodes, local = np.unique(m.offsets[lo * es: hi * es], return_inverse=True)
        q = np.ascontiguousarray(qd2[:, lo:hi]).reshape(-1)
        n = int(nodes.size)
        return nodes, orc.mass_apply(3, hi - lo, P, Q, 1, n, n, local.astype(np.int32), q, u_h[nodes])

    out = np.zeros(m.num_nodes)
    with cf.ThreadPoolExecutor(max_workers=min(len(bounds), os.cpu_count() or 1)) as ex:
        for nodes, vloc in ex.map(chunk, bounds):
            out[nodes] += vloc
    return out


@pytest.mark.parametrize("precision", ["fp32_ir", "bf16_ir", "fp64"])
def test_full_size_solve_residual_against_oracle(fem, cuda, orc, precision):
    """The solve benchmark's configuration at its full size: 64^3 hexes, P=5,
    Q=6, three components (vector mass, 50.9M DoFs), rtol 1e-10.  The true
    residual ||f - M u|| / ||f|| of the returned u is recomputed with the
    oracle's apply, component by component over the whole mesh, and must meet
    rtol (1.05x margin for the two applies' rounding) and agree with the
    residual the solve reports."""
    import torch
    P, Q, nc = 5, 6, 3
    m = box_mesh((64, 64, 64), P, seed=1)
    N = m.num_nodes
    qd = qdata(fem, cuda, m, Q)
    op = fem.MassOperator(fem.Restriction(m.num_elem, P**3, nc, N, nc * N, m.offsets), fem.Basis(3, nc, P, Q), qd,
                          fem.QF.apply_mass_vector)
    g = torch.Generator(device=cuda).manual_seed(1)
    f = torch.rand(nc * N, dtype=torch.float64, device=cuda, generator=g) * 2 - 1
    u = torch.empty_like(f)
    info = op.solve(f, u, rtol=1e-10, max_iter=2000, precision=precision)
    assert info["rel_residual"] <= 1e-10, info
    qd_h, u_h, f_h = host(qd), host(u), host(f)
    del qd, u, f, op
    res2 = 0.0
    for k in range(nc):
        mu = _oracle_apply_chunked(orc, m, qd_h, u_h[k * N:(k + 1) * N], P, Q)
        res2 += float(np.sum((f_h[k * N:(k + 1) * N] - mu) ** 2))
    rel = np.sqrt(res2) / np.linalg.norm(f_h)
    assert rel <= 1.05e-10, (precision, rel, info)
    assert abs(rel - info["rel_residual"]) <= 0.05 * rel + 1e-14, (rel, info)
