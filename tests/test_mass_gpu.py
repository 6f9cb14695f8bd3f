"""Device parity: the fused mass kernels against the oracle (GPU).

Tolerances (FP64): the device contracts in another axis order and with FMA,
so values agree to rounding.  Every comparison is normwise,
max|x - x_oracle| <= TOL * max|x_oracle| with TOL = 1e-13 (the reference's
own GPU tolerance, tests/cuda/test-cuda-elem-restriction.cu:51-57); integer
and index work (gather, multiplicity, transpose map) is compared bitwise.
"""
import numpy as np
import pytest

from fe_demo_cpp_b200.mesh import box_mesh, component_layout, mesh_for_dofs, random_vector

pytestmark = pytest.mark.gpu
TOL = 1e-13


def close(got, want, tol=TOL):
    got, want = np.asarray(got), np.asarray(want)
    assert got.shape == want.shape
    scale = max(np.abs(want).max(), 1e-300)
    err = np.abs(got - want).max() / scale
    assert err <= tol, f"normwise relative error {err:.3e} > {tol:.0e}"


def dev(a, cuda, dtype=None):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a))
    return t.to(device=cuda, dtype=dtype) if dtype is not None else t.to(cuda)


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def build_qdata(fem, cuda, m, Q, quad_mode=0):
    import torch
    rx = fem.Restriction(m.num_elem, m.P**m.dim, m.dim, m.num_nodes, m.dim * m.num_nodes, m.offsets)
    bx = fem.Basis(m.dim, m.dim, m.P, Q, quad_mode)
    qd = torch.empty(Q**m.dim * m.num_elem, dtype=torch.float64, device=cuda)
    fem.mass_build(rx, bx, dev(m.coords, cuda), qd)
    return qd


SHAPES = [(1, (7,), 2, 3), (1, (300,), 5, 6), (2, (5, 4), 4, 5), (2, (9, 7), 3, 4), (3, (8, 8, 8), 4, 5),
          (3, (3, 3, 3), 5, 6), (3, (2, 3, 4), 2, 3), (3, (1, 1, 1), 6, 7), (3, (4, 3, 2), 8, 9), (3, (3, 2, 2), 7, 8)]


def _mesh(dim, shape, P, seed):
    if dim == 1:  # a perturbed 1D line: node x at GLL positions of perturbed cells
        n = shape[0]
        from fe_demo_cpp_b200.mesh import gll_nodes
        rng = np.random.default_rng([seed, 17])
        xv = np.linspace(0, 1, n + 1)
        xv[1:-1] += rng.uniform(-0.1 / n, 0.1 / n, n - 1)
        s = (gll_nodes(P) + 1) / 2
        nodes = np.concatenate([xv[e] + (xv[e + 1] - xv[e]) * s[(0 if e == 0 else 1):] for e in range(n)])
        offs = np.array([e * (P - 1) + i for e in range(n) for i in range(P)], dtype=np.int32)

        class M1:
            pass
        m = M1()
        m.dim, m.P, m.num_elem, m.num_nodes, m.offsets, m.coords = 1, P, n, n * (P - 1) + 1, offs, nodes
        return m
    return box_mesh(shape, P, seed=seed)


@pytest.mark.parametrize("dim,shape,P,Q", SHAPES)
def test_build_qdata_matches_oracle(fem, cuda, orc, dim, shape, P, Q):
    """J = sum_p G_qp x_p is formed from O(1) absolute coordinates whose
    differences are O(h): the reference and the device both lose about
    log10(1/h) digits to that cancellation (with different rounding), so
    qdata is compared at TOL / h, h = 1 / (elements per side)."""
    m = _mesh(dim, shape, P, seed=3)
    qd = host(build_qdata(fem, cuda, m, Q))
    want = orc.mass_build(dim, m.num_elem, P, Q, m.num_nodes, m.offsets, m.coords)
    close(qd, want, TOL * max(shape))


@pytest.mark.parametrize("variant", [1, 2, 3, 4, 5, 6, 7],
                         ids=["simple", "pipelined", "paired", "prefetch", "occupancy", "narrow", "element"])
@pytest.mark.parametrize("scatter", [0, 1], ids=["atomic", "deterministic"])
@pytest.mark.parametrize("dim,shape,P,Q", SHAPES)
def test_apply_matches_oracle(fem, cuda, orc, dim, shape, P, Q, scatter, variant):
    import torch
    if variant in (2, 3, 4, 5, 6, 7) and dim != 3:
        pytest.skip("the pipelined, paired, prefetching, occupancy, narrow and element kernels are 3D only")
    if variant == 7 and P > 3:
        pytest.skip("the element-per-thread kernel covers P <= 3")
    m = _mesh(dim, shape, P, seed=5)
    qd = build_qdata(fem, cuda, m, Q)
    qd_h = host(qd)
    ru = fem.Restriction(m.num_elem, P**dim, 1, m.num_nodes, m.num_nodes, m.offsets, scatter)
    bu = fem.Basis(dim, 1, P, Q)
    op = fem.MassOperator(ru, bu, qd)
    op.set_kernel(variant)
    assert op.info()["kernel"] == fem.KernelVariant(variant).name
    u = random_vector(m.num_nodes, 6)
    v = torch.full((m.num_nodes,), 7.0, dtype=torch.float64, device=cuda)  # garbage: apply overwrites
    op.apply(dev(u, cuda), v)
    op.check()
    want = orc.mass_apply(dim, m.num_elem, P, Q, 1, m.num_nodes, m.num_nodes, m.offsets, qd_h, u)
    close(host(v), want)


@pytest.mark.parametrize("interleaved", [False, True], ids=["blocked", "interleaved"])
@pytest.mark.parametrize("P,Q", [(3, 4), (5, 6)])
def test_three_components(fem, cuda, orc, P, Q, interleaved):
    import torch
    m = box_mesh((3, 2, 2), P, seed=7)
    qd = build_qdata(fem, cuda, m, Q)
    qd_h = host(qd)
    offs, cs, l_size = component_layout(m, 3, interleaved)
    u = random_vector(l_size, 8)
    ru = fem.Restriction(m.num_elem, P**3, 3, cs, l_size, offs)
    bu = fem.Basis(3, 3, P, Q)
    for (qf, vector), variant in [(q, k) for q in ((fem.QF.apply_mass_vector, True), (fem.QF.apply_mass, False))
                                  for k in (1, 2, 3, 4, 5, 6)]:
        op = fem.MassOperator(ru, bu, qd, qf)
        op.set_kernel(variant)
        v = torch.empty(l_size, dtype=torch.float64, device=cuda)
        op.apply(dev(u, cuda), v)
        want = orc.mass_apply(3, m.num_elem, P, Q, 3, cs, l_size, offs, qd_h, u, vector=vector)
        close(host(v), want)
        if not vector:  # the reference apply_mass leaves components 1, 2 at exactly 0
            comp = np.zeros(l_size, dtype=bool)
            for k in (1, 2):
                comp[offs.astype(np.int64) + k * cs] = True
            assert np.all(host(v)[comp] == 0.0)


def test_golden_config1_matches_reference(fem, cuda, golden):
    """8^3 hexes, P=4, Q=5, seed 1: v against the reference's own output."""
    import torch
    name = "mass_d3_8x8x8_P4_Q5_s1"
    m = box_mesh((8, 8, 8), 4, seed=1)
    assert m.digest() == str(golden[name + "_mesh_sha"])
    qd = build_qdata(fem, cuda, m, 5)
    close(host(qd).reshape(-1, m.num_elem).sum(0), golden[name + "_qdata_elemsum"], TOL * 8)
    for scatter in (0, 1):
        op = fem.MassOperator(fem.Restriction(m.num_elem, 64, 1, m.num_nodes, m.num_nodes, m.offsets, scatter),
                              fem.Basis(3, 1, 4, 5), qd)
        v = torch.empty(m.num_nodes, dtype=torch.float64, device=cuda)
        op.apply(dev(random_vector(m.num_nodes, 1), cuda), v)
        close(host(v), golden[name + "_v"])


def test_deterministic_is_bitwise_reproducible(fem, cuda):
    import torch
    m = box_mesh((10, 9, 8), 4, seed=9)
    qd = build_qdata(fem, cuda, m, 5)
    op = fem.MassOperator(fem.Restriction(m.num_elem, 64, 1, m.num_nodes, m.num_nodes, m.offsets, 1),
                          fem.Basis(3, 1, 4, 5), qd)
    u = dev(random_vector(m.num_nodes, 2), cuda)
    first = None
    for _ in range(5):
        v = torch.empty(m.num_nodes, dtype=torch.float64, device=cuda)
        op.apply(u, v)
        if first is None:
            first = host(v)
        else:
            assert np.array_equal(host(v), first)


def test_apply_add_and_host_path(fem, cuda):
    import torch
    m = box_mesh((5, 4, 3), 5, seed=4)
    qd = build_qdata(fem, cuda, m, 6)
    op = fem.MassOperator(fem.Restriction(m.num_elem, 125, 1, m.num_nodes, m.num_nodes, m.offsets),
                          fem.Basis(3, 1, 5, 6), qd)
    u = random_vector(m.num_nodes, 3)
    v = torch.empty(m.num_nodes, dtype=torch.float64, device=cuda)
    op.apply(dev(u, cuda), v)
    v1 = host(v)
    base = random_vector(m.num_nodes, 4)
    w = dev(base, cuda)
    op.apply_add(dev(u, cuda), w)
    close(host(w), base + v1, 1e-15 * 10)
    v_host = op.apply_host(u)
    close(v_host, v1, 1e-15 * 10)


def test_tail_tiles_and_single_element(fem, cuda, orc):
    import torch
    for shape in [(1, 1, 1), (3, 1, 1), (9, 1, 1), (17, 1, 1)]:
        m = box_mesh(shape, 4, seed=1)
        qd = build_qdata(fem, cuda, m, 5)
        op = fem.MassOperator(fem.Restriction(m.num_elem, 64, 1, m.num_nodes, m.num_nodes, m.offsets),
                              fem.Basis(3, 1, 4, 5), qd)
        u = random_vector(m.num_nodes, 2)
        v = torch.empty(m.num_nodes, dtype=torch.float64, device=cuda)
        op.apply(dev(u, cuda), v)
        close(host(v), orc.mass_apply(3, m.num_elem, 4, 5, 1, m.num_nodes, m.num_nodes, m.offsets, host(qd), u))


@pytest.mark.parametrize("P,Q", [(2, 3), (3, 4), (4, 5), (5, 6), (6, 7), (8, 9)])
def test_pipelined_equals_simple_on_many_tiles(fem, cuda, P, Q):
    """Several tiles per persistent CTA (a mesh larger than one wave), the
    deterministic mode so that variants contracting in the same order compare
    bitwise (the variants the shape has).  At P >= 4 the one-tile and the
    pipelined kernels use the even-odd contractions (regrouped sums):
    those two are bitwise equal to each other and normwise within 1e-14 of the
    others, which stay bitwise equal among themselves."""
    import torch
    m = box_mesh((40, 30, 20), P, seed=8)
    qd = build_qdata(fem, cuda, m, Q)
    op = fem.MassOperator(fem.Restriction(m.num_elem, P**3, 1, m.num_nodes, m.num_nodes, m.offsets, 1),
                          fem.Basis(3, 1, P, Q), qd)
    u = dev(random_vector(m.num_nodes, 2), cuda)
    out = {}
    for variant in (1, 2, 3, 4, 5, 6, 7):
        try:
            op.set_kernel(variant)
        except fem.FemUnsupported:
            continue
        v = torch.empty(m.num_nodes, dtype=torch.float64, device=cuda)
        op.apply(u, v)
        op.check()
        out[variant] = host(v)
    assert len(out) >= 5
    even_odd = P >= 4
    eo_group = {1, 2} if even_odd else set()
    direct = [k for k in out if k not in eo_group]
    for group in (sorted(eo_group & set(out)), direct):
        for variant in group[1:]:
            assert np.array_equal(out[group[0]], out[variant]), (group[0], variant)
    if eo_group and direct:
        for variant in eo_group & set(out):
            close(out[variant], out[direct[0]], 1e-14)


def test_autotune_picks_a_variant_and_keeps_parity(fem, cuda, orc):
    import torch
    m = box_mesh((12, 10, 9), 5, seed=3)
    qd = build_qdata(fem, cuda, m, 6)
    op = fem.MassOperator(fem.Restriction(m.num_elem, 125, 1, m.num_nodes, m.num_nodes, m.offsets),
                          fem.Basis(3, 1, 5, 6), qd)
    u = dev(random_vector(m.num_nodes, 1), cuda)
    scratch = torch.empty_like(u)
    name, ms = op.autotune(u, scratch, reps=3)
    assert name in ("simple", "pipelined", "paired", "prefetch", "occupancy", "narrow", "element") and ms > 0
    assert op.info()["kernel"] == name
    v = torch.empty_like(u)
    op.apply(u, v)
    close(host(v), orc.mass_apply(3, m.num_elem, 5, 6, 1, m.num_nodes, m.num_nodes, m.offsets, host(qd), host(u)))
    # a new plan of the same shape starts from the tuned choice
    op2 = fem.MassOperator(fem.Restriction(m.num_elem, 125, 1, m.num_nodes, m.num_nodes, m.offsets),
                           fem.Basis(3, 1, 5, 6), qd)
    assert op2.info()["kernel"] == name


def test_pipelined_unavailable_where_smem_does_not_fit(fem, cuda):
    import torch
    m = box_mesh((1, 1, 1), 8, seed=0)
    op = fem.MassOperator(fem.Restriction(1, 512, 1, m.num_nodes, m.num_nodes, m.offsets), fem.Basis(3, 1, 8, 10),
                          torch.zeros(1000, dtype=torch.float64, device=cuda))
    assert op.info()["kernel"] in ("simple", "paired")
    with pytest.raises(fem.FemUnsupported):
        op.set_kernel(2)


def test_unsupported_shape_fails_loudly(fem, cuda):
    import torch
    m = box_mesh((1, 1, 1), 9, seed=0)
    r = fem.Restriction(1, 729, 1, m.num_nodes, m.num_nodes, m.offsets)
    b = fem.Basis(3, 1, 9, 10)
    qd = torch.zeros(1000, dtype=torch.float64, device=cuda)
    with pytest.raises(fem.FemUnsupported):
        fem.MassOperator(r, b, qd)


def test_argument_errors(fem, cuda):
    import torch
    m = box_mesh((2, 2, 2), 3, seed=0)
    r = fem.Restriction(8, 27, 1, m.num_nodes, m.num_nodes, m.offsets)
    b = fem.Basis(3, 1, 3, 4)
    with pytest.raises(ValueError):
        fem.MassOperator(r, b, torch.zeros(10, dtype=torch.float64, device=cuda))  # qdata size
    op = fem.MassOperator(r, b, torch.zeros(64 * 8, dtype=torch.float64, device=cuda))
    with pytest.raises(ValueError):
        op.apply(torch.zeros(5, dtype=torch.float64, device=cuda),
                 torch.zeros(m.num_nodes, dtype=torch.float64, device=cuda))
    with pytest.raises(ValueError):
        fem.MassOperator(r, fem.Basis(3, 1, 4, 5), torch.zeros(125 * 8, dtype=torch.float64, device=cuda))


@pytest.mark.parametrize("P", [2, 3, 4, 5, 6, 7, 8])
@pytest.mark.parametrize("nc", [1, 3])
def test_order_sweep_parity(fem, cuda, orc, P, nc):
    """The order-sweep family (P = 2..8, Q = P+1, num_comp 1 and 3) at small size."""
    import torch
    m = box_mesh((3, 2, 2), P, seed=P)
    Q = P + 1
    qd = build_qdata(fem, cuda, m, Q)
    offs, cs, l_size = component_layout(m, nc, interleaved=False)
    u = random_vector(l_size, 40 + P)
    op = fem.MassOperator(fem.Restriction(m.num_elem, P**3, nc, cs, l_size, offs), fem.Basis(3, nc, P, Q), qd,
                          fem.QF.apply_mass_vector)
    v = torch.empty(l_size, dtype=torch.float64, device=cuda)
    op.apply(dev(u, cuda), v)
    close(host(v), orc.mass_apply(3, m.num_elem, P, Q, nc, cs, l_size, offs, host(qd), u, vector=True))


def test_full_size_properties(fem, cuda, orc):
    """~64M DoFs (100^3 hexes, P=5, Q=6): size-independent properties, and the
    whole mesh through the oracle.

    The oracle runs the elements in chunks of ten z-slabs (each chunk a
    self-contained mesh with its nodes renumbered compactly), in parallel
    threads; the chunks' contributions are then added into the global vector
    in chunk order, so the reference sum over elements is formed in one fixed
    order and every DoF of the device result is checked."""
    import concurrent.futures as cf
    import os

    import torch
    shape = mesh_for_dofs(64_000_000, 5)
    m = box_mesh(shape, 5, seed=1)
    N = m.num_nodes
    qd = build_qdata(fem, cuda, m, 6)
    qsum = float(qd.sum())
    assert abs(qsum - 1.0) <= 1e-11  # volume of the unit box
    ru = fem.Restriction(m.num_elem, 125, 1, N, N, m.offsets)
    bu = fem.Basis(3, 1, 5, 6)
    op = fem.MassOperator(ru, bu, qd)
    ones = torch.ones(N, dtype=torch.float64, device=cuda)
    v = torch.empty(N, dtype=torch.float64, device=cuda)
    op.apply(ones, v)
    assert abs(float(v.sum()) - 1.0) <= 1e-11  # 1^T M 1
    del ones
    g = torch.Generator(device=cuda).manual_seed(5)
    u = torch.rand(N, dtype=torch.float64, device=cuda, generator=g) * 2 - 1
    w = torch.rand(N, dtype=torch.float64, device=cuda, generator=g) * 2 - 1
    Mu, Mw = torch.empty_like(u), torch.empty_like(u)
    op.apply(u, Mu)
    op.apply(w, Mw)
    a, b = float(w @ Mu), float(u @ Mw)
    assert abs(a - b) <= 1e-12 * abs(a)  # symmetry
    Mlin = torch.empty_like(u)
    op.apply(2.0 * u - 3.0 * w, Mlin)
    err = float((Mlin - (2.0 * Mu - 3.0 * Mw)).abs().max() / Mlin.abs().max())
    assert err <= 1e-13  # linearity
    del w, Mw, Mlin
    # every element through the oracle, chunked by z-slabs
    nx, ny, nz = shape
    ne_slab = nx * ny
    qd_h = host(qd).reshape(216, m.num_elem)
    u_h = host(u)
    bounds = [(z0 * ne_slab, min(nz, z0 + 10) * ne_slab) for z0 in range(0, nz, 10)]

    def chunk(lo_hi):
        lo, hi = lo_hi
        sub = m.offsets[lo * 125: hi * 125]
        nodes, local = np.unique(sub, return_inverse=True)
        q = np.ascontiguousarray(qd_h[:, lo:hi]).reshape(-1)
        n = int(nodes.size)
        return nodes, orc.mass_apply(3, hi - lo, 5, 6, 1, n, n, local.astype(np.int32), q, u_h[nodes])

    want = np.zeros(N)
    with cf.ThreadPoolExecutor(max_workers=min(len(bounds), os.cpu_count() or 1)) as ex:
        for nodes, vloc in ex.map(chunk, bounds):  # results in chunk order
            want[nodes] += vloc
    close(host(Mu), want)
