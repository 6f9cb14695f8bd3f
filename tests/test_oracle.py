"""Pins the oracle (oracle/fem_oracle.c) to the reference.

Three kinds of evidence, all on the CPU:
  * fixtures written by the reference itself (tests/golden/make_golden.py):
    the restatement must reproduce them bitwise;
  * the known answers of the reference's own tests, restated (file:line cited);
  * the live reference build (oracle/_ref), where it exists, on fresh inputs.
"""
import hashlib

import numpy as np
import pytest

from fe_demo_cpp_b200.mesh import box_mesh, component_layout, random_vector


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# ---------------------------------------------------------------------------
# fixtures from the reference
# ---------------------------------------------------------------------------
def test_basis_matches_reference_fixtures_bitwise(orc, golden):
    n = 0
    for key in golden.files:
        if key.startswith("basis_") and key.endswith("_qref"):
            stem = key[: -len("_qref")]
            _, p, q, m = stem.split("_")
            P, Q, mode = int(p[1:]), int(q[1:]), int(m[1:])
            got = orc.basis(3, 1, P, Q, mode)
            for arr, suffix in zip(got, ("_qref", "_qw", "_B", "_G")):
                assert np.array_equal(arr, golden[stem + suffix]), (stem, suffix)
            n += 1
    assert n > 50


def _case(name):
    # mass_d{dim}_{shape}_P{P}_Q{Q}_s{seed}
    parts = name.split("_")
    dim = int(parts[1][1:])
    shape = tuple(int(s) for s in parts[2].split("x"))
    return dim, shape, int(parts[3][1:]), int(parts[4][1:]), int(parts[5][1:])


def test_mass_operator_matches_reference_fixtures_bitwise(orc, golden):
    for name in golden["mass_cases"]:
        dim, shape, P, Q, seed = _case(str(name))
        m = box_mesh(shape, P, seed=seed)
        assert m.digest() == str(golden[name + "_mesh_sha"]), f"{name}: mesh generator drifted"
        qd = orc.mass_build(dim, m.num_elem, P, Q, m.num_nodes, m.offsets, m.coords)
        assert sha(qd) == str(golden[name + "_qdata_sha"]), name
        u = random_vector(m.num_nodes, seed)
        v = orc.mass_apply(dim, m.num_elem, P, Q, 1, m.num_nodes, m.num_nodes, m.offsets, qd, u)
        assert sha(v) == str(golden[name + "_v_sha"]), name
        if name + "_v" in golden.files:
            assert np.array_equal(v, golden[name + "_v"])


def test_mass_volume_is_one(golden):
    # the perturbation keeps the unit box: sum(qdata) = 1^T M 1 = 1
    for name in golden["mass_cases"]:
        vol = golden[name + "_volume"]
        np.testing.assert_allclose(vol, 1.0, rtol=0, atol=1e-12)


def test_three_components_match_reference_fixtures_bitwise(orc, golden):
    m = box_mesh((3, 2, 2), 3, seed=7)
    qd = orc.mass_build(3, m.num_elem, 3, 4, m.num_nodes, m.offsets, m.coords)
    assert np.array_equal(qd, golden["c3_qdata"])
    for inter in (False, True):
        tag = "inter" if inter else "blocked"
        offs, cs, l_size = component_layout(m, 3, inter)
        u = random_vector(l_size, 8)
        v_ref = orc.mass_apply(3, m.num_elem, 3, 4, 3, cs, l_size, offs, qd, u)
        assert np.array_equal(v_ref, golden[f"c3_{tag}_v_ref"])
        v_vec = orc.mass_apply(3, m.num_elem, 3, 4, 3, cs, l_size, offs, qd, u, vector=True)
        assert np.array_equal(v_vec, golden[f"c3_{tag}_v_vector"])
        assert np.array_equal(orc.gather(m.num_elem, 27, 3, cs, offs, u), golden[f"c3_{tag}_gather"])
        e_in = random_vector(3 * 27 * m.num_elem, 9)
        got = orc.scatter_add(m.num_elem, 27, 3, cs, offs, e_in, np.ones(l_size))
        assert np.array_equal(got, golden[f"c3_{tag}_scatter"])
        assert np.array_equal(orc.multiplicity(m.num_elem, 27, 3, cs, l_size, offs), golden[f"c3_{tag}_mult"])


def test_apply_mass_reference_quirk_component_zero_only(golden):
    # include/qfunctions/mass.hpp:45-51 loops over component 0 only, so the
    # reference's v is exactly 0 on components 1 and 2
    m = box_mesh((3, 2, 2), 3, seed=7)
    v = golden["c3_blocked_v_ref"]
    assert np.all(v[m.num_nodes:] == 0.0)
    assert np.array_equal(v[: m.num_nodes], golden["c3_blocked_v_vector"][: m.num_nodes])


def test_basis_actions_match_reference_fixtures_bitwise(orc, golden):
    for dim in (1, 2, 3):
        for nc in (1, 3):
            P, Q, ne = 3, 5, 2
            _, w1, B, G = orc.basis(dim, nc, P, Q)
            u = random_vector(nc * P**dim * ne, 10 + dim)
            w = random_vector(nc * Q**dim * ne, 20 + dim)
            g = random_vector(dim * nc * Q**dim * ne, 30 + dim)
            key = f"bapply_d{dim}_c{nc}"
            assert np.array_equal(orc.interp(dim, nc, P, Q, B, ne, 0, u), golden[key + "_interp"])
            assert np.array_equal(orc.interp(dim, nc, P, Q, B, ne, 1, w), golden[key + "_interpT"])
            assert np.array_equal(orc.grad(dim, nc, P, Q, B, G, ne, 0, u), golden[key + "_grad"])
            assert np.array_equal(orc.grad(dim, nc, P, Q, B, G, ne, 1, g), golden[key + "_gradT"])
            assert np.array_equal(orc.weight(dim, Q, w1, ne), golden[key + "_weight"])


# ---------------------------------------------------------------------------
# the live reference build, fresh inputs
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("dim,shape,P,Q", [(3, (3, 3, 2), 4, 5), (3, (2, 2, 3), 6, 7), (2, (6, 3), 5, 6),
                                           (3, (2, 2, 2), 3, 3)])
def test_oracle_equals_live_reference(orc, ref, dim, shape, P, Q):
    m = box_mesh(shape, P, seed=11)
    qd_o = orc.mass_build(dim, m.num_elem, P, Q, m.num_nodes, m.offsets, m.coords)
    qd_r = ref.mass_build(dim, m.num_elem, P, Q, m.num_nodes, dim * m.num_nodes, m.offsets, m.coords)
    assert np.array_equal(qd_o, qd_r)
    u = random_vector(m.num_nodes, 12)
    v_o = orc.mass_apply(dim, m.num_elem, P, Q, 1, m.num_nodes, m.num_nodes, m.offsets, qd_o, u)
    v_r = ref.mass_apply(dim, m.num_elem, P, Q, 1, m.num_nodes, m.num_nodes, m.offsets, qd_r, u)
    assert np.array_equal(v_o, v_r)


def test_chunked_reference_plan_matches_unchunked(ref):
    import oracle
    m = box_mesh((6, 5, 4), 4, seed=3)
    qd = ref.mass_build(3, m.num_elem, 4, 5, m.num_nodes, 3 * m.num_nodes, m.offsets, m.coords)
    u = random_vector(m.num_nodes, 4)
    v1 = ref.mass_apply(3, m.num_elem, 4, 5, 1, m.num_nodes, m.num_nodes, m.offsets, qd, u)
    plan = oracle.RefPlan(ref, 3, m.num_elem, 4, 5, m.num_nodes, m.offsets, qd, 4)
    plan2 = oracle.RefPlan(ref, 3, m.num_elem, 4, 5, m.num_nodes, m.offsets, None, 3, coords=m.coords)
    np.testing.assert_allclose(plan2.apply(u), v1, rtol=0, atol=1e-15 * np.abs(v1).max())
    plan2.close()
    v4 = plan.apply(u)
    plan.close()
    np.testing.assert_allclose(v4, v1, rtol=0, atol=1e-15 * np.abs(v1).max())


# ---------------------------------------------------------------------------
# known answers of the reference's tests, restated
# ---------------------------------------------------------------------------
def test_gauss_legendre_known_answers(orc):
    # tests/test-basis.cpp:12-59: weights sum to 2, points sorted in [-1,1],
    # exact for degree <= 2Q-1
    for Q in range(1, 6):
        x, w = orc.gauss_legendre(Q)
        assert abs(w.sum() - 2.0) <= 1e-12
        assert np.all(np.diff(x) > 0) and np.all(np.abs(x) <= 1)
        for k in range(2 * Q):
            exact = 2.0 / (k + 1) if k % 2 == 0 else 0.0
            assert abs(np.sum(w * x**k) - exact) <= 1e-10


def test_gauss_lobatto_known_answers(orc):
    # tests/test-basis.cpp:65-107
    for P in range(2, 6):
        x, w = orc.gauss_lobatto(P)
        assert abs(x[0] + 1) <= 1e-12 and abs(x[-1] - 1) <= 1e-12
        assert np.all(np.diff(x) > 0)
        assert abs(w.sum() - 2.0) <= 1e-12
    x, _ = orc.gauss_lobatto(3)
    np.testing.assert_allclose(x, [-1, 0, 1], atol=1e-12)


def test_lagrange_known_answers(orc):
    # tests/test-basis.cpp:113-162
    nodes = np.array([-1.0, 0.0, 1.0])
    B, _ = orc.lagrange_matrices(nodes, nodes)
    np.testing.assert_allclose(B.reshape(3, 3), np.eye(3), atol=1e-10)
    nodes = np.array([-1.0, -0.3, 0.4, 1.0])
    pts = np.array([-1.0, -0.6, 0.0, 0.55, 1.0])
    B, G = orc.lagrange_matrices(nodes, pts)
    np.testing.assert_allclose(B.reshape(5, 4).sum(1), 1.0, atol=1e-10)
    np.testing.assert_allclose(G.reshape(5, 4).sum(1), 0.0, atol=1e-10)
    pts = np.array([-1.0, -0.5, 0.0, 0.5, 1.0])
    B, G = orc.lagrange_matrices(np.array([-1.0, 1.0]), pts)
    np.testing.assert_allclose(B.reshape(5, 2), np.stack([(1 - pts) / 2, (1 + pts) / 2], 1), atol=1e-12)
    np.testing.assert_allclose(G.reshape(5, 2), [[-0.5, 0.5]] * 5, atol=1e-12)


def test_linear_reference_stiffness(orc):
    # tests/test-basis.cpp:181-206: K_ref = [[.5,-.5],[-.5,.5]]
    _, w, _, G = orc.basis(1, 1, 2, 2)
    G = G.reshape(2, 2)
    K = np.einsum("q,qi,qj->ij", w, G, G)
    np.testing.assert_allclose(K, [[0.5, -0.5], [-0.5, 0.5]], atol=1e-10)


def test_contraction_known_answers(orc):
    # tests/test-tensor-contract.cpp:19-86, t = [[1,2,3],[4,5,6]]
    t = np.array([1, 2, 3, 4, 5, 6], dtype=float)
    assert np.allclose(orc.contract(1, 3, 1, 2, t, 0, [2, -1, 3]), [9, 21])
    assert np.allclose(orc.contract(2, 3, 1, 2, t, 0, [2, -1, 3, 1, 1, 1]), [9, 21, 6, 15])
    assert np.allclose(orc.contract(1, 3, 2, 2, t, 0, [2, 1, -1, 1, 3, 1]), [9, 6, 21, 15])
    assert np.allclose(orc.contract(1, 3, 1, 2, t, 0, [2, -1, 3], v=[100.0, 200.0]), [109, 221])
    assert np.allclose(orc.contract(1, 2, 1, 3, t, 1, [9, 21]), [93, 123, 153])


def test_weight_known_answers(orc):
    # tests/test-tensor-contract.cpp:577-633
    for d in (1, 2, 3):
        _, w, _, _ = orc.basis(d, 3, 3, 5)
        assert abs(orc.weight(d, 5, w, 2).sum() - 2 * 2.0**d) <= 1e-12
    q, w, _, _ = orc.basis(3, 1, 3, 4)
    v = orc.weight(3, 4, w, 1)
    X = np.meshgrid(q, q, q, indexing="ij")  # z, y, x
    integral = np.sum(v.reshape(4, 4, 4) * X[2] ** 2 * X[1] ** 4 * (1 + X[0]))
    assert abs(integral - (2 / 3) * (2 / 5) * 2) <= 1e-13


def test_adjoint_identities(orc):
    # tests/test-tensor-contract.cpp:543-575
    dim, nc, ne, P, Q = 3, 3, 2, 3, 5
    _, _, B, G = orc.basis(dim, nc, P, Q)
    rng = np.random.default_rng(33)
    u = rng.uniform(-0.5, 0.5, nc * P**dim * ne)
    w = rng.uniform(-0.5, 0.5, nc * Q**dim * ne)
    g = rng.uniform(-0.5, 0.5, dim * nc * Q**dim * ne)
    assert abs(orc.interp(dim, nc, P, Q, B, ne, 0, u) @ w - u @ orc.interp(dim, nc, P, Q, B, ne, 1, w)) <= 1e-10
    assert abs(orc.grad(dim, nc, P, Q, B, G, ne, 0, u) @ g - u @ orc.grad(dim, nc, P, Q, B, G, ne, 1, g)) <= 1e-10


def test_restriction_known_answers(orc):
    # tests/test-elem-restriction.cpp:21-116
    offs = [0, 1, 1, 2]
    assert np.array_equal(orc.gather(2, 2, 1, 1, offs, [10.0, 20.0, 30.0]), [10, 20, 20, 30])
    assert np.array_equal(orc.scatter_add(2, 2, 1, 1, offs, [10.0, 20, 20, 30], np.zeros(3)), [10, 40, 30])
    assert np.array_equal(orc.scatter_add(2, 2, 1, 1, offs, [10.0, 20, 20, 30], [100.0, 200, 300]), [110, 240, 330])
    L = np.arange(200, dtype=float)
    assert np.array_equal(orc.gather(2, 2, 2, 100, [0, 1, 2, 3], L), [0, 2, 1, 3, 100, 102, 101, 103])


def test_multiplicity_known_answers(orc):
    # tests/test-elem-restriction.cpp:180-228 (libCEED t209)
    offs = [e * 3 + j for e in range(3) for j in range(4)]
    m = orc.multiplicity(3, 4, 1, 1, 10, offs)
    assert np.array_equal(m, [2.0 if (0 < i < 9 and i % 3 == 0) else 1.0 for i in range(10)])
    m = orc.multiplicity(2, 2, 2, 5, 12, [0, 1, 1, 2])
    assert np.array_equal(m, [1, 2, 1, 0, 0, 1, 2, 1, 0, 0, 0, 0])


def test_strided_known_answers(orc):
    # tests/test-elem-restriction.cpp:302-345
    L = np.arange(24, dtype=float)
    assert np.array_equal(orc.strided(0, 3, 4, 2, [3, 12, 1], L, np.zeros(24)), L)  # backend = identity
    L = np.arange(12, dtype=float)
    assert np.array_equal(orc.strided(0, 2, 3, 2, [1, 3, 6], L, np.zeros(12)), [0, 6, 1, 7, 2, 8, 3, 9, 4, 10, 5, 11])
    assert np.array_equal(orc.strided(1, 2, 2, 1, [2, 4, 1], [1.0, 2, 3, 4], [10.0, 20, 30, 40]), [11, 22, 33, 44])


def test_transpose_map_known_answers(orc):
    # tests/cuda/test-cuda-elem-restriction.cu:87-121
    lvi, to, ti = orc.transpose_map(2, 2, 3, [0, 1, 1, 2])
    assert lvi.tolist() == [0, 1, 2] and to.tolist() == [0, 1, 3, 4] and ti.tolist() == [0, 1, 2, 3]
    lvi, to, ti = orc.transpose_map(2, 2, 6, [2, 4, 5, 2])
    assert lvi.tolist() == [2, 4, 5] and to.tolist() == [0, 2, 3, 4] and ti.tolist() == [0, 3, 1, 2]


def _mesh1d_qdata(orc, h0, h1):
    # tests/test-operator.cpp:57-74: 2 linear elements, P=2, Q=3, qdata = w*h/2
    _, w, _, _ = orc.basis(1, 1, 2, 3)
    qd = orc.weight(1, 3, w, 2)
    qd[0::2] *= h0 / 2
    qd[1::2] *= h1 / 2
    return qd


def test_operator_known_answers_1d(orc):
    # tests/test-operator.cpp:256-286
    offs = [0, 1, 1, 2]
    qd = _mesh1d_qdata(orc, 1, 1)
    v = orc.mass_apply(1, 2, 2, 3, 1, 1, 3, offs, qd, np.ones(3))
    np.testing.assert_allclose(v, [0.5, 1.0, 0.5], rtol=1e-12)
    v = orc.mass_apply(1, 2, 2, 3, 1, 1, 3, offs, qd, np.array([0.0, 1, 2]))
    np.testing.assert_allclose(v, [1 / 6, 1.0, 5 / 6], rtol=1e-12)
    qd_build = orc.mass_build(1, 2, 2, 3, 3, offs, np.array([0.0, 1, 3]))
    np.testing.assert_allclose(qd_build, _mesh1d_qdata(orc, 1, 2), rtol=1e-12)


def test_operator_known_answers_2d(orc):
    # tests/test-operator.cpp:86-121, 288-329: distorted 2-quad mesh of area 5
    offs = [0, 1, 3, 4, 1, 2, 4, 5]
    coords = np.array([0, 1, 3, 0.5, 1, 2.5, 0, 0, 0, 2, 2, 2], dtype=float)
    qd = orc.mass_build(2, 2, 2, 3, 6, offs, coords)
    assert abs(qd.sum() - 5.0) <= 1e-12
    v = orc.mass_apply(2, 2, 2, 3, 1, 1, 6, offs, qd, np.ones(6))
    assert abs(v.sum() - 5.0) <= 1e-12
    u = np.array([0.37 * i - 1.3 + 0.01 * (i % 7) * (i % 5) for i in range(6)])
    w = -0.7 * u
    assert abs(w @ orc.mass_apply(2, 2, 2, 3, 1, 1, 6, offs, qd, u) - u @ orc.mass_apply(2, 2, 2, 3, 1, 1, 6, offs, qd, w)) <= 1e-12
