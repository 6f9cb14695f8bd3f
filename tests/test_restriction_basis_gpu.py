"""Device parity of the standalone restriction and basis kernels (GPU).

Cases follow the reference's CUDA tests
(tests/cuda/test-cuda-elem-restriction.cu:177-248): gathers and multiplicity
are bit-exact; the atomic scatter adds in a run-dependent order (normwise
1e-13, out starting at 1 to check it adds); the deterministic scatter sums in
the reference's order and is bitwise equal to the CPU scatter from a zero
start, and bitwise reproducible run to run.
"""
import numpy as np
import pytest

from fe_demo_cpp_b200.mesh import random_vector

pytestmark = pytest.mark.gpu
TOL = 1e-13


def close(got, want, tol=TOL):
    scale = max(np.abs(want).max(), 1e-300)
    err = np.abs(np.asarray(got) - np.asarray(want)).max() / scale
    assert err <= tol, f"normwise relative error {err:.3e} > {tol:.0e}"


def box_restriction(nx, ny, nz, P, nc, interleaved):
    """tests/cuda/test-cuda-elem-restriction.cu:24-42 restated."""
    Nx, Ny, Nz = nx * (P - 1) + 1, ny * (P - 1) + 1, nz * (P - 1) + 1
    n = Nx * Ny * Nz
    ns = nc if interleaved else 1
    cs = 1 if interleaved else n
    offs = []
    for ez in range(nz):
        for ey in range(ny):
            for ex in range(nx):
                for iz in range(P):
                    for iy in range(P):
                        for ix in range(P):
                            gx, gy, gz = ex * (P - 1) + ix, ey * (P - 1) + iy, ez * (P - 1) + iz
                            offs.append((gx + Nx * (gy + Ny * gz)) * ns)
    return nx * ny * nz, P**3, nc, cs, n * nc, np.array(offs, dtype=np.int32)


def wiggly(n, phase):
    i = np.arange(n)
    return np.sin(0.37 * i + phase) + 1e-3 * np.cos(11.0 * i)


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(cuda)


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


SMALL = [(2, 2, 1, 1, 3, [0, 1, 1, 2]), (2, 2, 1, 1, 6, [2, 4, 5, 2]), (2, 4, 2, 6, 12, [0, 1, 3, 4, 1, 2, 4, 5])]


def _cases():
    out = [tuple(c) for c in SMALL]
    for inter in (False, True):
        out.append(box_restriction(4, 3, 2, 2, 1, inter))
        out.append(box_restriction(3, 3, 3, 3, 3, inter))
        out.append(box_restriction(20, 20, 20, 3, 1, inter))
    return out


CASES = _cases()
IDS = [f"ne{c[0]}_es{c[1]}_nc{c[2]}_cs{c[3]}" for c in CASES]


@pytest.mark.parametrize("mode", [0, 1], ids=["atomic", "deterministic"])
@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_offset_restriction_matches_cpu(fem, cuda, orc, case, mode):
    import torch
    ne, es, nc, cs, l_size, offs = case
    offs = np.asarray(offs, dtype=np.int32)
    r = fem.Restriction(ne, es, nc, cs, l_size, offs, mode)
    # gather: exact
    l_in = wiggly(l_size, 0.1)
    e_out = torch.empty(nc * es * ne, dtype=torch.float64, device=cuda)
    r.apply(0, dev(l_in, cuda), e_out)
    assert np.array_equal(host(e_out), orc.gather(ne, es, nc, cs, offs, l_in))
    # scatter-add into 1
    e_in = wiggly(nc * es * ne, 0.7)
    l_out = dev(np.ones(l_size), cuda)
    r.apply(1, dev(e_in, cuda), l_out)
    close(host(l_out), orc.scatter_add(ne, es, nc, cs, offs, e_in, np.ones(l_size)))
    # from zero, the deterministic scatter is the CPU's sum order: bitwise
    l0 = dev(np.zeros(l_size), cuda)
    r.apply(1, dev(e_in, cuda), l0)
    want0 = orc.scatter_add(ne, es, nc, cs, offs, e_in, np.zeros(l_size))
    if mode == 1:
        assert np.array_equal(host(l0), want0)
    else:
        close(host(l0), want0)
    # multiplicity: exact integer counts
    m = torch.empty(l_size, dtype=torch.float64, device=cuda)
    r.multiplicity(m)
    assert np.array_equal(host(m), orc.multiplicity(ne, es, nc, cs, l_size, offs))


def test_deterministic_scatter_bitwise_reproducible(fem, cuda, orc):
    import torch
    ne, es, nc, cs, l_size, offs = box_restriction(16, 16, 16, 3, 3, True)
    r = fem.Restriction(ne, es, nc, cs, l_size, offs, 1)
    e = dev(wiggly(nc * es * ne, 0.3), cuda)
    first = None
    for _ in range(5):
        l = torch.zeros(l_size, dtype=torch.float64, device=cuda)
        r.apply(1, e, l)
        res = host(l)
        if first is None:
            first = res
        else:
            assert np.array_equal(res, first)
    assert np.array_equal(first, orc.scatter_add(ne, es, nc, cs, offs, host(e), np.zeros(l_size)))


def test_device_transpose_map_equals_host_map(fem, cuda, orc):
    ne, es, nc, cs, l_size, offs = box_restriction(2, 2, 1, 2, 3, True)
    r = fem.Restriction(ne, es, nc, cs, l_size, offs, 1)
    got = r.transpose_map()
    want = orc.transpose_map(ne, es, l_size, offs)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("strides", [None, [3, 1, 24]], ids=["backend", "user"])
def test_strided_restriction_matches_cpu(fem, cuda, orc, strides):
    import torch
    ne, es, nc = (5, 27, 7) if strides is None else (4, 8, 3)
    l_size = ne * es * nc
    s = [ne, es * ne, 1] if strides is None else strides
    r = fem.Restriction.strided_create(ne, es, nc, l_size, strides)
    l_in = wiggly(l_size, 0.1)
    e_out = torch.empty(l_size, dtype=torch.float64, device=cuda)
    r.apply(0, dev(l_in, cuda), e_out)
    assert np.array_equal(host(e_out), orc.strided(0, ne, es, nc, s, l_in, np.zeros(l_size)))
    e_in = wiggly(l_size, 0.7)
    l_out = dev(np.ones(l_size), cuda)
    r.apply(1, dev(e_in, cuda), l_out)
    assert np.array_equal(host(l_out), orc.strided(1, ne, es, nc, s, e_in, np.ones(l_size)))
    m = torch.empty(l_size, dtype=torch.float64, device=cuda)
    r.multiplicity(m)
    assert np.array_equal(host(m), np.ones(l_size))


def test_restriction_apply_size_errors(fem, cuda):
    import torch
    r = fem.Restriction(2, 2, 1, 1, 3, [0, 1, 1, 2])
    z = lambda n: torch.zeros(n, dtype=torch.float64, device=cuda)  # noqa: E731
    with pytest.raises(ValueError):
        r.apply(0, z(4), z(4))   # in must be l_size = 3
    with pytest.raises(ValueError):
        r.apply(1, z(3), z(3))   # in must be e_size = 4
    with pytest.raises(ValueError):
        r.apply(1, z(4), z(4))   # out must already be l_size = 3


@pytest.mark.parametrize("dim,nc,P,Q,ne", [(1, 1, 3, 5, 4), (2, 2, 3, 5, 3), (3, 3, 3, 5, 2), (3, 1, 5, 6, 37),
                                           (3, 3, 8, 9, 5), (2, 1, 16, 16, 2)])
def test_basis_apply_matches_oracle(fem, cuda, orc, dim, nc, P, Q, ne):
    import torch
    b = fem.Basis(dim, nc, P, Q)
    _, w1, B, G = orc.basis(dim, nc, P, Q)
    pn, qn = nc * P**dim * ne, nc * Q**dim * ne
    u = random_vector(pn, 1)
    w = random_vector(qn, 2)
    g = random_vector(dim * qn, 3)
    for t_mode, ev, inp, n_out, want in [
        (0, 1, u, qn, orc.interp(dim, nc, P, Q, B, ne, 0, u)),
        (1, 1, w, pn, orc.interp(dim, nc, P, Q, B, ne, 1, w)),
        (0, 2, u, dim * qn, orc.grad(dim, nc, P, Q, B, G, ne, 0, u)),
        (1, 2, g, pn, orc.grad(dim, nc, P, Q, B, G, ne, 1, g)),
    ]:
        out = torch.full((n_out,), 5.0, dtype=torch.float64, device=cuda)  # stale: overwritten
        b.apply(ne, t_mode, ev, dev(inp, cuda), out)
        close(host(out), want)
    wts = torch.empty(Q**dim * ne, dtype=torch.float64, device=cuda)
    b.apply(ne, 0, 3, None, wts)
    assert np.array_equal(host(wts), orc.weight(dim, Q, w1, ne))
    with pytest.raises(ValueError):
        b.apply(ne, 1, 3, None, wts)  # Weight rejects Transpose


def test_basis_manufactured_interp_and_grad_3d(fem, cuda):
    """tests/test-tensor-contract.cpp:233-309: P = Q = 16, spectral accuracy."""
    import torch
    P = Q = 16
    nodes = fem.gauss_lobatto_points(P)
    q, _, _, _ = fem.tensor_h1_lagrange(3, 1, P, Q)
    Z, Y, X = np.meshgrid(nodes, nodes, nodes, indexing="ij")
    u = (np.sin(X) + np.cos(X * Y) + X * Y * Z).reshape(-1)
    b = fem.Basis(3, 1, P, Q)
    v = torch.empty(Q**3, dtype=torch.float64, device=cuda)
    b.apply(1, 0, 1, dev(u, cuda), v)
    Zq, Yq, Xq = np.meshgrid(q, q, q, indexing="ij")
    np.testing.assert_allclose(host(v), (np.sin(Xq) + np.cos(Xq * Yq) + Xq * Yq * Zq).reshape(-1), atol=1e-11)
    gv = torch.empty(3 * Q**3, dtype=torch.float64, device=cuda)
    b.apply(1, 0, 2, dev(u, cuda), gv)
    gv = host(gv).reshape(3, -1)
    np.testing.assert_allclose(gv[0], (np.cos(Xq) - Yq * np.sin(Xq * Yq) + Yq * Zq).reshape(-1), atol=1e-11)
    np.testing.assert_allclose(gv[1], (-Xq * np.sin(Xq * Yq) + Xq * Zq).reshape(-1), atol=1e-11)
    np.testing.assert_allclose(gv[2], (Xq * Yq).reshape(-1), atol=1e-11)
