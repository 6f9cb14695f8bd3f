"""A basis whose interpolation matrix is not centro-symmetric (GPU).

Lagrange bases on GLL nodes evaluated at Gauss points satisfy
B[Q-1-q][P-1-p] = B[q][p], and the fused kernels then take the even-odd
contractions.  A caller can hand the C++ drop-in any interp_1d
(TensorBasis fields filled in by hand, fem_b200_basis_create_from); the plans
must detect the broken symmetry and keep the direct contractions.  Here B is
perturbed by 1e-3 in a few entries and the mass apply (3D P = 6 and 7, 2D
P = 8), the standalone interp / interp^T, and one batch class are compared
with the oracle at the FP64 tolerance of the other device tests (normwise
1e-13).
"""
import numpy as np
import pytest

from fe_demo_cpp_b200.mesh import box_mesh, random_vector

pytestmark = pytest.mark.gpu
TOL = 1e-13


def close(got, want, tol=TOL):
    scale = max(np.abs(want).max(), 1e-300)
    err = np.abs(got - want).max() / scale
    assert err <= tol, f"normwise relative error {err:.3e} > {tol:.0e}"


def perturbed_basis(fem, dim, nc, P, Q):
    q_ref, w, B, G = fem.tensor_h1_lagrange(dim, nc, P, Q)
    B = np.array(B, dtype=np.float64).reshape(Q, P)
    B[0, 1] += 1e-3
    B[Q // 2, P - 2] -= 2e-3
    B[Q - 1, 0] += 5e-4
    asym = np.abs(B - B[::-1, ::-1]).max()
    assert asym > 1e-4  # really not centro-symmetric
    return fem.Basis.from_matrices(dim, nc, P, Q, w, B, G), B


@pytest.mark.parametrize("dim,shape,P", [(3, (3, 2, 2), 6), (3, (2, 2, 2), 7), (2, (6, 5), 8)])
def test_mass_apply_asymmetric_interp(fem, cuda, orc, dim, shape, P):
    import torch
    Q = P + 1
    m = box_mesh(shape, P, seed=P)
    # geometric factors from the regular basis, then the operator on the perturbed one
    rx = fem.Restriction(m.num_elem, P**dim, dim, m.num_nodes, dim * m.num_nodes, m.offsets)
    qd = torch.empty(Q**dim * m.num_elem, dtype=torch.float64, device=cuda)
    fem.mass_build(rx, fem.Basis(dim, dim, P, Q), torch.from_numpy(m.coords).to(cuda), qd)
    bu, B = perturbed_basis(fem, dim, 1, P, Q)
    N = m.num_nodes
    op = fem.MassOperator(fem.Restriction(m.num_elem, P**dim, 1, N, N, m.offsets), bu, qd)
    u = random_vector(N, 70 + P)
    v = torch.empty(N, dtype=torch.float64, device=cuda)
    op.apply(torch.from_numpy(u).to(cuda), v)
    torch.cuda.synchronize()
    qd_h = qd.cpu().numpy()
    want = orc.mass_apply(dim, m.num_elem, P, Q, 1, N, N, m.offsets, qd_h, u, interp_1d=B)
    close(v.cpu().numpy(), want)
    # the symmetric basis gives a different operator: the perturbation is seen
    want_sym = orc.mass_apply(dim, m.num_elem, P, Q, 1, N, N, m.offsets, qd_h, u)
    assert np.abs(want - want_sym).max() > 1e-6 * np.abs(want).max()


@pytest.mark.parametrize("P", [6, 7])
def test_basis_interp_asymmetric(fem, cuda, orc, P):
    import torch
    Q, ne = P + 1, 37
    b, B = perturbed_basis(fem, 3, 1, P, Q)
    rng = np.random.default_rng(P)
    u = rng.uniform(-1, 1, P**3 * ne)
    y = torch.empty(Q**3 * ne, dtype=torch.float64, device=cuda)
    b.apply(ne, 0, 1, torch.from_numpy(u).to(cuda), y)
    torch.cuda.synchronize()
    close(y.cpu().numpy(), orc.interp(3, 1, P, Q, B.reshape(-1), ne, 0, u))
    q = rng.uniform(-1, 1, Q**3 * ne)
    x = torch.empty(P**3 * ne, dtype=torch.float64, device=cuda)
    b.apply(ne, 1, 1, torch.from_numpy(q).to(cuda), x)
    torch.cuda.synchronize()
    close(x.cpu().numpy(), orc.interp(3, 1, P, Q, B.reshape(-1), ne, 1, q))


def test_batch_class_asymmetric(fem, cuda, orc):
    import torch
    P, Q = 6, 7
    m = box_mesh((2, 2, 3), P, seed=11)
    rx = fem.Restriction(m.num_elem, P**3, 3, m.num_nodes, 3 * m.num_nodes, m.offsets)
    qd = torch.empty(Q**3 * m.num_elem, dtype=torch.float64, device=cuda)
    fem.mass_build(rx, fem.Basis(3, 3, P, Q), torch.from_numpy(m.coords).to(cuda), qd)
    bu, B = perturbed_basis(fem, 3, 1, P, Q)
    N = m.num_nodes
    ops = [fem.MassOperator(fem.Restriction(m.num_elem, P**3, 1, N, N, m.offsets), bu, qd) for _ in range(2)]
    us = [torch.from_numpy(random_vector(N, 90 + i)).to(cuda) for i in range(2)]
    vs = [torch.empty(N, dtype=torch.float64, device=cuda) for _ in range(2)]
    batch = fem.Batch(ops)
    batch.bind(us, vs)
    batch.apply()
    torch.cuda.synchronize()
    qd_h = qd.cpu().numpy()
    for uu, vv in zip(us, vs):
        want = orc.mass_apply(3, m.num_elem, P, Q, 1, N, N, m.offsets, qd_h, uu.cpu().numpy(), interp_1d=B)
        close(vv.cpu().numpy(), want)
