"""The mass apply in FP32 and BF16 storage (GPU), against the FP64 apply of
the same (rounded) inputs.

* FP32: u, v and qdata in FP32.  Against the FP64 apply of u rounded to FP32:
  normwise 1e-5 (FP32 rounding of qdata and of the sums).
* BF16: u and qdata in BF16, FP32 arithmetic.  Against the FP64 apply, with
  qdata rounded to BF16 the same way, of u rounded to BF16: normwise 1e-5 (what
  is left is FP32 arithmetic); against the unrounded qdata: 1e-2 (BF16 has an
  8-bit significand).
"""
import numpy as np
import pytest

from fe_demo_cpp_b200.mesh import box_mesh, component_layout, gll_nodes, random_vector

pytestmark = pytest.mark.gpu


def norm_err(got, want):
    return float((got.double() - want).abs().max() / want.abs().max())


class _Line:
    pass


def mesh(dim, shape, P, seed):
    if dim > 1:
        return box_mesh(shape, P, seed=seed)
    n = shape[0]
    rng = np.random.default_rng([seed, 17])
    xv = np.linspace(0, 1, n + 1)
    xv[1:-1] += rng.uniform(-0.1 / n, 0.1 / n, n - 1)
    s = (gll_nodes(P) + 1) / 2
    m = _Line()
    m.dim, m.P, m.num_elem, m.num_nodes = 1, P, n, n * (P - 1) + 1
    m.coords = np.concatenate([xv[e] + (xv[e + 1] - xv[e]) * s[(0 if e == 0 else 1):] for e in range(n)])
    m.offsets = np.array([e * (P - 1) + i for e in range(n) for i in range(P)], dtype=np.int32)
    return m


def operators(fem, cuda, dim, shape, P, Q, nc, scatter):
    import torch
    m = mesh(dim, shape, P, seed=7)
    rx = fem.Restriction(m.num_elem, P**dim, dim, m.num_nodes, dim * m.num_nodes, m.offsets)
    qd = torch.empty(Q**dim * m.num_elem, dtype=torch.float64, device=cuda)
    fem.mass_build(rx, fem.Basis(dim, dim, P, Q), torch.from_numpy(m.coords).to(cuda), qd)
    offs, cs, l_size = (m.offsets, m.num_nodes, m.num_nodes) if nc == 1 else component_layout(m, nc, False)
    qf = fem.QF.apply_mass_vector

    def make(q):
        return fem.MassOperator(fem.Restriction(m.num_elem, P**dim, nc, cs, l_size, offs, scatter),
                                fem.Basis(dim, nc, P, Q), q, qf)
    return make(qd), make(qd.to(torch.bfloat16).double()), l_size


CASES = [(1, (40,), 4, 5, 1), (2, (9, 7), 3, 4, 2), (3, (6, 5, 4), 4, 5, 1), (3, (4, 4, 3), 5, 6, 3),
         (3, (3, 3, 2), 6, 7, 1), (3, (2, 2, 2), 8, 9, 1)]


@pytest.mark.parametrize("scatter", [0, 1], ids=["atomic", "deterministic"])
@pytest.mark.parametrize("dim,shape,P,Q,nc", CASES)
def test_fp32_and_bf16_storage(fem, cuda, dim, shape, P, Q, nc, scatter):
    import torch
    op, op_q16, n = operators(fem, cuda, dim, shape, P, Q, nc, scatter)
    u = torch.from_numpy(random_vector(n, 3)).to(cuda)
    # FP32
    u32 = u.float()
    v32 = torch.full((n,), 9.0, dtype=torch.float32, device=cuda)  # overwritten
    op.apply_f32(u32, v32)
    want = torch.empty_like(u)
    op.apply(u32.double(), want)
    assert norm_err(v32, want) <= 1e-5
    # BF16
    u16 = u.to(torch.bfloat16)
    v16 = torch.full((n,), 9.0, dtype=torch.float32, device=cuda)
    op.apply_bf16(u16, v16)
    op_q16.apply(u16.double(), want)
    assert norm_err(v16, want) <= 1e-5
    op.apply(u16.double(), want)
    assert norm_err(v16, want) <= 1e-2
    if scatter == 1:  # deterministic: the same bits again
        again = torch.empty_like(v32)
        op.apply_f32(u32, again)
        assert torch.equal(again, v32)


def test_reduced_storage_argument_errors(fem, cuda):
    import torch
    op, _, n = operators(fem, cuda, 3, (2, 2, 2), 3, 4, 1, 0)
    with pytest.raises(ValueError):
        op.apply_f32(torch.zeros(n, dtype=torch.float64, device=cuda), torch.zeros(n, dtype=torch.float32,
                                                                                  device=cuda))
    with pytest.raises(ValueError):
        op.apply_bf16(torch.zeros(n + 1, dtype=torch.bfloat16, device=cuda),
                      torch.zeros(n, dtype=torch.float32, device=cuda))
