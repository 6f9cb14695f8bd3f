"""The mass apply with its 1D contractions on the tensor cores (GPU).

fem_b200_tc_selftest checks the tcgen05 layer itself: one TF32 MMA with the
operands staged as the applies stage them, against the host product of the
TF32-rounded inputs (relative 1e-6: FP32 rounding of the sums).

The applies (3D, P = 6..8, Q = P..8) against the FP64 oracle of the same
rounded inputs, normwise:
* FP32 storage, 3xTF32 (split): 1e-5, the tolerance of the SIMT FP32 apply
  (every operand carried as two TF32 parts: FP32-level products);
* FP32 storage, one TF32 part: 4e-3 (each of the six contractions rounds its
  input to TF32, relative 2^-11);
* BF16 storage (u and qdata BF16), one TF32 part: 4e-3 against the FP64 apply
  of the BF16-rounded u and qdata.
Tiles with fewer than 8 elements, one and three components, and the shapes
without a tensor-core kernel (an unsupported-shape error, not a fallback).
"""
import numpy as np
import pytest

from fe_demo_cpp_b200.mesh import box_mesh, component_layout

pytestmark = pytest.mark.gpu

CASES = [((3, 3, 2), 6, 7, 1), ((2, 2, 3), 6, 7, 3), ((2, 2, 2), 7, 8, 1), ((3, 2, 3), 7, 7, 3),
         ((3, 2, 2), 8, 8, 1), ((2, 3, 2), 6, 6, 1), ((5, 4, 3), 6, 8, 1)]


def norm_err(got, want):
    return float(np.abs(got - want).max() / np.abs(want).max())


def setup(fem, cuda, orc, shape, P, Q, nc):
    import torch
    m = box_mesh(shape, P, seed=P + nc)
    rx = fem.Restriction(m.num_elem, P**3, 3, m.num_nodes, 3 * m.num_nodes, m.offsets)
    qd = torch.empty(Q**3 * m.num_elem, dtype=torch.float64, device=cuda)
    fem.mass_build(rx, fem.Basis(3, 3, P, Q), torch.from_numpy(m.coords).to(cuda), qd)
    offs, cs, l_size = (m.offsets, m.num_nodes, m.num_nodes) if nc == 1 else component_layout(m, nc, False)
    op = fem.MassOperator(fem.Restriction(m.num_elem, P**3, nc, cs, l_size, offs), fem.Basis(3, nc, P, Q), qd,
                          fem.QF.apply_mass_vector)
    u = np.random.default_rng(P * 10 + nc).uniform(-1, 1, l_size)

    def oracle(uu, qq):
        return orc.mass_apply(3, m.num_elem, P, Q, nc, cs, l_size, offs, qq, uu, vector=True)
    return op, u, qd.cpu().numpy(), oracle, l_size


def test_tc_selftest(fem, cuda):
    import ctypes as C
    from fe_demo_cpp_b200 import _lib
    err = C.c_double(-1.0)
    _lib.check(_lib.load().fem_b200_tc_selftest(C.byref(err)))
    assert 0.0 <= err.value <= 1e-6, f"tensor-core self-test relative error {err.value:.3e}"


@pytest.mark.parametrize("shape,P,Q,nc", CASES)
@pytest.mark.parametrize("split", [True, False])
def test_tc_f32_apply(fem, cuda, orc, shape, P, Q, nc, split):
    import torch
    op, u, qd, oracle, n = setup(fem, cuda, orc, shape, P, Q, nc)
    u32 = u.astype(np.float32)
    v = torch.full((n,), float("nan"), dtype=torch.float32, device=cuda)
    for _ in range(2):  # twice: v is overwritten, not accumulated
        op.apply_f32_tc(torch.from_numpy(u32).to(cuda), v, split=split)
    op.check()
    got = v.double().cpu().numpy()
    want = oracle(u32.astype(np.float64), qd)
    tol = 1e-5 if split else 4e-3
    assert norm_err(got, want) <= tol, f"normwise error {norm_err(got, want):.3e} > {tol}"
    if not split:
        assert norm_err(got, want) > 1e-8  # the single-part form does round (the split one is not a copy of it)


@pytest.mark.parametrize("shape,P,Q,nc", CASES)
def test_tc_bf16_apply(fem, cuda, orc, shape, P, Q, nc):
    import torch
    op, u, qd, oracle, n = setup(fem, cuda, orc, shape, P, Q, nc)
    ub = torch.from_numpy(u).to(cuda).to(torch.bfloat16)
    v = torch.empty(n, dtype=torch.float32, device=cuda)
    op.apply_bf16_tc(ub, v)
    op.check()
    qd16 = torch.from_numpy(qd).to(torch.bfloat16).double().numpy()
    want = oracle(ub.double().cpu().numpy(), qd16)
    assert norm_err(v.double().cpu().numpy(), want) <= 4e-3


def test_tc_unsupported_shapes(fem, cuda, orc):
    import torch
    for shape, P, Q in [((2, 2, 2), 5, 6), ((2, 2, 2), 8, 9)]:
        op, u, qd, oracle, n = setup(fem, cuda, orc, shape, P, Q, 1)
        v = torch.empty(n, dtype=torch.float32, device=cuda)
        with pytest.raises(fem.FemUnsupported):
            op.apply_f32_tc(torch.from_numpy(u.astype(np.float32)).to(cuda), v)
