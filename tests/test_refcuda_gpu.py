"""The restriction stages against the reference's own CUDA kernels (GPU):
src/cuda/cuda-elem-restriction.cu built from its sources for sm_100a
(oracle/_ref/libfemrefcuda.so).  Gather and the deterministic scatter are
compared bitwise (same values, same summation order); the atomic scatter
normwise to 1e-14 (addition order differs run to run in both)."""
import numpy as np
import pytest

from fe_demo_cpp_b200.mesh import box_mesh, component_layout, random_vector

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refcuda():
    import oracle
    if not oracle.refcuda_available():
        pytest.skip("the reference CUDA build (oracle/_ref/libfemrefcuda.so) is not present")
    return oracle


@pytest.mark.parametrize("nc,interleaved", [(1, False), (3, False), (3, True)])
def test_restriction_matches_reference_cuda(fem, cuda, refcuda, nc, interleaved):
    import torch
    P = 4
    m = box_mesh((5, 4, 3), P, seed=2)
    offs, cs, l_size = component_layout(m, nc, interleaved) if nc > 1 else (m.offsets, m.num_nodes, m.num_nodes)
    es = P**3
    for det in (False, True):
        ours = fem.Restriction(m.num_elem, es, nc, cs, l_size, offs, 1 if det else 0)
        ref = refcuda.RefCudaRestriction(m.num_elem, es, nc, cs, l_size, offs, det)
        l = random_vector(l_size, 5)
        # gather
        e = torch.empty(ref.e_size, dtype=torch.float64, device=cuda)
        ours.apply(0, torch.from_numpy(l).to(cuda), e)
        ref.set_l(l)
        ref.apply(False)
        assert np.array_equal(e.cpu().numpy(), ref.get_e())
        # scatter-add into zero
        ev = random_vector(ref.e_size, 6)
        got = torch.zeros(l_size, dtype=torch.float64, device=cuda)
        ours.apply(1, torch.from_numpy(ev).to(cuda), got)
        ref.set_e(ev)
        ref.zero_l()
        ref.apply(True)
        want = ref.get_l()
        if det:
            assert np.array_equal(got.cpu().numpy(), want)
        else:
            assert np.abs(got.cpu().numpy() - want).max() <= 1e-14 * np.abs(want).max()
        ref.close()
