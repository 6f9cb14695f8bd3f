"""The allocation-free basis apply (fem_b200_basis_apply_static).

fem_b200_basis_apply allocates its pass buffers with cudaMalloc on first use;
callers being captured into a CUDA graph, or whose device memory belongs to
another allocator, cannot let it.  fem_b200_basis_apply_static computes the
same thing with its buffers in a fixed 16 MiB device array compiled into the
library.  Here it is called through the C ABI twice in a row and compared with
the allocating entry point, at the tolerance of the other device tests
(normwise 1e-13), and a call that needs more than the array holds must fail
with an argument error.  Dimension-3 calls run the fused one-pass kernels,
which need no scratch, so they are not bounded by the array (the 2000-element
case below would need 2,592,000 doubles through the generic passes).  This
file runs last so that a failure here cannot stop the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _close(got, want):
    scale = max(np.abs(want).max(), 1e-300)
    err = np.abs(got - want).max() / scale
    assert err <= TOL, f"normwise relative error {err:.3e} > {TOL:.0e}"


CASES = [(3, 3, 5, 6, 40), (3, 3, 5, 6, 2000), (3, 1, 4, 5, 100), (2, 2, 3, 4, 50), (1, 1, 6, 7, 30)]


@pytest.mark.parametrize("dim,nc,P,Q,ne", CASES)
def test_static_scratch_matches_allocating_basis_apply(fem, cuda, dim, nc, P, Q, ne):
    import torch
    from fe_demo_cpp_b200 import _lib
    lib = _lib.load()
    b = C.c_void_p()
    _lib.check(lib.fem_b200_basis_create(dim, nc, P, Q, 0, C.byref(b)))
    try:
        stream = torch.cuda.current_stream().cuda_stream
        pn, qn = nc * P**dim * ne, nc * Q**dim * ne
        g = torch.Generator(device=cuda).manual_seed(dim * 100 + P)
        # (t_mode, eval_mode, n_in, n_out): interp and grad, both directions
        for t_mode, eval_mode, n_in, n_out in [(0, 1, pn, qn), (1, 1, qn, pn), (0, 2, pn, dim * qn),
                                                (1, 2, dim * qn, pn)]:
            u = torch.rand(n_in, dtype=torch.float64, device=cuda, generator=g) * 2 - 1
            ref = torch.empty(n_out, dtype=torch.float64, device=cuda)
            _lib.check(lib.fem_b200_basis_apply(b, ne, t_mode, eval_mode, u.data_ptr(), n_in, ref.data_ptr(), n_out,
                                                stream))
            for _ in range(2):  # two calls in a row through the shared array
                out = torch.full((n_out,), float("nan"), dtype=torch.float64, device=cuda)
                _lib.check(lib.fem_b200_basis_apply_static(b, ne, t_mode, eval_mode, u.data_ptr(), n_in,
                                                           out.data_ptr(), n_out, stream))
                torch.cuda.synchronize()
                _close(out.cpu().numpy(), ref.cpu().numpy())
    finally:
        lib.fem_b200_basis_destroy(b)


def test_static_scratch_rejects_sizes_beyond_its_maximum(fem, cuda):
    import torch
    from fe_demo_cpp_b200 import _lib
    lib = _lib.load()
    b = C.c_void_p()
    _lib.check(lib.fem_b200_basis_create(2, 3, 5, 6, 0, C.byref(b)))
    try:
        ne = 10000  # dim 2 runs the generic passes: 2 * 3 * 6^2 * 10000 = 2,160,000 doubles > 2,097,152
        u = torch.zeros(3 * 25 * ne, dtype=torch.float64, device=cuda)
        v = torch.zeros(3 * 36 * ne, dtype=torch.float64, device=cuda)
        rc = lib.fem_b200_basis_apply_static(b, ne, 0, 1, u.data_ptr(), u.numel(), v.data_ptr(), v.numel(),
                                             torch.cuda.current_stream().cuda_stream)
        assert rc == _lib.ERROR_ARGUMENT
        assert "static scratch" in lib.fem_b200_last_error().decode()
    finally:
        lib.fem_b200_basis_destroy(b)
