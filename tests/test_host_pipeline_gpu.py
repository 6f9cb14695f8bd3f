"""The host-memory apply with its copies pipelined against element chunks
(GPU).

operator_apply on host vectors (src/operator.cpp:148-182) runs, for plans of
at least two chunks with the atomic scatter, as a pipeline: u copied in by
node span, the operator's kernel per element chunk, v copied out as it
becomes final.  Each case compares it with the device apply of the same plan
(normwise, TOL: the atomic scatter adds in a run-dependent order), and one
case with the oracle.  Cases: page-locked and pageable host buffers, every
3D kernel variant, blocked and interleaved vector fields, the reference's
component-0-only apply_mass on a 3-component field, node numberings that
defeat the pipeline (scrambled, elements in reverse), 2D, the chunk setting,
mixed page-locked / pageable pairs, and a mesh large enough that the
pageable staging ring wraps and splits copies across slots.
"""
import numpy as np
import pytest

from fe_demo_cpp_b200.mesh import box_mesh, component_layout, random_vector

pytestmark = pytest.mark.gpu
TOL = 1e-14

# 28 x 26 x 24 = 17,472 hexes: 2,184 tiles of 8, five chunks of up to 512 tiles
SHAPE3 = (28, 26, 24)


def close(got, want, tol=TOL):
    scale = max(np.abs(want).max(), 1e-300)
    err = np.abs(np.asarray(got) - np.asarray(want)).max() / scale
    assert err <= tol, f"normwise relative error {err:.3e} > {tol:.0e}"


def _qdata(fem, cuda, m, Q):
    import torch
    rx = fem.Restriction(m.num_elem, m.P**m.dim, m.dim, m.num_nodes, m.dim * m.num_nodes, m.offsets)
    bx = fem.Basis(m.dim, m.dim, m.P, Q)
    qd = torch.empty(Q**m.dim * m.num_elem, dtype=torch.float64, device=cuda)
    fem.mass_build(rx, bx, torch.from_numpy(m.coords).to(cuda), qd)
    return qd


def _both(fem, cuda, op, l_size, seed, pinned, pinned_v=None):
    """(host apply, device apply) of the same u; `pinned` / `pinned_v`: the
    host u / v page-locked (v like u unless given), else pageable."""
    import torch
    pinned_v = pinned if pinned_v is None else pinned_v
    u = random_vector(l_size, seed)
    v_dev = torch.empty(l_size, dtype=torch.float64, device=cuda)
    op.apply(torch.from_numpy(u).to(cuda), v_dev)
    torch.cuda.synchronize()
    u_h = torch.from_numpy(u).pin_memory() if pinned else torch.from_numpy(u.copy())
    v_h = torch.full((l_size,), np.nan, dtype=torch.float64)
    if pinned_v:
        v_h = v_h.pin_memory()
    op.apply_host(u_h.numpy(), v_h.numpy())
    return v_h.numpy().copy(), v_dev.cpu().numpy()


@pytest.fixture(scope="module")
def mesh3(fem, cuda):
    m = box_mesh(SHAPE3, 3, seed=5)
    return m, _qdata(fem, cuda, m, 4)


def _scalar_op(fem, m, qd, offs=None):
    return fem.MassOperator(fem.Restriction(m.num_elem, 27, 1, m.num_nodes, m.num_nodes,
                                            m.offsets if offs is None else offs),
                            fem.Basis(3, 1, 3, 4), qd)


@pytest.mark.parametrize("pinned", [True, False], ids=["page-locked", "pageable"])
@pytest.mark.parametrize("variant", ["simple", "pipelined", "paired", "prefetch", "occupancy", "narrow", "element"])
def test_pipelined_host_apply_every_variant(fem, cuda, mesh3, variant, pinned):
    m, qd = mesh3
    op = _scalar_op(fem, m, qd)
    try:
        op.set_kernel(fem.KernelVariant[variant])
    except Exception as e:  # a variant not compiled for this (P, Q)
        pytest.skip(f"{variant}: {e}")
    got, want = _both(fem, cuda, op, m.num_nodes, 11, pinned)
    assert np.isfinite(got).all()
    close(got, want)


def test_pipelined_host_apply_matches_oracle(fem, cuda, orc, mesh3):
    m, qd = mesh3
    op = _scalar_op(fem, m, qd)
    u = random_vector(m.num_nodes, 12)
    got = op.apply_host(u)
    want = orc.mass_apply(3, m.num_elem, 3, 4, 1, m.num_nodes, m.num_nodes, m.offsets, qd.cpu().numpy(), u)
    close(got, want, 1e-13)


@pytest.mark.parametrize("pinned", [True, False], ids=["page-locked", "pageable"])
@pytest.mark.parametrize("layout", ["blocked", "interleaved"])
@pytest.mark.parametrize("qf", ["apply_mass_vector", "apply_mass"])
def test_pipelined_host_apply_vector_fields(fem, cuda, mesh3, layout, qf, pinned):
    m, qd = mesh3
    offs, cs, l_size = component_layout(m, 3, interleaved=layout == "interleaved")
    op = fem.MassOperator(fem.Restriction(m.num_elem, 27, 3, cs, l_size, offs), fem.Basis(3, 3, 3, 4), qd,
                          fem.QF[qf])
    got, want = _both(fem, cuda, op, l_size, 13, pinned)
    close(got, want)
    if qf == "apply_mass":  # the reference's apply_mass: components 1, 2 of v stay zero
        comp = np.arange(l_size) % 3 if layout == "interleaved" else np.arange(l_size) // m.num_nodes
        assert not got[comp > 0].any()


@pytest.mark.parametrize("order", ["scrambled-nodes", "reversed-elements"])
def test_pipelined_host_apply_unfavourable_numbering(fem, cuda, mesh3, order):
    """Numberings where later elements do not use later nodes: the pipeline
    degenerates to copy-in, apply, copy-out, and stays exact."""
    import torch
    m, qd = mesh3
    if order == "scrambled-nodes":
        perm = np.random.default_rng(3).permutation(m.num_nodes).astype(np.int32)
        offs = perm[m.offsets]
        qd_o = qd
    else:
        offs = m.offsets.reshape(m.num_elem, 27)[::-1].reshape(-1).copy()
        q = qd.cpu().numpy().reshape(-1, m.num_elem)  # qdata is [q][e]: reverse the elements
        qd_o = torch.from_numpy(np.ascontiguousarray(q[:, ::-1]).reshape(-1)).to(cuda)
    op = _scalar_op(fem, m, qd_o, offs)
    got, want = _both(fem, cuda, op, m.num_nodes, 14, False)
    close(got, want)


def test_pipelined_host_apply_2d(fem, cuda):
    m = box_mesh((260, 260), 3, seed=6)  # 67,600 quads: 2,113 tiles of 32, five chunks
    qd = _qdata(fem, cuda, m, 4)
    op = fem.MassOperator(fem.Restriction(m.num_elem, 9, 1, m.num_nodes, m.num_nodes, m.offsets),
                          fem.Basis(2, 1, 3, 4), qd)
    for pinned in (True, False):
        got, want = _both(fem, cuda, op, m.num_nodes, 15, pinned)
        close(got, want)


def test_host_chunk_setting(fem, cuda, mesh3):
    """1 = unpipelined; 2, 3 and the default cut the same plan differently;
    every cut gives the device result."""
    m, qd = mesh3
    op = _scalar_op(fem, m, qd)
    for chunks in (1, 2, 3, 0):
        op.set_host_chunks(chunks)
        got, want = _both(fem, cuda, op, m.num_nodes, 16 + chunks, chunks % 2 == 0)
        close(got, want)
    with pytest.raises(Exception):
        op.set_host_chunks(-1)


@pytest.mark.parametrize("pinned_u,pinned_v", [(True, False), (False, True)], ids=["u-locked", "v-locked"])
def test_pipelined_host_apply_mixed_memory(fem, cuda, mesh3, pinned_u, pinned_v):
    m, qd = mesh3
    op = _scalar_op(fem, m, qd)
    got, want = _both(fem, cuda, op, m.num_nodes, 21, pinned_u, pinned_v)
    close(got, want)


def test_pageable_staging_ring_wraps(fem, cuda):
    """140^3 hexes at P = 2 (2.8M nodes, 343,000 tiles): 24 chunks give dozens
    of ring pieces a direction (the 6-slot ring wraps); 2 chunks give copies of
    1.4M nodes, split over slots of 1M doubles."""
    m = box_mesh((140, 140, 140), 2, seed=7)
    qd = _qdata(fem, cuda, m, 3)
    op = fem.MassOperator(fem.Restriction(m.num_elem, 8, 1, m.num_nodes, m.num_nodes, m.offsets),
                          fem.Basis(3, 1, 2, 3), qd)
    for chunks in (0, 2):
        op.set_host_chunks(chunks)
        for rep in range(2):  # the second call reuses the ring and its events
            got, want = _both(fem, cuda, op, m.num_nodes, 30 + rep, False)
            close(got, want)
