"""Seeded structured box meshes: the inputs of the mass operator.

A box [0,1]^dim split into nx x ny (x nz) elements, P Gauss-Lobatto nodes per
direction per element, lexicographic local nodes (x fastest) and elements
(x fastest), the numbering of the reference's own test meshes
(tests/cuda/test-cuda-elem-restriction.cu:24-42 ``box_restriction``).

Interior mesh vertices are moved by U[-f*h, f*h] per coordinate (h the element
size, f = 0.1 by default) from ``seed``; boundary vertices stay put, so the
domain, and its volume 1, do not change.  High-order nodes are placed by the
multilinear map of the element's perturbed corners, so neighbouring elements
agree on their shared faces and every element stays valid.

All arithmetic is element-wise IEEE double (numpy ufuncs, no reductions), and
the random streams are numpy PCG64 from fixed seeds, so a mesh is bitwise
reproducible from (shape, P, seed, perturb).
"""
from __future__ import annotations

import hashlib
import math
from dataclasses import dataclass

import numpy as np


def gll_nodes(P: int) -> np.ndarray:
    """Gauss-Lobatto-Legendre nodes on [-1, 1] (ascending), by Newton on P'_{P-1}.

    Only used to place mesh nodes; the basis matrices are built by the library.
    """
    if P < 2:
        raise ValueError("P must be >= 2")
    n = P - 1
    x = np.empty(P)
    x[0], x[-1] = -1.0, 1.0
    for i in range(1, P - 1):
        t = -math.cos(math.pi * i / n)
        for _ in range(100):
            # P_n, P_n' and P_n'' by recurrence at t
            p0, p1 = 1.0, t
            for k in range(2, n + 1):
                p0, p1 = p1, ((2 * k - 1) * t * p1 - (k - 1) * p0) / k
            dp = n * (t * p1 - p0) / (t * t - 1.0)
            d2p = (2.0 * t * dp - n * (n + 1) * p1) / (1.0 - t * t)
            step = dp / d2p
            t -= step
            if abs(step) < 1e-16:
                break
        x[i] = t
    # exact symmetry
    for i in range(P // 2):
        x[P - 1 - i] = -x[i]
    if P % 2:
        x[P // 2] = 0.0
    return x


@dataclass
class BoxMesh:
    dim: int
    shape: tuple            # elements per direction (nx, ny[, nz])
    P: int
    num_elem: int
    num_nodes: int          # scalar nodes, N_L for one component
    offsets: np.ndarray     # int32 [num_elem * P^dim], row e holds element e's nodes
    coords: np.ndarray      # float64 [dim * num_nodes], blocked: component k at k*num_nodes
    node_shape: tuple       # nodes per direction (Nx, Ny[, Nz])

    @property
    def elem_size(self) -> int:
        return self.P ** self.dim

    def digest(self) -> str:
        h = hashlib.sha256()
        h.update(np.ascontiguousarray(self.offsets).tobytes())
        h.update(np.ascontiguousarray(self.coords).tobytes())
        return h.hexdigest()


def box_mesh(shape, P: int, seed: int = 0, perturb: float = 0.1) -> BoxMesh:
    """Build a perturbed box mesh; ``shape`` = (nx, ny) or (nx, ny, nz)."""
    shape = tuple(int(s) for s in shape)
    dim = len(shape)
    if dim not in (2, 3) or min(shape) < 1 or P < 2:
        raise ValueError("shape must have 2 or 3 positive entries and P >= 2")
    nodes_per = tuple(n * (P - 1) + 1 for n in shape)
    num_nodes = int(np.prod(nodes_per, dtype=np.int64))
    num_elem = int(np.prod(shape, dtype=np.int64))
    if num_nodes * dim >= 2**31 or num_elem * P**dim >= 2**31:
        raise ValueError("mesh too large for int32 offsets")

    # --- offsets: e = ex + nx*(ey + ny*ez), i = ix + P*(iy + P*iz)
    e_idx = np.meshgrid(*[np.arange(n, dtype=np.int32) for n in reversed(shape)], indexing="ij")
    e_idx = [a.reshape(-1, 1) for a in reversed(e_idx)]           # ex, ey, ez (x fastest)
    i_idx = np.meshgrid(*[np.arange(P, dtype=np.int32)] * dim, indexing="ij")
    i_idx = [a.reshape(1, -1) for a in reversed(i_idx)]           # ix, iy, iz (x fastest)
    g = np.zeros((num_elem, P**dim), dtype=np.int32)
    stride = 1
    for d in range(dim):
        g += (e_idx[d] * (P - 1) + i_idx[d]) * np.int32(stride)
        stride *= nodes_per[d]
    offsets = g.reshape(-1)
    del g, e_idx, i_idx

    # --- vertices with interior perturbation
    h = [1.0 / n for n in shape]
    vshape = tuple(n + 1 for n in reversed(shape))                # (nz+1, ny+1, nx+1) for 3D
    rng = np.random.default_rng([int(seed), 17])
    verts = []
    grids = np.meshgrid(*[np.arange(n + 1) for n in reversed(shape)], indexing="ij")
    grids = list(reversed(grids))                                 # index along x, y, z
    interior = np.ones(vshape, dtype=bool)
    for d in range(dim):
        interior &= (grids[d] > 0) & (grids[d] < shape[d])
    for d in range(dim):
        base = grids[d] * h[d]
        delta = rng.uniform(-perturb * h[d], perturb * h[d], size=vshape)
        verts.append(np.where(interior, base + delta, base))
    del grids

    # --- high-order nodes by the multilinear map of each element's corners
    gll = gll_nodes(P)
    s1d = (gll + 1.0) * 0.5                                       # [0, 1]
    gi = [np.arange(N) for N in nodes_per]
    el = [np.minimum(a // (P - 1), n - 1) for a, n in zip(gi, shape)]
    loc = [a - e * (P - 1) for a, e in zip(gi, el)]
    s = [s1d[l] for l in loc]
    # broadcast shapes in (z, y, x) order
    def along(d, arr):
        sh = [1] * dim
        sh[dim - 1 - d] = arr.shape[0]
        return arr.reshape(sh)
    coords = np.empty((dim,) + tuple(reversed(nodes_per)))
    for c in range(dim):
        acc = np.zeros(tuple(reversed(nodes_per)))
        for corner in range(2**dim):
            bits = [(corner >> d) & 1 for d in range(dim)]
            w = None
            idx = []
            for d in range(dim):
                wd = along(d, s[d] if bits[d] else 1.0 - s[d])
                w = wd if w is None else w * wd
                idx.append(along(d, el[d] + bits[d]))
            acc += w * verts[c][tuple(reversed(idx))]
        coords[c] = acc
    coords = coords.reshape(-1)
    return BoxMesh(dim=dim, shape=shape, P=P, num_elem=num_elem, num_nodes=num_nodes,
                   offsets=offsets, coords=coords, node_shape=nodes_per)


def random_vector(n: int, seed: int, stream: int = 1) -> np.ndarray:
    """uniform[-1, 1] float64 vector from (seed, stream)."""
    return np.random.default_rng([int(seed), int(stream)]).uniform(-1.0, 1.0, int(n))


def component_layout(mesh: BoxMesh, num_comp: int, interleaved: bool = False):
    """Offsets and comp_stride for a num_comp-component field on ``mesh``.

    blocked: node stride 1, comp_stride = num_nodes; interleaved: node stride
    num_comp, comp_stride 1 (the two layouts of the reference's
    ``box_restriction``).  Returns (offsets, comp_stride, l_size).
    """
    if interleaved and num_comp > 1:
        return (mesh.offsets * np.int32(num_comp)).astype(np.int32), 1, mesh.num_nodes * num_comp
    return mesh.offsets, mesh.num_nodes, mesh.num_nodes * num_comp


def mesh_for_dofs(target_dofs: int, P: int, dim: int = 3):
    """Elements per side so that (n*(P-1)+1)^dim is close to target_dofs."""
    n = max(1, round((target_dofs ** (1.0 / dim) - 1) / (P - 1)))
    return (n,) * dim
