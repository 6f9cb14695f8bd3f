"""Seeded perturbed box meshes generated on the device (torch), for large
benchmark sweeps where the host generator (mesh.box_mesh) would dominate the
run time.  Same construction as mesh.box_mesh -- lexicographic elements and
local nodes, interior vertices moved by U[-f*h, f*h] per coordinate, nodes
placed by the trilinear map of the perturbed corners -- but the random stream
is torch's (seeded), so the meshes are not bitwise those of box_mesh.
"""
from __future__ import annotations

from dataclasses import dataclass

from .mesh import gll_nodes


@dataclass
class DeviceMesh:
    dim: int
    shape: tuple
    P: int
    num_elem: int
    num_nodes: int
    offsets: "object"  # torch.int32 [num_elem * P^dim] on the device
    coords: "object"   # torch.float64 [dim * num_nodes], blocked


def box_mesh_device_2d(shape, P: int, seed: int = 0, perturb: float = 0.1, device="cuda") -> DeviceMesh:
    """The quadrilateral form: shape = (nx, ny), nodes by the bilinear map;
    coords [2 * num_nodes], blocked."""
    import torch
    nx, ny = (int(s) for s in shape)
    Nx, Ny = nx * (P - 1) + 1, ny * (P - 1) + 1
    num_nodes = Nx * Ny
    num_elem = nx * ny
    if num_nodes * 2 >= 2**31 or num_elem * P**2 >= 2**31:
        raise ValueError("mesh too large for int32 offsets")
    dev = torch.device(device)
    i32 = dict(dtype=torch.int32, device=dev)
    # offsets[e, i] = gx + Nx*gy, e = ex + nx*ey, i = ix + P*iy
    ex = torch.arange(nx, **i32).view(1, nx)
    ey = torch.arange(ny, **i32).view(ny, 1)
    base = (ex * (P - 1) + Nx * (ey * (P - 1))).reshape(-1, 1)
    ix = torch.arange(P, **i32).view(1, P)
    iy = torch.arange(P, **i32).view(P, 1)
    offsets = (base + (ix + Nx * iy).reshape(1, -1)).reshape(-1)
    g = torch.Generator(device=dev).manual_seed(int(seed) * 7919 + 17)
    f64 = dict(dtype=torch.float64, device=dev)
    vy, vx = torch.meshgrid(torch.arange(ny + 1, **f64), torch.arange(nx + 1, **f64), indexing="ij")
    interior = (vx > 0) & (vx < nx) & (vy > 0) & (vy < ny)
    verts = []
    for base_v, n in ((vx, nx), (vy, ny)):
        h = 1.0 / n
        delta = (torch.rand(base_v.shape, generator=g, **f64) * 2 - 1) * (perturb * h)
        verts.append(torch.where(interior, base_v * h + delta, base_v * h))
    s1d = torch.tensor((gll_nodes(P) + 1.0) * 0.5, **f64)

    def axis(N, n):
        gi = torch.arange(N, device=dev)
        el = torch.clamp(gi // (P - 1), max=n - 1)
        return el, s1d[gi - el * (P - 1)]
    elx, sx = axis(Nx, nx)
    ely, sy = axis(Ny, ny)
    coords = torch.empty(2, Ny, Nx, **f64)
    for c in range(2):
        acc = torch.zeros(Ny, Nx, **f64)
        for corner in range(4):
            bx, by = corner & 1, (corner >> 1) & 1
            w = (sy if by else 1 - sy).view(-1, 1) * (sx if bx else 1 - sx).view(1, -1)
            acc += w * verts[c][(ely + by).view(-1, 1), (elx + bx).view(1, -1)]
        coords[c] = acc
    return DeviceMesh(2, (nx, ny), P, num_elem, num_nodes, offsets, coords.reshape(-1))


def box_mesh_device(shape, P: int, seed: int = 0, perturb: float = 0.1, device="cuda") -> DeviceMesh:
    """shape = (nx, ny, nz) hexahedra, or (nx, ny) quadrilaterals (box_mesh_device_2d)."""
    import torch
    if len(shape) == 2:
        return box_mesh_device_2d(shape, P, seed, perturb, device)
    nx, ny, nz = (int(s) for s in shape)
    Nx, Ny, Nz = nx * (P - 1) + 1, ny * (P - 1) + 1, nz * (P - 1) + 1
    num_nodes = Nx * Ny * Nz
    num_elem = nx * ny * nz
    if num_nodes * 3 >= 2**31 or num_elem * P**3 >= 2**31:
        raise ValueError("mesh too large for int32 offsets")
    dev = torch.device(device)
    i32 = dict(dtype=torch.int32, device=dev)
    # offsets[e, i] = gx + Nx*(gy + Ny*gz), e = ex + nx*(ey + ny*ez), i = ix + P*(iy + P*iz)
    ex = torch.arange(nx, **i32).view(1, 1, nx)
    ey = torch.arange(ny, **i32).view(1, ny, 1)
    ez = torch.arange(nz, **i32).view(nz, 1, 1)
    base = ((ex * (P - 1)) + Nx * ((ey * (P - 1)) + Ny * (ez * (P - 1)))).reshape(-1, 1)
    ix = torch.arange(P, **i32).view(1, 1, P)
    iy = torch.arange(P, **i32).view(1, P, 1)
    iz = torch.arange(P, **i32).view(P, 1, 1)
    local = (ix + Nx * (iy + Ny * iz)).reshape(1, -1)
    offsets = (base + local).reshape(-1)
    # perturbed vertices, (nz+1, ny+1, nx+1) per coordinate
    g = torch.Generator(device=dev).manual_seed(int(seed) * 7919 + 17)
    f64 = dict(dtype=torch.float64, device=dev)
    vz, vy, vx = torch.meshgrid(torch.arange(nz + 1, **f64), torch.arange(ny + 1, **f64),
                                torch.arange(nx + 1, **f64), indexing="ij")
    interior = (vx > 0) & (vx < nx) & (vy > 0) & (vy < ny) & (vz > 0) & (vz < nz)
    verts = []
    for base_v, n in ((vx, nx), (vy, ny), (vz, nz)):
        h = 1.0 / n
        delta = (torch.rand(base_v.shape, generator=g, **f64) * 2 - 1) * (perturb * h)
        verts.append(torch.where(interior, base_v * h + delta, base_v * h))
    # node positions by the trilinear map of each element's corners
    s1d = torch.tensor((gll_nodes(P) + 1.0) * 0.5, **f64)

    def axis(N, n):
        gi = torch.arange(N, device=dev)
        el = torch.clamp(gi // (P - 1), max=n - 1)
        return el, s1d[gi - el * (P - 1)]
    elx, sx = axis(Nx, nx)
    ely, sy = axis(Ny, ny)
    elz, sz = axis(Nz, nz)
    coords = torch.empty(3, Nz, Ny, Nx, **f64)
    for c in range(3):
        acc = torch.zeros(Nz, Ny, Nx, **f64)
        for corner in range(8):
            bx, by, bz = corner & 1, (corner >> 1) & 1, (corner >> 2) & 1
            w = ((sz if bz else 1 - sz).view(-1, 1, 1) * (sy if by else 1 - sy).view(1, -1, 1)
                 * (sx if bx else 1 - sx).view(1, 1, -1))
            vc = verts[c][(elz + bz).view(-1, 1, 1), (ely + by).view(1, -1, 1), (elx + bx).view(1, 1, -1)]
            acc += w * vc
        coords[c] = acc
    return DeviceMesh(3, (nx, ny, nz), P, num_elem, num_nodes, offsets, coords.reshape(-1))
