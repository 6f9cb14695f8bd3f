"""Generate tests/golden/*.npz from the reference library itself.

    python tests/golden/make_golden.py

Runs the compiled reference (oracle/_ref/libfemref.so, built from
fe-demo-cpp's own src/*.cpp by oracle/Makefile) through its public API on
seeded inputs and stores its outputs.  Large outputs are stored as a SHA-256
of their bytes plus a few reductions; the C restatement (oracle/) is pinned
to these fixtures bitwise, and the device path to the restatement.  Inputs
are regenerated from seeds by fe_demo_cpp_b200.mesh (their digest is stored
too, so a drift of the generator is caught).
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from fe_demo_cpp_b200.mesh import box_mesh, component_layout, random_vector  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    oracle.build(with_ref=True)
    ref = oracle.ref()
    out = {}

    # -- 1D rules and basis matrices
    for P in range(2, 10):
        for Q in (P - 1, P, P + 1, P + 2):
            if Q < 1:
                continue
            for mode in (0, 1):
                if mode == 1 and Q < 2:
                    continue
                q, w, B, G = ref.basis(3, 1, P, Q, mode)
                key = f"basis_P{P}_Q{Q}_m{mode}"
                out[key + "_qref"], out[key + "_qw"], out[key + "_B"], out[key + "_G"] = q, w, B, G

    # -- mass operator on seeded perturbed meshes (dim, shape, P, Q, seed)
    cases = [(3, (8, 8, 8), 4, 5, 1), (3, (3, 2, 2), 3, 4, 2), (3, (2, 2, 2), 5, 6, 3), (2, (5, 4), 4, 5, 4),
             (3, (4, 3, 2), 2, 3, 5), (3, (2, 1, 1), 8, 9, 6)]
    names = []
    for dim, shape, P, Q, seed in cases:
        m = box_mesh(shape, P, seed=seed)
        name = f"mass_d{dim}_{'x'.join(map(str, shape))}_P{P}_Q{Q}_s{seed}"
        names.append(name)
        qd = ref.mass_build(dim, m.num_elem, P, Q, m.num_nodes, dim * m.num_nodes, m.offsets, m.coords)
        u = random_vector(m.num_nodes, seed)
        v = ref.mass_apply(dim, m.num_elem, P, Q, 1, m.num_nodes, m.num_nodes, m.offsets, qd, u)
        ones = ref.mass_apply(dim, m.num_elem, P, Q, 1, m.num_nodes, m.num_nodes, m.offsets, qd,
                              np.ones(m.num_nodes))
        out[name + "_mesh_sha"] = m.digest()
        out[name + "_qdata_sha"] = sha(qd)
        out[name + "_v_sha"] = sha(v)
        out[name + "_qdata_elemsum"] = qd.reshape(-1, m.num_elem).sum(axis=0)
        out[name + "_volume"] = np.array([qd.sum(), ones.sum()])
        if m.num_nodes <= 20000:
            out[name + "_v"] = v
        if qd.size <= 5000:
            out[name + "_qdata"] = qd
    out["mass_cases"] = np.array(names)

    # -- num_comp = 3 on one small mesh, blocked and interleaved
    m = box_mesh((3, 2, 2), 3, seed=7)
    qd = ref.mass_build(3, m.num_elem, 3, 4, m.num_nodes, 3 * m.num_nodes, m.offsets, m.coords)
    out["c3_qdata"] = qd
    for inter in (False, True):
        offs, cs, l_size = component_layout(m, 3, inter)
        u = random_vector(l_size, 8)
        tag = "inter" if inter else "blocked"
        out[f"c3_{tag}_v_ref"] = ref.mass_apply(3, m.num_elem, 3, 4, 3, cs, l_size, offs, qd, u)
        out[f"c3_{tag}_v_vector"] = ref.mass_apply(3, m.num_elem, 3, 4, 3, cs, l_size, offs, qd, u, vector=True)
        # restriction gather / scatter / multiplicity of the 3-component field
        out[f"c3_{tag}_gather"] = ref.gather(m.num_elem, 27, 3, cs, l_size, offs, u)
        e_in = random_vector(3 * 27 * m.num_elem, 9)
        out[f"c3_{tag}_scatter"] = ref.scatter_add(m.num_elem, 27, 3, cs, l_size, offs, e_in, np.ones(l_size))
        out[f"c3_{tag}_mult"] = ref.multiplicity(m.num_elem, 27, 3, cs, l_size, offs)

    # -- basis actions (interp / grad / weight, both directions), dims 1-3
    for dim in (1, 2, 3):
        for nc in (1, 3):
            P, Q, ne = 3, 5, 2
            u = random_vector(nc * P**dim * ne, 10 + dim)
            w = random_vector(nc * Q**dim * ne, 20 + dim)
            g = random_vector(dim * nc * Q**dim * ne, 30 + dim)
            key = f"bapply_d{dim}_c{nc}"
            out[key + "_interp"] = ref.basis_apply(dim, nc, P, Q, ne, 0, 1, u)
            out[key + "_interpT"] = ref.basis_apply(dim, nc, P, Q, ne, 1, 1, w)
            out[key + "_grad"] = ref.basis_apply(dim, nc, P, Q, ne, 0, 2, u)
            out[key + "_gradT"] = ref.basis_apply(dim, nc, P, Q, ne, 1, 2, g)
            out[key + "_weight"] = ref.basis_apply(dim, nc, P, Q, ne, 0, 3, None)

    path = os.path.join(HERE, "reference_outputs.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes,", len(out), "arrays")


if __name__ == "__main__":
    main()
