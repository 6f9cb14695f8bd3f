"""CPU tests of libfem_b200's host side: it loads without a GPU, exports every
entry point of include/fem_b200.h, and its set-up (basis, validation,
transpose map) matches the oracle bitwise and raises the reference's errors.
No device compute runs here."""
import ctypes
import os
import re

import numpy as np
import pytest

from fe_demo_cpp_b200.mesh import box_mesh

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "fem_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(fem_b200_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol(fem):
    syms = header_symbols()
    assert len(syms) >= 25
    lib = ctypes.CDLL(fem.LIB_PATH)
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    # and the Python binding declares exactly these
    from fe_demo_cpp_b200 import _lib
    assert sorted(_lib.SIGNATURES) == syms


def test_python_constants_match_the_header():
    """The Python mirror's solve precisions and kernel variants carry the
    header's values (FEM_B200_SOLVE_*, FEM_B200_KERNEL_*)."""
    from fe_demo_cpp_b200.api import SOLVE_PRECISIONS, KernelVariant
    text = open(os.path.join(ROOT, "include", "fem_b200.h")).read()
    solve = {k.lower(): int(v) for k, v in re.findall(r"#define FEM_B200_SOLVE_(\w+) (\d+)", text)}
    assert solve == SOLVE_PRECISIONS
    kern = {k.lower(): int(v) for k, v in re.findall(r"#define FEM_B200_KERNEL_(\w+) (\d+)", text)}
    assert kern == {v.name: int(v) for v in KernelVariant}


def test_loads_without_gpu_and_reports_device_count(fem):
    n = fem.load().fem_b200_device_count()
    assert n >= 0


def test_basis_bitwise_equals_oracle(fem, orc):
    for dim in (1, 2, 3):
        for P in range(2, 12):
            for Q in range(1, 13):
                for mode in (0, 1):
                    if mode == 1 and Q < 2:
                        continue
                    got = fem.tensor_h1_lagrange(dim, 1, P, Q, mode)
                    want = orc.basis(dim, 1, P, Q, mode)
                    for a, b in zip(got, want):
                        assert np.array_equal(a, b), (dim, P, Q, mode)


def test_basis_matches_reference_fixtures(fem, golden):
    for key in golden.files:
        if key.startswith("basis_") and key.endswith("_B"):
            _, p, q, m, _ = key.split("_")
            got = fem.tensor_h1_lagrange(3, 1, int(p[1:]), int(q[1:]), int(m[1:]))
            assert np.array_equal(got[2], golden[key])


def test_quadrature_entry_points(fem, orc):
    for Q in range(1, 10):
        a, b = fem.gauss_legendre_quadrature(Q), orc.gauss_legendre(Q)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    for Q in range(2, 10):
        a, b = fem.gauss_lobatto_points(Q, weights=True), orc.gauss_lobatto(Q)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    nodes, pts = np.array([-1.0, -0.3, 0.4, 1.0]), np.array([-1.0, -0.6, 0.0, 0.55, 1.0])
    got, want = fem.lagrange_basis_matrix(nodes, pts), orc.lagrange_matrices(nodes, pts)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_basis_argument_errors(fem):
    # src/basis.cpp:202-216 and the quadrature guards
    for args in [(0, 1, 2, 2), (4, 1, 2, 2), (3, 0, 2, 2), (3, 4, 2, 2), (3, 1, 1, 2), (3, 1, 2, 0)]:
        with pytest.raises(ValueError):
            fem.tensor_h1_lagrange(*args)
    with pytest.raises(ValueError):
        fem.gauss_legendre_quadrature(0)
    with pytest.raises(ValueError):
        fem.gauss_lobatto_points(1)


def test_offset_restriction_validation(fem):
    # tests/test-elem-restriction.cpp:123-173
    chk = fem.check_offset_restriction
    ok = [0, 1, 1, 2]
    for args in [(0, 2, 1, 1, 3, []), (2, 0, 1, 1, 3, []), (2, 2, 0, 1, 3, ok), (2, 2, 1, 1, 0, ok),
                 (2, 2, 2, 0, 200, ok), (2, 2, 1, 1, 3, [0, 1, 1]), (2, 2, 1, 1, 3, [0, 1, 1, 2, 2]),
                 (2, 2, 1, 1, 3, [0, 1, 1, 3]), (2, 2, 1, 1, 3, [0, -1, 1, 2]), (1, 2, 2, 100, 3, [0, 1]),
                 (1, 2, 2, 2, 3, [0, 1])]:
        with pytest.raises(ValueError):
            chk(*args)
    chk(2, 2, 1, 0, 3, ok)          # comp_stride irrelevant for one component
    chk(1, 2, 2, 2, 4, [0, 1])      # exactly fitting


def test_strided_restriction_validation(fem):
    # tests/test-elem-restriction.cpp:262-280
    chk = fem.check_strided_restriction
    for args in [(0, 4, 1, 8), (2, 0, 1, 8), (2, 4, 0, 8), (2, 4, 1, 0), (2, 4, 2, 15)]:
        with pytest.raises(ValueError):
            chk(*args)
    chk(2, 4, 2, 16)
    chk(2, 3, 2, 12, [1, 3, 6])
    with pytest.raises(ValueError):
        chk(2, 3, 2, 11, [1, 3, 6])
    with pytest.raises(ValueError):
        chk(2, 3, 2, 12, [-1, 3, 6])


def test_transpose_map_known_answers_and_oracle(fem, orc):
    # tests/cuda/test-cuda-elem-restriction.cu:87-121
    lvi, to, ti = fem.transpose_map(2, 2, 3, [0, 1, 1, 2])
    assert lvi.tolist() == [0, 1, 2] and to.tolist() == [0, 1, 3, 4] and ti.tolist() == [0, 1, 2, 3]
    lvi, to, ti = fem.transpose_map(2, 2, 6, [2, 4, 5, 2])
    assert lvi.tolist() == [2, 4, 5] and to.tolist() == [0, 2, 3, 4] and ti.tolist() == [0, 3, 1, 2]
    m = box_mesh((3, 2, 2), 3, seed=0)
    got = fem.transpose_map(m.num_elem, 27, m.num_nodes, m.offsets)
    want = orc.transpose_map(m.num_elem, 27, m.num_nodes, m.offsets)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)
    # every E-node appears once, under its own L-node (test-cuda-elem-restriction.cu:107-121)
    lvi, to, ti = got
    seen = np.zeros(m.num_elem * 27, int)
    for n in range(len(lvi)):
        for t in ti[to[n]:to[n + 1]]:
            assert m.offsets[t] == lvi[n]
            seen[t] += 1
    assert np.all(seen == 1)


def test_mesh_generator_is_a_valid_box(fem):
    m = box_mesh((4, 3, 2), 4, seed=2)
    assert m.offsets.min() == 0 and m.offsets.max() == m.num_nodes - 1
    xs = m.coords.reshape(3, -1)
    assert np.all(xs >= 0) and np.all(xs <= 1)
    # neighbours along x share their face nodes
    o = m.offsets.reshape(m.num_elem, 4, 4, 4)
    assert np.array_equal(o[0, :, :, 3], o[1, :, :, 0])
    assert box_mesh((4, 3, 2), 4, seed=2).digest() == m.digest()


def test_server_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors of fem_b200_request / fem_b200_result have the C
    header's field offsets and sizes (compiled with gcc, no GPU)."""
    import ctypes as C
    import subprocess
    from fe_demo_cpp_b200.api import _Request, _Result
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "fem_b200.h"', 'int main(void) {']
    for ty, cls in (("fem_b200_request", _Request), ("fem_b200_result", _Result)):
        lines.append(f'printf("{ty} %zu\\n", sizeof({ty}));')
        for name, _ in cls._fields_:
            lines.append(f'printf("{ty}.{name} %zu\\n", offsetof({ty}, {name}));')
    lines += ["return 0;", "}"]
    src, exe = tmp_path / "layout.c", tmp_path / "layout"
    src.write_text("\n".join(lines))
    subprocess.run(["gcc", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                       check=True).stdout.splitlines())
    for ty, cls in (("fem_b200_request", _Request), ("fem_b200_result", _Result)):
        assert int(out[ty]) == C.sizeof(cls)
        for name, _ in cls._fields_:
            assert int(out[f"{ty}.{name}"]) == getattr(cls, name).offset, (ty, name)
