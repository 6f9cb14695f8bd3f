"""The oracle: CPU checkers for the mass operator path.  TEST INFRASTRUCTURE.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg load
this package, and only to check or to time the CPU path; the product library
(fe_demo_cpp_b200) never imports it and has no CPU fallback.

Two libraries, both built by ``oracle/Makefile``:

* ``_lib/liboracle.so`` -- fem_oracle.c, a C restatement of the reference
  algorithm (each function cites the reference file:line it follows);
* ``_ref/libfemref.so`` -- the reference's own src/*.cpp compiled where they
  lie, driven through its public C++ API by ref_driver.cpp.  Present wherever
  it was built (it is not in git; it travels with the working tree).
* ``_ref/libfemrefcuda.so`` -- the reference's own CUDA restriction
  (src/cuda/cuda-elem-restriction.cu) for sm_100a, driven by
  ref_cuda_driver.cu: the GPU baseline of the restriction stages.

``orc`` wraps the restatement, ``ref`` the reference build; both take and
return numpy arrays.  The restatement is pinned to the reference by
tests/test_oracle.py (bitwise, and against tests/golden/).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_lib", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libfemref.so")
REFCUDA_SO = os.path.join(HERE, "_ref", "libfemrefcuda.so")
# The fe-demo-cpp source tree the reference build compiles from: the
# FE_DEMO_CPP_SRC environment variable, else its checkout location on the
# build container.  Absent on machines that only run the prebuilt libraries.
REF_SOURCE = os.environ.get("FE_DEMO_CPP_SRC", "/root/reference")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64 = C.c_int64


def build(with_ref: bool | None = None) -> None:
    """Compile the restatement (and the reference build when its sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if with_ref is None:
        with_ref = os.path.isdir(os.path.join(REF_SOURCE, "src"))
    elif with_ref and not os.path.isdir(os.path.join(REF_SOURCE, "src")):
        raise FileNotFoundError(f"oracle: fe-demo-cpp sources not found at {REF_SOURCE!r} "
                                "(set FE_DEMO_CPP_SRC to the source tree)")
    if with_ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref", "refcuda", f"REF={REF_SOURCE}"], check=True)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class _Orc:
    """The C restatement (fem_oracle.c)."""

    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            build(with_ref=False)
        L = C.CDLL(path)
        L.orc_gauss_legendre.argtypes = [C.c_int, _dp, _dp]
        L.orc_gauss_lobatto.argtypes = [C.c_int, _dp, C.c_void_p]
        L.orc_lagrange_matrices.argtypes = [C.c_int, _dp, C.c_int, _dp, _dp, _dp]
        L.orc_tensor_h1_lagrange.argtypes = [C.c_int] * 5 + [_dp] * 4
        L.orc_offset_apply.argtypes = [C.c_int, _i64, C.c_int, C.c_int, _i64, _ip, _dp, _dp]
        L.orc_strided_apply.argtypes = [C.c_int, _i64, C.c_int, C.c_int, np.ctypeslib.ndpointer(np.int64), _dp, _dp]
        L.orc_offset_multiplicity.argtypes = [_i64, C.c_int, C.c_int, _i64, _i64, _ip, _dp]
        L.orc_transpose_map.argtypes = [_i64, C.c_int, _i64, _ip, _ip, _ip, _ip]
        L.orc_transpose_map.restype = _i64
        L.orc_contract.argtypes = [_i64, C.c_int, _i64, C.c_int, _dp, C.c_int, C.c_int, _dp, _dp]
        L.orc_interp.argtypes = [C.c_int] * 4 + [_dp, _i64, C.c_int, _dp, _dp]
        L.orc_grad.argtypes = [C.c_int] * 4 + [_dp, _dp, _i64, C.c_int, _dp, _dp]
        L.orc_weight.argtypes = [C.c_int, C.c_int, _dp, _i64, _dp]
        L.orc_build_mass_qf.argtypes = [C.c_int, _i64, _dp, _dp, _dp]
        L.orc_apply_mass_qf.argtypes = [_i64, _dp, _dp, _dp]
        L.orc_mass_apply.argtypes = [C.c_int, _i64, C.c_int, C.c_int, C.c_int, _i64, _i64, _ip, _dp, _dp, _dp, _dp,
                                     C.c_int, C.c_int]
        L.orc_mass_apply_vector.argtypes = [C.c_int, _i64, C.c_int, C.c_int, C.c_int, _i64, _i64, _ip, _dp, _dp, _dp,
                                            _dp]
        L.orc_mass_build.argtypes = [C.c_int, _i64, C.c_int, C.c_int, _i64, _ip, _dp, _dp, _dp, _dp, _dp]
        self.L = L

    # -- 1D rules / basis
    def gauss_legendre(self, Q):
        x, w = np.zeros(Q), np.zeros(Q)
        if self.L.orc_gauss_legendre(Q, x, w):
            raise ValueError("Q must be positive")
        return x, w

    def gauss_lobatto(self, Q):
        x, w = np.zeros(Q), np.zeros(Q)
        if self.L.orc_gauss_lobatto(Q, x, w.ctypes.data):
            raise ValueError("Q must be > 1")
        return x, w

    def lagrange_matrices(self, nodes, pts):
        nodes, pts = _f64(nodes), _f64(pts)
        B = np.zeros(len(pts) * len(nodes))
        G = np.zeros_like(B)
        self.L.orc_lagrange_matrices(len(nodes), nodes, len(pts), pts, B, G)
        return B, G

    def basis(self, dim, num_comp, P, Q, quad_mode=0):
        """(q_ref, q_weight, interp[Q*P], grad[Q*P]) of the tensor H1 Lagrange basis."""
        q, w, B, G = np.zeros(Q), np.zeros(Q), np.zeros(Q * P), np.zeros(Q * P)
        if self.L.orc_tensor_h1_lagrange(dim, num_comp, P, Q, quad_mode, q, w, B, G):
            raise ValueError("bad basis arguments")
        return q, w, B, G

    # -- restriction
    def gather(self, ne, es, nc, comp_stride, offsets, l_vec):
        out = np.zeros(nc * es * ne)
        self.L.orc_offset_apply(0, ne, es, nc, comp_stride, _i32(offsets), _f64(l_vec), out)
        return out

    def scatter_add(self, ne, es, nc, comp_stride, offsets, e_vec, l_out):
        l_out = _f64(l_out).copy()
        self.L.orc_offset_apply(1, ne, es, nc, comp_stride, _i32(offsets), _f64(e_vec), l_out)
        return l_out

    def strided(self, t_mode, ne, es, nc, strides, inp, out):
        out = _f64(out).copy()
        self.L.orc_strided_apply(t_mode, ne, es, nc, np.asarray(strides, dtype=np.int64), _f64(inp), out)
        return out

    def multiplicity(self, ne, es, nc, comp_stride, l_size, offsets):
        m = np.zeros(l_size)
        self.L.orc_offset_multiplicity(ne, es, nc, comp_stride, l_size, _i32(offsets), m)
        return m

    def transpose_map(self, ne, es, l_size, offsets):
        lv = np.zeros(l_size, np.int32)
        to = np.zeros(l_size + 1, np.int32)
        ti = np.zeros(max(ne * es, 1), np.int32)
        n = self.L.orc_transpose_map(ne, es, l_size, _i32(offsets), lv, to, ti)
        return lv[:n].copy(), to[:n + 1].copy(), ti[:ne * es].copy()

    # -- basis action
    def contract(self, A, B, Cc, J, t, t_mode, u, v=None):
        out = np.zeros(A * J * Cc) if v is None else _f64(v).copy()
        self.L.orc_contract(A, B, Cc, J, _f64(t), t_mode, 0 if v is None else 1, _f64(u), out)
        return out

    def interp(self, dim, nc, P, Q, interp_1d, ne, t_mode, u):
        n_out = nc * (P if t_mode else Q) ** dim * ne
        v = np.zeros(n_out)
        self.L.orc_interp(dim, nc, P, Q, _f64(interp_1d), ne, t_mode, _f64(u), v)
        return v

    def grad(self, dim, nc, P, Q, interp_1d, grad_1d, ne, t_mode, u):
        n_out = nc * P**dim * ne if t_mode else dim * nc * Q**dim * ne
        v = np.zeros(n_out)
        self.L.orc_grad(dim, nc, P, Q, _f64(interp_1d), _f64(grad_1d), ne, t_mode, _f64(u), v)
        return v

    def weight(self, dim, Q, q_weight_1d, ne):
        v = np.zeros(Q**dim * ne)
        self.L.orc_weight(dim, Q, _f64(q_weight_1d), ne, v)
        return v

    # -- mass operator
    def mass_build(self, dim, ne, P, Q, comp_stride, offsets, coords, quad_mode=0):
        _, w, B, G = self.basis(dim, dim, P, Q, quad_mode)
        qd = np.zeros(Q**dim * ne)
        if self.L.orc_mass_build(dim, ne, P, Q, comp_stride, _i32(offsets), B, G, w, _f64(coords), qd):
            raise RuntimeError("orc_mass_build failed")
        return qd

    def mass_apply(self, dim, ne, P, Q, nc, comp_stride, l_size, offsets, qdata, u, quad_mode=0, vector=False,
                   interp_1d=None):
        """v = M u.  vector=False: the reference apply_mass (component 0 only
        for nc > 1); vector=True: every component (nc scalar applies).
        interp_1d: a caller-given [Q][P] interpolation matrix in place of the
        Lagrange basis's."""
        _, _, B, _ = self.basis(dim, nc, P, Q, quad_mode)
        if interp_1d is not None:
            B = _f64(interp_1d).reshape(B.shape)
        v = np.zeros(l_size)
        if vector:
            rc = self.L.orc_mass_apply_vector(dim, ne, P, Q, nc, comp_stride, l_size, _i32(offsets), B, _f64(qdata),
                                              _f64(u), v)
        else:
            rc = self.L.orc_mass_apply(dim, ne, P, Q, nc, comp_stride, l_size, _i32(offsets), B, _f64(qdata),
                                       _f64(u), v, 1, -1)
        if rc:
            raise RuntimeError("orc_mass_apply failed")
        return v


class _Ref:
    """The reference library itself (ref_driver.cpp over src/*.cpp)."""

    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            build(with_ref=True)
        L = C.CDLL(path)
        L.ref_last_error.restype = C.c_char_p
        L.ref_gauss_legendre.argtypes = [C.c_int, _dp, _dp]
        L.ref_gauss_lobatto.argtypes = [C.c_int, _dp, C.c_void_p]
        L.ref_tensor_h1_lagrange.argtypes = [C.c_int] * 5 + [_dp] * 4
        L.ref_basis_apply.argtypes = [C.c_int] * 8 + [_dp, C.c_long, _dp, C.c_long]
        L.ref_offset_apply.argtypes = [C.c_int] * 5 + [_ip, C.c_int, _dp, _dp]
        L.ref_multiplicity.argtypes = [C.c_int] * 5 + [_ip, _dp]
        L.ref_mass_build.argtypes = [C.c_int] * 6 + [_ip, _dp, _dp]
        L.ref_mass_apply.argtypes = [C.c_int] * 7 + [_ip, _dp, _dp, _dp]
        L.ref_mass_apply_vector.argtypes = [C.c_int] * 7 + [_ip, _dp, _dp, _dp]
        L.ref_plan_create.argtypes = [C.c_int, C.c_long, C.c_int, C.c_int, C.c_long, _ip, C.c_void_p, C.c_void_p,
                                      C.c_int]
        L.ref_plan_create.restype = C.c_void_p
        L.ref_plan_apply.argtypes = [C.c_void_p, _dp, _dp]
        L.ref_plan_destroy.argtypes = [C.c_void_p]
        self.L = L

    def _check(self, rc):
        if rc:
            msg = self.L.ref_last_error().decode()
            raise (ValueError if rc == 1 else RuntimeError)(msg)

    def gauss_legendre(self, Q):
        x, w = np.zeros(Q), np.zeros(Q)
        self._check(self.L.ref_gauss_legendre(Q, x, w))
        return x, w

    def gauss_lobatto(self, Q):
        x, w = np.zeros(Q), np.zeros(Q)
        self._check(self.L.ref_gauss_lobatto(Q, x, w.ctypes.data))
        return x, w

    def basis(self, dim, num_comp, P, Q, quad_mode=0):
        q, w, B, G = np.zeros(Q), np.zeros(Q), np.zeros(Q * P), np.zeros(Q * P)
        self._check(self.L.ref_tensor_h1_lagrange(dim, num_comp, P, Q, quad_mode, q, w, B, G))
        return q, w, B, G

    def basis_apply(self, dim, nc, P, Q, ne, t_mode, eval_mode, u, quad_mode=0):
        """eval_mode: 1 Interp, 2 Grad, 3 Weight (the reference EvalMode values)."""
        if eval_mode == 3:
            n_v = Q**dim * ne
        elif t_mode:
            n_v = nc * P**dim * ne
        else:
            n_v = (dim if eval_mode == 2 else 1) * nc * Q**dim * ne
        u = _f64(u) if u is not None and len(u) else np.zeros(1)
        v = np.zeros(n_v)
        self._check(self.L.ref_basis_apply(dim, nc, P, Q, quad_mode, ne, t_mode, eval_mode, u, len(u), v, n_v))
        return v

    def gather(self, ne, es, nc, comp_stride, l_size, offsets, l_vec):
        out = np.zeros(nc * es * ne)
        self._check(self.L.ref_offset_apply(ne, es, nc, comp_stride, l_size, _i32(offsets), 0, _f64(l_vec), out))
        return out

    def scatter_add(self, ne, es, nc, comp_stride, l_size, offsets, e_vec, l_out):
        l_out = _f64(l_out).copy()
        self._check(self.L.ref_offset_apply(ne, es, nc, comp_stride, l_size, _i32(offsets), 1, _f64(e_vec), l_out))
        return l_out

    def multiplicity(self, ne, es, nc, comp_stride, l_size, offsets):
        m = np.zeros(l_size)
        self._check(self.L.ref_multiplicity(ne, es, nc, comp_stride, l_size, _i32(offsets), m))
        return m

    def mass_build(self, dim, ne, P, Q, comp_stride, l_size, offsets, coords):
        qd = np.zeros(Q**dim * ne)
        self._check(self.L.ref_mass_build(dim, ne, P, Q, comp_stride, l_size, _i32(offsets), _f64(coords), qd))
        return qd

    def mass_apply(self, dim, ne, P, Q, nc, comp_stride, l_size, offsets, qdata, u, vector=False):
        v = np.zeros(l_size)
        f = self.L.ref_mass_apply_vector if vector else self.L.ref_mass_apply
        self._check(f(dim, ne, P, Q, nc, comp_stride, l_size, _i32(offsets), _f64(qdata), _f64(u), v))
        return v


class RefPlan:
    """Threaded, element-chunked reference apply (scalar mass) for timing."""

    def __init__(self, ref: _Ref, dim, ne, P, Q, l_size, offsets, qdata=None, n_chunks=1, coords=None):
        """qdata ([q][e]) given, or None to build it per chunk from coords
        (blocked, comp_stride = l_size) with the reference build operator."""
        self.ref, self.l_size = ref, l_size
        qd = None if qdata is None else _f64(qdata)
        xc = None if coords is None else _f64(coords)
        self.h = ref.L.ref_plan_create(dim, ne, P, Q, l_size, _i32(offsets), None if qd is None else qd.ctypes.data,
                                       None if xc is None else xc.ctypes.data, n_chunks)
        if not self.h:
            raise RuntimeError(ref.L.ref_last_error().decode())

    def apply(self, u, v=None):
        v = np.zeros(self.l_size) if v is None else v
        self.ref._check(self.ref.L.ref_plan_apply(self.h, _f64(u), v))
        return v

    def close(self):
        if self.h:
            self.ref.L.ref_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


_orc = None
_ref = None


def orc() -> _Orc:
    global _orc
    if _orc is None:
        _orc = _Orc()
    return _orc


def ref() -> _Ref:
    global _ref
    if _ref is None:
        _ref = _Ref()
    return _ref


class RefCudaRestriction:
    """The reference's CUDA restriction (fem::cuda::elem_restriction_*) on a
    host offsets array, with its own device L- and E-vectors; numpy in and out.
    apply() launches on the default stream, asynchronously, as the reference."""

    def __init__(self, num_elem, elem_size, num_comp, comp_stride, l_size, offsets, deterministic=False):
        self.L = _refcuda_lib()
        self.h = C.c_void_p()
        self._check(self.L.refcuda_create(num_elem, elem_size, num_comp, comp_stride, l_size, _i32(offsets),
                                          int(bool(deterministic)), C.byref(self.h)))
        ls, es = _i64(0), _i64(0)
        self._check(self.L.refcuda_sizes(self.h, C.byref(ls), C.byref(es)))
        self.l_size, self.e_size = ls.value, es.value

    def _check(self, rc):
        if rc:
            raise RuntimeError(self.L.refcuda_last_error().decode())

    def set_l(self, l):
        self._check(self.L.refcuda_set_l(self.h, _f64(l)))

    def set_e(self, e):
        self._check(self.L.refcuda_set_e(self.h, _f64(e)))

    def zero_l(self):
        self._check(self.L.refcuda_zero_l(self.h))

    def apply(self, transpose):
        self._check(self.L.refcuda_apply(self.h, int(bool(transpose))))

    def get_l(self):
        out = np.empty(self.l_size)
        self._check(self.L.refcuda_get_l(self.h, out))
        return out

    def get_e(self):
        out = np.empty(self.e_size)
        self._check(self.L.refcuda_get_e(self.h, out))
        return out

    def close(self):
        if self.h:
            self.L.refcuda_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_refcuda = None


def _refcuda_lib():
    global _refcuda
    if _refcuda is None:
        L = C.CDLL(REFCUDA_SO)
        L.refcuda_last_error.restype = C.c_char_p
        L.refcuda_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _ip, C.c_int, C.c_void_p]
        for name in ("refcuda_set_l", "refcuda_set_e", "refcuda_get_l", "refcuda_get_e"):
            getattr(L, name).argtypes = [C.c_void_p, _dp]
        for name in ("refcuda_zero_l", "refcuda_destroy"):
            getattr(L, name).argtypes = [C.c_void_p]
        L.refcuda_apply.argtypes = [C.c_void_p, C.c_int]
        L.refcuda_sizes.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        _refcuda = L
    return _refcuda


def refcuda_available() -> bool:
    return os.path.exists(REFCUDA_SO)


def ref_available() -> bool:
    return os.path.exists(REF_SO) or os.path.isdir(os.path.join(REF_SOURCE, "src"))


def compact_submesh(offsets, elem_size, num_elem_sample, coords=None, dim=None, num_nodes=None):
    """The first ``num_elem_sample`` elements as a self-contained mesh.

    Returns (local_offsets int32, n_local, global_nodes, local_coords) with
    the used nodes renumbered 0..n_local-1 (increasing global order) and, if
    coords (blocked, comp_stride = num_nodes) are given, their coordinates in
    the same blocked layout with comp_stride = n_local.  Used to time the
    reference on a bounded sample of a large workload.
    """
    sub = np.ascontiguousarray(offsets[: num_elem_sample * elem_size])
    nodes, local = np.unique(sub, return_inverse=True)
    local = local.astype(np.int32)
    loc_coords = None
    if coords is not None:
        loc_coords = np.concatenate([coords[k * num_nodes + nodes] for k in range(dim)])
    return local, int(nodes.size), nodes, loc_coords
