"""Python objects over the libfem_b200 C ABI (tests, benchmarks, scripting).

Device arrays are torch CUDA tensors (float64 / int32, contiguous); host
arrays are numpy.  Each object owns one C handle and releases it on close()
or garbage collection.  Names follow the reference API (fe-demo-cpp):
restriction gather/scatter, tensor basis, the mass operator and its
geometric-factor build.
"""
from __future__ import annotations

import ctypes as C
from enum import IntEnum

import numpy as np

from . import _lib
from ._lib import call


class ContractMode(IntEnum):
    NoTranspose = 0
    Transpose = 1


class EvalMode(IntEnum):
    None_ = 0
    Interp = 1
    Grad = 2
    Weight = 3


class QuadMode(IntEnum):
    Gauss = 0
    GaussLobatto = 1


class ScatterMode(IntEnum):
    Atomic = 0
    Deterministic = 1


# fem_b200_mass_solve's precision argument (FEM_B200_SOLVE_*)
SOLVE_PRECISIONS = {"fp64": 0, "fp32_ir": 1, "bf16_ir": 2}


class KernelVariant(IntEnum):
    auto = 0
    simple = 1
    pipelined = 2
    paired = 3
    prefetch = 4
    occupancy = 5
    narrow = 6
    element = 7


class QF(IntEnum):
    """Device QFunctions of the mass operator."""
    apply_mass = 0          # the reference apply_mass: component 0 only
    apply_mass_vector = 1   # every component


def _ptr(a) -> int:
    if a is None:
        return 0
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    return int(a)


def _n(a) -> int:
    return int(a.size) if isinstance(a, np.ndarray) else int(a.numel())


def _check_dev(a, dtype_name="float64"):
    if a is None:
        return
    if isinstance(a, np.ndarray) or not getattr(a, "is_cuda", False):
        raise ValueError("expected a CUDA tensor")
    if str(a.dtype) != f"torch.{dtype_name}":
        raise ValueError(f"expected a {dtype_name} tensor, got {a.dtype}")


def _stream(stream) -> int:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return int(getattr(stream, "cuda_stream", stream))


# ---------------------------------------------------------------------------
# host set-up (no GPU)
# ---------------------------------------------------------------------------
def gauss_legendre_quadrature(Q: int):
    x, w = np.zeros(max(Q, 0)), np.zeros(max(Q, 0))
    call("fem_b200_gauss_legendre", Q, _ptr(x), _ptr(w))
    return x, w


def gauss_lobatto_points(Q: int, weights: bool = False):
    x, w = np.zeros(max(Q, 1)), np.zeros(max(Q, 1))
    call("fem_b200_gauss_lobatto", Q, _ptr(x), _ptr(w) if weights else 0)
    return (x, w) if weights else x


def lagrange_basis_matrix(nodes, eval_points):
    nodes = np.ascontiguousarray(nodes, dtype=np.float64)
    pts = np.ascontiguousarray(eval_points, dtype=np.float64)
    B = np.zeros(len(pts) * len(nodes))
    G = np.zeros_like(B)
    call("fem_b200_lagrange_basis_matrix", len(nodes), _ptr(nodes), len(pts), _ptr(pts), _ptr(B), _ptr(G))
    return B, G


def tensor_h1_lagrange(dim, num_comp, P, Q, quad_mode=QuadMode.Gauss):
    """(q_ref[Q], q_weight[Q], interp[Q*P], grad[Q*P]) of the tensor H1 Lagrange basis."""
    q, w = np.zeros(max(Q, 1)), np.zeros(max(Q, 1))
    B, G = np.zeros(max(Q * P, 1)), np.zeros(max(Q * P, 1))
    call("fem_b200_tensor_h1_lagrange", dim, num_comp, P, Q, int(quad_mode), _ptr(q), _ptr(w), _ptr(B), _ptr(G))
    return q[:Q], w[:Q], B[:Q * P], G[:Q * P]


def check_offset_restriction(num_elem, elem_size, num_comp, comp_stride, l_size, offsets) -> None:
    offsets = np.ascontiguousarray(offsets, dtype=np.int32)
    call("fem_b200_restriction_check_offset", num_elem, elem_size, num_comp, comp_stride, l_size, _ptr(offsets),
         offsets.size)


def check_strided_restriction(num_elem, elem_size, num_comp, l_size, strides=None) -> None:
    s = None if strides is None else np.ascontiguousarray(strides, dtype=np.int32)
    call("fem_b200_restriction_check_strided", num_elem, elem_size, num_comp, l_size, _ptr(s))


def transpose_map(num_elem, elem_size, l_size, offsets):
    """(l_vec_indices, t_offsets, t_indices) of an offset restriction, on the host."""
    offsets = np.ascontiguousarray(offsets, dtype=np.int32)
    lvi = np.zeros(l_size, np.int32)
    to = np.zeros(l_size + 1, np.int32)
    ti = np.zeros(max(num_elem * elem_size, 1), np.int32)
    n = C.c_int(0)
    call("fem_b200_transpose_map", num_elem, elem_size, l_size, _ptr(offsets), _ptr(lvi), _ptr(to), _ptr(ti),
         C.addressof(n))
    return lvi[:n.value].copy(), to[:n.value + 1].copy(), ti[:num_elem * elem_size].copy()


# ---------------------------------------------------------------------------
# device objects
# ---------------------------------------------------------------------------
class _Handle:
    _destroy = ""

    def __init__(self):
        self.h = C.c_void_p(0)

    def close(self):
        if self.h and self.h.value:
            _lib.load()
            getattr(_lib.load(), self._destroy)(self.h)
            self.h = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Restriction(_Handle):
    """Device element restriction (offset or strided)."""
    _destroy = "fem_b200_restriction_destroy"

    def __init__(self, num_elem, elem_size, num_comp, comp_stride, l_size, offsets,
                 scatter_mode=ScatterMode.Atomic):
        super().__init__()
        offsets = np.ascontiguousarray(offsets, dtype=np.int32)
        call("fem_b200_restriction_create_offset", num_elem, elem_size, num_comp, comp_stride, l_size,
             _ptr(offsets), int(scatter_mode), C.addressof(self.h))
        self.strided = False
        self.num_elem, self.elem_size, self.num_comp = num_elem, elem_size, num_comp
        self.comp_stride, self.l_size = comp_stride, l_size
        self.e_size = num_comp * elem_size * num_elem
        self.scatter_mode = ScatterMode(scatter_mode)

    @classmethod
    def strided_create(cls, num_elem, elem_size, num_comp, l_size, strides=None):
        self = cls.__new__(cls)
        _Handle.__init__(self)
        s = None if strides is None else np.ascontiguousarray(strides, dtype=np.int32)
        call("fem_b200_restriction_create_strided", num_elem, elem_size, num_comp, l_size, _ptr(s),
             C.addressof(self.h))
        self.strided = True
        self.num_elem, self.elem_size, self.num_comp = num_elem, elem_size, num_comp
        self.comp_stride, self.l_size = 0, l_size
        self.e_size = num_comp * elem_size * num_elem
        self.scatter_mode = ScatterMode.Atomic
        return self

    def apply(self, t_mode, inp, out, stream=None):
        """NoTranspose: out = E in (overwritten).  Transpose: out += E^T in."""
        _check_dev(inp)
        _check_dev(out)
        call("fem_b200_restriction_apply", self.h, int(t_mode), _ptr(inp), _n(inp), _ptr(out), _n(out),
             _stream(stream))

    def multiplicity(self, mult, stream=None):
        _check_dev(mult)
        call("fem_b200_restriction_multiplicity", self.h, _ptr(mult), _n(mult), _stream(stream))

    def transpose_map(self):
        lvi = np.zeros(self.l_size, np.int32)
        to = np.zeros(self.l_size + 1, np.int32)
        ti = np.zeros(self.num_elem * self.elem_size, np.int32)
        n = C.c_int(0)
        call("fem_b200_restriction_transpose_map", self.h, _ptr(lvi), _ptr(to), _ptr(ti), C.addressof(n))
        return lvi[:n.value].copy(), to[:n.value + 1].copy(), ti


class Basis(_Handle):
    """Device tensor-product H1 Lagrange basis."""
    _destroy = "fem_b200_basis_destroy"

    def __init__(self, dim, num_comp, P, Q, quad_mode=QuadMode.Gauss):
        super().__init__()
        call("fem_b200_basis_create", dim, num_comp, P, Q, int(quad_mode), C.addressof(self.h))
        self.dim, self.num_comp, self.P, self.Q, self.quad_mode = dim, num_comp, P, Q, QuadMode(quad_mode)

    @classmethod
    def from_matrices(cls, dim, num_comp, P, Q, q_weight_1d, interp_1d, grad_1d):
        """A basis from caller-given 1D data (q_weight_1d[Q], interp_1d and
        grad_1d [Q][P] row-major), as the reference's TensorBasis whose fields
        the caller filled in (include/basis.hpp:28-40)."""
        self = cls.__new__(cls)
        _Handle.__init__(self)
        w = np.ascontiguousarray(q_weight_1d, dtype=np.float64)
        B = np.ascontiguousarray(interp_1d, dtype=np.float64)
        G = np.ascontiguousarray(grad_1d, dtype=np.float64)
        if w.size != Q or B.size != Q * P or G.size != Q * P:
            raise ValueError("Basis.from_matrices: q_weight_1d needs Q entries, interp_1d and grad_1d Q*P")
        call("fem_b200_basis_create_from", dim, num_comp, P, Q, _ptr(w), _ptr(B), _ptr(G), C.addressof(self.h))
        self.dim, self.num_comp, self.P, self.Q, self.quad_mode = dim, num_comp, P, Q, None
        return self

    def host_data(self):
        return tensor_h1_lagrange(self.dim, self.num_comp, self.P, self.Q, self.quad_mode)

    def apply(self, num_elem, t_mode, eval_mode, u, v, stream=None):
        if u is not None:
            _check_dev(u)
        _check_dev(v)
        call("fem_b200_basis_apply", self.h, num_elem, int(t_mode), int(eval_mode), _ptr(u),
             0 if u is None else _n(u), _ptr(v), _n(v), _stream(stream))


def mass_build(rx: Restriction, bx: Basis, x, qdata, stream=None) -> None:
    """qdata ([q][e], device) = det(dx/dX) * w from coordinates x (device)."""
    _check_dev(x)
    _check_dev(qdata)
    call("fem_b200_mass_build", rx.h, bx.h, _ptr(x), _n(x), _ptr(qdata), _n(qdata), _stream(stream))


class MassOperator(_Handle):
    """v = M u, the fused mass operator (its own copy of qdata)."""
    _destroy = "fem_b200_mass_destroy"

    def __init__(self, ru: Restriction, bu: Basis, qdata, qf=QF.apply_mass):
        super().__init__()
        _check_dev(qdata)
        call("fem_b200_mass_create", ru.h, bu.h, _ptr(qdata), _n(qdata), int(qf), C.addressof(self.h))
        self.l_size = ru.l_size
        self.qf = QF(qf)

    def apply(self, u, v, stream=None):
        _check_dev(u)
        _check_dev(v)
        call("fem_b200_mass_apply", self.h, _ptr(u), _n(u), _ptr(v), _n(v), _stream(stream))

    def apply_add(self, u, v, stream=None):
        _check_dev(u)
        _check_dev(v)
        call("fem_b200_mass_apply_add", self.h, _ptr(u), _n(u), _ptr(v), _n(v), _stream(stream))

    def apply_host(self, u: np.ndarray, v: np.ndarray | None = None, stream=None) -> np.ndarray:
        u = np.ascontiguousarray(u, dtype=np.float64)
        v = np.empty(self.l_size) if v is None else v
        call("fem_b200_mass_apply_host", self.h, _ptr(u), u.size, _ptr(v), v.size, _stream(stream))
        return v

    def info(self):
        launches, tile, variant = C.c_int(0), C.c_int(0), C.c_int(0)
        nbytes = C.c_int64(0)
        call("fem_b200_mass_info", self.h, C.addressof(launches), C.addressof(tile), C.addressof(nbytes),
             C.addressof(variant))
        return {"launches_per_apply": launches.value, "tile_elems": tile.value, "device_bytes": nbytes.value,
                "kernel": KernelVariant(variant.value).name}

    def set_kernel(self, variant) -> None:
        call("fem_b200_mass_set_kernel", self.h, int(variant))

    def set_host_chunks(self, chunks: int) -> None:
        """Chunks of apply_host's copy pipeline: 0 default, 1 unpipelined, n about n."""
        call("fem_b200_mass_set_host_chunks", self.h, int(chunks))

    def autotune(self, u, v, reps: int = 10, stream=None):
        """Time every kernel variant on (u, v) (v is scratch), keep the fastest;
        returns (variant name, ms per apply)."""
        _check_dev(u)
        _check_dev(v)
        chosen, ms = C.c_int(0), C.c_float(0.0)
        call("fem_b200_mass_autotune", self.h, _ptr(u), _n(u), _ptr(v), _n(v), int(reps), C.addressof(chosen),
             C.addressof(ms), _stream(stream))
        return KernelVariant(chosen.value).name, ms.value

    def apply_f32(self, u, v, stream=None):
        """v = M u in FP32 storage and arithmetic (float32 device tensors)."""
        _check_dev(u, "float32")
        _check_dev(v, "float32")
        call("fem_b200_mass_apply_f32", self.h, _ptr(u), _n(u), _ptr(v), _n(v), _stream(stream))

    def apply_f32_tc(self, u, v, split=True, stream=None):
        """v = M u in FP32 storage with the 1D contractions on the tensor cores
        (TF32 inputs, FP32 accumulation; split: 3xTF32, FP32-level accuracy)."""
        _check_dev(u, "float32")
        _check_dev(v, "float32")
        call("fem_b200_mass_apply_f32_tc", self.h, _ptr(u), _n(u), _ptr(v), _n(v), 1 if split else 0,
             _stream(stream))

    def apply_bf16_tc(self, u, v, stream=None):
        """v (float32) = M u, u (bfloat16) and qdata in BF16, contractions on the tensor cores."""
        _check_dev(u, "bfloat16")
        _check_dev(v, "float32")
        call("fem_b200_mass_apply_bf16_tc", self.h, _ptr(u), _n(u), _ptr(v), _n(v), _stream(stream))

    def apply_bf16(self, u, v, stream=None):
        """v (float32) = M u with u (bfloat16) and qdata in BF16 storage, FP32 arithmetic."""
        _check_dev(u, "bfloat16")
        _check_dev(v, "float32")
        call("fem_b200_mass_apply_bf16", self.h, _ptr(u), _n(u), _ptr(v), _n(v), _stream(stream))

    def diagonal(self, diag, stream=None) -> None:
        """diag (device, l_size) = the assembled diagonal of M."""
        _check_dev(diag)
        call("fem_b200_mass_diagonal", self.h, _ptr(diag), _n(diag), _stream(stream))

    def solve(self, f, u, rtol=1e-10, max_iter=1000, precision="fp64", stream=None) -> dict:
        """Solve M u = f (device arrays) by Jacobi PCG; precision 'fp64',
        'fp32_ir' (FP32 inner PCG in FP64 iterative refinement) or 'bf16_ir'
        (BF16-storage inner PCG, FP32 arithmetic, in FP64 refinement)."""
        _check_dev(f)
        _check_dev(u)
        prec = SOLVE_PRECISIONS[precision]
        its, outer, rel = C.c_int(0), C.c_int(0), C.c_double(0.0)
        call("fem_b200_mass_solve", self.h, _ptr(f), _n(f), _ptr(u), _n(u), float(rtol), int(max_iter), prec,
             C.addressof(its), C.addressof(outer), C.addressof(rel), _stream(stream))
        return {"iterations": its.value, "refinements": outer.value, "rel_residual": rel.value}

    def check(self, stream=None) -> None:
        """Synchronise and raise if a device-side wait of the plan's kernels ran out."""
        call("fem_b200_mass_check", self.h, _stream(stream))


class Batch(_Handle):
    """Many mass operators applied together, v_i = M_i u_i, as one captured
    CUDA graph (fem_b200_batch_*).  precision 'fp64' or 'fp32' (FP32 vectors
    and qdata).  The operators must outlive the batch."""
    _destroy = "fem_b200_batch_destroy"

    def __init__(self, ops, precision="fp64"):
        super().__init__()
        if precision not in ("fp64", "fp32"):
            raise ValueError("batch precision must be 'fp64' or 'fp32'")
        self.ops = list(ops)  # keeps the operators alive
        self.precision = precision
        arr = (C.c_void_p * len(self.ops))(*[op.h.value for op in self.ops])
        call("fem_b200_batch_create", C.addressof(arr), len(self.ops), {"fp64": 0, "fp32": 1}[precision],
             C.addressof(self.h))
        self._bound = None

    def bind(self, us, vs, stream=None) -> None:
        dt = "float64" if self.precision == "fp64" else "float32"
        assert len(us) == len(self.ops) and len(vs) == len(self.ops)
        for op, u, v in zip(self.ops, us, vs):
            _check_dev(u, dt)
            _check_dev(v, dt)
            if _n(u) != op.l_size or _n(v) != op.l_size:
                raise ValueError("batch bind: vector sizes must equal each operator's l_size")
        ua = (C.c_void_p * len(us))(*[_ptr(u) for u in us])
        va = (C.c_void_p * len(vs))(*[_ptr(v) for v in vs])
        call("fem_b200_batch_bind", self.h, C.addressof(ua), C.addressof(va), _stream(stream))
        self._bound = (list(us), list(vs))  # keeps the bound tensors alive

    def apply(self, graph=True, stream=None) -> None:
        call("fem_b200_batch_apply", self.h, int(bool(graph)), _stream(stream))

    def autotune(self, reps=5, stream=None) -> None:
        call("fem_b200_batch_autotune", self.h, int(reps), _stream(stream))

    MODES = {"auto": 0, "classes": 1, "persistent": 2}

    def set_mode(self, mode: str) -> None:
        """'persistent': one kernel launch for the whole batch; 'classes': one
        kernel per class; 'auto': the former where it applies, unless
        autotuning found the latter faster."""
        call("fem_b200_batch_set_mode", self.h, self.MODES[mode])

    def check(self, stream=None) -> None:
        call("fem_b200_batch_check", self.h, _stream(stream))

    def info(self) -> dict:
        nc, gk, pc, br = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0)
        tiles, dofs = C.c_int64(0), C.c_int64(0)
        call("fem_b200_batch_info", self.h, C.addressof(nc), C.addressof(tiles), C.addressof(dofs),
             C.addressof(gk), C.addressof(pc), C.addressof(br))
        return {"classes": nc.value, "tiles": tiles.value, "dofs": dofs.value, "graph_kernels": gk.value,
                "persistent_classes": pc.value, "graph_branches": br.value}


class _Request(C.Structure):
    """fem_b200_request (include/fem_b200.h)."""
    _fields_ = [("kind", C.c_int), ("dim", C.c_int), ("P", C.c_int), ("Q", C.c_int), ("num_comp", C.c_int),
                ("shape", C.c_int * 3), ("perturb", C.c_double), ("seed", C.c_uint64),
                ("num_elem", C.c_int), ("num_nodes", C.c_int), ("offsets", C.c_void_p), ("coords", C.c_void_p),
                ("f", C.c_void_p), ("rtol", C.c_double), ("max_iter", C.c_int), ("precision", C.c_int),
                ("scatter_mode", C.c_int), ("u_out", C.c_void_p), ("f_out", C.c_void_p)]


class _Result(C.Structure):
    """fem_b200_result (include/fem_b200.h)."""
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("refinements", C.c_int),
                ("rel_residual", C.c_double), ("t_submit", C.c_double), ("t_start", C.c_double),
                ("t_end", C.c_double), ("dofs", C.c_int64), ("device_bytes", C.c_int64),
                ("message", C.c_char * 256)]


class Server(_Handle):
    """Served mass solves (fem_b200_server_*): requests admitted by a device-
    memory budget into `slots` concurrent workers; see include/fem_b200.h."""
    _destroy = "fem_b200_server_destroy"

    def __init__(self, slots: int = 4, hbm_budget: int = 120 << 30):
        super().__init__()
        call("fem_b200_server_create", int(slots), int(hbm_budget), C.addressof(self.h))
        self._keep = {}  # host arrays a queued request still reads or writes

    def _submit(self, req, keep):
        rid = C.c_int64(0)
        call("fem_b200_server_submit", self.h, C.addressof(req), C.addressof(rid))
        self._keep[rid.value] = keep
        return rid.value

    @staticmethod
    def _common(req, dim, P, Q, num_comp, rtol, max_iter, precision, deterministic, u_out, f_out):
        req.dim, req.P, req.Q, req.num_comp = int(dim), int(P), int(Q if Q is not None else P + 1), int(num_comp)
        req.rtol, req.max_iter = float(rtol), int(max_iter)
        req.precision = SOLVE_PRECISIONS[precision]
        req.scatter_mode = 1 if deterministic else 0
        for name, a in (("u_out", u_out), ("f_out", f_out)):
            if a is not None:
                if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]):
                    raise ValueError(f"{name} must be a contiguous float64 numpy array")
                setattr(req, name, a.ctypes.data)

    def submit_box(self, dim, shape, P, Q=None, num_comp=1, seed=0, perturb=0.1, rtol=1e-10, max_iter=2000,
                   precision="fp32_ir", deterministic=False, u_out=None, f_out=None) -> int:
        """A box [0,1]^dim of `shape` elements generated on the device, f ~ U[-1,1]."""
        req = _Request()
        req.kind = 0
        self._common(req, dim, P, Q, num_comp, rtol, max_iter, precision, deterministic, u_out, f_out)
        for d, n in enumerate(shape):
            req.shape[d] = int(n)
        req.perturb, req.seed = float(perturb), int(seed)
        return self._submit(req, (u_out, f_out))

    def submit_mesh(self, dim, P, offsets, coords, f, Q=None, num_comp=1, rtol=1e-10, max_iter=2000,
                    precision="fp32_ir", deterministic=False, u_out=None) -> int:
        """A mesh from host arrays: offsets [num_elem*P^dim] int32, coordinates
        blocked [dim*num_nodes], f blocked [num_comp*num_nodes]."""
        offsets = np.ascontiguousarray(offsets, dtype=np.int32)
        coords = np.ascontiguousarray(coords, dtype=np.float64)
        f = np.ascontiguousarray(f, dtype=np.float64)
        req = _Request()
        req.kind = 1
        self._common(req, dim, P, Q, num_comp, rtol, max_iter, precision, deterministic, u_out, None)
        req.num_elem = offsets.size // (int(P) ** int(dim))
        req.num_nodes = coords.size // int(dim)
        if f.size != req.num_nodes * int(num_comp):
            raise ValueError("submit_mesh: f must have num_comp * num_nodes entries")
        req.offsets, req.coords, req.f = offsets.ctypes.data, coords.ctypes.data, f.ctypes.data
        return self._submit(req, (offsets, coords, f, u_out))

    def wait(self, rid: int, timeout=None) -> dict:
        res = _Result()
        call("fem_b200_server_wait", self.h, int(rid), -1.0 if timeout is None else float(timeout),
             C.addressof(res))
        self._keep.pop(rid, None)
        return {"status": res.status, "iterations": res.iterations, "refinements": res.refinements,
                "rel_residual": res.rel_residual, "t_submit": res.t_submit, "t_start": res.t_start,
                "t_end": res.t_end, "dofs": res.dofs, "device_bytes": res.device_bytes,
                "message": res.message.decode()}

    def stats(self) -> dict:
        sub, comp, pend, use, peak = (C.c_int64(0) for _ in range(5))
        run = C.c_int(0)
        call("fem_b200_server_stats", self.h, C.addressof(sub), C.addressof(comp), C.addressof(run),
             C.addressof(pend), C.addressof(use), C.addressof(peak))
        return {"submitted": sub.value, "completed": comp.value, "running": run.value, "pending": pend.value,
                "bytes_in_use": use.value, "bytes_peak": peak.value}


class ShardPlan(_Handle):
    """This rank's part of a mesh split into contiguous element ranges, through
    the C ABI (fem_b200_shard_*): sizes, the compact local numbering, the
    nodes shared with each peer, and the device pack / rank-ordered
    unpack-add of the interface exchange (the caller moves the segments)."""
    _destroy = "fem_b200_shard_destroy"

    def __init__(self, offsets, elem_size: int, world: int, rank: int):
        super().__init__()
        offsets = np.ascontiguousarray(offsets, dtype=np.int32)
        call("fem_b200_shard_create", offsets.size // elem_size, elem_size, _ptr(offsets), int(world), int(rank),
             C.addressof(self.h))
        e0, e1, nn, npeer = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0)
        tot = C.c_int64(0)
        call("fem_b200_shard_sizes", self.h, C.addressof(e0), C.addressof(e1), C.addressof(nn), C.addressof(npeer),
             C.addressof(tot))
        self.e0, self.e1, self.num_nodes, self.shared_total = e0.value, e1.value, nn.value, tot.value
        self.num_elem = self.e1 - self.e0
        self.offsets = np.zeros(self.num_elem * elem_size, np.int32)
        self.l2g = np.zeros(self.num_nodes, np.int64)
        owned = np.zeros(self.num_nodes, np.uint8)
        call("fem_b200_shard_local", self.h, _ptr(self.offsets), _ptr(self.l2g), _ptr(owned))
        self.owned = owned.astype(bool)
        self.peers = []  # (peer rank, local indices)
        for i in range(npeer.value):
            q, cnt = C.c_int(0), C.c_int64(0)
            call("fem_b200_shard_peer", self.h, i, C.addressof(q), C.addressof(cnt), None)
            idx = np.zeros(cnt.value, np.int64)
            call("fem_b200_shard_peer", self.h, i, None, None, _ptr(idx))
            self.peers.append((q.value, idx))

    def pack(self, v, send, num_comp=1, stream=None):
        _check_dev(v)
        _check_dev(send)
        call("fem_b200_shard_pack", self.h, _ptr(v), _n(v), int(num_comp), _ptr(send), _n(send), _stream(stream))

    def unpack_add(self, recv, v, num_comp=1, stream=None):
        _check_dev(recv)
        _check_dev(v)
        call("fem_b200_shard_unpack_add", self.h, _ptr(recv), _n(recv), int(num_comp), _ptr(v), _n(v),
             _stream(stream))
