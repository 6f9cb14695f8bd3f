"""ctypes binding of libfem_b200.so (the C ABI in include/fem_b200.h).

The library is built in-tree by ``python -m fe_demo_cpp_b200.build``.  There
is no fallback: if the library is missing, loading fails with an error that
says how to build it.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libfem_b200.so")

SUCCESS, ERROR_ARGUMENT, ERROR_CUDA, ERROR_UNSUPPORTED, NOT_READY = 0, 1, 2, 3, 4

_i, _i64, _p, _dp, _ip = C.c_int, C.c_int64, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)

# name -> argtypes (every entry point of include/fem_b200.h)
SIGNATURES = {
    "fem_b200_last_error": ([], C.c_char_p),
    "fem_b200_version": ([], _i),
    "fem_b200_device_count": ([], _i),
    "fem_b200_gauss_legendre": ([_i, _p, _p], _i),
    "fem_b200_gauss_lobatto": ([_i, _p, _p], _i),
    "fem_b200_lagrange_basis_matrix": ([_i, _p, _i, _p, _p, _p], _i),
    "fem_b200_tensor_h1_lagrange": ([_i, _i, _i, _i, _i, _p, _p, _p, _p], _i),
    "fem_b200_restriction_check_offset": ([_i, _i, _i, _i, _i, _p, _i64], _i),
    "fem_b200_restriction_check_strided": ([_i, _i, _i, _i, _p], _i),
    "fem_b200_transpose_map": ([_i, _i, _i, _p, _p, _p, _p, _p], _i),
    "fem_b200_restriction_create_offset": ([_i, _i, _i, _i, _i, _p, _i, _p], _i),
    "fem_b200_restriction_create_strided": ([_i, _i, _i, _i, _p, _p], _i),
    "fem_b200_restriction_destroy": ([_p], _i),
    "fem_b200_restriction_sizes": ([_p, _p, _p, _p, _p, _p], _i),
    "fem_b200_restriction_transpose_map": ([_p, _p, _p, _p, _p], _i),
    "fem_b200_restriction_apply": ([_p, _i, _p, _i64, _p, _i64, _p], _i),
    "fem_b200_restriction_multiplicity": ([_p, _p, _i64, _p], _i),
    "fem_b200_basis_create": ([_i, _i, _i, _i, _i, _p], _i),
    "fem_b200_basis_create_from": ([_i, _i, _i, _i, _p, _p, _p, _p], _i),
    "fem_b200_basis_destroy": ([_p], _i),
    "fem_b200_basis_apply": ([_p, _i, _i, _i, _p, _i64, _p, _i64, _p], _i),
    "fem_b200_basis_apply_static": ([_p, _i, _i, _i, _p, _i64, _p, _i64, _p], _i),
    "fem_b200_malloc": ([_p, C.c_size_t], _i),
    "fem_b200_free": ([_p], _i),
    "fem_b200_memcpy": ([_p, _p, C.c_size_t, _i, _p], _i),
    "fem_b200_memset_zero": ([_p, C.c_size_t, _p], _i),
    "fem_b200_synchronize": ([_p], _i),
    "fem_b200_device_info": ([_i, _p, _i, _p, _p], _i),
    "fem_b200_offset_gather": ([_i, _i, _i, _i, _p, _p, _p, _p], _i),
    "fem_b200_offset_scatter_add": ([_i, _i, _i, _i, _p, _p, _p, _p], _i),
    "fem_b200_transpose_scatter_add": ([_i, _i, _i, _i, _i, _p, _p, _p, _p, _p, _p], _i),
    "fem_b200_strided_apply": ([_i, _i, _i, _i, _p, _p, _p, _p], _i),
    "fem_b200_contract": ([_i64, _i, _i64, _i, _p, _i, _i, _p, _p, _p], _i),
    "fem_b200_qfunction_apply_mass": ([_i64, _p, _p, _p, _p], _i),
    "fem_b200_qfunction_build_mass": ([_i, _i64, _p, _p, _p, _p], _i),
    "fem_b200_mass_build": ([_p, _p, _p, _i64, _p, _i64, _p], _i),
    "fem_b200_mass_create": ([_p, _p, _p, _i64, _i, _p], _i),
    "fem_b200_mass_destroy": ([_p], _i),
    "fem_b200_mass_apply": ([_p, _p, _i64, _p, _i64, _p], _i),
    "fem_b200_mass_apply_add": ([_p, _p, _i64, _p, _i64, _p], _i),
    "fem_b200_mass_apply_host": ([_p, _p, _i64, _p, _i64, _p], _i),
    "fem_b200_mass_info": ([_p, _p, _p, _p, _p], _i),
    "fem_b200_mass_set_kernel": ([_p, _i], _i),
    "fem_b200_mass_apply_f32_tc": ([_p, _p, _i64, _p, _i64, _i, _p], _i),
    "fem_b200_mass_apply_bf16_tc": ([_p, _p, _i64, _p, _i64, _p], _i),
    "fem_b200_tc_selftest": ([_p], _i),
    "fem_b200_mass_set_host_chunks": ([_p, _i], _i),
    "fem_b200_mass_check": ([_p, _p], _i),
    "fem_b200_mass_diagonal": ([_p, _p, _i64, _p], _i),
    "fem_b200_mass_solve": ([_p, _p, _i64, _p, _i64, C.c_double, _i, _i, _p, _p, _p, _p], _i),
    "fem_b200_mass_apply_f32": ([_p, _p, _i64, _p, _i64, _p], _i),
    "fem_b200_mass_apply_bf16": ([_p, _p, _i64, _p, _i64, _p], _i),
    "fem_b200_batch_create": ([_p, _i, _i, _p], _i),
    "fem_b200_batch_bind": ([_p, _p, _p, _p], _i),
    "fem_b200_batch_apply": ([_p, _i, _p], _i),
    "fem_b200_batch_autotune": ([_p, _i, _p], _i),
    "fem_b200_batch_set_mode": ([_p, _i], _i),
    "fem_b200_batch_check": ([_p, _p], _i),
    "fem_b200_shard_create": ([_i, _i, _p, _i, _i, _p], _i),
    "fem_b200_shard_sizes": ([_p, _p, _p, _p, _p, _p], _i),
    "fem_b200_shard_local": ([_p, _p, _p, _p], _i),
    "fem_b200_shard_peer": ([_p, _i, _p, _p, _p], _i),
    "fem_b200_shard_pack": ([_p, _p, _i64, _i, _p, _i64, _p], _i),
    "fem_b200_shard_unpack_add": ([_p, _p, _i64, _i, _p, _i64, _p], _i),
    "fem_b200_shard_destroy": ([_p], _i),
    "fem_b200_batch_info": ([_p, _p, _p, _p, _p, _p, _p], _i),
    "fem_b200_batch_destroy": ([_p], _i),
    "fem_b200_server_create": ([_i, _i64, _p], _i),
    "fem_b200_server_submit": ([_p, _p, _p], _i),
    "fem_b200_server_wait": ([_p, _i64, C.c_double, _p], _i),
    "fem_b200_server_stats": ([_p, _p, _p, _p, _p, _p, _p], _i),
    "fem_b200_server_destroy": ([_p], _i),
    "fem_b200_mass_autotune": ([_p, _p, _i64, _p, _i64, _i, _p, _p, _p], _i),
}

_lib = None


class FemError(RuntimeError):
    """A CUDA or device-path failure reported by libfem_b200."""


class FemUnsupported(FemError):
    """A valid request the device path does not implement (no CPU fallback)."""


def load(path: str = LIB_PATH) -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FemError(f"{path} is missing: build it with `python -m fe_demo_cpp_b200.build` "
                       "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (argtypes, restype) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = restype
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc == SUCCESS:
        return
    msg = load().fem_b200_last_error().decode()
    if rc == ERROR_ARGUMENT:
        raise ValueError(msg)
    if rc == ERROR_UNSUPPORTED:
        raise FemUnsupported(msg)
    if rc == NOT_READY:
        raise TimeoutError("the request has not finished within the timeout")
    raise FemError(msg)


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))
