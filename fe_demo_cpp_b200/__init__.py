"""fe_demo_cpp_b200: the fe-demo-cpp matrix-free mass operator on B200 (sm_100a).

The compute path is libfem_b200.so (hand-written CUDA + a C ABI, see
include/fem_b200.h); the C++ drop-in for the reference API is header-only
under include/fem/.  This Python package binds the C ABI (``api``), builds
the library in-tree (``build``) and makes the seeded benchmark meshes
(``mesh``).
"""
from ._lib import FemError, FemUnsupported, LIB_PATH, load  # noqa: F401
from .api import (  # noqa: F401
    QF,
    Basis,
    Batch,
    ContractMode,
    EvalMode,
    KernelVariant,
    MassOperator,
    QuadMode,
    Restriction,
    ScatterMode,
    Server,
    ShardPlan,
    check_offset_restriction,
    check_strided_restriction,
    gauss_legendre_quadrature,
    gauss_lobatto_points,
    lagrange_basis_matrix,
    mass_build,
    tensor_h1_lagrange,
    transpose_map,
)
