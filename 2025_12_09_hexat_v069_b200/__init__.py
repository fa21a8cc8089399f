"""B200-native (sm_100a) inner-solve library for HEXA(T) v069.

The compute path is libhexat_b200.so (hand-written CUDA, C ABI in
include/hexat_b200.h); this package is its Python host side: ctypes binding
(_lib), reference-shaped entry points (api), mesh/boundary set-up in the
reference's layout (mesh, boundary), the OC loop driver (topopt) and the
synthetic workloads (workloads).
"""
from . import boundary, mesh, workloads  # noqa: F401
from ._lib import Context, HexatError, default_opts, load  # noqa: F401

__all__ = ["Context", "HexatError", "default_opts", "load", "mesh", "boundary", "workloads"]
