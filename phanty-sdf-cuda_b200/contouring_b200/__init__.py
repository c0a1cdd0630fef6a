"""B200-native dual-contouring backend (drop-in for the reference's IDualContouringBackend).

Public names mirror the reference module ``_contouring_cpp_module`` (src/cpp/bindings.cpp):
``DenseSdfGrid``, ``DenseSdfGridDevice``, ``DualContouringMesh``, ``DualContouringStats``,
``ContouringOptions``, ``ContouringMethod``, ``NormalComputationMode``; the new backends are
``B200DualContouringBackend`` and, for the reference's sparse CUDA backends,
``B200SparseDualContouringBackend`` / ``B200SparseMvdcDualContouringBackend``.
"""
from .backend import (B200DualContouringBackend, B200SparseDualContouringBackend,
                      B200SparseMvdcDualContouringBackend, ContouringMethod, ContouringOptions, DcbError,
                      DenseSdfGrid, DenseSdfGridDevice, DualContouringMesh, DualContouringStats,
                      MeshSdfStats, NormalComputationMode, PostprocessStats, mesh_to_sdf_cuda, mesh_to_sdf_tensor,
                      postprocess_mesh, postprocess_mesh_tensor)
from . import _lib


def __getattr__(name):
    # torch is imported only by the differentiable path
    if name in ("dual_contour", "DualContourFunction"):
        from . import autograd
        return getattr(autograd, name)
    raise AttributeError(name)

__all__ = ["B200DualContouringBackend", "B200SparseDualContouringBackend", "B200SparseMvdcDualContouringBackend",
           "NormalComputationMode", "ContouringMethod", "ContouringOptions", "DcbError",
           "DenseSdfGrid", "DenseSdfGridDevice", "DualContouringMesh", "DualContouringStats",
           "MeshSdfStats", "mesh_to_sdf_cuda", "mesh_to_sdf_tensor", "dual_contour", "DualContourFunction",
           "PostprocessStats", "postprocess_mesh", "postprocess_mesh_tensor"]
