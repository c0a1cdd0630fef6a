"""The reference CLI's file formats (src/cpp/dc_cli.cpp:17-47) on the C ABI's native readers and
writers: the binary ``.sdf`` grid and the OBJ mesh.

``read_sdf`` returns a :class:`DenseSdfGrid` like the reference's ``read_sdf``; ``read_obj`` /
``obj_grid`` / ``read_obj_to_sdf`` are the CLI's OBJ -> SDF ingestion (dc_cli.cpp:121-203) with the
conversion on the GPU; ``read_sdf_tensor``
reads straight into pinned host memory and uploads it to a CUDA tensor for ``extract_tensor``
(the torch path of ``extract_device``, src/cpp/bindings.cpp:223-227); ``write_obj`` formats the
mesh in parallel slices with the reference's text (6 significant digits, 1-based indices)."""
import ctypes
import os

import numpy as np

from . import _lib
from .backend import DenseSdfGrid, DualContouringMesh


def _path(p):
    return os.fsencode(os.fspath(p))


def read_sdf_header(path):
    """(dims, spacing, origin) of a ``.sdf`` file."""
    h = _lib.DcbGrid()
    _lib.check(_lib.lib().dcb_read_sdf(_path(path), ctypes.byref(h), None, 0))
    return (h.nx, h.ny, h.nz), (h.vx, h.vy, h.vz), (h.ox, h.oy, h.oz)


def _read_into(path, buf, n):
    h = _lib.DcbGrid()
    _lib.check(_lib.lib().dcb_read_sdf(_path(path), ctypes.byref(h), buf, n))


def read_sdf(path):
    """``read_sdf`` (dc_cli.cpp:31-47): a :class:`DenseSdfGrid` with float32 values."""
    dims, sp, org = read_sdf_header(path)
    n = dims[0] * dims[1] * dims[2]
    vals = np.empty(n, np.float32)
    _read_into(path, vals.ctypes.data, n)
    return DenseSdfGrid(*dims, *sp, *org, values=vals)


def read_sdf_tensor(path, device="cuda"):
    """The grid of a ``.sdf`` file as a CUDA float32 tensor, read into pinned host memory and
    copied asynchronously; returns ``(values, dims, spacing, origin)`` for ``extract_tensor``."""
    import torch
    dims, sp, org = read_sdf_header(path)
    n = dims[0] * dims[1] * dims[2]
    host = torch.empty(n, dtype=torch.float32, pin_memory=True)
    _read_into(path, host.data_ptr(), n)
    return host.to(device, non_blocking=True), dims, sp, org


def write_sdf(path, grid):
    """The inverse of :func:`read_sdf` (``grid.values`` on the host)."""
    vals = np.ascontiguousarray(np.asarray(grid.values, dtype=np.float32).reshape(-1))
    g = _lib.DcbGrid(int(grid.nx), int(grid.ny), int(grid.nz), float(grid.vx), float(grid.vy), float(grid.vz),
                     float(grid.ox), float(grid.oy), float(grid.oz), vals.ctypes.data)
    _lib.check(_lib.lib().dcb_write_sdf(_path(path), ctypes.byref(g)))


def write_obj(path, vertices, faces=None, verts_per_face=4, threads=0):
    """``write_obj`` (dc_cli.cpp:17-29). ``vertices`` may be a :class:`DualContouringMesh`
    (its faces are quads), or float32 vertices (N, 3) with int32 faces (M, verts_per_face);
    numpy arrays or torch tensors (copied to the host)."""
    if isinstance(vertices, DualContouringMesh):
        faces = vertices.faces
        vertices = vertices.vertices
        verts_per_face = 4
    V = np.ascontiguousarray(_host(vertices), dtype=np.float32).reshape(-1)
    F = np.ascontiguousarray(_host(faces if faces is not None else np.zeros(0, np.int32)), dtype=np.int32).reshape(-1)
    nv, nf = V.size // 3, F.size // verts_per_face
    _lib.check(_lib.lib().dcb_write_obj(_path(path), V.ctypes.data if nv else None, nv,
                                        F.ctypes.data if nf else None, nf, int(verts_per_face), int(threads)))


def _host(a):
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def read_obj(path):
    """The OBJ reading of ``read_obj_to_sdf`` (dc_cli.cpp:121-158): float32 vertices (N, 3) and
    int32 triangles (M, 3) (polygons fanned from their first vertex)."""
    L = _lib.lib()
    nv, nt = ctypes.c_int64(), ctypes.c_int64()
    _lib.check(L.dcb_read_obj(_path(path), None, 0, None, 0, ctypes.byref(nv), ctypes.byref(nt)))
    V = np.empty((nv.value, 3), np.float32)
    T = np.empty((nt.value, 3), np.int32)
    _lib.check(L.dcb_read_obj(_path(path), V.ctypes.data, nv.value, T.ctypes.data, nt.value,
                              ctypes.byref(nv), ctypes.byref(nt)))
    return V, T


def obj_grid(vertices, res):
    """(dims, spacing, origin) of the grid ``read_obj_to_sdf`` puts around a mesh
    (dc_cli.cpp:160-184): the bounding box grown by 8% of its diagonal, res points per axis."""
    V = np.ascontiguousarray(_host(vertices), dtype=np.float32).reshape(-1)
    g = _lib.DcbGrid()
    _lib.check(_lib.lib().dcb_obj_grid(V.ctypes.data if V.size else None, V.size // 3, int(res), ctypes.byref(g)))
    return (g.nx, g.ny, g.nz), (g.vx, g.vy, g.vz), (g.ox, g.oy, g.oz)


def read_obj_to_sdf(backend, path, res, voxelize_first=False, voxel_res=256):
    """``read_obj_to_sdf`` (dc_cli.cpp:121-203): the OBJ's signed distance grid, computed on the
    GPU; returns ``(DenseSdfGrid, milliseconds of the conversion)``."""
    from .backend import mesh_to_sdf_cuda
    V, T = read_obj(path)
    dims, sp, org = obj_grid(V, res)
    return mesh_to_sdf_cuda(backend, V, T, *dims, *org, *sp, voxelize_first=voxelize_first, voxel_res=voxel_res)
