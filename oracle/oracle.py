"""ctypes wrapper around the CPU oracle library (TEST INFRASTRUCTURE ONLY).

The oracle is the FP64 C++ restatement in ``oracle/dc_oracle.cpp`` of the reference's
``CpuDualContouringBackend::extract`` (src/cpp/dc_backend.cpp:51-125), and the float
restatement in ``oracle/mts_oracle.cpp`` of its mesh -> SDF conversion
(src/cuda/mesh_to_sdf_cuda.cu:740-1009), and ``oracle/sparse_oracle.cpp``: the float restatement of the reference's sparse (brick) and
multi-vertex GPU backends (src/cuda/dc_cuda_sparse.cu), and ``oracle/dc_adjoint_oracle.cpp``: the per-cell
FP64 vertex as a template run with double (for finite differences) and with dual numbers
(the FP64 reference Jacobian of each vertex with respect to its 4x4x4 stencil).  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference legs import this
module, and only as the checker or the CPU baseline, never as the product path.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_DC_LIB = os.path.join(_HERE, "_build", "libdc_oracle.so")
_MTS_LIB = os.path.join(_HERE, "_build", "libmts_oracle.so")
_ADJ_LIB = os.path.join(_HERE, "_build", "libdc_adjoint_oracle.so")
_OURS_LIB = os.path.join(_HERE, "_build", "libours_oracle.so")
_SPARSE_LIB = os.path.join(_HERE, "_build", "libsparse_oracle.so")
_POST_LIB = os.path.join(_HERE, "_build", "libpost_oracle.so")
_libs = {}


def build():
    """Compile the oracle libraries with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


class _Stats(ctypes.Structure):
    _fields_ = [("total_cells", ctypes.c_int64), ("active_cells", ctypes.c_int64),
                ("vertex_count", ctypes.c_int64), ("face_count", ctypes.c_int64),
                ("total_ms", ctypes.c_double)]


def _load(path):
    if path not in _libs:
        if not os.path.exists(path):
            build()
        _libs[path] = ctypes.CDLL(path)
    return _libs[path]


def _dc():
    lib = _load(_DC_LIB)
    if not getattr(lib, "_typed", False):
        lib.dco_extract.restype = ctypes.c_void_p
        lib.dco_extract.argtypes = [ctypes.c_int] * 3 + [ctypes.c_float] * 6 + [
            ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.POINTER(_Stats)]
        lib.dco_num_vertices.restype = ctypes.c_int64
        lib.dco_num_vertices.argtypes = [ctypes.c_void_p]
        lib.dco_num_faces.restype = ctypes.c_int64
        lib.dco_num_faces.argtypes = [ctypes.c_void_p]
        lib.dco_copy.restype = None
        lib.dco_copy.argtypes = [ctypes.c_void_p] * 6
        lib.dco_free.restype = None
        lib.dco_free.argtypes = [ctypes.c_void_p]
        lib.dco_extract_pos.restype = ctypes.c_void_p
        lib.dco_extract_pos.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p] * 4 + [
            ctypes.c_double, ctypes.c_int, ctypes.POINTER(_Stats)]
        lib._typed = True
    return lib


def _collect(lib, h, st):
    if not h:
        raise ValueError("oracle rejected the grid")
    try:
        nv = lib.dco_num_vertices(h)
        nf = lib.dco_num_faces(h)
        V = np.empty((nv, 3), np.float64)
        F = np.empty((nf, 4), np.int32)
        cells = np.empty(nv, np.int64)
        eig = np.empty((nv, 3), np.float64)
        nrows = np.empty(nv, np.int32)
        lib.dco_copy(h, V.ctypes.data, F.ctypes.data, cells.ctypes.data, eig.ctypes.data,
                     nrows.ctypes.data)
    finally:
        lib.dco_free(h)
    stats = {k: getattr(st, k) for k, _ in _Stats._fields_}
    return {"V": V, "F": F, "cells": cells, "eig": eig, "nrows": nrows, "stats": stats}


def dc_extract_positions(values, dims, px, py, pz, svd_threshold=0.01, threads=0):
    """Like dc_extract, with explicit float64 grid-point coordinates per axis."""
    nx, ny, nz = (int(d) for d in dims)
    vals = np.ascontiguousarray(np.asarray(values, dtype=np.float32).reshape(-1))
    axes = [np.ascontiguousarray(np.asarray(a, dtype=np.float64)) for a in (px, py, pz)]
    if vals.size != nx * ny * nz or [a.size for a in axes] != [nx, ny, nz]:
        raise ValueError("shape mismatch")
    lib = _dc()
    st = _Stats()
    h = lib.dco_extract_pos(nx, ny, nz, axes[0].ctypes.data, axes[1].ctypes.data, axes[2].ctypes.data,
                            vals.ctypes.data, float(svd_threshold), int(threads), ctypes.byref(st))
    return _collect(lib, h, st)


def dc_extract(values, dims, spacing, origin, svd_threshold=0.01, threads=0):
    """Run the restated CPU dual contouring on a dense x-fastest float32 grid.

    ``values`` has ``nx*ny*nz`` float32 entries, index ``i + nx*(j + ny*k)``.
    Returns a dict with FP64 vertices ``V`` (nv,3), int32 quads ``F`` (nf,4), the linear
    index of each vertex's cell ``cells``, the eigenvalues of each cell's A^T A ``eig``,
    the Hermite row count ``nrows`` and ``stats``.
    """
    nx, ny, nz = (int(d) for d in dims)
    vals = np.ascontiguousarray(np.asarray(values, dtype=np.float32).reshape(-1))
    if vals.size != nx * ny * nz:
        raise ValueError("values has %d entries, expected %d" % (vals.size, nx * ny * nz))
    lib = _dc()
    st = _Stats()
    h = lib.dco_extract(nx, ny, nz, float(spacing[0]), float(spacing[1]), float(spacing[2]),
                        float(origin[0]), float(origin[1]), float(origin[2]),
                        vals.ctypes.data, float(svd_threshold), int(threads), ctypes.byref(st))
    if not h:
        raise ValueError("oracle rejected the grid")
    try:
        nv = lib.dco_num_vertices(h)
        nf = lib.dco_num_faces(h)
        V = np.empty((nv, 3), np.float64)
        F = np.empty((nf, 4), np.int32)
        cells = np.empty(nv, np.int64)
        eig = np.empty((nv, 3), np.float64)
        nrows = np.empty(nv, np.int32)
        lib.dco_copy(h, V.ctypes.data, F.ctypes.data, cells.ctypes.data, eig.ctypes.data,
                     nrows.ctypes.data)
    finally:
        lib.dco_free(h)
    stats = {k: getattr(st, k) for k, _ in _Stats._fields_}
    return {"V": V, "F": F, "cells": cells, "eig": eig, "nrows": nrows, "stats": stats}


def triangulate(V, F):
    """triangulate_v1 (src/cpp/contouring.cpp:88-113) with orient_triangles_for_quad
    (:40-86): quad (a,b,c,d) -> (a,b,c), (a,c,d), each flipped when its normal points against
    the quad normal (pb-pa)x(pd-pa) [fallback (pc-pa)x(pd-pa) below 1e-24; none below that
    too]. V are the FP64 vertices, F the quads; returns int32 triangles (2 per quad)."""
    F = np.asarray(F, np.int64).reshape(-1, 4)
    V = np.asarray(V, np.float64)
    a, b, c, d = F[:, 0], F[:, 1], F[:, 2], F[:, 3]
    pa, pb, pc, pd = V[a], V[b], V[c], V[d]

    def dot(u, v):
        return (u[:, 0] * v[:, 0] + u[:, 1] * v[:, 1]) + u[:, 2] * v[:, 2]
    qn = np.cross(pb - pa, pd - pa)
    fb = dot(qn, qn) < 1e-24
    qn[fb] = np.cross(pc - pa, pd - pa)[fb]
    orient = ~(dot(qn, qn) < 1e-24)
    flip0 = orient & (dot(np.cross(pb - pa, pc - pa), qn) < 0.0)
    flip1 = orient & (dot(np.cross(pc - pa, pd - pa), qn) < 0.0)
    T = np.empty((len(F), 2, 3), np.int64)
    T[:, 0, 0], T[:, 0, 1], T[:, 0, 2] = a, np.where(flip0, c, b), np.where(flip0, b, c)
    T[:, 1, 0], T[:, 1, 1], T[:, 1, 2] = a, np.where(flip1, d, c), np.where(flip1, c, d)
    return T.reshape(-1, 3).astype(np.int32)


class _MtsStats(ctypes.Structure):
    _fields_ = [("num_bins", ctypes.c_int64), ("bin_entries", ctypes.c_int64),
                ("band_points", ctypes.c_int64), ("exterior_filled", ctypes.c_int64)]


def _mts():
    lib = _load(_MTS_LIB)
    if not getattr(lib, "_typed", False):
        common = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64] + [ctypes.c_int] * 3 + \
                 [ctypes.c_float] * 6
        lib.mts_compute.argtypes = common + [ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(_MtsStats)]
        lib.mts_compute.restype = ctypes.c_int
        lib.mts_band_values.argtypes = common + [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p]
        lib.mts_band_values.restype = ctypes.c_int
        lib.mts_compute_voxelized.argtypes = common + [ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                       ctypes.POINTER(_MtsStats), ctypes.c_void_p]
        lib.mts_compute_voxelized.restype = ctypes.c_int
        lib._typed = True
    return lib


def _mesh_args(V, F):
    V = np.ascontiguousarray(np.asarray(V, np.float32).reshape(-1, 3))
    F = np.ascontiguousarray(np.asarray(F, np.int32).reshape(-1, 3))
    if len(F) and (F.min() < 0 or F.max() >= len(V)):
        raise ValueError("face index out of range")
    return V, F


def mesh_to_sdf(V, F, dims, origin, spacing, threads=0):
    """The whole mesh -> SDF conversion; returns (float32 values, nx*ny*nz, x fastest; stats)."""
    V, F = _mesh_args(V, F)
    nx, ny, nz = (int(d) for d in dims)
    out = np.empty(nx * ny * nz, np.float32)
    st = _MtsStats()
    rc = _mts().mts_compute(V.ctypes.data, len(V), F.ctypes.data, len(F), nx, ny, nz,
                            *[float(x) for x in origin], *[float(x) for x in spacing], int(threads),
                            out.ctypes.data, ctypes.byref(st))
    if rc != 0:
        raise ValueError("oracle rejected the input")
    return out, {k: getattr(st, k) for k, _ in _MtsStats._fields_}


def mesh_to_sdf_voxelized(V, F, dims, origin, spacing, voxel_res=256, threads=0, return_solid=False):
    """The conversion with voxelize_first: far points signed by a voxel_res^3 solid. Returns
    (float32 values, stats), plus the solid (uint8, (vres, vres, vres) z-major) if asked."""
    V, F = _mesh_args(V, F)
    nx, ny, nz = (int(d) for d in dims)
    out = np.empty(nx * ny * nz, np.float32)
    st = _MtsStats()
    vr = max(32, min(2048, int(voxel_res)))
    solid = np.empty(vr ** 3, np.uint8) if return_solid else None
    rc = _mts().mts_compute_voxelized(V.ctypes.data, len(V), F.ctypes.data, len(F), nx, ny, nz,
                                      *[float(x) for x in origin], *[float(x) for x in spacing], int(voxel_res),
                                      int(threads), out.ctypes.data, ctypes.byref(st),
                                      solid.ctypes.data if return_solid else None)
    if rc != 0:
        raise ValueError("oracle rejected the input")
    stats = {k: getattr(st, k) for k, _ in _MtsStats._fields_}
    if return_solid:
        return out, stats, solid.reshape(vr, vr, vr)
    return out, stats


def mesh_band_values(V, F, dims, origin, spacing, idx, threads=0):
    """Band values (before the sign fill and relaxation) at the listed linear point indices."""
    V, F = _mesh_args(V, F)
    nx, ny, nz = (int(d) for d in dims)
    idx = np.ascontiguousarray(np.asarray(idx, np.int64))
    out = np.empty(len(idx), np.float32)
    rc = _mts().mts_band_values(V.ctypes.data, len(V), F.ctypes.data, len(F), nx, ny, nz,
                                *[float(x) for x in origin], *[float(x) for x in spacing],
                                idx.ctypes.data, len(idx), int(threads), out.ctypes.data)
    if rc != 0:
        raise ValueError("oracle rejected the input")
    return out


def _adj():
    lib = _load(_ADJ_LIB)
    if not getattr(lib, "_typed", False):
        args = [ctypes.c_int] * 3 + [ctypes.c_void_p] * 6 + [ctypes.c_int64, ctypes.c_double, ctypes.c_void_p]
        lib.dca_cell_vertices.argtypes = args + [ctypes.c_void_p, ctypes.c_int]
        lib.dca_cell_vertices.restype = ctypes.c_int
        lib.dca_cell_jacobians.argtypes = args + [ctypes.c_void_p, ctypes.c_int]
        lib.dca_cell_jacobians.restype = ctypes.c_int
        lib._typed = True
    return lib


def _adj_args(values, dims, axes, cells):
    nx, ny, nz = (int(d) for d in dims)
    v = np.asarray(values).reshape(-1)
    if v.dtype == np.float64:
        vf, vd = None, np.ascontiguousarray(v)
    else:
        vf, vd = np.ascontiguousarray(v, dtype=np.float32), None
    ax = [np.ascontiguousarray(np.asarray(a, np.float64)) for a in axes]
    if (vf if vf is not None else vd).size != nx * ny * nz or [a.size for a in ax] != [nx, ny, nz]:
        raise ValueError("shape mismatch")
    cells = np.ascontiguousarray(np.asarray(cells, np.int64))
    keep = (vf, vd, ax, cells)
    ptr = lambda a: None if a is None else a.ctypes.data
    return keep, [nx, ny, nz, ax[0].ctypes.data, ax[1].ctypes.data, ax[2].ctypes.data, ptr(vf), ptr(vd),
                  cells.ctypes.data, len(cells)]


def cell_vertices(values, dims, axes, cells, svd_threshold=0.01, threads=0, return_kept=False):
    """FP64 vertices of the listed active cells (linear i + cx*(j + cy*k)); ``values`` float32
    or float64 (nx*ny*nz, x fastest), ``axes`` the float64 grid-point coordinates per axis.
    With ``return_kept`` also the number of eigenvalues each cell's solve keeps."""
    keep, args = _adj_args(values, dims, axes, cells)
    out = np.empty((len(keep[3]), 3), np.float64)
    kept = np.empty(len(keep[3]), np.int32)
    if _adj().dca_cell_vertices(*args, float(svd_threshold), out.ctypes.data, kept.ctypes.data, int(threads)) != 0:
        raise ValueError("oracle rejected the grid")
    return (out, kept) if return_kept else out


def cell_jacobians(values, dims, axes, cells, svd_threshold=0.01, threads=0):
    """(vertices (n,3), jac (n,3,64)): the FP64 reference Jacobian of each listed cell's vertex
    with respect to the values of its stencil, slot s = grid point (i-1+s%4, j-1+(s//4)%4,
    k-1+s//16), by forward-mode automatic differentiation."""
    keep, args = _adj_args(values, dims, axes, cells)
    n = len(keep[3])
    out = np.empty((n, 3), np.float64)
    jac = np.empty((n, 3, 64), np.float64)
    if _adj().dca_cell_jacobians(*args, float(svd_threshold), out.ctypes.data, jac.ctypes.data, int(threads)) != 0:
        raise ValueError("oracle rejected the grid")
    return out, jac


def vertex_vjp(values, dims, axes, cells, grad_vertices, svd_threshold=0.01, threads=0):
    """FP64 reference adjoint: d(loss)/d(grid values) (float64, nx*ny*nz) from
    d(loss)/d(vertices) of the listed cells, as the sum of J^T g over the cells."""
    nx, ny, nz = (int(d) for d in dims)
    cells = np.asarray(cells, np.int64)
    _, jac = cell_jacobians(values, dims, axes, cells, svd_threshold, threads)
    contrib = np.einsum("nds,nd->ns", jac, np.asarray(grad_vertices, np.float64))
    cx, cy = nx - 1, ny - 1
    i, j, k = cells % cx, (cells // cx) % cy, cells // (cx * cy)
    s = np.arange(64)
    gi = i[:, None] - 1 + s % 4
    gj = j[:, None] - 1 + (s // 4) % 4
    gk = k[:, None] - 1 + s // 16
    inside = (gi >= 0) & (gi < nx) & (gj >= 0) & (gj < ny) & (gk >= 0) & (gk < nz)
    if np.any(contrib[~inside] != 0.0):
        raise AssertionError("derivative with respect to a point outside the grid")
    out = np.zeros(nx * ny * nz, np.float64)
    np.add.at(out, (gi + nx * (gj + ny * gk))[inside], contrib[inside])
    return out


class _OursOpts(ctypes.Structure):
    _fields_ = [("outer_iters", ctypes.c_int), ("inner_iters", ctypes.c_int), ("mu", ctypes.c_double),
                ("dc_weight", ctypes.c_double), ("sphere_weight", ctypes.c_double),
                ("svd_threshold", ctypes.c_double), ("hermite_update", ctypes.c_int), ("batch_size", ctypes.c_int),
                ("new_hermite_pos_weight", ctypes.c_double), ("new_face_pos_weight", ctypes.c_double),
                ("new_hermite_normal_weight", ctypes.c_double), ("seed", ctypes.c_uint64)]


def ours(values, dims, spacing, origin, outer_iters=100, inner_iters=100, mu=0.1, dc_weight=0.02,
         sphere_weight=1.0, svd_threshold=0.01, hermite_update=True, batch_size=200000,
         new_hermite_pos_weight=0.2, new_face_pos_weight=0.2, new_hermite_normal_weight=0.2, seed=0x5eed,
         threads=0):
    """The restated outer/inner refinement (ContouringMethod::Ours) on a dense float32 grid:
    dict with FP64 vertices ``V``, wound quads ``F`` and the active ``cells``."""
    lib = _load(_OURS_LIB)
    if not getattr(lib, "_typed", False):
        lib.dco_ours.restype = ctypes.c_void_p
        lib.dco_ours.argtypes = [ctypes.c_int] * 3 + [ctypes.c_float] * 6 + [
            ctypes.c_void_p, ctypes.POINTER(_OursOpts), ctypes.c_int, ctypes.POINTER(_Stats)]
        lib.dco_num_vertices.restype = ctypes.c_int64
        lib.dco_num_vertices.argtypes = [ctypes.c_void_p]
        lib.dco_num_faces.restype = ctypes.c_int64
        lib.dco_num_faces.argtypes = [ctypes.c_void_p]
        lib.dco_copy.restype = None
        lib.dco_copy.argtypes = [ctypes.c_void_p] * 6
        lib.dco_free.restype = None
        lib.dco_free.argtypes = [ctypes.c_void_p]
        lib._typed = True
    nx, ny, nz = (int(d) for d in dims)
    vals = np.ascontiguousarray(np.asarray(values, dtype=np.float32).reshape(-1))
    if vals.size != nx * ny * nz:
        raise ValueError("shape mismatch")
    o = _OursOpts(int(outer_iters), int(inner_iters), float(mu), float(dc_weight), float(sphere_weight),
                  float(svd_threshold), int(bool(hermite_update)), int(batch_size), float(new_hermite_pos_weight),
                  float(new_face_pos_weight), float(new_hermite_normal_weight), int(seed))
    st = _Stats()
    h = lib.dco_ours(nx, ny, nz, float(spacing[0]), float(spacing[1]), float(spacing[2]),
                     float(origin[0]), float(origin[1]), float(origin[2]), vals.ctypes.data, ctypes.byref(o),
                     int(threads), ctypes.byref(st))
    return _collect(lib, h, st)


SPARSE_STATS = ("total_bricks", "active_bricks", "active_cells", "qef_fallbacks", "clamps", "invalid",
                "ambiguous_cells", "multi_vertex_cells", "one_vertex_cells", "two_vertex_cells",
                "split_rejections", "faces_skipped")


def _sparse():
    lib = _load(_SPARSE_LIB)
    if not getattr(lib, "_typed", False):
        lib.sdo_extract.restype = ctypes.c_void_p
        lib.sdo_extract.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 3 + [ctypes.c_float] * 6 + [ctypes.c_int] * 4
        for f in ("sdo_num_vertices", "sdo_num_faces", "sdo_num_cells"):
            getattr(lib, f).restype = ctypes.c_int64
            getattr(lib, f).argtypes = [ctypes.c_void_p]
        lib.sdo_copy.restype = None
        lib.sdo_copy.argtypes = [ctypes.c_void_p] * 7
        lib.sdo_free.restype = None
        lib.sdo_free.argtypes = [ctypes.c_void_p]
        lib._typed = True
    return lib


def sparse_extract(values, dims, spacing, origin, brick_size=8, mvdc=False, normal_mode=0, threads=0):
    """The reference's sparse brick backend (mvdc=False) or its multi-vertex variant
    (mvdc=True), restated in float. Returns V (float32), vertex normals N (float32, the
    multi-vertex variant's per-vertex normals), quads F (int32), the active cells' linear
    indices, each active cell's first vertex, and the counters of SPARSE_STATS."""
    lib = _sparse()
    v = np.ascontiguousarray(values, dtype=np.float32).reshape(-1)
    nx, ny, nz = (int(d) for d in dims)
    assert v.size == nx * ny * nz
    h = lib.sdo_extract(v.ctypes.data, nx, ny, nz, *(float(x) for x in spacing), *(float(x) for x in origin),
                        int(brick_size), int(bool(mvdc)), int(normal_mode), int(threads))
    if not h:
        raise ValueError("sparse oracle rejected the grid")
    try:
        nv, nf, nc = lib.sdo_num_vertices(h), lib.sdo_num_faces(h), lib.sdo_num_cells(h)
        V = np.empty((nv, 3), np.float32)
        N = np.empty((nv, 3), np.float32)
        F = np.empty((nf, 4), np.int32)
        cells = np.empty(nc, np.int64)
        vstart = np.empty(nc, np.int32)
        st = np.zeros(len(SPARSE_STATS), np.int64)
        lib.sdo_copy(h, V.ctypes.data, N.ctypes.data, F.ctypes.data, cells.ctypes.data, vstart.ctypes.data,
                     st.ctypes.data)
    finally:
        lib.sdo_free(h)
    return {"V": V, "N": N, "F": F, "cells": cells, "vstart": vstart, "stats": dict(zip(SPARSE_STATS, st.tolist()))}


def ref_sparse(d_values_ptr, dims, spacing, origin, brick_size=8, normal_mode=0, mvdc=False, exact=True):
    """The reference's own sparse CUDA backend (src/cuda/dc_cuda_sparse.cu), built from its
    source into ``oracle/_ref/`` (``make -C oracle ref``): ``exact`` selects the build without
    FMA contraction (the parity pin), otherwise the build as shipped (the speed bar). Runs on
    the current CUDA device on a device grid; returns V, F, the counters of SPARSE_STATS plus
    vertex and face counts, and the reference's own stage times (total, marking+compaction,
    QEF, faces; ms). Returns None when the library was not built or the grid is refused."""
    name = "libref_sparse_exact.so" if exact else "libref_sparse.so"
    path = os.path.join(_HERE, "_ref", name)
    if not os.path.exists(path):
        return None
    if path not in _libs:
        lib = ctypes.CDLL(path)
        lib.refsparse_run.restype = ctypes.c_void_p
        lib.refsparse_run.argtypes = [ctypes.c_int] * 3 + [ctypes.c_float] * 6 + [ctypes.c_void_p] + [ctypes.c_int] * 3
        for f in ("refsparse_num_vertices", "refsparse_num_faces"):
            getattr(lib, f).restype = ctypes.c_int64
            getattr(lib, f).argtypes = [ctypes.c_void_p]
        lib.refsparse_copy.restype = None
        lib.refsparse_copy.argtypes = [ctypes.c_void_p] * 5
        lib.refsparse_free.restype = None
        lib.refsparse_free.argtypes = [ctypes.c_void_p]
        _libs[path] = lib
    lib = _libs[path]
    nx, ny, nz = (int(d) for d in dims)
    h = lib.refsparse_run(nx, ny, nz, *(float(x) for x in spacing), *(float(x) for x in origin),
                          ctypes.c_void_p(int(d_values_ptr)), int(brick_size), int(normal_mode), int(bool(mvdc)))
    if not h:
        return None
    try:
        nv, nf = lib.refsparse_num_vertices(h), lib.refsparse_num_faces(h)
        V = np.empty((nv, 3), np.float32)
        F = np.empty((nf, 4), np.int32)
        st = np.zeros(16, np.int64)
        times = np.zeros(4, np.float64)
        lib.refsparse_copy(h, V.ctypes.data, F.ctypes.data, st.ctypes.data, times.ctypes.data)
    finally:
        lib.refsparse_free(h)
    stats = dict(zip(SPARSE_STATS, st[:12].tolist()))
    stats.update(vertex_count=int(st[12]), face_count=int(st[13]))
    return {"V": V, "F": F, "stats": stats, "times": times.tolist()}


def ref_cpu_extract(values, dims, spacing, origin, timeout=600):
    """The reference's OWN CPU dual contouring backend (CpuDualContouringBackend::extract,
    src/cpp/dc_backend.cpp:51-125), compiled from its sources into oracle/_ref/ref_cpu_dc
    (``make -C oracle ref``) with stand-in Eigen headers (JacobiSVD restated). Host float32
    values in; returns (V float32 nv x 3, F int32 nf x 4, active_cells), or None when the
    program was not built. Single-threaded and about 2-3 KB per cell, like the reference:
    keep grids small (<= ~96^3)."""
    import subprocess
    import tempfile
    exe = os.path.join(_HERE, "_ref", "ref_cpu_dc")
    if not os.path.exists(exe):
        return None
    v = np.ascontiguousarray(np.asarray(values, np.float32).reshape(-1))
    nx, ny, nz = (int(d) for d in dims)
    with tempfile.TemporaryDirectory() as td:
        gp, op = os.path.join(td, "g.sdf"), os.path.join(td, "o.bin")
        with open(gp, "wb") as f:
            f.write(np.array([nx, ny, nz], np.int32).tobytes())
            f.write(np.array(list(spacing) + list(origin), np.float32).tobytes())
            f.write(v.tobytes())
        r = subprocess.run([exe, gp, op], capture_output=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError("ref_cpu_dc failed (%d): %s" % (r.returncode, r.stderr.decode()[-500:]))
        buf = open(op, "rb").read()
    nv, nf, vpf = np.frombuffer(buf, np.int64, 3, 0)
    pos = 24
    V = np.frombuffer(buf, np.float32, 3 * int(nv), pos).reshape(-1, 3).copy()
    pos += 12 * int(nv)
    F = np.frombuffer(buf, np.int32, int(vpf * nf), pos).reshape(-1, int(vpf)).copy()
    pos += 4 * int(vpf * nf)
    active = int(np.frombuffer(buf, np.int64, 1, pos)[0])
    return V, F, active


def ref_dense_mesh(d_values_ptr, dims, spacing, origin, exact=True):
    """The reference's own dense CUDA backend (CudaDualContouringBackend::extract_device,
    src/cuda/dc_cuda.cu:652-847) from ``oracle/_ref/`` (``make -C oracle ref``) on a device grid
    of the current CUDA device: returns its vertices (float32, nv x 3) and quads (int32, nf x 4)
    in its own order, or None when the library was not built or the grid exceeds its 32-bit
    indices. Its active-cell numbering and its unordered quad set follow the CPU semantics; its
    vertex positions (clamped into the cell, no normal averaging), quad order and winding do
    not."""
    name = "libref_dc_cuda_exact.so" if exact else "libref_dc_cuda.so"
    path = os.path.join(_HERE, "_ref", name)
    if not os.path.exists(path):
        return None
    key = path + ":dense"
    if key not in _libs:
        lib = ctypes.CDLL(path)
        lib.refdc_extract_mesh.argtypes = [ctypes.c_int] * 3 + [ctypes.c_float] * 6 + \
            [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
             ctypes.c_void_p, ctypes.c_void_p]
        lib.refdc_extract_mesh.restype = ctypes.c_int
        _libs[key] = lib
    lib = _libs[key]
    nx, ny, nz = (int(d) for d in dims)
    nv, nf = ctypes.c_int64(0), ctypes.c_int64(0)
    args = [nx, ny, nz, *(float(x) for x in spacing), *(float(x) for x in origin), ctypes.c_void_p(int(d_values_ptr))]
    rc = lib.refdc_extract_mesh(*args, None, 0, None, 0, ctypes.byref(nv), ctypes.byref(nf))
    if rc == -3:
        V = np.empty((nv.value, 3), np.float32)
        F = np.empty((nf.value, 4), np.int32)
        rc = lib.refdc_extract_mesh(*args, V.ctypes.data, nv.value, F.ctypes.data, nf.value,
                                    ctypes.byref(nv), ctypes.byref(nf))
    elif rc == 0:
        V, F = np.empty((0, 3), np.float32), np.empty((0, 4), np.int32)
    if rc != 0:
        return None
    return V, F


def ref_mesh_to_sdf(V, F, dims, origin, spacing, voxelize_first=False, voxel_res=256, exact=True):
    """The reference's own CUDA mesh -> SDF conversion (compute_mesh_sdf_device_cuda,
    src/cuda/mesh_to_sdf_cuda.cu:740-1009) from ``oracle/_ref/`` (``make -C oracle ref``):
    ``exact`` selects the build without FMA contraction. Host arrays in; returns (float32
    values, its own milliseconds), or None when the library was not built."""
    name = "libref_dc_cuda_exact.so" if exact else "libref_dc_cuda.so"
    path = os.path.join(_HERE, "_ref", name)
    if not os.path.exists(path):
        return None
    key = path + ":sdf"
    if key not in _libs:
        lib = ctypes.CDLL(path)
        lib.refsdf_compute_ex.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int] + \
            [ctypes.c_int] * 3 + [ctypes.c_float] * 6 + [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        lib.refsdf_compute_ex.restype = ctypes.c_int
        _libs[key] = lib
    lib = _libs[key]
    V, F = _mesh_args(V, F)
    nx, ny, nz = (int(d) for d in dims)
    out = np.empty(nx * ny * nz, np.float32)
    ms = ctypes.c_float()
    rc = lib.refsdf_compute_ex(V.ctypes.data, len(V), F.ctypes.data, len(F), nx, ny, nz,
                               *[float(x) for x in origin], *[float(x) for x in spacing],
                               1 if voxelize_first else 0, int(voxel_res), ctypes.byref(ms), out.ctypes.data)
    if rc != 0:
        return None
    return out, ms.value


# ---- mesh post-pass: oracle/post_oracle.cpp restates postprocess_mesh (src/cpp/dc_backend.cpp:127-558)
POST_STATS = ("welded_vertices", "welded_faces", "components", "kept_faces", "boundary_edges", "loops_found",
              "loops_filled", "fill_vertices", "fill_faces", "vertex_count", "face_count")


def _post_lib(path, prefix):
    lib = _load(path)
    if not getattr(lib, "_post_typed", False):
        run = getattr(lib, prefix + "_run")
        run.restype = ctypes.c_void_p
        run.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int]
        for name in ("_num_vertices", "_num_faces"):
            f = getattr(lib, prefix + name)
            f.restype = ctypes.c_int64
            f.argtypes = [ctypes.c_void_p]
        getattr(lib, prefix + "_free").argtypes = [ctypes.c_void_p]
        lib._post_typed = True
    return lib


def _post_call(lib, prefix, V, F, close_holes, remove_floaters, with_stats):
    V = np.ascontiguousarray(V, dtype=np.float32).reshape(-1, 3)
    F = np.ascontiguousarray(F, dtype=np.int32).reshape(-1, 4)
    h = getattr(lib, prefix + "_run")(V.ctypes.data if V.size else None, V.shape[0],
                                     F.ctypes.data if F.size else None, F.shape[0], int(close_holes), int(remove_floaters))
    if not h:
        raise ValueError("invalid mesh")
    try:
        nv, nf = getattr(lib, prefix + "_num_vertices")(h), getattr(lib, prefix + "_num_faces")(h)
        Vo = np.empty((nv, 3), np.float32)
        Fo = np.empty((nf, 4), np.int32)
        if with_stats:
            st = np.zeros(len(POST_STATS), np.int64)
            lib.ppo_copy(ctypes.c_void_p(h), Vo.ctypes.data_as(ctypes.c_void_p), Fo.ctypes.data_as(ctypes.c_void_p),
                         st.ctypes.data_as(ctypes.c_void_p))
            return Vo, Fo, dict(zip(POST_STATS, st.tolist()))
        lib.refpost_copy(ctypes.c_void_p(h), Vo.ctypes.data_as(ctypes.c_void_p), Fo.ctypes.data_as(ctypes.c_void_p))
        return Vo, Fo
    finally:
        getattr(lib, prefix + "_free")(ctypes.c_void_p(h))


def postprocess_mesh(V, F, close_holes=True, remove_floaters=True):
    """The oracle's post-pass: (vertices, quads, stats dict) for quads in."""
    if not os.path.exists(_POST_LIB):
        build()
    return _post_call(_post_lib(_POST_LIB, "ppo"), "ppo", V, F, close_holes, remove_floaters, True)


_REF_POST_LIB = os.path.join(_HERE, "_ref", "libref_post.so")


def ref_postprocess_mesh(V, F, close_holes=True, remove_floaters=True):
    """The reference's own postprocess_mesh compiled from its source (oracle/_ref/libref_post.so,
    `make -C oracle ref`); None when that library was not built."""
    if not os.path.exists(_REF_POST_LIB):
        return None
    return _post_call(_post_lib(_REF_POST_LIB, "refpost"), "refpost", V, F, close_holes, remove_floaters, False)
