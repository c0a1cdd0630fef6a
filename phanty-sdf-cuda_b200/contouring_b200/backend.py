"""Host-side mirror of the reference's Python/C++ backend API for the B200 engine.

The reference exposes (src/cpp/bindings.cpp:127-268, module ``_contouring_cpp_module``):
``DenseSdfGrid`` (nx..oz, values), ``DualContouringMesh`` (vertices, faces),
``DualContouringStats`` and backends whose ``extract(grid)`` returns ``(mesh, stats)`` and
whose CUDA variant also has ``extract_device(grid_device)``. This module provides the same
names and call shapes for the new backend, :class:`B200DualContouringBackend`, on top of the
C ABI in ``include/dcb.h``. Differences: ``vertices`` / ``faces`` are flat numpy arrays
(float32 / int32) instead of Python lists, and errors raise :class:`DcbError` instead of
terminating the process (the reference exits on CUDA errors: src/cuda/dc_cuda.cu:14-20).
"""
import ctypes
import enum
import time

import numpy as np

from . import _lib
from ._lib import DcbError


class ContouringMethod(enum.IntEnum):
    """ContouringMethod (include/contouring.h:21-25)."""
    MarchingCubes = 0
    DualContouring = 1
    Ours = 2


class NormalComputationMode(enum.IntEnum):
    """NormalComputationMode (include/dc_cuda.h:5-9) of the sparse backends."""
    FiniteDifference = 0
    EdgeGradient = 1
    PrecomputedGradient = 2


class ContouringOptions:
    """ContouringOptions (include/contouring.h:27-41) plus the B200 precision knobs."""

    def __init__(self):
        self.method = ContouringMethod.DualContouring
        self.verbose = False
        self.mu = 0.1
        self.dc_weight = 0.02
        self.sphere_weight = 1.0
        self.svd_threshold = 0.01
        self.outer_iters = 100
        self.inner_iters = 100
        self.hermite_update = True
        self.new_hermite_pos_weight = 0.2
        self.new_face_pos_weight = 0.2
        self.new_hermite_normal_weight = 0.2
        self.batch_size = 200000
        d = _lib.DcbOpts()
        try:
            _lib.lib().dcb_default_opts(ctypes.byref(d))
            self.fp64_escalation_cond = d.fp64_escalation_cond
            self.fp64_threshold_band = d.fp64_threshold_band
        except ImportError:
            self.fp64_escalation_cond = 1e6
            self.fp64_threshold_band = 0.01
        self.emit_triangles = False
        self.force_fp64 = False
        self.seed = 0x5eed
        # the sparse backends (set by B200SparseDualContouringBackend): 0 dense, 1 sparse,
        # 2 sparse with up to two vertices per cell
        self.sparse = 0
        self.brick_size = 8
        self.normal_mode = NormalComputationMode.FiniteDifference

    def to_c(self):
        o = _lib.default_opts()
        if int(self.method) == ContouringMethod.MarchingCubes:
            raise DcbError(_lib.DCB_ERR_NOT_SUPPORTED, "marching cubes is not part of this engine")
        o.method = _lib.DCB_METHOD_OURS if int(self.method) == ContouringMethod.Ours else _lib.DCB_METHOD_DUAL_CONTOURING
        o.outer_iters = int(self.outer_iters)
        o.inner_iters = int(self.inner_iters)
        o.mu = float(self.mu)
        o.dc_weight = float(self.dc_weight)
        o.sphere_weight = float(self.sphere_weight)
        o.svd_threshold = float(self.svd_threshold)
        o.fp64_escalation_cond = float(self.fp64_escalation_cond)
        o.fp64_threshold_band = float(self.fp64_threshold_band)
        o.emit_triangles = 1 if self.emit_triangles else 0
        o.force_fp64 = 1 if self.force_fp64 else 0
        o.hermite_update = 1 if self.hermite_update else 0
        o.batch_size = int(self.batch_size)
        o.new_hermite_pos_weight = float(self.new_hermite_pos_weight)
        o.new_face_pos_weight = float(self.new_face_pos_weight)
        o.new_hermite_normal_weight = float(self.new_hermite_normal_weight)
        o.seed = int(self.seed)
        o.brick_size = int(self.brick_size)
        o.normal_mode = int(self.normal_mode)
        if self.sparse:
            o.method = _lib.DCB_METHOD_SPARSE_MVDC if int(self.sparse) == 2 else _lib.DCB_METHOD_SPARSE
        return o


class DenseSdfGrid:
    """DenseSdfGrid (include/dc_backend.h:13-21): dense float32 grid, x fastest."""

    def __init__(self, nx=0, ny=0, nz=0, vx=0.0, vy=0.0, vz=0.0, ox=0.0, oy=0.0, oz=0.0, values=None):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.vx, self.vy, self.vz = vx, vy, vz
        self.ox, self.oy, self.oz = ox, oy, oz
        self.values = values if values is not None else []

    @classmethod
    def from_tuple(cls, t):
        values, dims, spacing, origin = t
        if hasattr(values, "detach"):
            values = values.detach().cpu().numpy()
        return cls(*dims, *spacing, *origin, values=np.asarray(values, np.float32).reshape(-1))


class DenseSdfGridDevice:
    """DenseSdfGridDevice (include/dc_cuda.h:24-29): ``d_values`` is a CUDA tensor or a raw
    device pointer (int). The grid is borrowed, never freed by the backend."""

    def __init__(self, nx=0, ny=0, nz=0, vx=0.0, vy=0.0, vz=0.0, ox=0.0, oy=0.0, oz=0.0, d_values=None):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.vx, self.vy, self.vz = vx, vy, vz
        self.ox, self.oy, self.oz = ox, oy, oz
        self.d_values = d_values

    def pointer(self):
        v = self.d_values
        if v is None:
            return 0
        if hasattr(v, "data_ptr"):
            if not v.is_cuda or v.dtype.__repr__() != "torch.float32" or not v.is_contiguous():
                raise DcbError(_lib.DCB_ERR_INVALID_ARGUMENT, "d_values must be a contiguous float32 CUDA tensor")
            if v.numel() != self.nx * self.ny * self.nz:
                raise DcbError(_lib.DCB_ERR_INVALID_ARGUMENT, "d_values has the wrong number of elements")
            return v.data_ptr()
        return int(v)


class DualContouringMesh:
    """DualContouringMesh (include/dc_backend.h:23-26): xyz per vertex, 4 ints per quad."""

    def __init__(self, vertices=None, faces=None):
        self.vertices = vertices if vertices is not None else np.zeros(0, np.float32)
        self.faces = faces if faces is not None else np.zeros(0, np.int32)


class DualContouringStats:
    """DualContouringStats (include/dc_backend.h:44-78) plus the engine's own counters."""
    _FIELDS = ("backend", "nx", "ny", "nz", "total_cells", "active_cells", "total_bricks", "active_bricks",
               "upload_ms", "marking_ms", "compaction_ms", "active_brick_marking_ms",
               "active_brick_compaction_ms", "active_cell_marking_ms", "active_cell_compaction_ms",
               "qef_ms", "face_emission_ms", "face_count_ms", "face_prefix_sum_ms", "face_fill_ms",
               "download_ms", "total_ms", "vertex_count", "face_count", "qef_fallback_count",
               "clamp_count", "invalid_count", "ambiguous_cells", "multi_vertex_cells",
               "one_vertex_cells", "two_vertex_cells", "split_rejection_count", "bad_qef_count",
               "faces_skipped_due_to_missing_cluster")

    def __init__(self):
        for f in self._FIELDS:
            setattr(self, f, "" if f == "backend" else 0)
        self.escalated_fp64_cells = 0
        self.winding_fp64_faces = 0
        self.rank_hist = [0, 0, 0, 0]

    @classmethod
    def from_c(cls, st):
        s = cls()
        s.backend = "b200"
        for f in ("nx", "ny", "nz", "total_cells", "active_cells", "vertex_count", "face_count",
                  "upload_ms", "marking_ms", "compaction_ms", "qef_ms", "face_emission_ms",
                  "download_ms", "total_ms", "qef_fallback_count", "clamp_count",
                  "escalated_fp64_cells", "winding_fp64_faces", "total_bricks", "active_bricks",
                  "invalid_count", "ambiguous_cells", "multi_vertex_cells", "one_vertex_cells",
                  "two_vertex_cells", "split_rejection_count", "active_brick_marking_ms",
                  "active_brick_compaction_ms", "active_cell_marking_ms", "active_cell_compaction_ms",
                  "face_count_ms", "face_prefix_sum_ms", "face_fill_ms", "bad_qef_count"):
            setattr(s, f, getattr(st, f))
        s.faces_skipped_due_to_missing_cluster = st.faces_skipped
        s.rank_hist = list(st.rank_hist)
        return s

    def as_dict(self):
        d = {f: getattr(self, f) for f in self._FIELDS}
        d.update(escalated_fp64_cells=self.escalated_fp64_cells, winding_fp64_faces=self.winding_fp64_faces,
                 rank_hist=list(self.rank_hist))
        return d


def _host_array(n, dtype):
    """A host array for a mesh download: page-locked (torch's caching host allocator, so the
    copy runs at full DMA speed and repeated calls reuse blocks) when torch with CUDA is
    present, else ordinary memory."""
    try:
        import torch
        if torch.cuda.is_available():
            tdt = torch.float32 if dtype == np.float32 else torch.int32
            return torch.empty(max(n, 0), dtype=tdt, pin_memory=True).numpy()
    except ImportError:
        pass
    return np.empty(n, dtype)


def _current_stream():
    try:
        import torch
        if torch.cuda.is_available() and torch.cuda.is_initialized():
            return torch.cuda.current_stream().cuda_stream
    except ImportError:
        pass
    return 0


class B200DualContouringBackend:
    """The B200 backend. ``extract`` has the semantics of the reference's
    ``CpuDualContouringBackend::extract`` (src/cpp/dc_backend.cpp:51-125)."""

    def __init__(self, device=0, options=None):
        self._L = _lib.lib()
        h = ctypes.c_void_p()
        _lib.check(self._L.dcb_create(ctypes.byref(h), int(device)))
        self._h = h
        self.device = int(device)
        self.options = options if options is not None else ContouringOptions()
        self._last_nv = 0
        self._last_vpf = 4
        self._generation = 0          # counts extractions; a backward needs its forward's

    def close(self):
        if getattr(self, "_h", None):
            self._L.dcb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _grid_c(g, ptr):
        return _lib.DcbGrid(int(g.nx), int(g.ny), int(g.nz), float(g.vx), float(g.vy), float(g.vz),
                            float(g.ox), float(g.oy), float(g.oz), ptr)

    def extract(self, grid, stream=None):
        """Host grid in, host mesh out: returns ``(DualContouringMesh, DualContouringStats)``."""
        vals = np.ascontiguousarray(np.asarray(grid.values, dtype=np.float32).reshape(-1))
        if vals.size != int(grid.nx) * int(grid.ny) * int(grid.nz):
            raise DcbError(_lib.DCB_ERR_INVALID_ARGUMENT, "values has %d entries, expected nx*ny*nz" % vals.size)
        gc = self._grid_c(grid, vals.ctypes.data)
        st = _lib.DcbStats()
        md = _lib.DcbMeshDev()
        s = _current_stream() if stream is None else stream
        # upload + extraction; the mesh is then read once, straight into the returned arrays
        _lib.check(self._L.dcb_extract_upload(self._h, ctypes.byref(gc), ctypes.byref(self.options.to_c()),
                                              ctypes.byref(md), ctypes.byref(st), ctypes.c_void_p(s)), self._h)
        self._last_nv = md.vertex_count
        self._last_vpf = md.verts_per_face
        self._generation += 1
        nv, nf, vpf = md.vertex_count, md.face_count, md.verts_per_face
        V = _host_array(3 * nv, np.float32)
        F = _host_array(vpf * nf, np.int32)
        t0 = time.perf_counter()
        _lib.check(self._L.dcb_copy_mesh_to_host(self._h, V.ctypes.data if nv else None,
                                                 F.ctypes.data if nf else None, ctypes.c_void_p(s)), self._h)
        stats = DualContouringStats.from_c(st)
        stats.download_ms = (time.perf_counter() - t0) * 1e3
        stats.total_ms += stats.download_ms
        return DualContouringMesh(V, F), stats

    @staticmethod
    def _host_mesh(mh):
        nv, nf, vpf = mh.vertex_count, mh.face_count, mh.verts_per_face
        V = (np.ctypeslib.as_array(ctypes.cast(mh.vertices, ctypes.POINTER(ctypes.c_float)), shape=(3 * nv,)).copy()
             if nv else np.zeros(0, np.float32))
        F = (np.ctypeslib.as_array(ctypes.cast(mh.faces, ctypes.POINTER(ctypes.c_int32)), shape=(vpf * nf,)).copy()
             if nf else np.zeros(0, np.int32))
        return DualContouringMesh(V, F)

    def active_cells(self, stream=None):
        """Linear index (i + cx*(j + cy*k)) of the cell of every vertex of the last mesh."""
        n = self._last_nv
        out = np.empty(n, np.int64)
        s = _current_stream() if stream is None else stream
        _lib.check(self._L.dcb_copy_cells_to_host(self._h, out.ctypes.data if n else None, ctypes.c_void_p(s)), self._h)
        return out

    def extract_device(self, grid, stream=None):
        """Device grid in (``DenseSdfGridDevice``), host mesh out, like the reference's
        ``CudaDualContouringBackend::extract_device`` (src/cuda/dc_cuda.cu:652-847)."""
        V, F, stats = self.extract_tensor_ptr(grid, stream)
        nv, nf = stats.vertex_count, stats.face_count
        hv = np.empty(3 * nv, np.float32)
        hf = np.empty(self._last_vpf * nf, np.int32)
        s = _current_stream() if stream is None else stream
        _lib.check(self._L.dcb_copy_mesh_to_host(self._h, hv.ctypes.data if nv else None,
                                                 hf.ctypes.data if nf else None, ctypes.c_void_p(s)), self._h)
        return DualContouringMesh(hv, hf), stats

    def extract_tensor_ptr(self, grid, stream=None):
        """Run on a device grid; returns the handle-owned device pointers (valid until the
        next call) and the stats."""
        gc = self._grid_c(grid, grid.pointer())
        st = _lib.DcbStats()
        md = _lib.DcbMeshDev()
        s = _current_stream() if stream is None else stream
        _lib.check(self._L.dcb_extract_device(self._h, ctypes.byref(gc), ctypes.byref(self.options.to_c()),
                                              ctypes.byref(md), ctypes.byref(st), ctypes.c_void_p(s)), self._h)
        self._last_nv = md.vertex_count
        self._last_vpf = md.verts_per_face
        self._generation += 1
        return md.vertices, md.faces, DualContouringStats.from_c(st)

    def _grid_array(self, grids):
        arr = (_lib.DcbGrid * len(grids))()
        for b, (values, dims, spacing, origin) in enumerate(grids):
            d = DenseSdfGridDevice(*dims, *spacing, *origin, d_values=values)
            arr[b] = self._grid_c(d, d.pointer())
        return arr

    def batch_graph_create(self, grids, headroom=0.25, stream=None):
        """Capture the batched extraction of these device grids into a CUDA graph kept in the
        handle (their pointers and sizes stay fixed; the values may change between replays).
        Needs a stream other than the legacy default one (e.g. inside ``torch.cuda.stream``)."""
        s = _current_stream() if stream is None else stream
        _lib.check(self._L.dcb_batch_graph_create(self._h, self._grid_array(grids), len(grids),
                                                  ctypes.byref(self.options.to_c()), float(headroom),
                                                  ctypes.c_void_p(s)), self._h)
        self._graph_grids = grids          # the graph reads these tensors' memory
        self._generation += 1

    def batch_graph_launch(self, stream=None):
        """Enqueue one replay of the captured batch (returns at once)."""
        s = _current_stream() if stream is None else stream
        _lib.check(self._L.dcb_batch_graph_launch(self._h, ctypes.c_void_p(s)), self._h)

    def batch_graph_finish(self, stream=None):
        """Wait for the replays and publish the last one's mesh like ``extract_batch_ptr``."""
        st = _lib.DcbStats()
        out = _lib.DcbBatchMesh()
        s = _current_stream() if stream is None else stream
        _lib.check(self._L.dcb_batch_graph_finish(self._h, ctypes.byref(out), ctypes.byref(st), ctypes.c_void_p(s)),
                   self._h)
        self._last_nv = out.vertex_count
        self._last_vpf = out.verts_per_face
        self._generation += 1
        return out, DualContouringStats.from_c(st)

    def batch_graph_destroy(self):
        _lib.check(self._L.dcb_batch_graph_destroy(self._h), self._h)
        self._graph_grids = None

    def extract_batch_ptr(self, grids, stream=None):
        """Batched extraction into the handle's device buffers (valid until the next call);
        returns the raw ``DcbBatchMesh`` and the batch's stats."""
        n = len(grids)
        arr = (_lib.DcbGrid * n)()
        for b, (values, dims, spacing, origin) in enumerate(grids):
            d = DenseSdfGridDevice(*dims, *spacing, *origin, d_values=values)
            arr[b] = self._grid_c(d, d.pointer())
        st = _lib.DcbStats()
        out = _lib.DcbBatchMesh()
        s = _current_stream() if stream is None else stream
        _lib.check(self._L.dcb_extract_batch_device(self._h, arr, n, ctypes.byref(self.options.to_c()),
                                                    ctypes.byref(out), ctypes.byref(st), ctypes.c_void_p(s)), self._h)
        self._last_nv = out.vertex_count
        self._last_vpf = out.verts_per_face
        self._generation += 1
        return out, DualContouringStats.from_c(st)

    def autotune_mark(self, grids, stream=None):
        """Time the mark kernel's tilings on ``grids`` = [(CUDA float32 values, dims, spacing,
        origin)] and keep the fastest for this backend; returns (waves, narrow_cells, ms)."""
        n = len(grids)
        arr = (_lib.DcbGrid * n)()
        for b, (values, dims, spacing, origin) in enumerate(grids):
            d = DenseSdfGridDevice(*dims, *spacing, *origin, d_values=values)
            arr[b] = self._grid_c(d, d.pointer())
        w, nc, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
        s = _current_stream() if stream is None else stream
        _lib.check(self._L.dcb_autotune_mark(self._h, arr, n, ctypes.byref(w), ctypes.byref(nc), ctypes.byref(ms),
                                             ctypes.c_void_p(s)), self._h)
        return w.value, nc.value, ms.value

    def autotune_cells(self, grids, stream=None):
        """Time the vertex kernel's register caps and launch widths and the face kernel's launch
        widths on ``grids`` = [(CUDA float32 values, dims, spacing, origin)] with this backend's
        options, and keep the fastest; returns (qef_min_blocks, qef_blocks_per_sm,
        face_blocks_per_sm, ms)."""
        arr = self._grid_array(grids)
        m, q, f, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
        s = _current_stream() if stream is None else stream
        _lib.check(self._L.dcb_autotune_cells(self._h, arr, len(grids), ctypes.byref(self.options.to_c()),
                                              ctypes.byref(m), ctypes.byref(q), ctypes.byref(f), ctypes.byref(ms),
                                              ctypes.c_void_p(s)), self._h)
        self._generation += 1
        return m.value, q.value, f.value, ms.value

    def extract_batch(self, grids, stream=None):
        """Batched extraction of ``grids`` = [(CUDA float32 values, dims, spacing, origin)] in one
        pass of the pipeline. Returns ``[(V (nv,3) float32, F (nf,vpf) int32)]`` CUDA tensors per
        grid (faces index their own grid's vertices) and the batch's totals as stats."""
        s = _current_stream() if stream is None else stream
        out, stats = self.extract_batch_ptr(grids, s)
        return self._batch_meshes(out, len(grids), grids[0][0].device, s), stats

    def batch_graph_meshes(self, stream=None):
        """``batch_graph_finish`` with the per-grid tensors of ``extract_batch``."""
        s = _current_stream() if stream is None else stream
        out, stats = self.batch_graph_finish(s)
        grids = self._graph_grids
        return self._batch_meshes(out, len(grids), grids[0][0].device, s), stats

    def _batch_meshes(self, out, n, dev, s):
        import torch
        vpf = out.verts_per_face
        V = torch.empty((out.vertex_count, 3), dtype=torch.float32, device=dev)
        F = torch.empty((out.face_count, vpf), dtype=torch.int32, device=dev)
        _lib.check(self._L.dcb_copy_mesh_device(self._h, V.data_ptr() if V.numel() else None,
                                                F.data_ptr() if F.numel() else None, ctypes.c_void_p(s)), self._h)
        vo = [out.vertex_offset[b] for b in range(n + 1)]
        fo = [out.face_offset[b] for b in range(n + 1)]
        return [(V[vo[b]:vo[b + 1]], F[fo[b]:fo[b + 1]]) for b in range(n)]

    def extract_tensor(self, values, dims, spacing, origin):
        """torch convenience: CUDA float32 grid in, ``(V (nv,3) float32, F (nf,4) int32,
        stats)`` CUDA tensors out (copied from the handle's buffers)."""
        import torch
        g = DenseSdfGridDevice(*dims, *spacing, *origin, d_values=values)
        _, _, stats = self.extract_tensor_ptr(g)
        V = torch.empty((stats.vertex_count, 3), dtype=torch.float32, device=values.device)
        F = torch.empty((stats.face_count, self._last_vpf), dtype=torch.int32, device=values.device)
        s = torch.cuda.current_stream().cuda_stream
        _lib.check(self._L.dcb_copy_mesh_device(self._h, V.data_ptr() if V.numel() else None,
                                                F.data_ptr() if F.numel() else None, ctypes.c_void_p(s)), self._h)
        return V, F, stats


    def backward_tensor(self, values, dims, spacing, origin, grad_vertices, out=None, accumulate=False):
        """d(loss)/d(grid values) from d(loss)/d(vertices) of the LAST single-grid extraction on
        this backend, which must have run on ``values`` (unchanged) with the same options:
        float32 CUDA tensors in, a float32 CUDA tensor of nx*ny*nz out (``out`` if given; added
        to when ``accumulate``)."""
        import torch
        n = int(dims[0]) * int(dims[1]) * int(dims[2])
        dV = grad_vertices.to(torch.float32).contiguous()
        if dV.numel() != 3 * self._last_nv or not dV.is_cuda:
            raise DcbError(_lib.DCB_ERR_INVALID_ARGUMENT, "grad_vertices must be a CUDA tensor of (vertex_count, 3)")
        if out is None:
            out = torch.empty(n, dtype=torch.float32, device=values.device)
            accumulate = False
        elif out.numel() != n or out.dtype != torch.float32 or not out.is_cuda or not out.is_contiguous():
            raise DcbError(_lib.DCB_ERR_INVALID_ARGUMENT, "out must be a contiguous float32 CUDA tensor of nx*ny*nz")
        g = DenseSdfGridDevice(*dims, *spacing, *origin, d_values=values)
        gc = self._grid_c(g, g.pointer())
        s = torch.cuda.current_stream().cuda_stream
        _lib.check(self._L.dcb_backward(self._h, ctypes.byref(gc), ctypes.byref(self.options.to_c()),
                                        ctypes.c_void_p(dV.data_ptr() if dV.numel() else None),
                                        ctypes.c_void_p(out.data_ptr()), int(bool(accumulate)),
                                        ctypes.c_void_p(s)), self._h)
        return out


class B200SparseDualContouringBackend(B200DualContouringBackend):
    """Drop-in for ``CudaSparseDualContouringBackend(brick_size, normal_mode, chunk_size,
    multi_vertex_cells)`` (include/dc_cuda.h:37-53, src/cpp/bindings.cpp:229-249): brick
    culling, near-zero cells, thin edges, a float QEF clamped into the cell; with
    ``multi_vertex_cells`` up to two vertices per cell. ``chunk_size`` is accepted and, as in
    the reference's kernels, unused. ``extract`` / ``extract_device`` / ``extract_tensor``
    behave as on the dense backend; a backward pass and batches are dense-only."""

    def __init__(self, brick_size=8, normal_mode=NormalComputationMode.FiniteDifference, chunk_size=0,
                 multi_vertex_cells=False, device=0):
        super().__init__(device)
        self.brick_size = brick_size
        self.normal_mode = normal_mode
        self.chunk_size = chunk_size
        self.multi_vertex_cells = multi_vertex_cells

    @property
    def options(self):
        o = self._options
        o.sparse = 2 if self.multi_vertex_cells else 1
        o.brick_size = int(self.brick_size)
        o.normal_mode = int(self.normal_mode)
        return o

    @options.setter
    def options(self, value):
        self._options = value


class B200SparseMvdcDualContouringBackend(B200SparseDualContouringBackend):
    """Drop-in for ``CudaSparseMvdcDualContouringBackend(brick_size, normal_mode, chunk_size)``
    (include/dc_cuda.h:55-62): the sparse backend with up to two vertices per cell."""

    def __init__(self, brick_size=8, normal_mode=NormalComputationMode.FiniteDifference, chunk_size=0, device=0):
        super().__init__(brick_size, normal_mode, chunk_size, True, device)


class MeshSdfStats:
    """Counters and stage times (ms) of one mesh -> SDF conversion."""

    def __init__(self, st):
        for name, _ in _lib.DcbSdfStats._fields_:
            setattr(self, name, getattr(st, name))

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in _lib.DcbSdfStats._fields_}


def _sdf_call(backend, fn, Vp, nv, Fp, nf, dims, origin, spacing, outp, stream, voxelize_first, voxel_res):
    st = _lib.DcbSdfStats()
    s = _current_stream() if stream is None else stream
    _lib.check(fn(backend._h, ctypes.c_void_p(Vp), int(nv), ctypes.c_void_p(Fp), int(nf),
                  *[int(d) for d in dims], *[float(o) for o in origin], *[float(v) for v in spacing],
                  1 if voxelize_first else 0, int(voxel_res),
                  ctypes.c_void_p(outp), ctypes.byref(st), ctypes.c_void_p(s)), backend._h)
    return MeshSdfStats(st)


def mesh_to_sdf_tensor(backend, vertices, faces, dims, origin, spacing, out=None, stream=None,
                       voxelize_first=False, voxel_res=256):
    """``compute_mesh_sdf_device_cuda`` (src/cuda/mesh_to_sdf_cuda.cu:740-1009) on CUDA tensors:
    float32 (n,3) vertices and int32 (m,3) triangles in, a float32 CUDA tensor of nx*ny*nz
    signed distances (x fastest) out, with the conversion's stats. ``voxelize_first`` /
    ``voxel_res`` as in the reference: the points beyond the band take their sign from a
    voxel_res^3 solid."""
    import torch
    V = vertices.to(torch.float32).contiguous()
    F = faces.to(torch.int32).contiguous()
    if not (V.is_cuda and F.is_cuda):
        raise DcbError(_lib.DCB_ERR_INVALID_ARGUMENT, "vertices and faces must be CUDA tensors")
    n = int(dims[0]) * int(dims[1]) * int(dims[2])
    if out is None:
        out = torch.empty(n, dtype=torch.float32, device=V.device)
    elif out.numel() != n or out.dtype != torch.float32 or not out.is_cuda or not out.is_contiguous():
        raise DcbError(_lib.DCB_ERR_INVALID_ARGUMENT, "out must be a contiguous float32 CUDA tensor of nx*ny*nz")
    st = _sdf_call(backend, backend._L.dcb_mesh_to_sdf_device_ex, V.data_ptr(), V.shape[0], F.data_ptr(),
                   F.shape[0], dims, origin, spacing, out.data_ptr(), stream, voxelize_first, voxel_res)
    return out, st


def mesh_to_sdf_cuda(backend, vertices, faces, nx, ny, nz, ox, oy, oz, vx, vy, vz, voxelize_first=False,
                     voxel_res=256):
    """The reference module's ``mesh_to_sdf_cuda`` (src/cpp/bindings.cpp:270-276): host arrays in,
    ``(DenseSdfGrid, milliseconds)`` out."""
    V = np.ascontiguousarray(np.asarray(vertices, np.float32).reshape(-1, 3))
    F = np.ascontiguousarray(np.asarray(faces, np.int32).reshape(-1, 3))
    out = np.empty(int(nx) * int(ny) * int(nz), np.float32)
    st = _sdf_call(backend, backend._L.dcb_mesh_to_sdf_host_ex, V.ctypes.data, len(V), F.ctypes.data, len(F),
                   (nx, ny, nz), (ox, oy, oz), (vx, vy, vz), out.ctypes.data, None, voxelize_first, voxel_res)
    return DenseSdfGrid(nx, ny, nz, vx, vy, vz, ox, oy, oz, values=out), st.total_ms


class PostprocessStats:
    """Counters of one mesh post-pass (``dcb_post_stats``)."""

    def __init__(self, st):
        for name, _ in _lib.DcbPostStats._fields_:
            setattr(self, name, getattr(st, name))

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in _lib.DcbPostStats._fields_}


_default_backends = {}


def _default_backend(device=0):
    if device not in _default_backends:
        _default_backends[device] = B200DualContouringBackend(device=device)
    return _default_backends[device]


def postprocess_mesh_tensor(backend, vertices, faces, close_holes, remove_floaters, stream=None):
    """``postprocess_mesh`` (src/cpp/dc_backend.cpp:217-558) on CUDA tensors: float32 (n,3)
    vertices and int32 (m,4) quads in (e.g. the tensors of ``extract_tensor``); new tensors of
    the result and its ``PostprocessStats`` out."""
    import torch
    V = vertices.to(torch.float32).contiguous()
    F = faces.to(torch.int32).contiguous()
    if not (V.is_cuda and F.is_cuda):
        raise DcbError(_lib.DCB_ERR_INVALID_ARGUMENT, "vertices and faces must be CUDA tensors")
    if F.dim() != 2 or F.shape[1] != 4 or (V.numel() and (V.dim() != 2 or V.shape[1] != 3)):
        raise DcbError(_lib.DCB_ERR_INVALID_ARGUMENT, "expected (n,3) vertices and (m,4) quads")
    s = _current_stream() if stream is None else stream
    md = _lib.DcbMeshDev()
    st = _lib.DcbPostStats()
    L = backend._L
    _lib.check(L.dcb_postprocess_device(backend._h, V.data_ptr() if V.numel() else None, V.shape[0],
                                        F.data_ptr() if F.numel() else None, F.shape[0], int(bool(close_holes)),
                                        int(bool(remove_floaters)), ctypes.byref(md), ctypes.byref(st),
                                        ctypes.c_void_p(s)), backend._h)
    Vo = torch.empty((md.vertex_count, 3), dtype=torch.float32, device=V.device)
    Fo = torch.empty((md.face_count, 4), dtype=torch.int32, device=V.device)
    _lib.check(L.dcb_copy_post_mesh(backend._h, Vo.data_ptr() if Vo.numel() else None,
                                    Fo.data_ptr() if Fo.numel() else None, 0, ctypes.c_void_p(s)), backend._h)
    return Vo, Fo, PostprocessStats(st)


def postprocess_mesh(mesh, close_holes, remove_floaters, backend=None, stream=None):
    """The reference module's ``postprocess_mesh(mesh, close_holes, remove_floaters)``
    (src/cpp/bindings.cpp:145): a ``DualContouringMesh`` of quads in, the post-processed
    ``DualContouringMesh`` out (flat arrays, as ``extract`` returns them), computed on the GPU.
    The stats of the call are left in ``backend.last_postprocess_stats``."""
    backend = backend if backend is not None else _default_backend()
    V = np.ascontiguousarray(np.asarray(mesh.vertices, np.float32).reshape(-1))
    F = np.ascontiguousarray(np.asarray(mesh.faces, np.int32).reshape(-1))
    if V.size % 3 or F.size % 4:
        raise DcbError(_lib.DCB_ERR_INVALID_ARGUMENT, "expected xyz vertices and quads (4 indices per face)")
    s = _current_stream() if stream is None else stream
    md = _lib.DcbMeshDev()
    st = _lib.DcbPostStats()
    L = backend._L
    _lib.check(L.dcb_postprocess_host(backend._h, V.ctypes.data if V.size else None, V.size // 3,
                                      F.ctypes.data if F.size else None, F.size // 4, int(bool(close_holes)),
                                      int(bool(remove_floaters)), ctypes.byref(md), ctypes.byref(st),
                                      ctypes.c_void_p(s)), backend._h)
    Vo = _host_array(3 * md.vertex_count, np.float32)
    Fo = _host_array(4 * md.face_count, np.int32)
    _lib.check(L.dcb_copy_post_mesh(backend._h, Vo.ctypes.data if Vo.size else None, Fo.ctypes.data if Fo.size else None,
                                    1, ctypes.c_void_p(s)), backend._h)
    backend.last_postprocess_stats = PostprocessStats(st)
    return DualContouringMesh(Vo, Fo)
