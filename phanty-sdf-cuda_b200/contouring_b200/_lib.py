"""ctypes binding of libdcb.so (the C ABI declared in include/dcb.h).

The library is built in-tree next to this file. There is no fallback: if the shared
library is missing or no CUDA device is present, the calls raise.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdcb.so")

DCB_OK = 0
DCB_ERR_INVALID_ARGUMENT = -1
DCB_ERR_TOO_LARGE = -2
DCB_ERR_CUDA = -3
DCB_ERR_OUT_OF_MEMORY = -4
DCB_ERR_TIMEOUT = -5
DCB_ERR_NOT_SUPPORTED = -6
DCB_ERR_INTERNAL = -7

DCB_METHOD_DUAL_CONTOURING = 1
DCB_METHOD_OURS = 2
DCB_METHOD_SPARSE = 3
DCB_METHOD_SPARSE_MVDC = 4

# Every symbol include/dcb.h declares (checked by the CPU test suite).
EXPORTED = (
    "dcb_default_opts", "dcb_abi_version", "dcb_status_string", "dcb_last_error",
    "dcb_create", "dcb_destroy", "dcb_extract_device", "dcb_extract_host",
    "dcb_copy_mesh_to_host", "dcb_copy_mesh_device", "dcb_copy_cells_to_host",
    "dcb_mark_active_cells_noalloc", "dcb_mesh_to_sdf_device", "dcb_mesh_to_sdf_host",
    "dcb_extract_batch_device", "dcb_backward", "dcb_autotune_mark", "dcb_autotune_cells",
    "dcb_write_obj", "dcb_read_sdf", "dcb_write_sdf", "dcb_extract_upload", "dcb_mesh_to_sdf_device_ex",
    "dcb_mesh_to_sdf_host_ex", "dcb_batch_graph_create", "dcb_batch_graph_launch", "dcb_batch_graph_finish",
    "dcb_batch_graph_destroy", "dcb_postprocess_device", "dcb_postprocess_host", "dcb_copy_post_mesh",
    "dcb_read_obj", "dcb_obj_grid", "dcb_debug_fail_allocations")


class DcbGrid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("vx", ctypes.c_float), ("vy", ctypes.c_float), ("vz", ctypes.c_float),
                ("ox", ctypes.c_float), ("oy", ctypes.c_float), ("oz", ctypes.c_float),
                ("values", ctypes.c_void_p)]


class DcbOpts(ctypes.Structure):
    _fields_ = [("method", ctypes.c_int), ("outer_iters", ctypes.c_int), ("inner_iters", ctypes.c_int),
                ("mu", ctypes.c_double), ("dc_weight", ctypes.c_double), ("sphere_weight", ctypes.c_double),
                ("svd_threshold", ctypes.c_double), ("fp64_escalation_cond", ctypes.c_double),
                ("fp64_threshold_band", ctypes.c_double), ("emit_triangles", ctypes.c_int),
                ("force_fp64", ctypes.c_int), ("hermite_update", ctypes.c_int), ("batch_size", ctypes.c_int),
                ("new_hermite_pos_weight", ctypes.c_double), ("new_face_pos_weight", ctypes.c_double),
                ("new_hermite_normal_weight", ctypes.c_double), ("seed", ctypes.c_uint64),
                ("brick_size", ctypes.c_int), ("normal_mode", ctypes.c_int)]


class DcbStats(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("total_cells", ctypes.c_int64), ("active_cells", ctypes.c_int64),
                ("vertex_count", ctypes.c_int64), ("face_count", ctypes.c_int64),
                ("upload_ms", ctypes.c_float), ("marking_ms", ctypes.c_float),
                ("compaction_ms", ctypes.c_float), ("qef_ms", ctypes.c_float),
                ("face_emission_ms", ctypes.c_float), ("download_ms", ctypes.c_float),
                ("total_ms", ctypes.c_float), ("qef_fallback_count", ctypes.c_int64),
                ("clamp_count", ctypes.c_int64), ("escalated_fp64_cells", ctypes.c_int64),
                ("winding_fp64_faces", ctypes.c_int64), ("rank_hist", ctypes.c_int64 * 4),
                ("total_bricks", ctypes.c_int64), ("active_bricks", ctypes.c_int64),
                ("invalid_count", ctypes.c_int64), ("ambiguous_cells", ctypes.c_int64),
                ("multi_vertex_cells", ctypes.c_int64), ("one_vertex_cells", ctypes.c_int64),
                ("two_vertex_cells", ctypes.c_int64), ("split_rejection_count", ctypes.c_int64),
                ("faces_skipped", ctypes.c_int64),
                ("active_brick_marking_ms", ctypes.c_float), ("active_brick_compaction_ms", ctypes.c_float),
                ("active_cell_marking_ms", ctypes.c_float), ("active_cell_compaction_ms", ctypes.c_float),
                ("face_count_ms", ctypes.c_float), ("face_prefix_sum_ms", ctypes.c_float),
                ("face_fill_ms", ctypes.c_float), ("bad_qef_count", ctypes.c_int64)]


class DcbMeshDev(ctypes.Structure):
    _fields_ = [("vertex_count", ctypes.c_int64), ("face_count", ctypes.c_int64),
                ("verts_per_face", ctypes.c_int), ("vertices", ctypes.c_void_p),
                ("faces", ctypes.c_void_p), ("cell_coords", ctypes.c_void_p)]


class DcbMeshHost(ctypes.Structure):
    _fields_ = [("vertex_count", ctypes.c_int64), ("face_count", ctypes.c_int64),
                ("verts_per_face", ctypes.c_int), ("vertices", ctypes.c_void_p),
                ("faces", ctypes.c_void_p)]


class DcbBatchMesh(ctypes.Structure):
    _fields_ = [("vertex_count", ctypes.c_int64), ("face_count", ctypes.c_int64),
                ("verts_per_face", ctypes.c_int), ("vertices", ctypes.c_void_p),
                ("faces", ctypes.c_void_p), ("vertex_offset", ctypes.POINTER(ctypes.c_int64)),
                ("face_offset", ctypes.POINTER(ctypes.c_int64))]


class DcbSdfStats(ctypes.Structure):
    _fields_ = [("num_bins", ctypes.c_int64), ("bin_entries", ctypes.c_int64),
                ("flood_passes", ctypes.c_int64), ("exterior_points", ctypes.c_int64),
                ("bins_ms", ctypes.c_float), ("band_ms", ctypes.c_float), ("sign_ms", ctypes.c_float),
                ("relax_ms", ctypes.c_float), ("total_ms", ctypes.c_float)]


class DcbPostStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in (
        "welded_vertices", "welded_faces", "components", "kept_faces", "boundary_edges", "loops_found",
        "loops_filled", "fill_vertices", "fill_faces", "vertex_count", "face_count")] + [("total_ms", ctypes.c_float)]


class DcbError(RuntimeError):
    """A libdcb call returned a non-zero status."""

    def __init__(self, status, message):
        super().__init__("dcb status %d: %s" % (status, message))
        self.status = status


_lib = None


def lib():
    """Load libdcb.so once; raise if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libdcb.so not found at %s; run `make -C phanty-sdf-cuda_b200` "
                          "or __graft_entry__.build()" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    L.dcb_default_opts.argtypes = [P(DcbOpts)]
    L.dcb_default_opts.restype = None
    L.dcb_abi_version.argtypes = []
    L.dcb_abi_version.restype = ctypes.c_int
    L.dcb_status_string.argtypes = [ctypes.c_int]
    L.dcb_status_string.restype = ctypes.c_char_p
    L.dcb_last_error.argtypes = [ctypes.c_void_p]
    L.dcb_last_error.restype = ctypes.c_char_p
    L.dcb_write_obj.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                                ctypes.c_int, ctypes.c_int]
    L.dcb_write_obj.restype = ctypes.c_int
    L.dcb_read_sdf.argtypes = [ctypes.c_char_p, P(DcbGrid), ctypes.c_void_p, ctypes.c_int64]
    L.dcb_read_sdf.restype = ctypes.c_int
    L.dcb_write_sdf.argtypes = [ctypes.c_char_p, P(DcbGrid)]
    L.dcb_write_sdf.restype = ctypes.c_int
    L.dcb_read_obj.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                               P(ctypes.c_int64), P(ctypes.c_int64)]
    L.dcb_read_obj.restype = ctypes.c_int
    L.dcb_obj_grid.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, P(DcbGrid)]
    L.dcb_obj_grid.restype = ctypes.c_int
    L.dcb_create.argtypes = [P(ctypes.c_void_p), ctypes.c_int]
    L.dcb_create.restype = ctypes.c_int
    L.dcb_destroy.argtypes = [ctypes.c_void_p]
    L.dcb_destroy.restype = ctypes.c_int
    L.dcb_extract_device.argtypes = [ctypes.c_void_p, P(DcbGrid), P(DcbOpts), P(DcbMeshDev), P(DcbStats), ctypes.c_void_p]
    L.dcb_extract_device.restype = ctypes.c_int
    L.dcb_extract_host.argtypes = [ctypes.c_void_p, P(DcbGrid), P(DcbOpts), P(DcbMeshHost), P(DcbStats), ctypes.c_void_p]
    L.dcb_extract_host.restype = ctypes.c_int
    L.dcb_batch_graph_create.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, P(DcbOpts), ctypes.c_double,
                                         ctypes.c_void_p]
    L.dcb_batch_graph_create.restype = ctypes.c_int
    L.dcb_batch_graph_launch.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.dcb_batch_graph_launch.restype = ctypes.c_int
    L.dcb_batch_graph_finish.argtypes = [ctypes.c_void_p, P(DcbBatchMesh), P(DcbStats), ctypes.c_void_p]
    L.dcb_batch_graph_finish.restype = ctypes.c_int
    L.dcb_batch_graph_destroy.argtypes = [ctypes.c_void_p]
    L.dcb_batch_graph_destroy.restype = ctypes.c_int
    L.dcb_extract_upload.argtypes = [ctypes.c_void_p, P(DcbGrid), P(DcbOpts), P(DcbMeshDev), P(DcbStats), ctypes.c_void_p]
    L.dcb_extract_upload.restype = ctypes.c_int
    L.dcb_copy_mesh_to_host.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.dcb_copy_mesh_to_host.restype = ctypes.c_int
    L.dcb_copy_mesh_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.dcb_copy_mesh_device.restype = ctypes.c_int
    L.dcb_copy_cells_to_host.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.dcb_copy_cells_to_host.restype = ctypes.c_int
    L.dcb_debug_fail_allocations.argtypes = [ctypes.c_int64]
    L.dcb_debug_fail_allocations.restype = ctypes.c_int
    L.dcb_mark_active_cells_noalloc.argtypes = [P(DcbGrid), ctypes.c_void_p, ctypes.c_int64,
                                                P(ctypes.c_int64), ctypes.c_void_p]
    L.dcb_mark_active_cells_noalloc.restype = ctypes.c_int
    L.dcb_extract_batch_device.argtypes = [ctypes.c_void_p, P(DcbGrid), ctypes.c_int, P(DcbOpts), P(DcbBatchMesh),
                                           P(DcbStats), ctypes.c_void_p]
    L.dcb_extract_batch_device.restype = ctypes.c_int
    L.dcb_autotune_mark.argtypes = [ctypes.c_void_p, P(DcbGrid), ctypes.c_int, P(ctypes.c_int), P(ctypes.c_int),
                                    P(ctypes.c_float), ctypes.c_void_p]
    L.dcb_autotune_mark.restype = ctypes.c_int
    L.dcb_autotune_cells.argtypes = [ctypes.c_void_p, P(DcbGrid), ctypes.c_int, P(DcbOpts), P(ctypes.c_int),
                                     P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_float), ctypes.c_void_p]
    L.dcb_autotune_cells.restype = ctypes.c_int
    L.dcb_backward.argtypes = [ctypes.c_void_p, P(DcbGrid), P(DcbOpts), ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_int, ctypes.c_void_p]
    L.dcb_backward.restype = ctypes.c_int
    sdf_args = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64] + \
        [ctypes.c_int] * 3 + [ctypes.c_float] * 6 + [ctypes.c_void_p, P(DcbSdfStats), ctypes.c_void_p]
    for name in ("dcb_mesh_to_sdf_device", "dcb_mesh_to_sdf_host"):
        getattr(L, name).argtypes = sdf_args
        getattr(L, name).restype = ctypes.c_int
    sdf_ex_args = sdf_args[:14] + [ctypes.c_int, ctypes.c_int] + sdf_args[14:]   # after the 6 floats
    for name in ("dcb_mesh_to_sdf_device_ex", "dcb_mesh_to_sdf_host_ex"):
        getattr(L, name).argtypes = sdf_ex_args
        getattr(L, name).restype = ctypes.c_int
    post_args = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
                 ctypes.c_int, P(DcbMeshDev), P(DcbPostStats), ctypes.c_void_p]
    for name in ("dcb_postprocess_device", "dcb_postprocess_host"):
        getattr(L, name).argtypes = post_args
        getattr(L, name).restype = ctypes.c_int
    L.dcb_copy_post_mesh.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    L.dcb_copy_post_mesh.restype = ctypes.c_int
    _lib = L
    return L


def check(status, handle=None):
    if status != DCB_OK:
        L = lib()
        msg = L.dcb_status_string(status).decode()
        if handle:
            detail = L.dcb_last_error(handle)
            if detail:
                msg += ": " + detail.decode()
        raise DcbError(status, msg)


def default_opts(**overrides):
    o = DcbOpts()
    lib().dcb_default_opts(ctypes.byref(o))
    for k, v in overrides.items():
        if not hasattr(o, k):
            raise ValueError("Unknown option: %s" % k)
        setattr(o, k, v)
    return o
