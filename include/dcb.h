/*
 * dcb.h — C ABI of the B200 dual-contouring engine (libdcb.so).
 *
 * Plain pointers and sizes only; no C++ or torch types cross this boundary. A C++ class
 * implementing the reference's IDualContouringBackend (include/dc_backend.h:80-84), the
 * pybind / ctypes bindings and the CLI backend switch are thin layers over these calls.
 *
 * Conventions
 *   - Every entry point returns an int status: DCB_OK (0) or a negative DCB_ERR_* code.
 *     Nothing here calls exit() or traps the GPU (the reference exits the process on any
 *     CUDA error: src/cuda/dc_cuda.cu:14-20).
 *   - Grids are dense float32, x fastest: value(i,j,k) = values[i + nx*(j + ny*k)]
 *     (include/dc_backend.h:13-21; src/cpp/dc_backend.cpp:61).
 *   - Work is issued on the caller's stream; a handle owns its workspace and output
 *     buffers and must not be used from two host threads at once.
 */
#ifndef DCB_H_
#define DCB_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 4 adds, without changing earlier layouts: the batch CUDA-graph calls, the mesh post-pass
 * (dcb_postprocess_*, dcb_copy_post_mesh, dcb_post_stats) and the OBJ reader (dcb_read_obj,
 * dcb_obj_grid). */
#define DCB_ABI_VERSION 6

enum dcb_status {
    DCB_OK = 0,
    DCB_ERR_INVALID_ARGUMENT = -1,  /* null pointer, dims < 2, non-finite spacing, ... */
    DCB_ERR_TOO_LARGE = -2,         /* grid or mesh exceeds the index limits below     */
    DCB_ERR_CUDA = -3,              /* a CUDA runtime call failed (see dcb_last_error) */
    DCB_ERR_OUT_OF_MEMORY = -4,     /* device or pinned-host allocation failed          */
    DCB_ERR_TIMEOUT = -5,           /* a bounded device-side wait gave up               */
    DCB_ERR_NOT_SUPPORTED = -6,     /* option combination not implemented               */
    DCB_ERR_INTERNAL = -7           /* device-side consistency check failed             */
};

/* Limits: each grid axis <= 2^21 points and <= 65536 points along x; fewer than 2^31
 * vertices and faces (faces are int32 indices, as in DualContouringMesh::faces). */

/* Mirrors DenseSdfGrid (include/dc_backend.h:13-21) and DenseSdfGridDevice
 * (include/dc_cuda.h:24-29). `values` is a host pointer for dcb_extract_host and a
 * device pointer for dcb_extract_device (borrowed, never freed: dc_cuda.cu:679). */
typedef struct {
    int nx, ny, nz;
    float vx, vy, vz;
    float ox, oy, oz;
    const float* values;
} dcb_grid;

enum dcb_method {
    DCB_METHOD_DUAL_CONTOURING = 1,   /* ContouringMethod::DualContouring (contouring.h:21-25) */
    DCB_METHOD_OURS = 2,              /* outer/inner vertex refinement (contouring.cpp:1255-1328) */
    DCB_METHOD_SPARSE = 3,            /* CudaSparseDualContouringBackend (include/dc_cuda.h:37-53):
                                         brick culling, near-zero cells, thin edges, float QEF
                                         clamped into the cell (src/cuda/dc_cuda_sparse.cu)     */
    DCB_METHOD_SPARSE_MVDC = 4        /* CudaSparseMvdcDualContouringBackend (dc_cuda.h:55-62): the
                                         same with up to two vertices per cell                 */
};

/* Normal of a crossing edge's sample on the sparse backends (NormalComputationMode,
 * include/dc_cuda.h:5-9). PRECOMPUTED behaves as TRILINEAR: the reference passes no
 * precomputed gradients to its kernels (src/cuda/dc_cuda_sparse.cu:1306-1333). */
enum dcb_normal_mode {
    DCB_NORMAL_TRILINEAR = 0,         /* FiniteDifference: trilinear gradient at the sample */
    DCB_NORMAL_EDGE_GRADIENT = 1,     /* EdgeGradient: lerp of the end points' central differences */
    DCB_NORMAL_PRECOMPUTED = 2        /* PrecomputedGradient */
};

/* Mirrors ContouringOptions (include/contouring.h:27-41) plus the B200 precision knobs. */
typedef struct {
    int method;                   /* dcb_method; the reference CPU backend forces DC      */
    int outer_iters;              /* default 100 */
    int inner_iters;              /* default 100 */
    double mu;                    /* default 0.1 */
    double dc_weight;             /* default 0.02 */
    double sphere_weight;         /* default 1.0 */
    double svd_threshold;         /* default 0.01: singular values <= this are truncated */
    double fp64_escalation_cond;  /* FP32 solve escalates to FP64 when the condition
                                     estimate of the retained spectrum exceeds this      */
    double fp64_threshold_band;   /* ... or an eigenvalue lies within this relative band
                                     of svd_threshold (rank decision ambiguous in FP32)  */
    int emit_triangles;           /* 0: quads (DualContouringMesh), 1: triangulate_v1     */
    int force_fp64;               /* 1: every cell takes the FP64 path (testing)          */
    /* DCB_METHOD_OURS only (ContouringOptions, contouring.h:27-41): */
    int hermite_update;           /* default 1: PCA update of Hermite normals and points   */
    int batch_size;               /* default 200000: spheres per outer iteration at least */
    double new_hermite_pos_weight;    /* default 0.2 */
    double new_face_pos_weight;       /* default 0.2 */
    double new_hermite_normal_weight; /* default 0.2 */
    uint64_t seed;                /* random fill of the sphere batch (the reference draws
                                     from std::random_device; here it is seeded)          */
    /* DCB_METHOD_SPARSE / _MVDC only (CudaSparseDualContouringBackend's constructor): */
    int brick_size;               /* default 8 (dc_cli.cpp:217) */
    int normal_mode;              /* dcb_normal_mode, default DCB_NORMAL_TRILINEAR */
} dcb_opts;

/* Fill `o` with the reference defaults (contouring.h:27-41) and the B200 knobs. */
void dcb_default_opts(dcb_opts* o);

/* Field-compatible subset of DualContouringStats (include/dc_backend.h:44-78) plus the
 * counters this engine adds. Times are device-side (CUDA events) in milliseconds. */
typedef struct {
    int nx, ny, nz;
    int64_t total_cells;
    int64_t active_cells;
    int64_t vertex_count;
    int64_t face_count;
    float upload_ms;
    float marking_ms;        /* the mark kernel (active bits + segment counts) */
    float compaction_ms;     /* segment scan */
    float qef_ms;            /* rank expansion, Hermite + averaging + QEF (FP32 and FP64) */
    float face_emission_ms;  /* column scan + face scatter + ordering */
    float download_ms;
    float total_ms;
    int64_t qef_fallback_count;     /* cells solved on the FP64 path */
    int64_t clamp_count;            /* always 0: the CPU semantics never clamp */
    int64_t escalated_fp64_cells;   /* == qef_fallback_count */
    int64_t winding_fp64_faces;     /* faces whose orientation was re-decided in FP64 */
    int64_t rank_hist[4];           /* retained-rank histogram of the QEF solves */
    /* sparse backends (DualContouringStats, include/dc_backend.h:44-78); qef_fallback_count
     * then counts QEF solves that fell back to the centroid and clamp_count the vertices
     * clamped into their cell */
    int64_t total_bricks;
    int64_t active_bricks;
    int64_t invalid_count;
    int64_t ambiguous_cells;
    int64_t multi_vertex_cells;
    int64_t one_vertex_cells;
    int64_t two_vertex_cells;
    int64_t split_rejection_count;
    int64_t faces_skipped;          /* faces_skipped_due_to_missing_cluster */
    /* the remaining DualContouringStats fields: active cells are marked and compacted in one
     * pass (the brick times are 0, the cell times equal marking_ms / compaction_ms); faces
     * are counted (inside the vertex stage for dual contouring), their counts scanned, then
     * filled; bad_qef_count is always 0, as in the reference, which never increments it */
    float active_brick_marking_ms;
    float active_brick_compaction_ms;
    float active_cell_marking_ms;
    float active_cell_compaction_ms;
    float face_count_ms;
    float face_prefix_sum_ms;
    float face_fill_ms;
    int64_t bad_qef_count;
} dcb_stats;

/* Device-resident mesh; pointers are owned by the handle and stay valid until the next
 * extract call on that handle or dcb_destroy. */
typedef struct {
    int64_t vertex_count;
    int64_t face_count;
    int verts_per_face;      /* 4 for quads, 3 for triangles */
    float* vertices;         /* device, 3 floats per vertex */
    int32_t* faces;          /* device, verts_per_face ints per face */
    const uint64_t* cell_coords; /* device, per vertex: cell (i,j,k) packed i | j<<21 | k<<42 */
} dcb_mesh_dev;

/* Host mesh; pointers are owned by the handle (pinned) with the same lifetime. */
typedef struct {
    int64_t vertex_count;
    int64_t face_count;
    int verts_per_face;
    const float* vertices;
    const int32_t* faces;
} dcb_mesh_host;

typedef struct dcb_context* dcb_handle;

/* Create a handle bound to CUDA device `device`. */
int dcb_create(dcb_handle* out, int device);
int dcb_destroy(dcb_handle h);

/* Replaces CudaDualContouringBackend::extract_device (include/dc_cuda.h:31-35,
 * src/cuda/dc_cuda.cu:652-847): grid->values is a device pointer. */
int dcb_extract_device(dcb_handle h, const dcb_grid* grid, const dcb_opts* opts,
                       dcb_mesh_dev* out, dcb_stats* stats, void* cuda_stream);

/* Replaces IDualContouringBackend::extract (include/dc_backend.h:80-84;
 * CpuDualContouringBackend::extract src/cpp/dc_backend.cpp:51-125 is the semantics):
 * grid->values is a host pointer; upload, extraction and download all run on the stream
 * and the call returns after the mesh is on the host. */
int dcb_extract_host(dcb_handle h, const dcb_grid* grid, const dcb_opts* opts,
                     dcb_mesh_host* out, dcb_stats* stats, void* cuda_stream);

/* dcb_extract_host without the download: grid->values is a host pointer (pinned for full
 * bandwidth), the mesh stays in the handle's device buffers as with dcb_extract_device. The
 * caller then sizes its own host arrays (e.g. pinned) from `out` and calls
 * dcb_copy_mesh_to_host: one device-to-host copy, no staging through the handle. */
int dcb_extract_upload(dcb_handle h, const dcb_grid* grid, const dcb_opts* opts,
                       dcb_mesh_dev* out, dcb_stats* stats, void* cuda_stream);

/* Copy the last mesh of `h` into caller-owned host arrays (3*V floats, vpf*F ints). */
int dcb_copy_mesh_to_host(dcb_handle h, float* vertices, int32_t* faces, void* cuda_stream);

/* Copy the last mesh of `h` into caller-owned DEVICE arrays (e.g. torch CUDA tensors). */
int dcb_copy_mesh_device(dcb_handle h, float* vertices, int32_t* faces, void* cuda_stream);

/* Copy the linear cell index (i + cx*(j + cy*k), cx = nx-1, cy = ny-1, of the vertex's own
 * grid for a batch) of every vertex of the last mesh into a caller-owned host array of
 * vertex_count entries. */
int dcb_copy_cells_to_host(dcb_handle h, int64_t* cell_linear_index, void* cuda_stream);

/* Active-cell marking and compaction without any device allocation (no counterpart in
 * the reference). For callers that cannot let the library call cudaMalloc: applications
 * that hand out all device memory from their own budget or pool, and latency-sensitive
 * loops in which an allocation's implicit device synchronisation is not acceptable.
 * grid->values is a device pointer; `cells` is a caller-owned DEVICE array of `capacity`
 * entries that receives the linear index i + cx*(j + cy*k) (cx = nx-1, cy = ny-1) of every
 * active cell in ascending order, i.e. the vertex numbering of the extraction; `*count`
 * (host) receives the number of active cells. Returns DCB_ERR_TOO_LARGE with *count set
 * when capacity is too small, and DCB_ERR_TOO_LARGE when the grid's scratch exceeds the
 * fixed 16 MiB scratch array (a 450^3 grid fits; the bound is checked on every call).
 * Scratch lives in one file-scope device array shared by all calls on a device and kept
 * between calls: calls whose work overlaps on the GPU race. Every call looks the array's
 * address up in the current context (cudaGetSymbolAddress, no allocation); the first call on
 * a device may also load the library's device code, so make it before any stream capture.
 * Runs on the current device and the given stream and returns after the result is
 * complete. */
int dcb_mark_active_cells_noalloc(const dcb_grid* grid, int64_t* cells, int64_t capacity,
                                  int64_t* count, void* cuda_stream);

/* Test hook (no counterpart in the reference; the host-side failure injection of a forced
 * allocation failure): after `allowed` more device or page-locked host allocations, every
 * allocation the library attempts fails as cudaMalloc does when the device is out of memory,
 * so entry points return DCB_ERR_OUT_OF_MEMORY; allowed < 0 turns the hook off. Process-wide,
 * for tests; a handle stays usable after such a failure. Returns DCB_OK. */
int dcb_debug_fail_allocations(int64_t allowed);

/* ---- files either side of the extraction (src/cpp/dc_cli.cpp:17-47) -------------------- */

/* Replaces dc_cli's write_obj (dc_cli.cpp:17-29): "v x y z" lines (6 significant digits, the
 * C++ stream default) then "f ..." lines with 1-based indices, verts_per_face 4 (quads) or 3.
 * Host arrays. threads <= 0: all hardware threads format slices in parallel. */
int dcb_write_obj(const char* path, const float* vertices, int64_t num_vertices, const int32_t* faces,
                  int64_t num_faces, int verts_per_face, int threads);

/* Replaces dc_cli's read_sdf (dc_cli.cpp:31-47): int32 nx, ny, nz, float32 vx, vy, vz, ox, oy,
 * oz, then nx*ny*nz float32 values. With values == NULL only the header is read (to size the
 * caller's buffer, e.g. pinned host memory for an upload); otherwise `capacity` floats are
 * available and header->values is set to `values`. */
int dcb_read_sdf(const char* path, dcb_grid* header, float* values, int64_t capacity);

/* The inverse of dcb_read_sdf (host values). */
int dcb_write_sdf(const char* path, const dcb_grid* grid);

/* Replaces the OBJ reading of dc_cli's read_obj_to_sdf (dc_cli.cpp:121-158): "v" lines, "f"
 * lines with 1-based or negative indices (the leading integer of "v/vt/vn" tokens), polygons
 * fanned into triangles. Sets *num_vertices and *num_triangles; with vertices and triangles
 * NULL that is all, otherwise both arrays must hold the counts (DCB_ERR_TOO_LARGE if not).
 * A file without vertices or faces, or with an index out of range, is DCB_ERR_INVALID_ARGUMENT. */
int dcb_read_obj(const char* path, float* vertices, int64_t vertex_capacity, int32_t* triangles,
                 int64_t triangle_capacity, int64_t* num_vertices, int64_t* num_triangles);

/* The grid read_obj_to_sdf puts around a mesh (dc_cli.cpp:160-184): res points per axis over
 * the bounding box grown by 8% of its diagonal on every side (0.1 for a single point);
 * grid->values is set to NULL. The mesh -> SDF call then fills it (dcb_mesh_to_sdf_*_ex). */
int dcb_obj_grid(const float* vertices, int64_t num_vertices, int res, dcb_grid* grid);

/* ---- batches of grids ------------------------------------------------------------------- */

/* The meshes of a batch, concatenated grid by grid in device memory. Grid b's vertices are
 * vertices[3*vertex_offset[b] .. 3*vertex_offset[b+1]) and its faces
 * faces[vpf*face_offset[b] .. vpf*face_offset[b+1]); face indices count from the first vertex
 * of their own grid, so every grid's part is exactly its single-grid extraction. The offset
 * arrays (n+1 entries, host memory) and the device arrays are owned by the handle and stay
 * valid until the next extract call on it. */
typedef struct {
    int64_t vertex_count;
    int64_t face_count;
    int verts_per_face;
    float* vertices;
    int32_t* faces;
    const int64_t* vertex_offset;
    const int64_t* face_offset;
} dcb_batch_mesh;

/* Batched extraction (no counterpart in the reference, whose callers loop over grids): n
 * device grids of any sizes in one pass of the pipeline. Each kernel runs once over all
 * grids (the mark over all grids' tiles, the scans over all grids' segments and face
 * columns, the vertex and face kernels over one queue of all active cells), with two host
 * synchronisations per batch instead of two per grid. stats holds batch totals. */
int dcb_extract_batch_device(dcb_handle h, const dcb_grid* grids, int n, const dcb_opts* opts,
                             dcb_batch_mesh* out, dcb_stats* stats, void* cuda_stream);

/* ---- a batch pipeline captured in a CUDA graph -------------------------------------------- */

/* Captures the whole batched extraction of `grids` (device grids whose pointers, sizes and
 * spacing stay fixed; their values may change between launches) into a CUDA graph kept in
 * the handle. An eager run first sizes the buffers: capacity = active cells * (1 + headroom)
 * + 1024. The graph has no host synchronisation inside: the kernels read the active count
 * from device memory; counters and offsets are copied to pinned host memory as the graph's
 * last nodes. cuda_stream must not be the legacy default stream. The graph holds pointers into
 * the handle's workspace: any other extraction, backward or autotune call on the handle
 * invalidates it (launch then returns DCB_ERR_INVALID_ARGUMENT). */
int dcb_batch_graph_create(dcb_handle h, const dcb_grid* grids, int n, const dcb_opts* opts, double headroom,
                           void* cuda_stream);
/* Enqueues one replay on the stream (returns at once). */
int dcb_batch_graph_launch(dcb_handle h, void* cuda_stream);
/* Waits for the stream and publishes the last replay's mesh as dcb_extract_batch_device does;
 * DCB_ERR_TOO_LARGE when the grids had more active cells than the capacity (nothing was
 * extracted: recreate the graph). */
int dcb_batch_graph_finish(dcb_handle h, dcb_batch_mesh* out, dcb_stats* stats, void* cuda_stream);
int dcb_batch_graph_destroy(dcb_handle h);


/* Tile autotuner for the mark kernel (no counterpart in the reference): times the mark
 * launches of these device grids (one batch) for every combination of CTAs per resident
 * slot (waves 1, 2, 4, 8) and x-tile width (256-cell tiles for grids at most 0, 256, 512 or
 * 1024 cells wide, 1024-cell tiles otherwise), and keeps the fastest for this handle's later
 * extractions. The results of an extraction do not depend on the tiling. The chosen waves,
 * width limit and the median mark time (ms) are returned through the optional pointers. */
int dcb_autotune_mark(dcb_handle h, const dcb_grid* grids, int n, int* waves_out, int* narrow_cells_out,
                      float* best_ms_out, void* cuda_stream);

/* Autotuner for the vertex and face kernels (no counterpart in the reference): extracts these
 * device grids (one batch) repeatedly, first for every register cap of the FP32 vertex
 * kernel (4, 5 or 6 resident blocks of 128 threads per SM) with every launch width (8, 16 or
 * 32 blocks per SM of its grid-stride loop), timing the vertex stage, then for every width of
 * the face scatter (8, 16 or 32 blocks per SM), timing the face stage; keeps the fastest of
 * each for this handle's later extractions, batches and captured graphs. Cells and quads do not
 * depend on these choices; vertices may differ in the last float bits between register caps
 * (separately compiled kernels), within the same tolerance. The choices and the sum of the two
 * median stage times (ms) are returned through the optional pointers. opts may be null
 * (defaults); dual contouring only. */
int dcb_autotune_cells(dcb_handle h, const dcb_grid* grids, int n, const dcb_opts* opts, int* qef_min_blocks_out,
                       int* qef_blocks_per_sm_out, int* face_blocks_per_sm_out, float* best_ms_out,
                       void* cuda_stream);

/* ---- mesh -> signed distance grid ------------------------------------------------------ */

typedef struct {
    int64_t num_bins;          /* spatial bins (about 8 grid points a side) */
    int64_t bin_entries;       /* (bin, triangle) pairs */
    int64_t flood_passes;      /* exterior-flood launches until nothing changed */
    int64_t exterior_points;   /* far points that ended exterior (+10) */
    float bins_ms;             /* triangle records, binning, in-bin ordering */
    float band_ms;             /* closest-triangle distances near the surface */
    float sign_ms;             /* far / exterior masks and the exterior flood */
    float relax_ms;            /* far values and the 4 relaxation passes */
    float total_ms;
} dcb_sdf_stats;

/* Replaces compute_mesh_sdf_device_cuda (include/mesh_to_sdf.h; src/cuda/mesh_to_sdf_cuda.cu:
 * 740-1009, without voxelisation): vertices (float xyz) and faces (int32 triangles) are DEVICE
 * arrays; out_values is a caller-owned DEVICE array of nx*ny*nz floats (x fastest) that
 * receives the signed distances, ready for dcb_extract_device. Returns
 * DCB_ERR_INVALID_ARGUMENT if a face index is out of range. */
int dcb_mesh_to_sdf_device(dcb_handle h, const float* vertices, int64_t num_vertices, const int32_t* faces,
                           int64_t num_faces, int nx, int ny, int nz, float ox, float oy, float oz, float vx,
                           float vy, float vz, float* out_values, dcb_sdf_stats* stats, void* cuda_stream);

/* Replaces compute_mesh_sdf_cuda (same file): host vertices and faces in, host values out
 * (nx*ny*nz floats); returns after the values are on the host. */
int dcb_mesh_to_sdf_host(dcb_handle h, const float* vertices, int64_t num_vertices, const int32_t* faces,
                         int64_t num_faces, int nx, int ny, int nz, float ox, float oy, float oz, float vx,
                         float vy, float vz, float* out_values, dcb_sdf_stats* stats, void* cuda_stream);

/* The two calls above with the reference's remaining arguments of compute_mesh_sdf[_device]_cuda
 * (include/mesh_to_sdf.h; dc_cli's --voxelize-first / --voxel-res): voxelize_first != 0 takes
 * the sign of the points beyond the band from a voxel solid of voxel_res^3 voxels (clamped to
 * [32, 2048]; mesh_to_sdf_cuda.cu:458-577, 764-832) instead of the exterior flood and the
 * relaxation. voxelize_first = 0 is the plain conversion (voxel_res unused). */
int dcb_mesh_to_sdf_device_ex(dcb_handle h, const float* vertices, int64_t num_vertices, const int32_t* faces,
                              int64_t num_faces, int nx, int ny, int nz, float ox, float oy, float oz, float vx,
                              float vy, float vz, int voxelize_first, int voxel_res, float* out_values,
                              dcb_sdf_stats* stats, void* cuda_stream);
int dcb_mesh_to_sdf_host_ex(dcb_handle h, const float* vertices, int64_t num_vertices, const int32_t* faces,
                            int64_t num_faces, int nx, int ny, int nz, float ox, float oy, float oz, float vx,
                            float vy, float vz, int voxelize_first, int voxel_res, float* out_values,
                            dcb_sdf_stats* stats, void* cuda_stream);

/* ---- adjoint of the vertices ------------------------------------------------------------ */

/* Gradient of a loss with respect to the grid values, given its gradient with respect to the
 * vertices of the LAST single-grid extraction on this handle (no counterpart in the reference,
 * whose backends are forward-only). grid must be the grid that extraction ran on (device
 * values, unchanged since) and opts the same options. dL_dvertices is a device array of
 * 3*vertex_count floats; dL_dgrid a device array of nx*ny*nz floats that receives the
 * gradient (added to what it holds when accumulate != 0, else overwritten). Topology is held
 * fixed: the active cells, the Hermite edges and the rank of every cell's QEF solve are those
 * of the extraction. Each vertex is differentiated through its FP64 solve: the 4-cell averaged
 * Hermite normals, the trilinear gradients and crossings of the cell and its neighbours (the
 * 4x4x4 stencil), and the truncated pseudo-inverse by its implicit derivative. Sums into
 * dL_dgrid use float atomics, so their order (and the last bits) may vary between calls. */
int dcb_backward(dcb_handle h, const dcb_grid* grid, const dcb_opts* opts, const float* dL_dvertices,
                 float* dL_dgrid, int accumulate, void* cuda_stream);

/* Human-readable text of a status code and of the last error on this handle. */
const char* dcb_status_string(int status);
const char* dcb_last_error(dcb_handle h);

/* Version of the ABI compiled into the library. */
/* ---- mesh post-pass. Replaces postprocess_mesh (include/dc_backend.h:28;
 * src/cpp/dc_backend.cpp:217-558, its vertex weld merge_vertices_in_place :127-215): weld
 * vertices on a grid of 1e-5 box diagonals, drop faces left with < 3 distinct vertices, keep
 * only the largest face component (remove_floaters), fill boundary loops of 3..4096 vertices
 * with rings and a fan (close_holes), number vertices by first use and weld again (close_holes).
 * The result has the reference's vertices, faces and order, bit for bit. Quads in and out (4
 * int32 indices per face; a filled triangle repeats its last index). With neither flag, or an
 * empty mesh, the input is returned unchanged (out points at it). */
typedef struct {
    int64_t welded_vertices;      /* after the first weld */
    int64_t welded_faces;
    int64_t components;           /* face components (remove_floaters), else 0 */
    int64_t kept_faces;           /* faces of the kept component */
    int64_t boundary_edges;       /* edge uses that bound the mesh (one use; with both flags, also
                                     every use of a non-manifold edge) */
    int64_t loops_found;          /* loops the boundary walks closed */
    int64_t loops_filled;         /* of them, those with 3..4096 vertices */
    int64_t fill_vertices;        /* vertices and faces the fill added */
    int64_t fill_faces;
    int64_t vertex_count;         /* the result */
    int64_t face_count;
    float total_ms;
} dcb_post_stats;

/* vertices/faces are device pointers (e.g. the handle's own last mesh, quads only). The result
 * lives in buffers of the handle until the next post-pass call or dcb_destroy. */
int dcb_postprocess_device(dcb_handle h, const float* vertices, int64_t num_vertices, const int32_t* faces,
                           int64_t num_faces, int close_holes, int remove_floaters, dcb_mesh_dev* out,
                           dcb_post_stats* stats, void* cuda_stream);
/* The same from host arrays (uploaded on the stream); read the result with dcb_copy_post_mesh. */
int dcb_postprocess_host(dcb_handle h, const float* vertices, int64_t num_vertices, const int32_t* faces,
                         int64_t num_faces, int close_holes, int remove_floaters, dcb_mesh_dev* out,
                         dcb_post_stats* stats, void* cuda_stream);
/* Copy the last post-pass result into caller-owned arrays (3*V floats, 4*F ints): host arrays
 * when to_host is non-zero (returns after the copy), device arrays otherwise. */
int dcb_copy_post_mesh(dcb_handle h, float* vertices, int32_t* faces, int to_host, void* cuda_stream);

int dcb_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* DCB_H_ */
