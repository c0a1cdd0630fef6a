// dcb_kernels.cuh — parameter blocks and launchers of the dual-contouring kernels.
#pragma once
#include "dcb_common.cuh"

namespace dcb {

// One grid of a batch; a single extraction is a batch of one. The per-grid arrays of the
// pipeline (active bits, super ranks, segment counts, face columns) are concatenated grid
// by grid; the offsets below locate a grid's part. Vertex ranks are global over the batch
// (the segment scan runs over all grids), so the vertices of grid b are the contiguous
// ranks [vert_off[b], vert_off[b+1]).
struct GridSlot {
    GridDesc g;
    long long bits_off;            // first word of the grid's active bits (rows * W)
    long long super_off;           // first super word (rows * W8)
    long long seg_off;             // first segment (rows * nxt)
    long long col_off;             // first face column (3 * cx * cy)
    int R;                         // mark: cell rows per tile (point rows = R + 1 <= 8)
    int KZ;                        // mark: cell planes per tile
    int nxt;                       // mark: x-tiles of 1024 cells per row
    int nrb;                       // mark: row blocks
    int nzc;                       // mark: z-chunks
    int tw;                        // mark: cell words per x-tile (32, or 8 for narrow grids)
    float hmax;                    // largest cell width of the grid (world units)
    long long wt_off;              // first entry of the grid's cell-width tables (width_tables)
};

// Cell-width tables of a grid (k_width_tables): for each axis the widths of cells -1..n (n the
// cells along it), entry c + 1 for cell c, then their reciprocals: w_x, w_y, w_z, r_x, r_y, r_z.
__host__ __device__ inline long long width_table_len(int cx, int cy, int cz) {
    return 2LL * ((long long)cx + cy + cz + 6);
}

struct BatchTable {
    GridSlot s0;                           // the grid when n == 1 (read from kernel parameters)
    const GridSlot* slots;                 // [n], device
    int n;
    const long long* seg_off;              // [n+1] first segment per grid
    const long long* col_off;              // [n+1] first face column per grid
    const unsigned long long* vert_off;    // [n+1] first vertex rank per grid (after the scan)
    const uint32_t* cell_slot;             // [active] grid of every vertex rank (n > 1, after expand)
};

// Largest index b in [0, n) with offs[b] <= x (offsets ascending, offs[0] = 0).
template <typename T>
__device__ __forceinline__ int slot_search(const T* __restrict__ offs, int n, T x) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(offs + mid) <= x) lo = mid; else hi = mid - 1;
    }
    return lo;
}
// The hot kernels are instantiated twice: ONE (a single grid, its slot in the kernel
// parameters, as fast as a kernel without batch support) and batch (slots in global memory).
template <bool ONE>
__device__ __forceinline__ const GridSlot& slot_ref(const BatchTable& B, int gi) {
    return ONE ? B.s0 : B.slots[gi];
}
__device__ __forceinline__ int slot_of_rank(const BatchTable& B, unsigned long long r) {
    if (B.n == 1) return 0;
    return B.cell_slot ? (int)__ldg(B.cell_slot + r) : slot_search(B.vert_off, B.n, r);
}
__device__ __forceinline__ int slot_of_segment(const BatchTable& B, long long s) {
    return B.n == 1 ? 0 : slot_search(B.seg_off, B.n, s);
}
__device__ __forceinline__ int slot_of_column(const BatchTable& B, long long c) {
    return B.n == 1 ? 0 : slot_search(B.col_off, B.n, c);
}

// Device and pinned-host allocations of the library go through these two (dcb_api.cu); the test
// hook dcb_debug_fail_allocations makes them fail as if the device were out of memory.
cudaError_t dev_malloc(void** p, size_t bytes);
cudaError_t host_malloc(void** p, size_t bytes);

struct MarkParams {
    BatchTable B;
    const int* tile_slot;          // [m] the grids of this launch (all share load path and tile width)
    const long long* tile_off;     // [m+1] first tile of each of them
    int m;
    long long ntiles;
    uint32_t* bits;                // all grids' active bits
    uint32_t* seg_count;           // all grids' segment counts
    int* nonfinite;                // optional: set to 1 when a grid value is NaN or infinite
};
cudaError_t launch_mark(const MarkParams& P, int tw, cudaStream_t s);
int mark_tile_words();
int mark_narrow_tile_words();
int mark_ctas_per_sm(bool one);   // resident CTAs of the mark kernel per SM (single grid / batch)
int mark_max_rows();

struct ExpandParams {
    BatchTable B;
    long long nseg;                // segments of all grids
    const uint32_t* bits;
    const uint32_t* seg_count;
    const uint32_t* seg_start;     // exclusive scan of seg_count (global ranks)
    uint32_t* super;               // all grids' super ranks
    uint64_t* list;                // [active] packed cells, grid-local coordinates
    uint32_t* cell_slot;           // [active] grid of every vertex (batches only; may be null)
    long long list_cap;            // entries of list / cell_slot; <= 0: sized for every active cell
};
cudaError_t launch_expand(const ExpandParams& P, int num_sms, cudaStream_t s);

// vert_off[b] = seg_start[seg_off[b]] (b < n), vert_off[n] = total.
cudaError_t launch_vert_offsets(const BatchTable& B, const uint32_t* seg_start, const unsigned long long* total,
                                unsigned long long* vert_off, cudaStream_t s);
// face_off[b] = col_start[col_off[b]] (b < n), face_off[n] = total.
cudaError_t launch_face_offsets(const BatchTable& B, const uint32_t* col_start, const unsigned long long* total,
                                unsigned long long* face_off, cudaStream_t s);
// Global vertex ranks in the faces -> ranks within each face's grid (vpf ints per face).
cudaError_t launch_localize_faces(const unsigned long long* vert_off, const unsigned long long* face_off, int n,
                                  int* faces, int vpf, long long max_faces, int num_sms, cudaStream_t s);

// Error class of a stored vertex (cell widths, before the float rounding of the output):
// 0 = certified rank-1 FP32 solve (<= 2e-6), 1 = FP32 Jacobi (<= 1e-4), 2 = FP64 path.
enum VertexClass : uint8_t { kVcRank1 = 0, kVcJacobi = 1, kVcFp64 = 2 };

struct QefParams {
    BatchTable B;
    const uint64_t* list;
    long long nactive;             // active cells (capacity when live is set)
    const unsigned long long* live; // device count of active cells (a captured graph; above
                                    // nactive, nothing is processed), or null
    const float* wt;                // cell-width tables of every grid (k_width_tables)
    float* V;
    uint8_t* vclass;                // [active] VertexClass
    uint8_t* fmask;                 // bit a: cell owns a face on its min-corner edge a
    uint32_t* col_count;            // per grid [3][cx*cy]: col_off + a*cx*cy + i*cy + j
    uint32_t* esc_list;
    unsigned int* esc_count;
    uint32_t* hard_list;            // cells not certified rank 1
    float4* hard_data;              // [3 per hard cell]: A^T A (6), A^T b (3), centroid (3)
    unsigned int* hard_count;
    unsigned long long* rank_hist;  // [4]
    int* err;
    const int* nonfinite;           // device flag: the grid holds NaN or infinite values; every
                                    // cell then takes the FP64 path (may be null)
    float thr;
    float band;
    float cond_max;
    int force64;
};
// minb: k_cell_qef's register cap (resident blocks per SM: 4, 5 or 6); blocks_per_sm: the width
// of its grid-stride launch
cudaError_t launch_width_tables(const BatchTable& B, float* wt, cudaStream_t s);
cudaError_t launch_cell_qef(const QefParams& P, int num_sms, cudaStream_t s, int minb = 5, int blocks_per_sm = 32);
cudaError_t launch_cell_jacobi(const QefParams& P, long long max_items, int num_sms, cudaStream_t s);

struct Vertex64Params {
    BatchTable B;
    const uint64_t* list;
    const uint32_t* cells;          // ranks of the cells to solve
    const unsigned int* count;
    unsigned int cap;               // entries in cells; count may exceed it on overflow
    float* Vf;                      // optional: float vertex at [rank]
    uint8_t* vclass;                // optional: set to kVcFp64 at [rank] with Vf
    double* V64;                    // optional: double vertex at [item]
    double thr;
};
cudaError_t launch_vertex_fp64(const Vertex64Params& P, long long max_items, int num_sms, cudaStream_t s);

struct Winding64Params {
    BatchTable B;
    const uint4* items;             // {staging slot, axis | grid << 2, packed cell lo, packed cell hi}
    const unsigned int* count;
    unsigned int cap;
    int4* quads;                    // staging quads (rewritten in place)
    const int* v64_index;           // [rank] -> item in V64, or -1
    const double* V64;
    int* err;
};
cudaError_t launch_winding_fp64(const Winding64Params& P, long long max_items, int num_sms, cudaStream_t s);

cudaError_t launch_scan(const uint32_t* in, long long n, uint32_t* partials, uint32_t* out,
                        unsigned long long* grand_total, cudaStream_t s);
long long scan_partials_len(long long n);

struct FaceParams {
    BatchTable B;
    const uint64_t* list;
    long long nactive;             // active cells (capacity when live is set)
    const unsigned long long* live; // device count of active cells (a captured graph; above
                                    // nactive, nothing is processed), or null
    const uint8_t* fmask;
    const float* V;
    const uint8_t* vclass;
    const uint32_t* bits;
    const uint32_t* super;
    const uint32_t* col_start;     // per grid [3][cx*cy] (global column index)
    const uint32_t* col_count;
    uint32_t* col_fill;            // next free slot of each column (starts as a copy of col_start)
    int4* stage_quad;
    uint2* stage_key;              // {k, column}
    uint4* wind_items;             // {slot, axis | grid << 2, packed lo, packed hi}
    unsigned int* wind_count;
    unsigned long long wind_cap;
    int* v64_index;                // [rank] -> FP64 vertex slot (-1 none, -2 being claimed)
    uint32_t* v64_cells;           // cells whose FP64 vertex the windings need
    unsigned int* v64_count;
    unsigned long long v64_cap;
    int* err;
    float hmax;                    // unused: each grid's slot holds its own cell width
};
cudaError_t launch_face_scatter(const FaceParams& P, int num_sms, cudaStream_t s, int blocks_per_sm = 16);
cudaError_t launch_face_order(const int4* stage_quad, const uint2* stage_key, const uint32_t* col_start,
                              const uint32_t* col_count, const unsigned long long* nfaces, int4* faces,
                              long long max_faces, int num_sms, cudaStream_t s);

struct TriParams {
    BatchTable B;
    const int4* quads;             // final quads
    const unsigned long long* nquads;
    const float* V;
    const uint8_t* vclass;
    float hmax;                    // largest cell width of the batch (when grids are unknown)
    int* tris;                     // 2 triangles (6 ints) per quad
    uint32_t* items;               // quads whose orientation FP32 cannot settle
    unsigned int* item_count;
    unsigned int item_cap;
    int* v64_index;
    uint32_t* v64_cells;
    unsigned int* v64_count;
    unsigned long long v64_cap;
    int* err;
};
cudaError_t launch_triangulate(const TriParams& P, long long max_quads, int num_sms, cudaStream_t s);

struct Tri64Params {
    const int4* quads;
    const uint32_t* items;
    const unsigned int* count;
    unsigned int cap;
    const int* v64_index;
    const double* V64;
    int* tris;
    int* err;
};
cudaError_t launch_tri_fp64(const Tri64Params& P, long long max_items, int num_sms, cudaStream_t s);

// ---- adjoint of the vertices (dcb_vertex64.cu) ----
// One row (cell, local edge) of the adjoint's workspace: after the first pass the row's normal
// (a) and point (b); after the second their gradients. flags: 0 no sample, 1 row, 2 gradients.
struct AdjointRow {
    double a[3];
    double b[3];
    long long flags;
};
struct AdjointParams {
    GridDesc g;
    const uint64_t* list;
    long long nactive;
    const float* dV;               // [3 * active] d(loss)/d(vertex)
    float* dgrid;                  // [nx*ny*nz] d(loss)/d(grid value), accumulated
    AdjointRow* rows;              // [12 * active] workspace
    const uint32_t* bits;          // the extraction's active bits and super-word ranks
    const uint32_t* super;
    uint32_t* owners;              // [12 * active] rows (cell * 12 + edge) that own their edge
    unsigned int* owner_count;
    double thr;
};
cudaError_t launch_vertex_adjoint(const AdjointParams& P, int num_sms, cudaStream_t s);

// ---- outer/inner vertex refinement (dcb_ours.cu) ----
// FP64 state of one active cell (the Cell members the refinement uses, Cell.h:44-115).
struct OursCell {
    double v[3];          // vertex
    double hp[12][3];     // Hermite points, by local edge
    double hn[12][3];     // Hermite normals
    double fi[6][3];      // face points, by face (0:+X 1:-X 2:+Y 3:-Y 4:+Z 5:-Z)
    int hmask;            // edges with a Hermite sample
    int fmask;            // faces with a point
};
struct OursParams {
    GridDesc g;
    const uint64_t* list;
    long long nv;
    const uint32_t* bits;
    const uint32_t* super;
    const int4* dc_faces;           // the extraction's quads
    long long nq;
    float* out_V;                   // [3 nv] refined vertices
    int4* out_faces;                // [nq] quads, or [2 nq] triangles (6 ints per quad)
    double lo[3], hi[3];            // box of the Morton codes
    double gmin[3], gd[3];          // grid minimum and cell size (cell_diagonal, contouring.cpp:788-804)
    double cell_diag;
    int inner_iters;
    double mu, dc_weight, sphere_weight, thr, wface, wnormal, wpos;
    int* err;
    // workspace (set by ours_run)
    OursCell* cells;
    double* Vm;                     // [3 nv] the current mesh's vertices
    int4* quads;                    // [nq] canonical cell order of each quad
    double* gsum;                   // [3 nq] gradient sums of the quads' grid edges
    const uint32_t* sel;            // selected grid points (sphere centres)
    long long nsel;
    int* sel_cell;                  // [nsel] cell rank or -1
    unsigned int* cell_count;
    unsigned int* cell_start;
    unsigned int* cell_fill;
    uint32_t* cell_spheres;         // grid points by cell, by radius
    int* prev_tri;                  // [npts] closest triangle of each grid point last time
    uint32_t* heavy;                // cells with many spheres (a warp each)
    unsigned int* heavy_count;
    long long nt;                   // triangles
    unsigned long long* mkeys_sorted;
    uint32_t* tcode;                // triangles' 30-bit Morton codes and indices, then sorted
    uint32_t* tidx;
    uint32_t* tcode_sorted;
    uint32_t* tidx_sorted;
    int2* child;                    // internal nodes: children (< 0: ~leaf)
    int* parent;                    // [2 nt]: internal nodes, then leaves at nt - 1 + leaf
    float4* bmin;
    float4* bmax;
    unsigned int* flags;
    double* tri9;                   // [9 nt] triangle vertices
};
struct OursRun {
    OursParams P;
    void* workspace;
    size_t sort_bytes;
    int outer_iters;
    int hermite_update;
    long long batch_size;
    unsigned long long seed;
    int triangles;
    int num_sms;
};
size_t ours_workspace_bytes(long long nv, long long nq, long long npts, size_t* sort_bytes);
cudaError_t ours_run(OursRun& R, cudaStream_t s);

// ---- mesh -> SDF (dcb_mesh_sdf.cu) ----
struct SdfParams {
    int nx, ny, nz;
    float ox, oy, oz, vx, vy, vz;
    int gx, gy, gz;                // bins per axis
    float bdx, bdy, bdz;           // bin size
    float margin;                  // bounding-box growth of a triangle before binning
    float min_box;                 // smallest bin size
    long long nbins;
    int W;                         // 32-point words per x row (flood masks)
    const float* verts;
    const int* faces;
    long long nv, nf;
    float* tris;                   // sdf_tri_record_bytes() per triangle
    uint32_t* bin_count;
    uint32_t* bin_start;
    uint32_t* bin_fill;
    uint32_t* bin_scratch;         // bin entries as scattered
    uint32_t* bin_tris;            // bin entries in ascending triangle order
    uint8_t* bin_active;
    uint32_t* active_list;         // active bins (any order)
    unsigned int* active_count;
    unsigned int* work_next;       // next active bin for the band kernel
    int* axis_start;               // first point of every bin per axis: [gx+1][gy+1][gz+1]
    float* out;                    // nx*ny*nz values
    uint32_t* far;                 // [nz*ny][W] bits: value is far
    uint32_t* ext;                 // [nz*ny][W] bits: exterior
    int* err;
    // voxelize-first (mesh_to_sdf_cuda.cu:458-577, :764-832)
    int vres;                      // voxels per axis
    int Wv;                        // 32-voxel words per voxel row
    float vox_vx, vox_vy, vox_vz;  // voxel size (n*v)/vres
    uint32_t* vshell;              // [vres*vres][Wv] rasterised shell
    uint32_t* vfar;                // [vres*vres][Wv] outside the dilated shell (flood passes through)
    uint32_t* vext;                // [vres*vres][Wv] exterior (flood result)
};
void sdf_bin_geometry(SdfParams& P);
size_t sdf_tri_record_bytes();     // bytes of one triangle record in SdfParams::tris
cudaError_t launch_sdf_prep(const SdfParams& P, int num_sms, cudaStream_t s);
cudaError_t launch_sdf_bins(const SdfParams& P, int num_sms, cudaStream_t s);
cudaError_t launch_sdf_band(const SdfParams& P, int num_sms, cudaStream_t s);
cudaError_t launch_sdf_masks(const SdfParams& P, int num_sms, cudaStream_t s);
cudaError_t launch_sdf_flood(const SdfParams& P, int* changed, int num_sms, cudaStream_t s);
cudaError_t launch_sdf_finish(const SdfParams& P, unsigned long long* filled, float* tmp, int num_sms, cudaStream_t s);
cudaError_t launch_vox_raster(const SdfParams& P, int num_sms, cudaStream_t s);
cudaError_t launch_vox_dilate(const SdfParams& P, int num_sms, cudaStream_t s);
// the exterior flood of the voxel grid (k_flood on vfar / vext)
cudaError_t launch_vox_flood(const SdfParams& P, int* changed, int num_sms, cudaStream_t s);
cudaError_t launch_vox_sign(const SdfParams& P, unsigned long long* filled, int num_sms, cudaStream_t s);

// ---- sparse (brick) backends ------------------------------------------------------------

// SparseParams::counters slots: the reference's DualContouringStats counters of the sparse
// backends, then the scan totals.
enum SparseCounter {
    kScTotalBricks = 0, kScActiveBricks, kScActiveCells, kScFallback, kScClamp, kScInvalid, kScAmbiguous,
    kScMulti, kScOne, kScTwo, kScSplitReject, kScSkipped,
    kScCount,                      // counters kept per block in the kernels
    kScVertices = kScCount,        // total vertices (multi-vertex scan)
    kScFaces,                      // total faces (face scan)
    kScSlots = 16
};

struct SparseParams {
    GridDesc g;                    // W, W8: the dense path's bitmap layout
    int bs;                        // brick size (cells)
    int nbx, nby, nbz;             // bricks per axis
    int Wp;                        // point words per point row (32 points a word)
    int nxt;                       // cell-word segments of 32 words per cell row
    int mvdc;                      // up to two vertices per cell
    int normal_mode;               // 0 trilinear, 1 edge gradient (2 behaves as 0)
    float close;                   // 0.45f * vx: near-zero cells and thin edges
    uint32_t* pn;                  // [ny*nz][Wp] point words: value < 0
    uint32_t* pp;                  //   value > 0
    uint32_t* pc;                  //   |value| <= close
    uint8_t* brick;                // [nbx*nby*nbz] active flags
    uint32_t* bits;                // [cy*cz][W] active cells
    uint32_t* super;               // [cy*cz][W8] ranks (after the rank expansion)
    uint32_t* seg_count;           // [cy*cz][nxt]
    const uint64_t* list;          // [nactive] packed active cells, ascending
    long long nactive;
    uint32_t* vcount;              // multi-vertex: [nactive] vertices of the cell (1 or 2)
    const uint32_t* vstart;        // multi-vertex: [nactive] first vertex (scan of vcount)
    float* vtmp;                   // multi-vertex: [nactive][2][3] vertices before placing
    float* ntmp;                   // multi-vertex: [nactive][2][3] vertex normals
    float* V;                      // [vertices][3]
    float* N;                      // multi-vertex: [vertices][3]
    uint64_t* vcell;               // multi-vertex: [vertices] packed cell of each vertex
    uint32_t* fcount;              // [nactive] faces of the cell
    const uint32_t* fstart;        // [nactive] first face (scan of fcount)
    int4* stage;                   // [nactive][6] faces of each cell before the scan
    int4* faces;
    unsigned long long* counters;  // [kScSlots], indexed by SparseCounter
};
cudaError_t launch_sparse_mark(const SparseParams& P, int num_sms, cudaStream_t s);
cudaError_t launch_sparse_vertices(const SparseParams& P, int num_sms, cudaStream_t s);
cudaError_t launch_sparse_place(const SparseParams& P, int num_sms, cudaStream_t s);
cudaError_t launch_sparse_faces(const SparseParams& P, int num_sms, cudaStream_t s);
cudaError_t launch_sparse_compact(const SparseParams& P, int num_sms, cudaStream_t s);

// ---- mesh post-pass (dcb_post.cu): postprocess_mesh, src/cpp/dc_backend.cpp:127-558
struct PostBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

enum PostStatIndex {
    kPostWeldedVertices, kPostWeldedFaces, kPostComponents, kPostKeptFaces, kPostBoundaryEdges, kPostLoopsFound,
    kPostLoopsFilled, kPostFillVertices, kPostFillFaces, kPostVertexCount, kPostFaceCount, kPostNumStats
};

// Device workspace of the post-pass; kept by the handle between calls (buffers only grow).
struct PostWork {
    PostBuf count, key, key2, val, val2, u0, u1, u2, u3, ft, flag8, scratch;
    PostBuf Vw, Fw, kept, parent, csize, bnd;
    PostBuf deg, bot, top, pos, vparent, skey, sdeg, shead, soff, sgid, stack, lverts, lflag, lkey, llen;
    PostBuf lpos, lorder, lkey2, nvl, nfl, vb, fb, fillV, fillF;
    PostBuf first, fflag, slot, V1, F1, outV, outF, succ, indeg, cbad, clen, cbase, crank, jflags;
    PostBuf fscratch, frings, fcenters;
    unsigned long long fill_scap = 1ull << 23;   // ring vertices the fill scratch holds (grows)
    unsigned long long fill_rcap = 1ull << 20;   // ring records
    void* hcount = nullptr;             // page-locked copy of the device counters
};

struct PostRun {
    // in: a quad mesh on the device
    const float* V = nullptr;
    long long nv = 0;
    const int32_t* F = nullptr;
    long long nf = 0;
    int close_holes = 0, remove_floaters = 0;
    int num_sms = 148;
    // out: the result (the workspace's buffers, or the input when nothing is to be done)
    const float* out_V = nullptr;
    const int32_t* out_F = nullptr;
    long long nv_out = 0, nf_out = 0;
    long long stats[kPostNumStats] = {};
    int err = 0;                        // device-side findings: 1 face index out of range, 2 non-finite vertex,
                                        // 4 weld key out of range, 8 a bounded loop gave up, 16 fill did not converge
    int too_large = 0;
    const char* what = nullptr;         // the failing CUDA call
};

cudaError_t post_run(PostWork& W, PostRun& R, cudaStream_t s);
void post_release(PostWork& W);

}  // namespace dcb
