// dcb_kernels.cuh — parameter blocks and launchers of the dual-contouring kernels.
#pragma once
#include "dcb_common.cuh"

namespace dcb {

struct MarkParams {
    GridDesc g;
    int R;                         // cell rows per tile (point rows = R + 1 <= 8)
    int KZ;                        // cell planes per tile
    int nxt;                       // x-tiles of 1024 cells per row
    uint32_t* bits;                // [cy*cz][W]
    uint32_t* seg_count;           // [cz*cy*nxt] active cells per (plane, row, x-tile)
    int vec4;                      // rows are 16-byte aligned and nx % 4 == 0
};
cudaError_t launch_mark(const MarkParams& P, cudaStream_t s);
int mark_tile_words();
int mark_ctas_per_sm(int vec4);   // resident CTAs of the mark kernel per SM
int mark_max_rows();

struct ExpandParams {
    GridDesc g;
    int nxt;
    const uint32_t* bits;
    const uint32_t* seg_count;
    const uint32_t* seg_start;     // exclusive scan of seg_count
    uint32_t* super;               // [cy*cz][W8]
    uint64_t* list;                // [active]
};
cudaError_t launch_expand(const ExpandParams& P, int num_sms, cudaStream_t s);

// Error class of a stored vertex (cell widths, before the float rounding of the output):
// 0 = certified rank-1 FP32 solve (<= 2e-6), 1 = FP32 Jacobi (<= 1e-4), 2 = FP64 path.
enum VertexClass : uint8_t { kVcRank1 = 0, kVcJacobi = 1, kVcFp64 = 2 };

struct QefParams {
    GridDesc g;
    const uint64_t* list;
    long long nactive;
    float* V;
    uint8_t* vclass;                // [active] VertexClass
    uint8_t* fmask;                 // bit a: cell owns a face on its min-corner edge a
    uint32_t* col_count;            // [3][cx*cy]: a*cx*cy + i*cy + j
    uint32_t* esc_list;
    unsigned int* esc_count;
    uint32_t* hard_list;            // cells not certified rank 1
    float4* hard_data;              // [3 per hard cell]: A^T A (6), A^T b (3), centroid (3)
    unsigned int* hard_count;
    unsigned long long* rank_hist;  // [4]
    float thr;
    float band;
    float cond_max;
    int force64;
};
cudaError_t launch_cell_qef(const QefParams& P, int num_sms, cudaStream_t s);
cudaError_t launch_cell_jacobi(const QefParams& P, long long max_items, int num_sms, cudaStream_t s);

struct Vertex64Params {
    GridDesc g;
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
    GridDesc g;
    const uint4* items;             // {staging slot, axis, packed cell lo, packed cell hi}
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
    GridDesc g;
    const uint64_t* list;
    long long nactive;
    const uint8_t* fmask;
    const float* V;
    const uint8_t* vclass;
    const uint32_t* bits;
    const uint32_t* super;
    const uint32_t* col_start;     // [3][cx*cy]
    const uint32_t* col_count;
    uint32_t* col_fill;
    int4* stage_quad;
    uint2* stage_key;              // {k, column}
    uint4* wind_items;             // {slot, axis, packed lo, packed hi}
    unsigned int* wind_count;
    unsigned long long wind_cap;
    int* v64_index;                // [rank] -> FP64 vertex slot (-1 none, -2 being claimed)
    uint32_t* v64_cells;           // cells whose FP64 vertex the windings need
    unsigned int* v64_count;
    unsigned long long v64_cap;
    int* err;
    float hmax;                    // largest cell width (world units)
};
cudaError_t launch_face_scatter(const FaceParams& P, int num_sms, cudaStream_t s);
cudaError_t launch_face_order(const int4* stage_quad, const uint2* stage_key, const uint32_t* col_start,
                              const uint32_t* col_count, const unsigned long long* nfaces, int4* faces,
                              long long max_faces, int num_sms, cudaStream_t s);

struct TriParams {
    const int4* quads;             // final quads
    const unsigned long long* nquads;
    const float* V;
    const uint8_t* vclass;
    float hmax;
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
};
void sdf_bin_geometry(SdfParams& P);
size_t sdf_tri_record_bytes();     // bytes of one triangle record in SdfParams::tris
cudaError_t launch_sdf_prep(const SdfParams& P, int num_sms, cudaStream_t s);
cudaError_t launch_sdf_bins(const SdfParams& P, int num_sms, cudaStream_t s);
cudaError_t launch_sdf_band(const SdfParams& P, int num_sms, cudaStream_t s);
cudaError_t launch_sdf_masks(const SdfParams& P, int num_sms, cudaStream_t s);
cudaError_t launch_sdf_flood(const SdfParams& P, int* changed, int num_sms, cudaStream_t s);
cudaError_t launch_sdf_finish(const SdfParams& P, unsigned long long* filled, float* tmp, int num_sms, cudaStream_t s);

}  // namespace dcb
