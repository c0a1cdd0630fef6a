// dcb_api.cu — handle, workspace and the C ABI declared in include/dcb.h.
//
// Pipeline of one extraction (all on the caller's stream):
//   k_mark_zmarch    grid -> active bits, per-segment counts, a flag for non-finite
//                    values                                            (dcb_mark.cu)
//   scan             segment counts -> segment first ranks, total     (dcb_faces.cu)
//   [host reads the active count: sizes the vertex buffers]
//   k_expand_ranks   super-word ranks + packed active-cell list        (dcb_mark.cu)
//   k_cell_qef       Hermite + averaging + QEF (rank-1 certified), face masks, column
//                    counts; other cells listed                        (dcb_vertex.cu)
//   k_cell_jacobi    listed cells solved with FP32 Jacobi              (dcb_vertex.cu)
//   k_vertex_fp64    cells FP32 does not trust, re-solved in FP64      (dcb_vertex64.cu)
//   scan             column counts -> column starts, face total       (dcb_faces.cu)
//   k_face_scatter   quads into their columns, FP32 winding           (dcb_faces.cu)
//   k_vertex_fp64    FP64 vertices of the cells of uncertain windings  (dcb_vertex64.cu)
//   k_winding_fp64   uncertain windings re-decided in FP64            (dcb_vertex64.cu)
//   k_face_order     rank by k inside each column -> final face list  (dcb_faces.cu)
//   [host reads the face total and counters]
// The reference backend allocates and frees everything per call and synchronises after
// every stage (src/cuda/dc_cuda.cu:614-847); here buffers live in the handle and grow.
#include <cstdio>
#include <cstring>
#include <cmath>
#include <string>
#include <algorithm>
#include <atomic>
#include <vector>
#include "dcb_kernels.cuh"
#include "../../include/dcb.h"

namespace dcb {

// Small device-side counters, cleared at the start of every extraction.
struct Counters {
    int err;
    unsigned int esc_count;
    unsigned long long total_active;
    unsigned int wind_count;
    unsigned int hard_count;
    unsigned int v64_count;
    unsigned int tri_count;           // quads whose triangle orientation goes to FP64
    unsigned long long rank_hist[4];
    unsigned long long face_total;
    int nonfinite;                    // the mark met a NaN or infinite grid value
};

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

}  // namespace dcb

using namespace dcb;

struct dcb_context {
    int device = 0;
    int num_sms = 148;
    std::string last_error;
    cudaEvent_t ev[10] = {};
    bool substage_events = false;     // ev[8] / ev[9] hold the face sub-stages of the last call
    DevBuf grid, bits, super, list, seg_count, seg_start, counters, V, vclass, fmask, col_count, col_fill,
        col_start, partials, esc_list, hard_list, hard_data, stage_quad, stage_key, faces, wind_items,
        v64_index, v64_cells, V64, tris, tri_items, adj_rows, adj_owners, ours_ws, wt;
    // sparse backends
    DevBuf sp_words, sp_brick, sp_vcount, sp_vstart, sp_vtmp, sp_ntmp, sp_N, sp_vcell, sp_fcount, sp_fstart,
        sp_stage, sp_counters;
    void* h_sp_counters = nullptr;    // pinned copy of the sparse counters
    int last_kind = 0;                // last extraction: 0 dense dual contouring, 1 sparse
    // a captured batch graph (dcb_batch_graph_*): it holds pointers into this workspace, so
    // every call that may reallocate or rewrite the workspace bumps `gen` and invalidates it
    unsigned long long gen = 0;
    struct BatchGraphState* bg = nullptr;
    int cells_per_vertex = 0;         // 1: the vertex -> cell list is `sp_vcell` (two vertices per cell)
    // mesh -> SDF workspace
    DevBuf m_verts, m_faces, m_out, m_tris, m_bin_count, m_bin_start, m_bin_fill, m_bin_scratch, m_bin_tris,
        m_bin_active, m_active_list, m_axis_start, m_far, m_ext, m_tmp, m_partials, m_counters, m_vox;
    void* h_sdf_counters = nullptr;   // pinned SdfCounters
    void* h_counters = nullptr;       // pinned Counters
    void* hV = nullptr; size_t hV_bytes = 0;
    void* hF = nullptr; size_t hF_bytes = 0;
    int64_t nv = 0, nf = 0;           // vertices; output faces (quads or triangles)
    int vpf = 4;                      // output vertices per face
    int mark_ctas[2] = {0, 0};        // resident mark CTAs per SM: batch, single grid
    // mark tiling (dcb_autotune_mark): CTAs per resident mark slot, and the widest grid
    // (cells along x) that marches 256-cell x-tiles instead of 1024-cell ones
    int tune_waves = 4;
    int tune_narrow_cells = 256;
    // vertex and face kernels (dcb_autotune_cells): k_cell_qef's register cap (resident blocks
    // per SM its allocation allows) and grid-stride width, k_face_scatter's width (blocks per SM)
    int tune_qef_minb = 5;
    int tune_qef_bps = 32;
    int tune_face_bps = 16;
    int cx = 0, cy = 0, cz = 0;
    // batch layout table (device + pinned staging) and the last batch's per-grid offsets
    DevBuf table, cell_slot;
    void* h_table = nullptr; size_t h_table_bytes = 0;
    void* h_offsets = nullptr; size_t h_offsets_bytes = 0;
    int batch_n = 1;
    std::vector<int> batch_cx, batch_cy;
    std::vector<int64_t> vert_offsets, face_offsets;
    // mesh post-pass: workspace, uploaded host input, the last result
    PostWork post;
    DevBuf pp_in_V, pp_in_F;
    const float* pp_V = nullptr;
    const int32_t* pp_F = nullptr;
    int64_t pp_nv = 0, pp_nf = 0;
};

namespace dcb {

// dcb_debug_fail_allocations: < 0 off; otherwise the number of allocations still allowed before
// every further one fails.
std::atomic<long long> g_alloc_budget{-1};

static bool allocation_refused() {
    long long b = g_alloc_budget.load();
    while (b >= 0) {
        if (b == 0) return true;
        if (g_alloc_budget.compare_exchange_weak(b, b - 1)) return false;
    }
    return false;
}

cudaError_t dev_malloc(void** p, size_t bytes) {
    if (allocation_refused()) { *p = nullptr; return cudaErrorMemoryAllocation; }
    return cudaMalloc(p, bytes);
}

cudaError_t host_malloc(void** p, size_t bytes) {
    if (allocation_refused()) { *p = nullptr; return cudaErrorMemoryAllocation; }
    return cudaMallocHost(p, bytes);
}

}  // namespace dcb

namespace {

int fail(dcb_context* h, int code, const std::string& msg) {
    if (h) h->last_error = msg;
    return code;
}

int cuda_fail(dcb_context* h, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return fail(h, DCB_ERR_OUT_OF_MEMORY, m);
    return fail(h, DCB_ERR_CUDA, m);
}

#define DCB_TRY(h, expr, what)                                   \
    do {                                                         \
        cudaError_t e_ = (expr);                                 \
        if (e_ != cudaSuccess) return cuda_fail((h), e_, (what)); \
    } while (0)

cudaError_t ensure(DevBuf& b, size_t bytes) {
    if (bytes == 0) bytes = 256;
    if (b.bytes >= bytes) return cudaSuccess;
    if (b.p) { cudaFree(b.p); b.p = nullptr; b.bytes = 0; }
    const size_t want = bytes + bytes / 8;   // headroom for slowly growing workloads
    cudaError_t e = dev_malloc(&b.p, want);
    if (e != cudaSuccess) { cudaGetLastError(); return e; }
    b.bytes = want;
    return cudaSuccess;
}

cudaError_t ensure_host(void*& p, size_t& have, size_t bytes) {
    if (bytes == 0) bytes = 256;
    if (have >= bytes) return cudaSuccess;
    if (p) { cudaFreeHost(p); p = nullptr; have = 0; }
    const size_t want = bytes + bytes / 8;
    cudaError_t e = host_malloc(&p, want);
    if (e != cudaSuccess) { cudaGetLastError(); return e; }
    have = want;
    return cudaSuccess;
}

template <typename T> T* as(DevBuf& b) { return reinterpret_cast<T*>(b.p); }

// The output face array of the last extraction: quads, or their triangles.
int32_t* face_ptr(dcb_context* h) { return reinterpret_cast<int32_t*>(h->vpf == 3 ? h->tris.p : h->faces.p); }

bool finite_pos(float x) { return std::isfinite(x); }

int validate(dcb_context* h, const dcb_grid* g) {
    if (!h) return DCB_ERR_INVALID_ARGUMENT;
    if (!g || !g->values) return fail(h, DCB_ERR_INVALID_ARGUMENT, "grid or grid values is null");
    if (g->nx < 2 || g->ny < 2 || g->nz < 2) return fail(h, DCB_ERR_INVALID_ARGUMENT, "grid needs at least 2 points per axis");
    if (g->nx > 65536 || g->ny > (1 << 21) || g->nz > (1 << 21))
        return fail(h, DCB_ERR_TOO_LARGE, "grid axis exceeds the index limits (nx <= 65536, ny,nz <= 2^21)");
    if (!finite_pos(g->vx) || !finite_pos(g->vy) || !finite_pos(g->vz) || !finite_pos(g->ox) ||
        !finite_pos(g->oy) || !finite_pos(g->oz))
        return fail(h, DCB_ERR_INVALID_ARGUMENT, "grid spacing and origin must be finite");
    const double cells = (double)(g->nx - 1) * (double)(g->ny - 1) * (double)(g->nz - 1);
    if (cells >= 4.0e18) return fail(h, DCB_ERR_TOO_LARGE, "grid too large");
    return DCB_OK;
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) { cudaGetLastError(); return 0.f; }
    return ms;
}

// Host copy of a batch's layout (per-grid offsets of the concatenated arrays, mark tiling).
struct BatchLayout {
    std::vector<GridSlot> slots;
    std::vector<long long> seg_off, col_off;          // n + 1
    // mark launches: index 1 for 256-cell x-tiles, 0 for 1024-cell ones
    std::vector<int> tile_slot[2];                    // grids of each mark launch
    std::vector<long long> tile_off[2];               // their first tiles (+ total)
    long long bits = 0, super = 0, nseg = 0, ncol = 0, ncell = 0, wt = 0;
    float hmax = 0.f;
};

int layout_batch(dcb_context* h, const dcb_grid* in, int n, BatchLayout& L) {
    L.slots.resize(n);
    L.seg_off.assign(n + 1, 0);
    L.col_off.assign(n + 1, 0);
    for (int v = 0; v < 2; ++v) { L.tile_slot[v].clear(); L.tile_off[v].assign(1, 0); }
    for (int b = 0; b < n; ++b) {
        GridSlot& S = L.slots[b];
        GridDesc& g = S.g;
        g.nx = in[b].nx; g.ny = in[b].ny; g.nz = in[b].nz;
        g.cx = g.nx - 1; g.cy = g.ny - 1; g.cz = g.nz - 1;
        g.W = ((g.cx + 31) / 32 + 7) / 8 * 8;
        g.W8 = g.W / 8;
        g.vx = in[b].vx; g.vy = in[b].vy; g.vz = in[b].vz;
        g.ox = in[b].ox; g.oy = in[b].oy; g.oz = in[b].oz;
        g.v = in[b].values;
        const long long rows = (long long)g.cy * g.cz;
        // grids at most 256 cells wide march 256-cell x-tiles (less idle width)
        S.tw = g.cx <= h->tune_narrow_cells ? mark_narrow_tile_words() : mark_tile_words();
        S.nxt = (g.cx + 32 * S.tw - 1) / (32 * S.tw);
        S.R = std::min(mark_max_rows(), g.cy);
        S.nrb = (g.cy + S.R - 1) / S.R;
        // About four CTAs per resident slot, each marching 8..64 planes (a single long wave
        // measured slower at 1024^3: 0.887 vs 0.848 ms).
        if (h->mark_ctas[n == 1] == 0) h->mark_ctas[n == 1] = mark_ctas_per_sm(n == 1);
        const long long slots = (long long)h->num_sms * h->mark_ctas[n == 1] * h->tune_waves;
        S.KZ = (int)std::max(8LL, std::min(64LL, (g.cz * S.nxt * (long long)S.nrb + slots - 1) / slots));
        S.nzc = (g.cz + S.KZ - 1) / S.KZ;
        S.bits_off = L.bits;
        S.super_off = L.super;
        S.seg_off = L.nseg;
        S.col_off = L.ncol;
        L.seg_off[b] = L.nseg;
        L.col_off[b] = L.ncol;
        L.bits += rows * g.W;
        L.super += rows * g.W8;
        L.nseg += rows * S.nxt;
        L.ncol += 3LL * g.cx * g.cy;
        L.ncell += (long long)g.cx * rows;
        const int grp = S.tw == mark_narrow_tile_words() ? 1 : 0;
        L.tile_slot[grp].push_back(b);
        L.tile_off[grp].push_back(L.tile_off[grp].back() + (long long)S.nxt * S.nrb * S.nzc);
        S.hmax = std::max(std::fabs(g.vx), std::max(std::fabs(g.vy), std::fabs(g.vz)));
        S.wt_off = L.wt;
        L.wt += width_table_len(g.cx, g.cy, g.cz);
        L.hmax = std::max(L.hmax, S.hmax);
    }
    L.seg_off[n] = L.nseg;
    L.col_off[n] = L.ncol;
    for (int v = 0; v < 2; ++v)
        if (L.tile_off[v].back() > 0x7fffffffLL) return fail(h, DCB_ERR_TOO_LARGE, "grid too large for the tiling");
    if (L.nseg >= 0xffffffffLL || L.ncol >= 0xffffffffLL) return fail(h, DCB_ERR_TOO_LARGE, "batch too large");
    return DCB_OK;
}

// Device copy of the layout: slots | seg_off | col_off | vert_off | face_off | tile lists.
struct TableView {
    BatchTable B;
    unsigned long long* vert_off;
    unsigned long long* face_off;
    const int* tile_slot[2];
    const long long* tile_off[2];
};

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

// A captured batch pipeline (dcb_batch_graph_create): the graph, its layout and options, and
// the capacity its buffers were sized for.
struct BatchGraphState {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    BatchLayout L;
    TableView T;
    dcb_opts o;
    long long cap = 0;
    int n = 0;
    unsigned long long gen = 0;
};

namespace {

void destroy_graph(dcb_context* h) {
    if (!h->bg) return;
    if (h->bg->exec) cudaGraphExecDestroy(h->bg->exec);
    if (h->bg->graph) cudaGraphDestroy(h->bg->graph);
    delete h->bg;
    h->bg = nullptr;
}

int upload_table(dcb_context* h, const BatchLayout& L, cudaStream_t s, TableView& T) {
    const int n = (int)L.slots.size();
    const size_t o_slots = 0;
    const size_t o_seg = align_up(o_slots + sizeof(GridSlot) * n);
    const size_t o_col = align_up(o_seg + sizeof(long long) * (n + 1));
    const size_t o_vert = align_up(o_col + sizeof(long long) * (n + 1));
    const size_t o_face = align_up(o_vert + sizeof(unsigned long long) * (n + 1));
    size_t o_ts[2], o_to[2];
    size_t at = align_up(o_face + sizeof(unsigned long long) * (n + 1));
    for (int v = 0; v < 2; ++v) { o_ts[v] = at; at = align_up(at + sizeof(int) * L.tile_slot[v].size() + 1); }
    for (int v = 0; v < 2; ++v) { o_to[v] = at; at = align_up(at + sizeof(long long) * L.tile_off[v].size()); }
    const size_t total = at;
    DCB_TRY(h, ensure(h->table, total), "alloc batch table");
    DCB_TRY(h, ensure_host(h->h_table, h->h_table_bytes, total), "alloc pinned batch table");
    char* hb = reinterpret_cast<char*>(h->h_table);
    std::memcpy(hb + o_slots, L.slots.data(), sizeof(GridSlot) * n);
    std::memcpy(hb + o_seg, L.seg_off.data(), sizeof(long long) * (n + 1));
    std::memcpy(hb + o_col, L.col_off.data(), sizeof(long long) * (n + 1));
    for (int v = 0; v < 2; ++v) {
        std::memcpy(hb + o_ts[v], L.tile_slot[v].data(), sizeof(int) * L.tile_slot[v].size());
        std::memcpy(hb + o_to[v], L.tile_off[v].data(), sizeof(long long) * L.tile_off[v].size());
    }
    DCB_TRY(h, cudaMemcpyAsync(h->table.p, hb, total, cudaMemcpyHostToDevice, s), "upload batch table");
    char* db = reinterpret_cast<char*>(h->table.p);
    T.B.s0 = L.slots[0];
    T.B.slots = reinterpret_cast<const GridSlot*>(db + o_slots);
    T.B.n = n;
    T.B.seg_off = reinterpret_cast<const long long*>(db + o_seg);
    T.B.col_off = reinterpret_cast<const long long*>(db + o_col);
    T.vert_off = reinterpret_cast<unsigned long long*>(db + o_vert);
    T.face_off = reinterpret_cast<unsigned long long*>(db + o_face);
    T.B.vert_off = T.vert_off;
    T.B.cell_slot = nullptr;
    for (int v = 0; v < 2; ++v) {
        T.tile_slot[v] = reinterpret_cast<const int*>(db + o_ts[v]);
        T.tile_off[v] = reinterpret_cast<const long long*>(db + o_to[v]);
    }
    return DCB_OK;
}

// The mark launches of a batch (one per group of grids with the same load width and tile).
int launch_marks(dcb_context* h, const BatchLayout& L, const TableView& T, cudaStream_t s) {
    for (int v = 0; v < 2; ++v) {
        if (L.tile_slot[v].empty()) continue;
        MarkParams mp;
        mp.B = T.B; mp.tile_slot = T.tile_slot[v]; mp.tile_off = T.tile_off[v];
        mp.m = (int)L.tile_slot[v].size(); mp.ntiles = L.tile_off[v].back();
        mp.bits = as<uint32_t>(h->bits); mp.seg_count = as<uint32_t>(h->seg_count);
        mp.nonfinite = h->counters.p ? &as<Counters>(h->counters)->nonfinite : nullptr;
        DCB_TRY(h, launch_mark(mp, v ? mark_narrow_tile_words() : mark_tile_words(), s), "launch mark");
    }
    return DCB_OK;
}

// Runs the pipeline on n device-resident grids as one batch (a single extraction is n = 1);
// ev[1] must already be recorded. Vertices are numbered over the whole batch while running;
// for n > 1 the faces are rebased to their own grid's vertices at the end.
// Layout, table upload and the buffers whose sizes do not depend on the active count.
int batch_prepare(dcb_context* h, const dcb_grid* in, int n, cudaStream_t s, BatchLayout& L, TableView& T) {
    int rc = layout_batch(h, in, n, L);
    if (rc != DCB_OK) return rc;
    rc = upload_table(h, L, s, T);
    if (rc != DCB_OK) return rc;
    const long long nseg = L.nseg, ncol = L.ncol;

    DCB_TRY(h, ensure(h->bits, sizeof(uint32_t) * L.bits), "alloc bits");
    DCB_TRY(h, ensure(h->super, sizeof(uint32_t) * L.super), "alloc ranks");
    DCB_TRY(h, ensure(h->seg_count, sizeof(uint32_t) * nseg), "alloc segment counts");
    DCB_TRY(h, ensure(h->seg_start, sizeof(uint32_t) * nseg), "alloc segment starts");
    DCB_TRY(h, ensure(h->counters, sizeof(Counters)), "alloc counters");
    DCB_TRY(h, ensure(h->col_count, sizeof(uint32_t) * ncol), "alloc column counts");
    DCB_TRY(h, ensure(h->col_fill, sizeof(uint32_t) * ncol), "alloc column fill");
    DCB_TRY(h, ensure(h->col_start, sizeof(uint32_t) * ncol), "alloc column starts");
    DCB_TRY(h, ensure(h->wt, sizeof(float) * L.wt), "alloc cell-width tables");
    const long long plen = std::max(scan_partials_len(ncol), scan_partials_len(nseg));
    DCB_TRY(h, ensure(h->partials, sizeof(uint32_t) * std::max(1LL, plen)), "alloc scan");
    if (!h->h_counters) DCB_TRY(h, host_malloc(&h->h_counters, sizeof(Counters)), "alloc pinned counters");
    DCB_TRY(h, ensure_host(h->h_offsets, h->h_offsets_bytes, 2 * sizeof(unsigned long long) * (n + 1)), "alloc pinned offsets");


    return DCB_OK;
}

// The buffers for up to `cap` active cells.
int batch_alloc(dcb_context* h, int n, long long cap, const dcb_opts* o, TableView& T) {
    DCB_TRY(h, ensure(h->list, sizeof(uint64_t) * cap), "alloc active list");
    DCB_TRY(h, ensure(h->V, sizeof(float) * 3 * cap), "alloc vertices");
    DCB_TRY(h, ensure(h->fmask, cap), "alloc face masks");
    DCB_TRY(h, ensure(h->vclass, cap), "alloc vertex classes");
    DCB_TRY(h, ensure(h->esc_list, sizeof(uint32_t) * cap), "alloc escalation list");
    DCB_TRY(h, ensure(h->hard_list, sizeof(uint32_t) * cap), "alloc hard list");
    DCB_TRY(h, ensure(h->hard_data, sizeof(float4) * 3 * cap), "alloc hard data");
    DCB_TRY(h, ensure(h->stage_quad, sizeof(int4) * 3 * cap), "alloc face staging");
    DCB_TRY(h, ensure(h->stage_key, sizeof(uint2) * 3 * cap), "alloc face keys");
    DCB_TRY(h, ensure(h->faces, sizeof(int4) * 3 * cap), "alloc faces");
    DCB_TRY(h, ensure(h->v64_index, sizeof(int) * cap), "alloc fp64 index");
    if (n > 1) {
        DCB_TRY(h, ensure(h->cell_slot, sizeof(uint32_t) * cap), "alloc vertex grids");
        T.B.cell_slot = as<uint32_t>(h->cell_slot);
    }
    // Exact upper bounds: at most 3 faces per owner cell, one FP64 vertex per cell.
    const long long wind_cap = std::min(0x7fffffffLL, 3 * cap);
    const long long v64_cap = cap;
    DCB_TRY(h, ensure(h->wind_items, sizeof(uint4) * wind_cap), "alloc winding list");
    DCB_TRY(h, ensure(h->v64_cells, sizeof(uint32_t) * v64_cap), "alloc fp64 cells");
    DCB_TRY(h, ensure(h->V64, sizeof(double) * 3 * v64_cap), "alloc fp64 vertices");
    if (o->emit_triangles) {
        DCB_TRY(h, ensure(h->tris, sizeof(int) * 6 * 3 * cap), "alloc triangles");
        DCB_TRY(h, ensure(h->tri_items, sizeof(uint32_t) * wind_cap), "alloc triangle list");
    }
    return DCB_OK;
}

// The mark launches, the segment scan (total active count into the counters) and the
// first vertex of every grid.
int batch_mark(dcb_context* h, const BatchLayout& L, const TableView& T, cudaStream_t s, bool events) {
    Counters* dc = as<Counters>(h->counters);
    DCB_TRY(h, cudaMemsetAsync(h->counters.p, 0, sizeof(Counters), s), "memset counters");
    int rc = launch_marks(h, L, T, s);
    if (rc != DCB_OK) return rc;
    if (events) DCB_TRY(h, cudaEventRecord(h->ev[6], s), "event");
    DCB_TRY(h, launch_scan(as<uint32_t>(h->seg_count), L.nseg, as<uint32_t>(h->partials), as<uint32_t>(h->seg_start),
                           &dc->total_active, s), "launch segment scan");
    DCB_TRY(h, launch_vert_offsets(T.B, as<uint32_t>(h->seg_start), &dc->total_active, T.vert_off, s), "vertex offsets");
    if (events) DCB_TRY(h, cudaEventRecord(h->ev[2], s), "event");
    return DCB_OK;
}

// Handle state of a batch with nv vertices (the per-grid first vertices are in h_offsets).
void batch_state(dcb_context* h, const BatchLayout& L, int n, const dcb_opts* o, long long nv) {
    const unsigned long long* h_vert_off = reinterpret_cast<const unsigned long long*>(h->h_offsets);
    h->nv = nv;
    h->nf = 0;
    h->vpf = o->emit_triangles ? 3 : 4;
    h->cx = L.slots[0].g.cx;
    h->cy = L.slots[0].g.cy;
    h->cz = L.slots[0].g.cz;
    h->batch_n = n;
    h->last_kind = 0;
    h->cells_per_vertex = 0;
    h->batch_cx.resize(n); h->batch_cy.resize(n);
    h->vert_offsets.assign(n + 1, 0);
    h->face_offsets.assign(n + 1, 0);
    for (int b = 0; b < n; ++b) { h->batch_cx[b] = L.slots[b].g.cx; h->batch_cy[b] = L.slots[b].g.cy; }
    for (int b = 0; b <= n; ++b) h->vert_offsets[b] = (int64_t)h_vert_off[b];
}

// Everything after the mark for up to `cap` active cells: ranks and list, vertices, faces.
// With `live` (a device count, as in a captured graph) the kernels take the active count from
// there, bounded by cap; otherwise it is cap.
int batch_rest(dcb_context* h, const BatchLayout& L, TableView& T, const dcb_opts* o, cudaStream_t s, long long cap,
               const unsigned long long* live, bool events) {
    const int n = (int)L.slots.size();
    const long long nseg = L.nseg, ncol = L.ncol;
    Counters* dc = as<Counters>(h->counters);
    const long long wind_cap = std::min(0x7fffffffLL, 3 * cap);
    const long long v64_cap = cap;
    DCB_TRY(h, cudaMemsetAsync(h->col_count.p, 0, sizeof(uint32_t) * ncol, s), "memset");
    DCB_TRY(h, cudaMemsetAsync(h->v64_index.p, 0xff, sizeof(int) * cap, s), "memset");

    // 2) ranks + list, QEF with fused edge normals (rank-1 fast path, Jacobi list, FP64).
    ExpandParams xp;
    xp.B = T.B; xp.nseg = nseg; xp.bits = as<uint32_t>(h->bits); xp.seg_count = as<uint32_t>(h->seg_count);
    xp.seg_start = as<uint32_t>(h->seg_start); xp.super = as<uint32_t>(h->super); xp.list = as<uint64_t>(h->list);
    xp.cell_slot = n > 1 ? as<uint32_t>(h->cell_slot) : nullptr;
    xp.B.cell_slot = nullptr;                      // expand finds grids by segment
    xp.list_cap = cap;
    DCB_TRY(h, launch_expand(xp, h->num_sms, s), "launch expand");
    DCB_TRY(h, launch_width_tables(T.B, as<float>(h->wt), s), "launch width tables");
    QefParams qp;
    qp.B = T.B; qp.list = xp.list; qp.nactive = cap; qp.live = live; qp.V = as<float>(h->V); qp.vclass = as<uint8_t>(h->vclass);
    qp.fmask = as<uint8_t>(h->fmask); qp.col_count = as<uint32_t>(h->col_count);
    qp.wt = as<float>(h->wt);
    qp.esc_list = as<uint32_t>(h->esc_list); qp.esc_count = &dc->esc_count;
    qp.hard_list = as<uint32_t>(h->hard_list); qp.hard_data = as<float4>(h->hard_data); qp.hard_count = &dc->hard_count;
    qp.rank_hist = dc->rank_hist;
    qp.err = &dc->err;
    qp.nonfinite = &dc->nonfinite;
    qp.thr = (float)o->svd_threshold; qp.band = (float)o->fp64_threshold_band;
    qp.cond_max = (float)std::min(o->fp64_escalation_cond, 3.0e38); qp.force64 = o->force_fp64;
    DCB_TRY(h, launch_cell_qef(qp, h->num_sms, s, h->tune_qef_minb, h->tune_qef_bps), "launch qef");
    DCB_TRY(h, launch_cell_jacobi(qp, cap, h->num_sms, s), "launch jacobi");
    Vertex64Params v64;
    v64.B = T.B; v64.list = xp.list; v64.cells = qp.esc_list; v64.count = &dc->esc_count; v64.cap = (unsigned int)cap;
    v64.Vf = qp.V; v64.vclass = qp.vclass; v64.V64 = nullptr; v64.thr = o->svd_threshold;
    DCB_TRY(h, launch_vertex_fp64(v64, cap, h->num_sms, s), "launch vertex fp64");
    if (events) DCB_TRY(h, cudaEventRecord(h->ev[3], s), "event");
    // the faces were counted per column by k_cell_qef
    if (events) DCB_TRY(h, cudaEventRecord(h->ev[8], s), "event");

    // 3) faces: column scan, scatter with FP32 winding, FP64 re-decisions, in-column order.
    DCB_TRY(h, launch_scan(as<uint32_t>(h->col_count), ncol, as<uint32_t>(h->partials),
                           as<uint32_t>(h->col_start), &dc->face_total, s), "launch scan");
    DCB_TRY(h, cudaMemcpyAsync(h->col_fill.p, h->col_start.p, sizeof(uint32_t) * ncol, cudaMemcpyDeviceToDevice, s),
            "column slots");
    if (events) {
        DCB_TRY(h, cudaEventRecord(h->ev[9], s), "event");
        h->substage_events = true;
    }
    if (n > 1)
        DCB_TRY(h, launch_face_offsets(T.B, as<uint32_t>(h->col_start), &dc->face_total, T.face_off, s), "face offsets");
    FaceParams fp;
    fp.B = T.B; fp.list = xp.list; fp.nactive = cap; fp.live = live; fp.fmask = qp.fmask; fp.V = qp.V; fp.vclass = qp.vclass;
    fp.bits = xp.bits; fp.super = xp.super;
    fp.col_start = as<uint32_t>(h->col_start); fp.col_count = as<uint32_t>(h->col_count);
    fp.col_fill = as<uint32_t>(h->col_fill);
    fp.stage_quad = as<int4>(h->stage_quad); fp.stage_key = as<uint2>(h->stage_key);
    fp.wind_items = as<uint4>(h->wind_items); fp.wind_count = &dc->wind_count;
    fp.wind_cap = (unsigned long long)wind_cap;
    fp.v64_index = as<int>(h->v64_index); fp.v64_cells = as<uint32_t>(h->v64_cells);
    fp.v64_count = &dc->v64_count; fp.v64_cap = (unsigned long long)v64_cap;
    fp.err = &dc->err;
    fp.hmax = L.hmax;
    DCB_TRY(h, launch_face_scatter(fp, h->num_sms, s, h->tune_face_bps), "launch face scatter");
    Vertex64Params w64;
    w64.B = T.B; w64.list = xp.list; w64.cells = fp.v64_cells; w64.count = fp.v64_count; w64.cap = (unsigned int)v64_cap;
    w64.Vf = nullptr; w64.vclass = nullptr; w64.V64 = as<double>(h->V64); w64.thr = o->svd_threshold;
    DCB_TRY(h, launch_vertex_fp64(w64, v64_cap, h->num_sms, s), "launch fp64 vertices for windings");
    Winding64Params wp;
    wp.B = T.B; wp.items = fp.wind_items; wp.count = fp.wind_count; wp.cap = (unsigned int)wind_cap;
    wp.quads = fp.stage_quad; wp.v64_index = fp.v64_index; wp.V64 = w64.V64; wp.err = &dc->err;
    DCB_TRY(h, launch_winding_fp64(wp, wind_cap, h->num_sms, s), "launch winding fp64");
    DCB_TRY(h, launch_face_order(fp.stage_quad, fp.stage_key, fp.col_start, fp.col_count, &dc->face_total,
                                 as<int4>(h->faces), 3 * cap, h->num_sms, s), "launch face order");
    if (o->emit_triangles) {
        // 4) quads -> triangles; FP64 vertices for the quads FP32 cannot orient (the winding
        // pass's FP64 vertices are recomputed too: same values, and few).
        TriParams tp;
        tp.B = T.B;
        tp.quads = as<int4>(h->faces); tp.nquads = &dc->face_total; tp.V = qp.V; tp.vclass = qp.vclass;
        tp.hmax = fp.hmax; tp.tris = as<int>(h->tris); tp.items = as<uint32_t>(h->tri_items);
        tp.item_count = &dc->tri_count; tp.item_cap = (unsigned int)wind_cap;
        tp.v64_index = fp.v64_index; tp.v64_cells = fp.v64_cells; tp.v64_count = fp.v64_count;
        tp.v64_cap = fp.v64_cap; tp.err = &dc->err;
        DCB_TRY(h, launch_triangulate(tp, 3 * cap, h->num_sms, s), "launch triangulate");
        DCB_TRY(h, launch_vertex_fp64(w64, v64_cap, h->num_sms, s), "launch fp64 vertices for triangles");
        Tri64Params t64;
        t64.quads = tp.quads; t64.items = tp.items; t64.count = tp.item_count; t64.cap = tp.item_cap;
        t64.v64_index = fp.v64_index; t64.V64 = w64.V64; t64.tris = tp.tris; t64.err = &dc->err;
        DCB_TRY(h, launch_tri_fp64(t64, wind_cap, h->num_sms, s), "launch triangle fp64");
    }
    if (n > 1) {
        // 5) faces refer to vertices of their own grid
        if (o->emit_triangles)
            DCB_TRY(h, launch_localize_faces(T.vert_off, T.face_off, n, as<int>(h->tris), 3, 6 * cap, h->num_sms, s), "localize");
        else
            DCB_TRY(h, launch_localize_faces(T.vert_off, T.face_off, n, as<int>(h->faces), 4, 3 * cap, h->num_sms, s), "localize");
        DCB_TRY(h, cudaMemcpyAsync(reinterpret_cast<unsigned long long*>(h->h_offsets) + (n + 1), T.face_off, sizeof(unsigned long long) * (n + 1),
                                   cudaMemcpyDeviceToHost, s), "read face offsets");
    }
    return DCB_OK;
}

// After the last copy of the counters has arrived: errors, face counts and offsets, stats.
int batch_finish(dcb_context* h, int n, const dcb_opts* o, dcb_stats* st) {
    const Counters* hc = reinterpret_cast<const Counters*>(h->h_counters);
    const unsigned long long* h_face_off = reinterpret_cast<const unsigned long long*>(h->h_offsets) + (n + 1);
    if (hc->err == kErrNonFinite)
        return fail(h, DCB_ERR_INVALID_ARGUMENT,
                    "an infinite grid value at a quad edge's interpolation end: the reference CPU backend "
                    "cannot find that edge's Hermite sample and exits (contouring.cpp:590-594)");
    if (hc->err) {
        return fail(h, hc->err == kErrTimeout ? DCB_ERR_TIMEOUT : DCB_ERR_INTERNAL,
                    hc->err == kErrOverflow ? "FP64 work list overflow" : "device error flag set");
    }
    const int fpq = o->emit_triangles ? 2 : 1;
    h->vpf = o->emit_triangles ? 3 : 4;
    h->nf = (int64_t)hc->face_total * fpq;
    if (n > 1) for (int b = 0; b <= n; ++b) h->face_offsets[b] = (int64_t)h_face_off[b] * fpq;
    else { h->face_offsets[0] = 0; h->face_offsets[1] = h->nf; }
    if (st) {
        st->face_count = h->nf;
        st->qef_fallback_count = hc->esc_count;
        st->escalated_fp64_cells = hc->esc_count;
        st->winding_fp64_faces = hc->wind_count;
        for (int q = 0; q < 4; ++q) st->rank_hist[q] = (int64_t)hc->rank_hist[q];
        st->clamp_count = 0;
    }
    return DCB_OK;
}

// Active cells every per-cell buffer of the workspace holds (0 before the first extraction).
long long cell_capacity(const dcb_context* h, const dcb_opts* o) {
    long long c = (long long)(h->list.bytes / sizeof(uint64_t));
    auto lim = [&c](const DevBuf& b, size_t per) { c = std::min(c, (long long)(b.bytes / per)); };
    lim(h->V, 3 * sizeof(float)); lim(h->fmask, 1); lim(h->vclass, 1);
    lim(h->esc_list, sizeof(uint32_t)); lim(h->hard_list, sizeof(uint32_t)); lim(h->hard_data, 3 * sizeof(float4));
    lim(h->stage_quad, 3 * sizeof(int4)); lim(h->stage_key, 3 * sizeof(uint2)); lim(h->faces, 3 * sizeof(int4));
    lim(h->v64_index, sizeof(int)); lim(h->wind_items, 3 * sizeof(uint4)); lim(h->v64_cells, sizeof(uint32_t));
    lim(h->V64, 3 * sizeof(double));
    if (o->emit_triangles) { lim(h->tris, 18 * sizeof(int)); lim(h->tri_items, 3 * sizeof(uint32_t)); }
    return std::min(c, 0x7fffffffLL / 3);      // the winding list holds exactly 3 entries per cell
}

int run_batch(dcb_context* h, const dcb_grid* in, int n, const dcb_opts* o, cudaStream_t s, dcb_stats* st) {
    ++h->gen;
    BatchLayout L;
    TableView T;
    int rc = batch_prepare(h, in, n, s, L, T);
    if (rc != DCB_OK) return rc;
    Counters* dc = as<Counters>(h->counters);
    Counters* hc = reinterpret_cast<Counters*>(h->h_counters);
    unsigned long long* h_vert_off = reinterpret_cast<unsigned long long*>(h->h_offsets);

    // 1) mark: active bits + per-segment counts; scan -> segment starts and the total.
    rc = batch_mark(h, L, T, s, true);
    if (rc != DCB_OK) return rc;
    const long long cap = cell_capacity(h, o);
    if (cap > 0) {
        // 2) on the buffers of an earlier call, with no wait for the count: the kernels read it
        // on the device (above cap, every kernel past the mark does nothing)
        rc = batch_alloc(h, n, cap, o, T);
        if (rc != DCB_OK) return rc;
        rc = batch_rest(h, L, T, o, s, cap, &dc->total_active, true);
        if (rc != DCB_OK) return rc;
        DCB_TRY(h, cudaEventRecord(h->ev[4], s), "event");
        DCB_TRY(h, cudaMemcpyAsync(hc, dc, sizeof(Counters), cudaMemcpyDeviceToHost, s), "read counters");
        DCB_TRY(h, cudaMemcpyAsync(h_vert_off, T.vert_off, sizeof(unsigned long long) * (n + 1),
                                   cudaMemcpyDeviceToHost, s), "read vertex offsets");
        DCB_TRY(h, cudaStreamSynchronize(s), "pipeline");
        const long long nv = (long long)hc->total_active;
        if (nv >= 0x7fffffffLL) return fail(h, DCB_ERR_TOO_LARGE, "more than 2^31-1 vertices");
        batch_state(h, L, n, o, nv);
        if (st) {
            st->nx = L.slots[0].g.nx; st->ny = L.slots[0].g.ny; st->nz = L.slots[0].g.nz;
            st->total_cells = L.ncell; st->active_cells = nv; st->vertex_count = nv;
        }
        if (nv <= cap) return batch_finish(h, n, o, st);
        // more active cells than those buffers hold: the marks, counts and ranks stand; the rest
        // runs again below with buffers for nv cells (the counters past the mark start over)
        const Counters keep = *hc;
        std::memset(hc, 0, sizeof(Counters));
        hc->total_active = keep.total_active;
        hc->nonfinite = keep.nonfinite;
        DCB_TRY(h, cudaMemcpyAsync(dc, hc, sizeof(Counters), cudaMemcpyHostToDevice, s), "reset counters");
    }
    DCB_TRY(h, cudaMemcpyAsync(hc, dc, sizeof(Counters), cudaMemcpyDeviceToHost, s), "read count");
    DCB_TRY(h, cudaMemcpyAsync(h_vert_off, T.vert_off, sizeof(unsigned long long) * (n + 1), cudaMemcpyDeviceToHost, s),
            "read vertex offsets");
    DCB_TRY(h, cudaStreamSynchronize(s), "mark");
    const long long nv = (long long)hc->total_active;
    if (nv >= 0x7fffffffLL) return fail(h, DCB_ERR_TOO_LARGE, "more than 2^31-1 vertices");
    batch_state(h, L, n, o, nv);
    if (st) {
        st->nx = L.slots[0].g.nx; st->ny = L.slots[0].g.ny; st->nz = L.slots[0].g.nz;
        st->total_cells = L.ncell; st->active_cells = nv; st->vertex_count = nv;
    }
    if (nv == 0) {
        DCB_TRY(h, cudaEventRecord(h->ev[3], s), "event");
        DCB_TRY(h, cudaEventRecord(h->ev[4], s), "event");
        return DCB_OK;
    }
    rc = batch_alloc(h, n, nv, o, T);
    if (rc != DCB_OK) return rc;
    // 2) ranks + list, vertices, faces
    rc = batch_rest(h, L, T, o, s, nv, nullptr, true);
    if (rc != DCB_OK) return rc;
    DCB_TRY(h, cudaEventRecord(h->ev[4], s), "event");
    DCB_TRY(h, cudaMemcpyAsync(hc, dc, sizeof(Counters), cudaMemcpyDeviceToHost, s), "read counters");
    DCB_TRY(h, cudaStreamSynchronize(s), "pipeline");
    return batch_finish(h, n, o, st);
}

int run_pipeline(dcb_context* h, const dcb_grid* in, const dcb_opts* o, cudaStream_t s, dcb_stats* st) {
    return run_batch(h, in, 1, o, s, st);
}

// The outer/inner refinement (contouring.cpp:1255-1328): a dual-contouring extraction, then
// the refinement of its vertices; the mesh's topology is the extraction's.
int run_ours(dcb_context* h, const dcb_grid* in, const dcb_opts* o, cudaStream_t s, dcb_stats* st) {
    if (o->outer_iters < 0 || o->inner_iters < 0 || o->batch_size < 0 || !(o->mu >= 0.0) ||
        !std::isfinite(o->dc_weight) || !(o->sphere_weight >= 0.0) || !std::isfinite(o->new_face_pos_weight) ||
        !std::isfinite(o->new_hermite_pos_weight) || !std::isfinite(o->new_hermite_normal_weight))
        return fail(h, DCB_ERR_INVALID_ARGUMENT, "invalid refinement options");
    dcb_opts dc = *o;
    dc.method = DCB_METHOD_DUAL_CONTOURING;
    dc.emit_triangles = 0;
    dc.svd_threshold = 0.01;            // Cell::update's solve (Cell.cpp:314) ignores the options
    int rc = run_batch(h, in, 1, &dc, s, st);
    if (rc != DCB_OK) return rc;
    const long long nv = h->nv, nq = h->nf;
    const long long npts = (long long)in->nx * in->ny * in->nz;
    if (npts >= 0xffffffffLL) return fail(h, DCB_ERR_TOO_LARGE, "grid too large for the refinement");
    BatchLayout L;
    rc = layout_batch(h, in, 1, L);
    if (rc != DCB_OK) return rc;
    size_t sort_bytes = 0;
    const size_t ws = ours_workspace_bytes(nv, nq, npts, &sort_bytes);
    DCB_TRY(h, ensure(h->ours_ws, ws), "alloc refinement workspace");
    const bool tri = o->emit_triangles != 0;
    if (tri) DCB_TRY(h, ensure(h->tris, sizeof(int32_t) * 6 * (size_t)std::max(1LL, nq)), "alloc triangles");
    OursRun R;
    std::memset(&R, 0, sizeof(R));
    OursParams& P = R.P;
    P.g = L.slots[0].g;
    P.list = as<uint64_t>(h->list);
    P.nv = nv;
    P.bits = as<uint32_t>(h->bits);
    P.super = as<uint32_t>(h->super);
    P.dc_faces = as<int4>(h->faces);
    P.nq = nq;
    P.out_V = as<float>(h->V);
    P.out_faces = tri ? as<int4>(h->tris) : as<int4>(h->faces);
    // cell_diagonal (contouring.cpp:788-804) over the float grid positions
    const int n3[3] = {in->nx, in->ny, in->nz};
    const float o3[3] = {in->ox, in->oy, in->oz}, v3[3] = {in->vx, in->vy, in->vz};
    double hmin = 0.0;
    for (int a = 0; a < 3; ++a) {
        const double p0 = (double)(o3[a] + (float)0 * v3[a]);
        const double p1 = (double)(o3[a] + (float)(n3[a] - 1) * v3[a]);
        const double mn = std::min(p0, p1), mx = std::max(p0, p1);
        P.gmin[a] = mn;
        P.gd[a] = (mx - mn) / (double)(n3[a] - 1);
        P.lo[a] = mn;
        P.hi[a] = mx > mn ? mx : mn + 1.0;
        hmin = a == 0 ? P.gd[a] : std::min(hmin, P.gd[a]);
    }
    P.cell_diag = hmin * std::sqrt(3.0);
    P.inner_iters = o->inner_iters;
    P.mu = o->mu;
    P.dc_weight = o->dc_weight;
    P.sphere_weight = o->sphere_weight;
    P.thr = o->svd_threshold;
    P.wface = o->new_face_pos_weight;
    P.wnormal = o->new_hermite_normal_weight;
    P.wpos = o->new_hermite_pos_weight;
    Counters* dc_counters = as<Counters>(h->counters);
    P.err = &dc_counters->err;
    R.workspace = h->ours_ws.p;
    R.sort_bytes = sort_bytes;
    R.outer_iters = o->outer_iters;
    R.hermite_update = o->hermite_update;
    R.batch_size = o->batch_size;
    R.seed = o->seed;
    R.triangles = tri ? 1 : 0;
    R.num_sms = h->num_sms;
    DCB_TRY(h, cudaMemsetAsync(&dc_counters->err, 0, sizeof(int), s), "clear error flag");
    DCB_TRY(h, ours_run(R, s), "refinement");
    Counters* hc = reinterpret_cast<Counters*>(h->h_counters);
    DCB_TRY(h, cudaMemcpyAsync(hc, dc_counters, sizeof(Counters), cudaMemcpyDeviceToHost, s), "read counters");
    DCB_TRY(h, cudaEventRecord(h->ev[4], s), "event");
    DCB_TRY(h, cudaStreamSynchronize(s), "refinement");
    if (hc->err) return fail(h, DCB_ERR_INTERNAL, "refinement: BVH traversal stack overflow");
    h->vpf = tri ? 3 : 4;
    h->nf = tri ? 2 * nq : nq;
    if (st) { st->face_count = h->nf; st->vertex_count = nv; }
    return DCB_OK;
}

// The sparse (brick) backends (src/cuda/dc_cuda_sparse.cu:1171-1415) on one device grid:
// point words -> bricks -> active-cell bits, scan + rank expansion, vertices (and, for the
// multi-vertex variant, their scan and placement), faces into per-cell slots, scan,
// compaction. Two host read-backs: the active-cell count and the vertex and face totals.
int run_sparse(dcb_context* h, const dcb_grid* in, const dcb_opts* o, cudaStream_t s, dcb_stats* st) {
    ++h->gen;
    if (o->emit_triangles) return fail(h, DCB_ERR_NOT_SUPPORTED, "the sparse backends emit quads only");
    if (o->brick_size < 1 || o->brick_size > 4096) return fail(h, DCB_ERR_INVALID_ARGUMENT, "brick_size must be in [1, 4096]");
    if (o->normal_mode < 0 || o->normal_mode > 2) return fail(h, DCB_ERR_INVALID_ARGUMENT, "unknown normal_mode");
    if ((double)in->nx * in->ny * in->nz >= 2147483647.0)
        return fail(h, DCB_ERR_TOO_LARGE, "the sparse backends index points with 32-bit ints (as the reference)");
    const bool mvdc = o->method == DCB_METHOD_SPARSE_MVDC;
    GridSlot S{};
    GridDesc& g = S.g;
    g.nx = in->nx; g.ny = in->ny; g.nz = in->nz;
    g.cx = g.nx - 1; g.cy = g.ny - 1; g.cz = g.nz - 1;
    g.W = ((g.cx + 31) / 32 + 7) / 8 * 8;
    g.W8 = g.W / 8;
    g.vx = in->vx; g.vy = in->vy; g.vz = in->vz;
    g.ox = in->ox; g.oy = in->oy; g.oz = in->oz;
    g.v = in->values;
    S.tw = 32;
    S.nxt = (g.W + 31) / 32;
    SparseParams P{};
    P.g = g;
    P.bs = o->brick_size;
    P.nbx = (g.cx + P.bs - 1) / P.bs; P.nby = (g.cy + P.bs - 1) / P.bs; P.nbz = (g.cz + P.bs - 1) / P.bs;
    P.Wp = (g.nx + 31) / 32;
    P.nxt = S.nxt;
    P.mvdc = mvdc ? 1 : 0;
    P.normal_mode = o->normal_mode;
    P.close = 0.45f * g.vx;
    const long long prow = (long long)g.ny * g.nz, crow = (long long)g.cy * g.cz;
    const long long nb = (long long)P.nbx * P.nby * P.nbz, nseg = crow * S.nxt;
    DCB_TRY(h, ensure(h->sp_words, sizeof(uint32_t) * 3 * prow * P.Wp), "alloc point words");
    DCB_TRY(h, ensure(h->sp_brick, nb), "alloc brick flags");
    DCB_TRY(h, ensure(h->bits, sizeof(uint32_t) * crow * g.W), "alloc bits");
    DCB_TRY(h, ensure(h->super, sizeof(uint32_t) * crow * g.W8), "alloc ranks");
    DCB_TRY(h, ensure(h->seg_count, sizeof(uint32_t) * nseg), "alloc segment counts");
    DCB_TRY(h, ensure(h->seg_start, sizeof(uint32_t) * nseg), "alloc segment starts");
    DCB_TRY(h, ensure(h->sp_counters, sizeof(unsigned long long) * kScSlots), "alloc counters");
    if (!h->h_sp_counters) DCB_TRY(h, host_malloc(&h->h_sp_counters, sizeof(unsigned long long) * kScSlots), "alloc pinned counters");
    unsigned long long* dcn = as<unsigned long long>(h->sp_counters);
    unsigned long long* hcn = reinterpret_cast<unsigned long long*>(h->h_sp_counters);
    P.pn = as<uint32_t>(h->sp_words);
    P.pp = P.pn + prow * P.Wp;
    P.pc = P.pp + prow * P.Wp;
    P.brick = as<uint8_t>(h->sp_brick);
    P.bits = as<uint32_t>(h->bits);
    P.super = as<uint32_t>(h->super);
    P.seg_count = as<uint32_t>(h->seg_count);
    P.counters = dcn;

    // 1) point words, bricks, active-cell bits; scan -> the active count
    DCB_TRY(h, cudaMemsetAsync(dcn, 0, sizeof(unsigned long long) * kScSlots, s), "memset counters");
    DCB_TRY(h, launch_sparse_mark(P, h->num_sms, s), "launch sparse mark");
    DCB_TRY(h, cudaEventRecord(h->ev[6], s), "event");
    long long plen = std::max(1LL, scan_partials_len(nseg));
    DCB_TRY(h, ensure(h->partials, sizeof(uint32_t) * plen), "alloc scan");
    DCB_TRY(h, launch_scan(P.seg_count, nseg, as<uint32_t>(h->partials), as<uint32_t>(h->seg_start),
                           dcn + kScActiveCells, s), "launch segment scan");
    DCB_TRY(h, cudaEventRecord(h->ev[2], s), "event");
    DCB_TRY(h, cudaMemcpyAsync(hcn, dcn, sizeof(unsigned long long) * kScSlots, cudaMemcpyDeviceToHost, s), "read counts");
    DCB_TRY(h, cudaStreamSynchronize(s), "sparse mark");
    const long long na = (long long)hcn[kScActiveCells];
    if (na >= (mvdc ? 0x3fffffffLL : 0x7fffffffLL)) return fail(h, DCB_ERR_TOO_LARGE, "more than 2^31-1 vertices");

    h->last_kind = 1;
    h->cells_per_vertex = mvdc ? 1 : 0;
    h->nv = 0; h->nf = 0; h->vpf = 4;
    h->cx = g.cx; h->cy = g.cy; h->cz = g.cz;
    h->batch_n = 1;
    h->vert_offsets.assign(2, 0);
    h->face_offsets.assign(2, 0);
    if (st) {
        st->nx = g.nx; st->ny = g.ny; st->nz = g.nz;
        st->total_cells = (long long)g.cx * crow; st->active_cells = na;
        st->total_bricks = nb;
    }
    long long nverts = 0, nf = 0;
    if (na > 0) {
        // 2) ranks + list, vertices
        DCB_TRY(h, ensure(h->list, sizeof(uint64_t) * na), "alloc active list");
        DCB_TRY(h, ensure(h->V, sizeof(float) * 3 * (mvdc ? 2 * na : na)), "alloc vertices");
        DCB_TRY(h, ensure(h->sp_fcount, sizeof(uint32_t) * na), "alloc face counts");
        DCB_TRY(h, ensure(h->sp_fstart, sizeof(uint32_t) * na), "alloc face starts");
        DCB_TRY(h, ensure(h->sp_stage, sizeof(int4) * 6 * na), "alloc face staging");
        plen = std::max(plen, scan_partials_len(na));
        DCB_TRY(h, ensure(h->partials, sizeof(uint32_t) * plen), "alloc scan");
        ExpandParams xp{};
        xp.B.s0 = S; xp.B.n = 1;
        xp.nseg = nseg; xp.bits = P.bits; xp.seg_count = P.seg_count; xp.seg_start = as<uint32_t>(h->seg_start);
        xp.super = P.super; xp.list = as<uint64_t>(h->list); xp.cell_slot = nullptr;
        DCB_TRY(h, launch_expand(xp, h->num_sms, s), "launch expand");
        P.list = xp.list;
        P.nactive = na;
        P.V = as<float>(h->V);
        if (mvdc) {
            DCB_TRY(h, ensure(h->sp_vcount, sizeof(uint32_t) * na), "alloc vertex counts");
            DCB_TRY(h, ensure(h->sp_vstart, sizeof(uint32_t) * na), "alloc vertex starts");
            DCB_TRY(h, ensure(h->sp_vtmp, sizeof(float) * 6 * na), "alloc vertex staging");
            DCB_TRY(h, ensure(h->sp_ntmp, sizeof(float) * 6 * na), "alloc normal staging");
            DCB_TRY(h, ensure(h->sp_N, sizeof(float) * 6 * na), "alloc vertex normals");
            DCB_TRY(h, ensure(h->sp_vcell, sizeof(uint64_t) * 2 * na), "alloc vertex cells");
            P.vcount = as<uint32_t>(h->sp_vcount); P.vstart = as<uint32_t>(h->sp_vstart);
            P.vtmp = as<float>(h->sp_vtmp); P.ntmp = as<float>(h->sp_ntmp);
            P.N = as<float>(h->sp_N); P.vcell = as<uint64_t>(h->sp_vcell);
        }
        DCB_TRY(h, launch_sparse_vertices(P, h->num_sms, s), "launch sparse vertices");
        if (mvdc) {
            DCB_TRY(h, launch_scan(P.vcount, na, as<uint32_t>(h->partials), as<uint32_t>(h->sp_vstart),
                                   dcn + kScVertices, s), "launch vertex scan");
            DCB_TRY(h, launch_sparse_place(P, h->num_sms, s), "launch vertex placement");
        }
        DCB_TRY(h, cudaEventRecord(h->ev[3], s), "event");
        // 3) faces: per-cell staging with counts, scan, compaction
        P.fcount = as<uint32_t>(h->sp_fcount);
        P.fstart = as<uint32_t>(h->sp_fstart);
        P.stage = as<int4>(h->sp_stage);
        DCB_TRY(h, launch_sparse_faces(P, h->num_sms, s), "launch faces");
        DCB_TRY(h, cudaEventRecord(h->ev[8], s), "event");
        DCB_TRY(h, launch_scan(P.fcount, na, as<uint32_t>(h->partials), as<uint32_t>(h->sp_fstart),
                               dcn + kScFaces, s), "launch face scan");
        DCB_TRY(h, cudaEventRecord(h->ev[9], s), "event");
        h->substage_events = true;
        DCB_TRY(h, cudaMemcpyAsync(hcn, dcn, sizeof(unsigned long long) * kScSlots, cudaMemcpyDeviceToHost, s), "read totals");
        DCB_TRY(h, cudaStreamSynchronize(s), "sparse vertices");
        nverts = mvdc ? (long long)hcn[kScVertices] : na;
        nf = (long long)hcn[kScFaces];
        if (nf >= 0x7fffffffLL) return fail(h, DCB_ERR_TOO_LARGE, "more than 2^31-1 faces");
        DCB_TRY(h, ensure(h->faces, sizeof(int4) * std::max(1LL, nf)), "alloc faces");
        P.faces = as<int4>(h->faces);
        DCB_TRY(h, launch_sparse_compact(P, h->num_sms, s), "launch face compaction");
    } else {
        DCB_TRY(h, cudaEventRecord(h->ev[3], s), "event");
    }
    DCB_TRY(h, cudaEventRecord(h->ev[4], s), "event");
    DCB_TRY(h, cudaMemcpyAsync(hcn, dcn, sizeof(unsigned long long) * kScSlots, cudaMemcpyDeviceToHost, s), "read counters");
    DCB_TRY(h, cudaStreamSynchronize(s), "sparse faces");
    h->nv = nverts;
    h->nf = nf;
    h->vert_offsets[1] = nverts;
    h->face_offsets[1] = nf;
    if (st) {
        st->vertex_count = nverts;
        st->face_count = nf;
        st->active_bricks = (int64_t)hcn[kScActiveBricks];
        st->qef_fallback_count = (int64_t)hcn[kScFallback];
        st->clamp_count = (int64_t)hcn[kScClamp];
        st->invalid_count = (int64_t)hcn[kScInvalid];
        st->ambiguous_cells = (int64_t)hcn[kScAmbiguous];
        st->multi_vertex_cells = (int64_t)hcn[kScMulti];
        st->one_vertex_cells = (int64_t)hcn[kScOne];
        st->two_vertex_cells = (int64_t)hcn[kScTwo];
        st->split_rejection_count = (int64_t)hcn[kScSplitReject];
        st->faces_skipped = (int64_t)hcn[kScSkipped];
    }
    return DCB_OK;
}

// The extraction a method names, on a device grid.
int run_method(dcb_context* h, const dcb_grid* in, const dcb_opts* o, cudaStream_t s, dcb_stats* st) {
    h->substage_events = false;
    if (o->method == DCB_METHOD_SPARSE || o->method == DCB_METHOD_SPARSE_MVDC) return run_sparse(h, in, o, s, st);
    h->last_kind = 0;
    h->cells_per_vertex = 0;
    return o->method == DCB_METHOD_OURS ? run_ours(h, in, o, s, st) : run_pipeline(h, in, o, s, st);
}

bool known_method(int m) {
    return m == DCB_METHOD_DUAL_CONTOURING || m == DCB_METHOD_OURS || m == DCB_METHOD_SPARSE ||
           m == DCB_METHOD_SPARSE_MVDC;
}

void fill_times(dcb_context* h, dcb_stats* st, bool upload) {
    if (!st) return;
    st->upload_ms = upload ? elapsed(h->ev[0], h->ev[1]) : 0.f;
    st->marking_ms = elapsed(h->ev[1], h->ev[6]);       // the mark kernel alone
    st->compaction_ms = elapsed(h->ev[6], h->ev[2]);    // segment scan
    st->qef_ms = elapsed(h->ev[2], h->ev[3]);
    st->face_emission_ms = elapsed(h->ev[3], h->ev[4]);
    // DualContouringStats' finer stage times (include/dc_backend.h:44-78, filled by the
    // reference's sparse backend, dc_cuda_sparse.cu:1458-1467): active cells are marked and
    // compacted in one pass over the grid (no separate brick stage); faces are counted, their
    // counts scanned, then filled.
    st->active_brick_marking_ms = 0.f;
    st->active_brick_compaction_ms = 0.f;
    st->active_cell_marking_ms = st->marking_ms;
    st->active_cell_compaction_ms = st->compaction_ms;
    st->face_count_ms = h->substage_events ? elapsed(h->ev[3], h->ev[8]) : 0.f;
    st->face_prefix_sum_ms = h->substage_events ? elapsed(h->ev[8], h->ev[9]) : 0.f;
    st->face_fill_ms = h->substage_events ? elapsed(h->ev[9], h->ev[4]) : 0.f;
    // the reference declares and reports bad_qef_count but never increments it
    // (dc_cuda_sparse.cu:41, 1481)
    st->bad_qef_count = 0;
}

struct SdfCounters {
    int err;
    int changed;
    unsigned long long total_entries;
    unsigned long long exterior;
    unsigned int active_bins;
    unsigned int work_next;
};

bool finite_pos_spacing(float v) { return std::isfinite(v) && v > 0.f; }

// The mesh -> SDF pipeline on device arrays; out has nx*ny*nz floats.
int run_mesh_sdf(dcb_context* h, const float* d_verts, int64_t nv, const int32_t* d_faces, int64_t nf, int nx,
                 int ny, int nz, float ox, float oy, float oz, float vx, float vy, float vz, int voxelize_first,
                 int voxel_res, float* out, dcb_sdf_stats* st, cudaStream_t s) {
    if (nx < 1 || ny < 1 || nz < 1) return fail(h, DCB_ERR_INVALID_ARGUMENT, "grid needs at least 1 point per axis");
    if (nv < 0 || nf < 0 || (nf > 0 && (!d_verts || !d_faces)) || !out)
        return fail(h, DCB_ERR_INVALID_ARGUMENT, "null mesh or output array");
    if (nv > 0x7fffffffLL || nf > 0x7fffffffLL) return fail(h, DCB_ERR_TOO_LARGE, "more than 2^31-1 vertices or faces");
    if (!finite_pos_spacing(vx) || !finite_pos_spacing(vy) || !finite_pos_spacing(vz) || !std::isfinite(ox) ||
        !std::isfinite(oy) || !std::isfinite(oz))
        return fail(h, DCB_ERR_INVALID_ARGUMENT, "spacing must be finite and positive, origin finite");
    SdfParams P;
    std::memset(&P, 0, sizeof(P));
    P.nx = nx; P.ny = ny; P.nz = nz;
    P.ox = ox; P.oy = oy; P.oz = oz; P.vx = vx; P.vy = vy; P.vz = vz;
    sdf_bin_geometry(P);
    if (P.nbins > 0x7fffffffLL) return fail(h, DCB_ERR_TOO_LARGE, "too many bins");
    P.verts = d_verts; P.faces = d_faces; P.nv = nv; P.nf = nf; P.out = out;
    const long long rows = (long long)ny * nz;
    DCB_TRY(h, ensure(h->m_tris, sdf_tri_record_bytes() * (size_t)std::max<int64_t>(1, nf)), "alloc triangle records");
    DCB_TRY(h, ensure(h->m_bin_count, sizeof(uint32_t) * P.nbins), "alloc bins");
    DCB_TRY(h, ensure(h->m_bin_start, sizeof(uint32_t) * P.nbins), "alloc bins");
    DCB_TRY(h, ensure(h->m_bin_fill, sizeof(uint32_t) * P.nbins), "alloc bins");
    DCB_TRY(h, ensure(h->m_bin_active, P.nbins), "alloc bins");
    DCB_TRY(h, ensure(h->m_active_list, sizeof(uint32_t) * P.nbins), "alloc bins");
    DCB_TRY(h, ensure(h->m_axis_start, sizeof(int) * (P.gx + P.gy + P.gz + 3)), "alloc bins");
    DCB_TRY(h, ensure(h->m_partials, sizeof(uint32_t) * std::max(1LL, scan_partials_len(P.nbins))), "alloc scan");
    DCB_TRY(h, ensure(h->m_far, sizeof(uint32_t) * rows * P.W), "alloc masks");
    DCB_TRY(h, ensure(h->m_ext, sizeof(uint32_t) * rows * P.W), "alloc masks");
    DCB_TRY(h, ensure(h->m_tmp, sizeof(float) * (size_t)nx * ny * nz), "alloc relaxation buffer");
    DCB_TRY(h, ensure(h->m_counters, sizeof(SdfCounters)), "alloc counters");
    if (!h->h_sdf_counters) DCB_TRY(h, host_malloc(&h->h_sdf_counters, sizeof(SdfCounters)), "alloc pinned counters");
    SdfCounters* dc = as<SdfCounters>(h->m_counters);
    SdfCounters* hc = reinterpret_cast<SdfCounters*>(h->h_sdf_counters);
    P.tris = as<float>(h->m_tris);
    P.bin_count = as<uint32_t>(h->m_bin_count); P.bin_start = as<uint32_t>(h->m_bin_start);
    P.bin_fill = as<uint32_t>(h->m_bin_fill); P.bin_active = as<uint8_t>(h->m_bin_active);
    P.active_list = as<uint32_t>(h->m_active_list); P.axis_start = as<int>(h->m_axis_start);
    P.far = as<uint32_t>(h->m_far); P.ext = as<uint32_t>(h->m_ext); P.err = &dc->err;
    P.active_count = &dc->active_bins; P.work_next = &dc->work_next;

    cudaEvent_t* ev = h->ev;
    DCB_TRY(h, cudaEventRecord(ev[0], s), "event");
    DCB_TRY(h, cudaMemsetAsync(dc, 0, sizeof(SdfCounters), s), "memset");
    DCB_TRY(h, cudaMemsetAsync(P.bin_count, 0, sizeof(uint32_t) * P.nbins, s), "memset");
    DCB_TRY(h, cudaMemsetAsync(P.bin_fill, 0, sizeof(uint32_t) * P.nbins, s), "memset");
    DCB_TRY(h, launch_sdf_prep(P, h->num_sms, s), "launch triangle records");
    DCB_TRY(h, launch_scan(P.bin_count, P.nbins, as<uint32_t>(h->m_partials), P.bin_start, &dc->total_entries, s),
            "launch bin scan");
    DCB_TRY(h, cudaMemcpyAsync(hc, dc, sizeof(SdfCounters), cudaMemcpyDeviceToHost, s), "read counters");
    DCB_TRY(h, cudaStreamSynchronize(s), "bins");
    if (hc->err == kErrInvalid) return fail(h, DCB_ERR_INVALID_ARGUMENT, "a face index is out of range");
    const unsigned long long entries = hc->total_entries;
    if (entries >= 0xffffffffULL) return fail(h, DCB_ERR_TOO_LARGE, "more than 2^32-1 bin entries");
    DCB_TRY(h, ensure(h->m_bin_scratch, sizeof(uint32_t) * std::max(1ULL, entries)), "alloc bin entries");
    DCB_TRY(h, ensure(h->m_bin_tris, sizeof(uint32_t) * std::max(1ULL, entries)), "alloc bin entries");
    P.bin_scratch = as<uint32_t>(h->m_bin_scratch); P.bin_tris = as<uint32_t>(h->m_bin_tris);
    DCB_TRY(h, launch_sdf_bins(P, h->num_sms, s), "launch binning");
    DCB_TRY(h, cudaEventRecord(ev[1], s), "event");
    DCB_TRY(h, launch_sdf_band(P, h->num_sms, s), "launch band");
    DCB_TRY(h, cudaEventRecord(ev[2], s), "event");
    int64_t passes = 0;
    if (!voxelize_first) {
        DCB_TRY(h, launch_sdf_masks(P, h->num_sms, s), "launch masks");
        for (;;) {
            DCB_TRY(h, cudaMemsetAsync(&dc->changed, 0, sizeof(int), s), "memset");
            DCB_TRY(h, launch_sdf_flood(P, &dc->changed, h->num_sms, s), "launch flood");
            DCB_TRY(h, cudaMemcpyAsync(&hc->changed, &dc->changed, sizeof(int), cudaMemcpyDeviceToHost, s), "read flag");
            DCB_TRY(h, cudaStreamSynchronize(s), "flood");
            ++passes;
            if (!hc->changed) break;
            if (passes > 1000000) return fail(h, DCB_ERR_INTERNAL, "exterior flood did not converge");
        }
        DCB_TRY(h, cudaEventRecord(ev[3], s), "event");
        DCB_TRY(h, launch_sdf_finish(P, &dc->exterior, as<float>(h->m_tmp), h->num_sms, s), "launch finish");
    } else {
        // the voxel solid (:764-808): shell, dilation, exterior flood to its fixpoint; then the
        // far grid points take their sign from it (:826-832); no relaxation in this branch
        const int vr = std::max(32, std::min(2048, voxel_res));
        P.vres = vr;
        P.Wv = (vr + 31) / 32;
        P.vox_vx = ((float)nx * vx) / (float)vr;
        P.vox_vy = ((float)ny * vy) / (float)vr;
        P.vox_vz = ((float)nz * vz) / (float)vr;
        const size_t vwords = (size_t)vr * vr * P.Wv;
        DCB_TRY(h, ensure(h->m_vox, sizeof(uint32_t) * 3 * vwords), "alloc voxels");
        P.vshell = as<uint32_t>(h->m_vox);
        P.vfar = P.vshell + vwords;
        P.vext = P.vfar + vwords;
        DCB_TRY(h, cudaMemsetAsync(P.vshell, 0, sizeof(uint32_t) * vwords, s), "memset");
        DCB_TRY(h, launch_vox_raster(P, h->num_sms, s), "launch voxel raster");
        DCB_TRY(h, launch_vox_dilate(P, h->num_sms, s), "launch voxel dilation");
        for (;;) {
            DCB_TRY(h, cudaMemsetAsync(&dc->changed, 0, sizeof(int), s), "memset");
            DCB_TRY(h, launch_vox_flood(P, &dc->changed, h->num_sms, s), "launch voxel flood");
            DCB_TRY(h, cudaMemcpyAsync(&hc->changed, &dc->changed, sizeof(int), cudaMemcpyDeviceToHost, s), "read flag");
            DCB_TRY(h, cudaStreamSynchronize(s), "voxel flood");
            ++passes;
            if (!hc->changed) break;
            if (passes > 1000000) return fail(h, DCB_ERR_INTERNAL, "voxel flood did not converge");
        }
        DCB_TRY(h, cudaEventRecord(ev[3], s), "event");
        DCB_TRY(h, launch_vox_sign(P, &dc->exterior, h->num_sms, s), "launch voxel sign");
    }
    DCB_TRY(h, cudaEventRecord(ev[4], s), "event");
    DCB_TRY(h, cudaMemcpyAsync(hc, dc, sizeof(SdfCounters), cudaMemcpyDeviceToHost, s), "read counters");
    DCB_TRY(h, cudaStreamSynchronize(s), "mesh to sdf");
    if (hc->err) return fail(h, hc->err == kErrInvalid ? DCB_ERR_INVALID_ARGUMENT : DCB_ERR_INTERNAL, "device error flag set");
    if (st) {
        st->num_bins = P.nbins;
        st->bin_entries = (int64_t)entries;
        st->flood_passes = passes;
        st->exterior_points = (int64_t)hc->exterior;
        st->bins_ms = elapsed(ev[0], ev[1]);
        st->band_ms = elapsed(ev[1], ev[2]);
        st->sign_ms = elapsed(ev[2], ev[3]);
        st->relax_ms = voxelize_first ? 0.f : elapsed(ev[3], ev[4]);
        st->sign_ms += voxelize_first ? elapsed(ev[3], ev[4]) : 0.f;
        st->total_ms = elapsed(ev[0], ev[4]);
    }
    return DCB_OK;
}

}  // namespace

extern "C" {

void dcb_default_opts(dcb_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->method = DCB_METHOD_DUAL_CONTOURING;
    o->outer_iters = 100;
    o->inner_iters = 100;
    o->mu = 0.1;
    o->dc_weight = 0.02;
    o->sphere_weight = 1.0;
    o->svd_threshold = 0.01;
    o->fp64_escalation_cond = 1e6;
    o->fp64_threshold_band = 0.01;
    o->emit_triangles = 0;
    o->force_fp64 = 0;
    o->hermite_update = 1;
    o->batch_size = 200000;
    o->new_hermite_pos_weight = 0.2;
    o->new_face_pos_weight = 0.2;
    o->new_hermite_normal_weight = 0.2;
    o->seed = 0x5eed;
    o->brick_size = 8;
    o->normal_mode = DCB_NORMAL_TRILINEAR;
}

int dcb_debug_fail_allocations(int64_t allowed) {
    g_alloc_budget.store(allowed < 0 ? -1 : (long long)allowed);
    return DCB_OK;
}

int dcb_abi_version(void) { return DCB_ABI_VERSION; }

const char* dcb_status_string(int status) {
    switch (status) {
        case DCB_OK: return "ok";
        case DCB_ERR_INVALID_ARGUMENT: return "invalid argument";
        case DCB_ERR_TOO_LARGE: return "input exceeds index limits";
        case DCB_ERR_CUDA: return "CUDA error";
        case DCB_ERR_OUT_OF_MEMORY: return "out of memory";
        case DCB_ERR_TIMEOUT: return "device wait timed out";
        case DCB_ERR_NOT_SUPPORTED: return "not supported";
        case DCB_ERR_INTERNAL: return "internal error";
        default: return "unknown status";
    }
}

const char* dcb_last_error(dcb_handle h) { return h ? h->last_error.c_str() : "null handle"; }

int dcb_create(dcb_handle* out, int device) {
    if (!out) return DCB_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) { cudaGetLastError(); return DCB_ERR_CUDA; }
    if (device < 0 || device >= count) return DCB_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return DCB_ERR_CUDA; }
    dcb_context* h = new dcb_context();
    h->device = device;
    cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device);
    for (auto& ev : h->ev) {
        if (cudaEventCreate(&ev) != cudaSuccess) { cudaGetLastError(); delete h; return DCB_ERR_CUDA; }
    }
    *out = h;
    return DCB_OK;
}

int dcb_destroy(dcb_handle h) {
    if (!h) return DCB_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    DevBuf* bufs[] = {&h->grid, &h->bits, &h->super, &h->list, &h->seg_count, &h->seg_start, &h->counters,
                      &h->V, &h->vclass, &h->fmask, &h->col_count, &h->col_fill, &h->col_start,
                      &h->partials, &h->esc_list, &h->hard_list, &h->hard_data, &h->stage_quad,
                      &h->stage_key, &h->faces, &h->wind_items, &h->v64_index, &h->v64_cells, &h->V64,
                      &h->tris, &h->tri_items, &h->m_verts, &h->m_faces, &h->m_out, &h->m_tris,
                      &h->m_bin_count, &h->m_bin_start, &h->m_bin_fill, &h->m_bin_scratch, &h->m_bin_tris,
                      &h->m_bin_active, &h->m_active_list, &h->m_axis_start, &h->m_far, &h->m_ext, &h->m_tmp,
                      &h->m_partials, &h->m_counters, &h->m_vox, &h->table, &h->cell_slot, &h->adj_rows, &h->adj_owners, &h->ours_ws, &h->wt,
                      &h->sp_words, &h->sp_brick, &h->sp_vcount, &h->sp_vstart, &h->sp_vtmp, &h->sp_ntmp,
                      &h->sp_N, &h->sp_vcell, &h->sp_fcount, &h->sp_fstart, &h->sp_stage, &h->sp_counters};
    for (DevBuf* b : bufs) if (b->p) cudaFree(b->p);
    if (h->h_counters) cudaFreeHost(h->h_counters);
    if (h->h_sdf_counters) cudaFreeHost(h->h_sdf_counters);
    if (h->h_sp_counters) cudaFreeHost(h->h_sp_counters);
    destroy_graph(h);
    post_release(h->post);
    if (h->pp_in_V.p) cudaFree(h->pp_in_V.p);
    if (h->pp_in_F.p) cudaFree(h->pp_in_F.p);
    if (h->h_table) cudaFreeHost(h->h_table);
    if (h->h_offsets) cudaFreeHost(h->h_offsets);
    if (h->hV) cudaFreeHost(h->hV);
    if (h->hF) cudaFreeHost(h->hF);
    for (auto& ev : h->ev) if (ev) cudaEventDestroy(ev);
    delete h;
    return DCB_OK;
}

int dcb_extract_device(dcb_handle h, const dcb_grid* grid, const dcb_opts* opts, dcb_mesh_dev* out,
                       dcb_stats* stats, void* cuda_stream) {
    int rc = validate(h, grid);
    if (rc != DCB_OK) return rc;
    dcb_opts def;
    dcb_default_opts(&def);
    const dcb_opts* o = opts ? opts : &def;
    if (!known_method(o->method)) return fail(h, DCB_ERR_NOT_SUPPORTED, "unknown method");
    if (!(o->svd_threshold >= 0.0)) return fail(h, DCB_ERR_INVALID_ARGUMENT, "svd_threshold must be >= 0");
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return fail(h, DCB_ERR_CUDA, "set device"); }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(cuda_stream);
    if (stats) std::memset(stats, 0, sizeof(*stats));
    DCB_TRY(h, cudaEventRecord(h->ev[0], s), "event");
    DCB_TRY(h, cudaEventRecord(h->ev[1], s), "event");
    rc = run_method(h, grid, o, s, stats);
    if (rc != DCB_OK) return rc;
    fill_times(h, stats, false);
    if (stats) stats->total_ms = elapsed(h->ev[1], h->ev[4]);
    if (out) {
        out->vertex_count = h->nv;
        out->face_count = h->nf;
        out->verts_per_face = h->vpf;
        out->vertices = as<float>(h->V);
        out->faces = face_ptr(h);
        out->cell_coords = h->cells_per_vertex ? as<uint64_t>(h->sp_vcell) : as<uint64_t>(h->list);
    }
    return DCB_OK;
}

int dcb_extract_batch_device(dcb_handle h, const dcb_grid* grids, int n, const dcb_opts* opts,
                             dcb_batch_mesh* out, dcb_stats* stats, void* cuda_stream) {
    if (!h) return DCB_ERR_INVALID_ARGUMENT;
    if (!grids || n < 1) return fail(h, DCB_ERR_INVALID_ARGUMENT, "empty batch");
    for (int b = 0; b < n; ++b) {
        const int rc = validate(h, grids + b);
        if (rc != DCB_OK) return rc;
    }
    dcb_opts def;
    dcb_default_opts(&def);
    const dcb_opts* o = opts ? opts : &def;
    if (o->method != DCB_METHOD_DUAL_CONTOURING)
        return fail(h, DCB_ERR_NOT_SUPPORTED, "batches run dual contouring only");
    if (!(o->svd_threshold >= 0.0)) return fail(h, DCB_ERR_INVALID_ARGUMENT, "svd_threshold must be >= 0");
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return fail(h, DCB_ERR_CUDA, "set device"); }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(cuda_stream);
    if (stats) std::memset(stats, 0, sizeof(*stats));
    DCB_TRY(h, cudaEventRecord(h->ev[0], s), "event");
    DCB_TRY(h, cudaEventRecord(h->ev[1], s), "event");
    const int rc = run_batch(h, grids, n, o, s, stats);
    if (rc != DCB_OK) return rc;
    fill_times(h, stats, false);
    if (stats) stats->total_ms = elapsed(h->ev[1], h->ev[4]);
    if (out) {
        out->vertex_count = h->nv;
        out->face_count = h->nf;
        out->verts_per_face = h->vpf;
        out->vertices = as<float>(h->V);
        out->faces = face_ptr(h);
        out->vertex_offset = h->vert_offsets.data();
        out->face_offset = h->face_offsets.data();
    }
    return DCB_OK;
}

int dcb_extract_host(dcb_handle h, const dcb_grid* grid, const dcb_opts* opts, dcb_mesh_host* out,
                     dcb_stats* stats, void* cuda_stream) {
    int rc = validate(h, grid);
    if (rc != DCB_OK) return rc;
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return fail(h, DCB_ERR_CUDA, "set device"); }
    dcb_opts def;
    dcb_default_opts(&def);
    const dcb_opts* o = opts ? opts : &def;
    if (!known_method(o->method)) return fail(h, DCB_ERR_NOT_SUPPORTED, "unknown method");
    if (!(o->svd_threshold >= 0.0)) return fail(h, DCB_ERR_INVALID_ARGUMENT, "svd_threshold must be >= 0");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(cuda_stream);
    if (stats) std::memset(stats, 0, sizeof(*stats));
    const size_t npts = (size_t)grid->nx * grid->ny * grid->nz;
    DCB_TRY(h, ensure(h->grid, sizeof(float) * npts), "alloc grid");
    DCB_TRY(h, cudaEventRecord(h->ev[0], s), "event");
    DCB_TRY(h, cudaMemcpyAsync(h->grid.p, grid->values, sizeof(float) * npts, cudaMemcpyHostToDevice, s), "upload grid");
    DCB_TRY(h, cudaEventRecord(h->ev[1], s), "event");
    dcb_grid dg = *grid;
    dg.values = as<float>(h->grid);
    rc = run_method(h, &dg, o, s, stats);
    if (rc != DCB_OK) return rc;
    DCB_TRY(h, ensure_host(h->hV, h->hV_bytes, sizeof(float) * 3 * h->nv), "alloc host vertices");
    DCB_TRY(h, ensure_host(h->hF, h->hF_bytes, sizeof(int32_t) * h->vpf * h->nf), "alloc host faces");
    if (h->nv) DCB_TRY(h, cudaMemcpyAsync(h->hV, h->V.p, sizeof(float) * 3 * h->nv, cudaMemcpyDeviceToHost, s), "download vertices");
    if (h->nf) DCB_TRY(h, cudaMemcpyAsync(h->hF, face_ptr(h), sizeof(int32_t) * h->vpf * h->nf, cudaMemcpyDeviceToHost, s), "download faces");
    DCB_TRY(h, cudaEventRecord(h->ev[5], s), "event");
    DCB_TRY(h, cudaStreamSynchronize(s), "download");
    fill_times(h, stats, true);
    if (stats) {
        stats->download_ms = elapsed(h->ev[4], h->ev[5]);
        stats->total_ms = elapsed(h->ev[0], h->ev[5]);
    }
    if (out) {
        out->vertex_count = h->nv;
        out->face_count = h->nf;
        out->verts_per_face = h->vpf;
        out->vertices = reinterpret_cast<const float*>(h->hV);
        out->faces = reinterpret_cast<const int32_t*>(h->hF);
    }
    return DCB_OK;
}

int dcb_batch_graph_create(dcb_handle h, const dcb_grid* grids, int n, const dcb_opts* opts, double headroom,
                           void* cuda_stream) {
    if (!h) return DCB_ERR_INVALID_ARGUMENT;
    if (!grids || n < 1) return fail(h, DCB_ERR_INVALID_ARGUMENT, "empty batch");
    for (int b = 0; b < n; ++b) {
        const int rc = validate(h, grids + b);
        if (rc != DCB_OK) return rc;
    }
    dcb_opts def;
    dcb_default_opts(&def);
    const dcb_opts* o = opts ? opts : &def;
    if (o->method != DCB_METHOD_DUAL_CONTOURING) return fail(h, DCB_ERR_NOT_SUPPORTED, "batches run dual contouring only");
    if (!(o->svd_threshold >= 0.0)) return fail(h, DCB_ERR_INVALID_ARGUMENT, "svd_threshold must be >= 0");
    if (!(headroom >= 0.0) || headroom > 100.0) return fail(h, DCB_ERR_INVALID_ARGUMENT, "headroom must be in [0, 100]");
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return fail(h, DCB_ERR_CUDA, "set device"); }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(cuda_stream);
    if (s == 0) return fail(h, DCB_ERR_INVALID_ARGUMENT, "capture needs a stream other than the legacy default stream");
    destroy_graph(h);
    // an eager run sizes the capacity and leaves every size-independent buffer in place
    DCB_TRY(h, cudaEventRecord(h->ev[1], s), "event");
    int rc = run_batch(h, grids, n, o, s, nullptr);
    if (rc != DCB_OK) return rc;
    long long cap = (long long)((double)h->nv * (1.0 + headroom)) + 1024;
    cap = std::min(cap, 0x7ffffffeLL);
    BatchGraphState* g = new BatchGraphState();
    g->n = n; g->o = *o; g->cap = cap;
    rc = batch_prepare(h, grids, n, s, g->L, g->T);
    if (rc == DCB_OK) rc = batch_alloc(h, n, cap, o, g->T);
    if (rc == DCB_OK) {
        cudaError_t e = cudaStreamSynchronize(s);            // table upload done before the capture
        if (e != cudaSuccess) rc = cuda_fail(h, e, "prepare graph");
    }
    if (rc != DCB_OK) { delete g; return rc; }
    Counters* dc = as<Counters>(h->counters);
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) { delete g; return cuda_fail(h, e, "begin capture"); }
    rc = batch_mark(h, g->L, g->T, s, false);
    if (rc == DCB_OK) rc = batch_rest(h, g->L, g->T, o, s, cap, &dc->total_active, false);
    if (rc == DCB_OK) {
        e = cudaMemcpyAsync(h->h_counters, dc, sizeof(Counters), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(h->h_offsets, g->T.vert_off, sizeof(unsigned long long) * (n + 1),
                                cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) rc = cuda_fail(h, e, "capture read-back");
    }
    const cudaError_t ee = cudaStreamEndCapture(s, &g->graph);
    if (rc == DCB_OK && ee != cudaSuccess) rc = cuda_fail(h, ee, "end capture");
    if (rc == DCB_OK) {
        e = cudaGraphInstantiate(&g->exec, g->graph, 0);
        if (e != cudaSuccess) rc = cuda_fail(h, e, "instantiate graph");
    }
    if (rc != DCB_OK) {
        cudaGetLastError();
        if (g->graph) cudaGraphDestroy(g->graph);
        delete g;
        return rc;
    }
    g->gen = h->gen;
    h->bg = g;
    return DCB_OK;
}

int dcb_batch_graph_launch(dcb_handle h, void* cuda_stream) {
    if (!h) return DCB_ERR_INVALID_ARGUMENT;
    if (!h->bg) return fail(h, DCB_ERR_INVALID_ARGUMENT, "no batch graph: call dcb_batch_graph_create");
    if (h->bg->gen != h->gen)
        return fail(h, DCB_ERR_INVALID_ARGUMENT, "the handle was used for another call since the graph was captured");
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return fail(h, DCB_ERR_CUDA, "set device"); }
    DCB_TRY(h, cudaGraphLaunch(h->bg->exec, reinterpret_cast<cudaStream_t>(cuda_stream)), "launch graph");
    return DCB_OK;
}

int dcb_batch_graph_finish(dcb_handle h, dcb_batch_mesh* out, dcb_stats* stats, void* cuda_stream) {
    if (!h) return DCB_ERR_INVALID_ARGUMENT;
    if (!h->bg) return fail(h, DCB_ERR_INVALID_ARGUMENT, "no batch graph: call dcb_batch_graph_create");
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return fail(h, DCB_ERR_CUDA, "set device"); }
    DCB_TRY(h, cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(cuda_stream)), "graph");
    BatchGraphState* g = h->bg;
    const Counters* hc = reinterpret_cast<const Counters*>(h->h_counters);
    const long long nv = (long long)hc->total_active;
    if (nv > g->cap)
        return fail(h, DCB_ERR_TOO_LARGE, "the grids now have more active cells than the graph was built for; "
                                          "recreate it");
    if (stats) std::memset(stats, 0, sizeof(*stats));
    batch_state(h, g->L, g->n, &g->o, nv);
    if (stats) {
        stats->nx = g->L.slots[0].g.nx; stats->ny = g->L.slots[0].g.ny; stats->nz = g->L.slots[0].g.nz;
        stats->total_cells = g->L.ncell; stats->active_cells = nv; stats->vertex_count = nv;
    }
    const int rc = batch_finish(h, g->n, &g->o, stats);
    if (rc != DCB_OK) return rc;
    if (out) {
        out->vertex_count = h->nv;
        out->face_count = h->nf;
        out->verts_per_face = h->vpf;
        out->vertices = as<float>(h->V);
        out->faces = face_ptr(h);
        out->vertex_offset = h->vert_offsets.data();
        out->face_offset = h->face_offsets.data();
    }
    return DCB_OK;
}

int dcb_batch_graph_destroy(dcb_handle h) {
    if (!h) return DCB_ERR_INVALID_ARGUMENT;
    destroy_graph(h);
    return DCB_OK;
}

int dcb_extract_upload(dcb_handle h, const dcb_grid* grid, const dcb_opts* opts, dcb_mesh_dev* out,
                       dcb_stats* stats, void* cuda_stream) {
    int rc = validate(h, grid);
    if (rc != DCB_OK) return rc;
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return fail(h, DCB_ERR_CUDA, "set device"); }
    dcb_opts def;
    dcb_default_opts(&def);
    const dcb_opts* o = opts ? opts : &def;
    if (!known_method(o->method)) return fail(h, DCB_ERR_NOT_SUPPORTED, "unknown method");
    if (!(o->svd_threshold >= 0.0)) return fail(h, DCB_ERR_INVALID_ARGUMENT, "svd_threshold must be >= 0");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(cuda_stream);
    if (stats) std::memset(stats, 0, sizeof(*stats));
    const size_t npts = (size_t)grid->nx * grid->ny * grid->nz;
    DCB_TRY(h, ensure(h->grid, sizeof(float) * npts), "alloc grid");
    DCB_TRY(h, cudaEventRecord(h->ev[0], s), "event");
    DCB_TRY(h, cudaMemcpyAsync(h->grid.p, grid->values, sizeof(float) * npts, cudaMemcpyHostToDevice, s), "upload grid");
    DCB_TRY(h, cudaEventRecord(h->ev[1], s), "event");
    dcb_grid dg = *grid;
    dg.values = as<float>(h->grid);
    rc = run_method(h, &dg, o, s, stats);
    if (rc != DCB_OK) return rc;
    fill_times(h, stats, true);
    if (stats) stats->total_ms = elapsed(h->ev[0], h->ev[4]);
    if (out) {
        out->vertex_count = h->nv;
        out->face_count = h->nf;
        out->verts_per_face = h->vpf;
        out->vertices = as<float>(h->V);
        out->faces = face_ptr(h);
        out->cell_coords = h->cells_per_vertex ? as<uint64_t>(h->sp_vcell) : as<uint64_t>(h->list);
    }
    return DCB_OK;
}

int dcb_copy_mesh_to_host(dcb_handle h, float* vertices, int32_t* faces, void* cuda_stream) {
    if (!h) return DCB_ERR_INVALID_ARGUMENT;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(cuda_stream);
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return fail(h, DCB_ERR_CUDA, "set device"); }
    if (vertices && h->nv) DCB_TRY(h, cudaMemcpyAsync(vertices, h->V.p, sizeof(float) * 3 * h->nv, cudaMemcpyDeviceToHost, s), "copy vertices");
    if (faces && h->nf) DCB_TRY(h, cudaMemcpyAsync(faces, face_ptr(h), sizeof(int32_t) * h->vpf * h->nf, cudaMemcpyDeviceToHost, s), "copy faces");
    DCB_TRY(h, cudaStreamSynchronize(s), "copy mesh");
    return DCB_OK;
}

int dcb_copy_mesh_device(dcb_handle h, float* vertices, int32_t* faces, void* cuda_stream) {
    if (!h) return DCB_ERR_INVALID_ARGUMENT;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(cuda_stream);
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return fail(h, DCB_ERR_CUDA, "set device"); }
    if (vertices && h->nv) DCB_TRY(h, cudaMemcpyAsync(vertices, h->V.p, sizeof(float) * 3 * h->nv, cudaMemcpyDeviceToDevice, s), "copy vertices");
    if (faces && h->nf) DCB_TRY(h, cudaMemcpyAsync(faces, face_ptr(h), sizeof(int32_t) * h->vpf * h->nf, cudaMemcpyDeviceToDevice, s), "copy faces");
    return DCB_OK;
}

int dcb_copy_cells_to_host(dcb_handle h, int64_t* cell_linear_index, void* cuda_stream) {
    if (!h || (!cell_linear_index && h->nv)) return DCB_ERR_INVALID_ARGUMENT;
    if (h->nv == 0) return DCB_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(cuda_stream);
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return fail(h, DCB_ERR_CUDA, "set device"); }
    uint64_t* packed = reinterpret_cast<uint64_t*>(cell_linear_index);
    DCB_TRY(h, cudaMemcpyAsync(packed, h->cells_per_vertex ? h->sp_vcell.p : h->list.p, sizeof(uint64_t) * h->nv,
                               cudaMemcpyDeviceToHost, s), "copy cells");
    DCB_TRY(h, cudaStreamSynchronize(s), "copy cells");
    int b = 0;
    for (int64_t r = 0; r < h->nv; ++r) {
        while (h->batch_n > 1 && b + 1 < h->batch_n && r >= h->vert_offsets[b + 1]) ++b;
        const int64_t cx = h->batch_n > 1 ? h->batch_cx[b] : h->cx, cy = h->batch_n > 1 ? h->batch_cy[b] : h->cy;
        const uint64_t p = packed[r];
        const int64_t i = (int64_t)(p & 0x1FFFFF), j = (int64_t)((p >> 21) & 0x1FFFFF), k = (int64_t)(p >> 42);
        cell_linear_index[r] = i + cx * (j + cy * k);
    }
    return DCB_OK;
}

int dcb_autotune_mark(dcb_handle h, const dcb_grid* grids, int n, int* waves_out, int* narrow_cells_out,
                      float* best_ms_out, void* cuda_stream) {
    if (h) ++h->gen;                        // reuses the extraction workspace
    if (!h) return DCB_ERR_INVALID_ARGUMENT;
    if (!grids || n < 1) return fail(h, DCB_ERR_INVALID_ARGUMENT, "empty batch");
    for (int b = 0; b < n; ++b) {
        const int rc = validate(h, grids + b);
        if (rc != DCB_OK) return rc;
    }
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return fail(h, DCB_ERR_CUDA, "set device"); }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(cuda_stream);
    static const int kWaves[4] = {1, 2, 4, 8};
    static const int kNarrow[4] = {0, 256, 512, 1024};
    const int keep_w = h->tune_waves, keep_n = h->tune_narrow_cells;
    float best = 1e30f;
    int best_w = keep_w, best_n = keep_n;
    for (int a = 0; a < 4; ++a) {
        for (int c = 0; c < 4; ++c) {
            h->tune_waves = kWaves[a];
            h->tune_narrow_cells = kNarrow[c];
            BatchLayout L;
            int rc = layout_batch(h, grids, n, L);
            if (rc == DCB_OK) {
                TableView T;
                rc = upload_table(h, L, s, T);
                if (rc == DCB_OK) {
                    DCB_TRY(h, ensure(h->bits, sizeof(uint32_t) * L.bits), "alloc bits");
                    DCB_TRY(h, ensure(h->seg_count, sizeof(uint32_t) * L.nseg), "alloc segment counts");
                    float ms[3];
                    for (int r = 0; r < 4 && rc == DCB_OK; ++r) {       // one warm-up, three timed
                        DCB_TRY(h, cudaEventRecord(h->ev[0], s), "event");
                        rc = launch_marks(h, L, T, s);
                        DCB_TRY(h, cudaEventRecord(h->ev[1], s), "event");
                        DCB_TRY(h, cudaEventSynchronize(h->ev[1]), "autotune");
                        if (r > 0) ms[r - 1] = elapsed(h->ev[0], h->ev[1]);
                    }
                    if (rc == DCB_OK) {
                        std::sort(ms, ms + 3);
                        if (ms[1] < best) { best = ms[1]; best_w = kWaves[a]; best_n = kNarrow[c]; }
                    }
                }
            }
            if (rc != DCB_OK) { h->tune_waves = keep_w; h->tune_narrow_cells = keep_n; return rc; }
        }
    }
    h->tune_waves = best_w;
    h->tune_narrow_cells = best_n;
    if (waves_out) *waves_out = best_w;
    if (narrow_cells_out) *narrow_cells_out = best_n;
    if (best_ms_out) *best_ms_out = best;
    return DCB_OK;
}

int dcb_autotune_cells(dcb_handle h, const dcb_grid* grids, int n, const dcb_opts* opts, int* qef_min_blocks_out,
                       int* qef_blocks_per_sm_out, int* face_blocks_per_sm_out, float* best_ms_out, void* cuda_stream) {
    if (h) ++h->gen;                        // reuses the extraction workspace
    if (!h) return DCB_ERR_INVALID_ARGUMENT;
    if (!grids || n < 1) return fail(h, DCB_ERR_INVALID_ARGUMENT, "empty batch");
    for (int b = 0; b < n; ++b) {
        const int rc = validate(h, grids + b);
        if (rc != DCB_OK) return rc;
    }
    dcb_opts def;
    dcb_default_opts(&def);
    const dcb_opts* o = opts ? opts : &def;
    if (o->method != DCB_METHOD_DUAL_CONTOURING) return fail(h, DCB_ERR_NOT_SUPPORTED, "tunes the dual contouring kernels");
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return fail(h, DCB_ERR_CUDA, "set device"); }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(cuda_stream);
    // median of three timed extractions after one untimed: the vertex stage (expand, k_cell_qef,
    // Jacobi, FP64 vertices) or the face stage
    auto stage_ms = [&](bool faces, float& out) -> int {
        float ms[3];
        for (int r = 0; r < 4; ++r) {
            dcb_stats st;
            std::memset(&st, 0, sizeof(st));
            DCB_TRY(h, cudaEventRecord(h->ev[0], s), "event");
            DCB_TRY(h, cudaEventRecord(h->ev[1], s), "event");
            const int rc = run_batch(h, grids, n, o, s, &st);
            if (rc != DCB_OK) return rc;
            fill_times(h, &st, false);
            if (r > 0) ms[r - 1] = faces ? st.face_emission_ms : st.qef_ms;
        }
        std::sort(ms, ms + 3);
        out = ms[1];
        return DCB_OK;
    };
    static const int kMinB[3] = {4, 5, 6};
    static const int kWidth[3] = {8, 16, 32};
    const int keep_m = h->tune_qef_minb, keep_q = h->tune_qef_bps, keep_f = h->tune_face_bps;
    float best_q = 1e30f, best_f = 1e30f;
    int bm = keep_m, bq = keep_q, bf = keep_f;
    for (int a = 0; a < 3; ++a) {
        for (int w = 0; w < 3; ++w) {
            h->tune_qef_minb = kMinB[a];
            h->tune_qef_bps = kWidth[w];
            float t = 0.f;
            const int rc = stage_ms(false, t);
            if (rc != DCB_OK) { h->tune_qef_minb = keep_m; h->tune_qef_bps = keep_q; return rc; }
            if (t < best_q) { best_q = t; bm = kMinB[a]; bq = kWidth[w]; }
        }
    }
    h->tune_qef_minb = bm;
    h->tune_qef_bps = bq;
    for (int w = 0; w < 3; ++w) {
        h->tune_face_bps = kWidth[w];
        float t = 0.f;
        const int rc = stage_ms(true, t);
        if (rc != DCB_OK) { h->tune_face_bps = keep_f; return rc; }
        if (t < best_f) { best_f = t; bf = kWidth[w]; }
    }
    h->tune_face_bps = bf;
    if (qef_min_blocks_out) *qef_min_blocks_out = bm;
    if (qef_blocks_per_sm_out) *qef_blocks_per_sm_out = bq;
    if (face_blocks_per_sm_out) *face_blocks_per_sm_out = bf;
    if (best_ms_out) *best_ms_out = best_q + best_f;
    return DCB_OK;
}

int dcb_backward(dcb_handle h, const dcb_grid* grid, const dcb_opts* opts, const float* dL_dvertices,
                 float* dL_dgrid, int accumulate, void* cuda_stream) {
    int rc = validate(h, grid);
    if (rc != DCB_OK) return rc;
    dcb_opts def;
    dcb_default_opts(&def);
    const dcb_opts* o = opts ? opts : &def;
    if (o->method != DCB_METHOD_DUAL_CONTOURING) return fail(h, DCB_ERR_NOT_SUPPORTED, "the adjoint covers dual contouring only");
    if (!(o->svd_threshold >= 0.0)) return fail(h, DCB_ERR_INVALID_ARGUMENT, "svd_threshold must be >= 0");
    if (h->last_kind != 0 || h->batch_n != 1 || h->cx != grid->nx - 1 || h->cy != grid->ny - 1 || h->cz != grid->nz - 1)
        return fail(h, DCB_ERR_INVALID_ARGUMENT, "backward needs the grid of the last single-grid extraction");
    if (!dL_dgrid || (h->nv > 0 && !dL_dvertices)) return fail(h, DCB_ERR_INVALID_ARGUMENT, "null gradient array");
    ++h->gen;
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return fail(h, DCB_ERR_CUDA, "set device"); }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(cuda_stream);
    const size_t npts = (size_t)grid->nx * grid->ny * grid->nz;
    if (!accumulate) DCB_TRY(h, cudaMemsetAsync(dL_dgrid, 0, sizeof(float) * npts, s), "clear grid gradient");
    if (h->nv == 0) return DCB_OK;
    BatchLayout L;
    rc = layout_batch(h, grid, 1, L);
    if (rc != DCB_OK) return rc;
    if (12 * h->nv >= 0xffffffffLL) return fail(h, DCB_ERR_TOO_LARGE, "too many vertices for the adjoint");
    DCB_TRY(h, ensure(h->adj_rows, sizeof(AdjointRow) * 12 * (size_t)h->nv), "alloc adjoint rows");
    DCB_TRY(h, ensure(h->adj_owners, sizeof(uint32_t) * (12 * (size_t)h->nv + 64)), "alloc adjoint owners");
    AdjointParams P;
    P.rows = as<AdjointRow>(h->adj_rows);
    P.bits = as<uint32_t>(h->bits);
    P.super = as<uint32_t>(h->super);
    P.owners = as<uint32_t>(h->adj_owners);
    P.owner_count = as<uint32_t>(h->adj_owners) + 12 * (size_t)h->nv + 32;
    P.g = L.slots[0].g;
    P.list = as<uint64_t>(h->list);
    P.nactive = h->nv;
    P.dV = dL_dvertices;
    P.dgrid = dL_dgrid;
    P.thr = o->svd_threshold;
    DCB_TRY(h, launch_vertex_adjoint(P, h->num_sms, s), "launch vertex adjoint");
    return DCB_OK;
}

int dcb_mesh_to_sdf_device_ex(dcb_handle h, const float* vertices, int64_t num_vertices, const int32_t* faces,
                              int64_t num_faces, int nx, int ny, int nz, float ox, float oy, float oz, float vx,
                              float vy, float vz, int voxelize_first, int voxel_res, float* out_values,
                              dcb_sdf_stats* stats, void* cuda_stream) {
    if (!h) return DCB_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return fail(h, DCB_ERR_CUDA, "set device"); }
    if (stats) std::memset(stats, 0, sizeof(*stats));
    return run_mesh_sdf(h, vertices, num_vertices, faces, num_faces, nx, ny, nz, ox, oy, oz, vx, vy, vz,
                        voxelize_first, voxel_res, out_values, stats, reinterpret_cast<cudaStream_t>(cuda_stream));
}

int dcb_mesh_to_sdf_device(dcb_handle h, const float* vertices, int64_t num_vertices, const int32_t* faces,
                           int64_t num_faces, int nx, int ny, int nz, float ox, float oy, float oz, float vx,
                           float vy, float vz, float* out_values, dcb_sdf_stats* stats, void* cuda_stream) {
    return dcb_mesh_to_sdf_device_ex(h, vertices, num_vertices, faces, num_faces, nx, ny, nz, ox, oy, oz, vx, vy, vz,
                                     0, 256, out_values, stats, cuda_stream);
}

int dcb_mesh_to_sdf_host(dcb_handle h, const float* vertices, int64_t num_vertices, const int32_t* faces,
                         int64_t num_faces, int nx, int ny, int nz, float ox, float oy, float oz, float vx,
                         float vy, float vz, float* out_values, dcb_sdf_stats* stats, void* cuda_stream) {
    return dcb_mesh_to_sdf_host_ex(h, vertices, num_vertices, faces, num_faces, nx, ny, nz, ox, oy, oz, vx, vy, vz,
                                   0, 256, out_values, stats, cuda_stream);
}

int dcb_mesh_to_sdf_host_ex(dcb_handle h, const float* vertices, int64_t num_vertices, const int32_t* faces,
                            int64_t num_faces, int nx, int ny, int nz, float ox, float oy, float oz, float vx,
                            float vy, float vz, int voxelize_first, int voxel_res, float* out_values,
                            dcb_sdf_stats* stats, void* cuda_stream) {
    if (!h) return DCB_ERR_INVALID_ARGUMENT;
    if (!out_values || num_vertices < 0 || num_faces < 0 || (num_faces > 0 && (!vertices || !faces)))
        return fail(h, DCB_ERR_INVALID_ARGUMENT, "null mesh or output array");
    if (nx < 1 || ny < 1 || nz < 1) return fail(h, DCB_ERR_INVALID_ARGUMENT, "grid needs at least 1 point per axis");
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return fail(h, DCB_ERR_CUDA, "set device"); }
    if (stats) std::memset(stats, 0, sizeof(*stats));
    cudaStream_t s = reinterpret_cast<cudaStream_t>(cuda_stream);
    const size_t npts = (size_t)nx * ny * nz;
    DCB_TRY(h, ensure(h->m_verts, sizeof(float) * 3 * (size_t)std::max<int64_t>(1, num_vertices)), "alloc vertices");
    DCB_TRY(h, ensure(h->m_faces, sizeof(int32_t) * 3 * (size_t)std::max<int64_t>(1, num_faces)), "alloc faces");
    DCB_TRY(h, ensure(h->m_out, sizeof(float) * npts), "alloc values");
    if (num_vertices)
        DCB_TRY(h, cudaMemcpyAsync(h->m_verts.p, vertices, sizeof(float) * 3 * num_vertices, cudaMemcpyHostToDevice, s), "upload vertices");
    if (num_faces)
        DCB_TRY(h, cudaMemcpyAsync(h->m_faces.p, faces, sizeof(int32_t) * 3 * num_faces, cudaMemcpyHostToDevice, s), "upload faces");
    const int rc = run_mesh_sdf(h, as<float>(h->m_verts), num_vertices, as<int32_t>(h->m_faces), num_faces, nx, ny, nz,
                                ox, oy, oz, vx, vy, vz, voxelize_first, voxel_res, as<float>(h->m_out), stats, s);
    if (rc != DCB_OK) return rc;
    DCB_TRY(h, cudaMemcpyAsync(out_values, h->m_out.p, sizeof(float) * npts, cudaMemcpyDeviceToHost, s), "download values");
    DCB_TRY(h, cudaStreamSynchronize(s), "download values");
    return DCB_OK;
}

int dcb_postprocess_device(dcb_handle h, const float* vertices, int64_t num_vertices, const int32_t* faces,
                           int64_t num_faces, int close_holes, int remove_floaters, dcb_mesh_dev* out,
                           dcb_post_stats* stats, void* cuda_stream) {
    if (!h) return DCB_ERR_INVALID_ARGUMENT;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (out) std::memset(out, 0, sizeof(*out));
    h->pp_V = nullptr; h->pp_F = nullptr; h->pp_nv = 0; h->pp_nf = 0;
    if (num_vertices < 0 || num_faces < 0 || (num_vertices > 0 && !vertices) || (num_faces > 0 && !faces))
        return fail(h, DCB_ERR_INVALID_ARGUMENT, "null mesh arrays or negative counts");
    if (num_vertices >= 0x7fffffffLL || num_faces >= (1LL << 29))
        return fail(h, DCB_ERR_TOO_LARGE, "post-pass limits: < 2^31 vertices, < 2^29 quads");
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return fail(h, DCB_ERR_CUDA, "set device"); }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(cuda_stream);
    DCB_TRY(h, cudaEventRecord(h->ev[0], s), "event");
    PostRun R;
    R.V = vertices; R.nv = num_vertices; R.F = faces; R.nf = num_faces;
    R.close_holes = close_holes != 0; R.remove_floaters = remove_floaters != 0; R.num_sms = h->num_sms;
    const cudaError_t e = post_run(h->post, R, s);
    if (e != cudaSuccess) return cuda_fail(h, e, R.what ? R.what : "post-pass");
    if (R.err & 1) return fail(h, DCB_ERR_INVALID_ARGUMENT, "face index out of range");
    if (R.err & 2) return fail(h, DCB_ERR_INVALID_ARGUMENT, "non-finite vertex coordinate");
    if (R.err & 4) return fail(h, DCB_ERR_NOT_SUPPORTED, "vertices too close together for the weld step");
    if (R.err & 16) return fail(h, DCB_ERR_NOT_SUPPORTED, "a hole fill did not converge within 8192 rings");
    if (R.err) return fail(h, DCB_ERR_INTERNAL, "post-pass consistency check failed");
    if (R.too_large) return fail(h, DCB_ERR_TOO_LARGE, "filled mesh exceeds the index limits");
    DCB_TRY(h, cudaEventRecord(h->ev[4], s), "event");
    DCB_TRY(h, cudaEventSynchronize(h->ev[4]), "post-pass");
    h->pp_V = R.out_V; h->pp_F = R.out_F; h->pp_nv = R.nv_out; h->pp_nf = R.nf_out;
    if (stats) {
        int64_t* st = &stats->welded_vertices;
        for (int i = 0; i < kPostNumStats; ++i) st[i] = R.stats[i];
        stats->total_ms = elapsed(h->ev[0], h->ev[4]);
    }
    if (out) {
        out->vertex_count = R.nv_out;
        out->face_count = R.nf_out;
        out->verts_per_face = 4;
        out->vertices = const_cast<float*>(R.out_V);
        out->faces = const_cast<int32_t*>(R.out_F);
        out->cell_coords = nullptr;
    }
    return DCB_OK;
}

int dcb_postprocess_host(dcb_handle h, const float* vertices, int64_t num_vertices, const int32_t* faces,
                         int64_t num_faces, int close_holes, int remove_floaters, dcb_mesh_dev* out,
                         dcb_post_stats* stats, void* cuda_stream) {
    if (!h) return DCB_ERR_INVALID_ARGUMENT;
    if (num_vertices < 0 || num_faces < 0 || (num_vertices > 0 && !vertices) || (num_faces > 0 && !faces))
        return fail(h, DCB_ERR_INVALID_ARGUMENT, "null mesh arrays or negative counts");
    if (num_vertices >= 0x7fffffffLL || num_faces >= (1LL << 29))
        return fail(h, DCB_ERR_TOO_LARGE, "post-pass limits: < 2^31 vertices, < 2^29 quads");
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return fail(h, DCB_ERR_CUDA, "set device"); }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(cuda_stream);
    DCB_TRY(h, ensure(h->pp_in_V, sizeof(float) * 3 * (size_t)std::max<int64_t>(1, num_vertices)), "alloc vertices");
    DCB_TRY(h, ensure(h->pp_in_F, sizeof(int32_t) * 4 * (size_t)std::max<int64_t>(1, num_faces)), "alloc faces");
    if (num_vertices)
        DCB_TRY(h, cudaMemcpyAsync(h->pp_in_V.p, vertices, sizeof(float) * 3 * num_vertices, cudaMemcpyHostToDevice, s), "upload vertices");
    if (num_faces)
        DCB_TRY(h, cudaMemcpyAsync(h->pp_in_F.p, faces, sizeof(int32_t) * 4 * num_faces, cudaMemcpyHostToDevice, s), "upload faces");
    return dcb_postprocess_device(h, as<float>(h->pp_in_V), num_vertices, as<int32_t>(h->pp_in_F), num_faces,
                                  close_holes, remove_floaters, out, stats, cuda_stream);
}

int dcb_copy_post_mesh(dcb_handle h, float* vertices, int32_t* faces, int to_host, void* cuda_stream) {
    if (!h) return DCB_ERR_INVALID_ARGUMENT;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(cuda_stream);
    if (cudaSetDevice(h->device) != cudaSuccess) { cudaGetLastError(); return fail(h, DCB_ERR_CUDA, "set device"); }
    const cudaMemcpyKind kind = to_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (vertices && h->pp_nv)
        DCB_TRY(h, cudaMemcpyAsync(vertices, h->pp_V, sizeof(float) * 3 * h->pp_nv, kind, s), "copy vertices");
    if (faces && h->pp_nf)
        DCB_TRY(h, cudaMemcpyAsync(faces, h->pp_F, sizeof(int32_t) * 4 * h->pp_nf, kind, s), "copy faces");
    if (to_host) DCB_TRY(h, cudaStreamSynchronize(s), "copy mesh");
    return DCB_OK;
}

}  // extern "C"
