/* dc_b200.h — the B200 engine as one more IDualContouringBackend of the reference project.
 *
 * Header-only C++ over the C ABI of dcb.h. It compiles inside the reference's tree: put this
 * repository's include/ and the reference's include/ on the include path and link libdcb.so.
 * It replaces, call for call:
 *   CpuDualContouringBackend::extract (src/cpp/dc_backend.cpp:51-125; interface
 *     IDualContouringBackend, include/dc_backend.h:80-84)             -> dcb_extract_host
 *   CudaDualContouringBackend::extract_device (include/dc_cuda.h:31-35,
 *     src/cuda/dc_cuda.cu:652-847)                                      -> dcb_extract_device
 *   CudaSparse[Mvdc]DualContouringBackend (include/dc_cuda.h:37-62)     -> the same calls with
 *     method DCB_METHOD_SPARSE[_MVDC], brick_size and normal_mode.
 * Errors become std::runtime_error (the reference calls exit(EXIT_FAILURE), dc_cuda.cu:14-20).
 * The returned mesh is a copy: vertices xyz, faces 4 ints per quad (3 with emit_triangles). */
#pragma once
#include "dc_backend.h"
#include "dc_cuda.h"
#include "dcb.h"
#include <stdexcept>
#include <string>

class B200DualContouringBackend : public IDualContouringBackend {
public:
    /* method: DCB_METHOD_DUAL_CONTOURING (the CPU backend's semantics), DCB_METHOD_OURS,
     * DCB_METHOD_SPARSE or DCB_METHOD_SPARSE_MVDC (the cuda-sparse backends). */
    explicit B200DualContouringBackend(int device = 0, int method = DCB_METHOD_DUAL_CONTOURING,
                                       int brick_size = 8, int normal_mode = DCB_NORMAL_TRILINEAR) {
        check(dcb_create(&h_, device));
        dcb_default_opts(&o_);
        o_.method = method;
        o_.brick_size = brick_size;
        o_.normal_mode = normal_mode;
    }
    ~B200DualContouringBackend() override { dcb_destroy(h_); }
    B200DualContouringBackend(const B200DualContouringBackend&) = delete;
    B200DualContouringBackend& operator=(const B200DualContouringBackend&) = delete;

    /* The options of the next calls (dcb_default_opts gives the reference defaults). */
    dcb_opts& options() { return o_; }

    /* Host grid in, host mesh out (IDualContouringBackend::extract). */
    DualContouringMesh extract(const DenseSdfGrid& grid, DualContouringStats& stats) override {
        dcb_grid g{grid.nx, grid.ny, grid.nz, grid.vx, grid.vy, grid.vz,
                   grid.ox, grid.oy, grid.oz, grid.values.data()};
        dcb_mesh_host m{};
        dcb_stats s{};
        check(dcb_extract_host(h_, &g, &o_, &m, &s, nullptr));
        DualContouringMesh mesh;
        mesh.vertices.assign(m.vertices, m.vertices + 3 * m.vertex_count);
        mesh.faces.assign(m.faces, m.faces + m.verts_per_face * m.face_count);
        fill_stats(s, stats);
        return mesh;
    }

    /* Borrowed device grid in (never freed), host mesh out
     * (CudaDualContouringBackend::extract_device). */
    DualContouringMesh extract_device(const DenseSdfGridDevice& grid, DualContouringStats& stats) {
        dcb_grid g{grid.nx, grid.ny, grid.nz, grid.vx, grid.vy, grid.vz,
                   grid.ox, grid.oy, grid.oz, grid.d_values};
        dcb_mesh_dev d{};
        dcb_stats s{};
        check(dcb_extract_device(h_, &g, &o_, &d, &s, nullptr));
        DualContouringMesh mesh;
        mesh.vertices.resize(3 * d.vertex_count);
        mesh.faces.resize(d.verts_per_face * d.face_count);
        check(dcb_copy_mesh_to_host(h_, mesh.vertices.empty() ? nullptr : mesh.vertices.data(),
                                    mesh.faces.empty() ? nullptr : mesh.faces.data(), nullptr));
        fill_stats(s, stats);
        return mesh;
    }

    /* Every DualContouringStats field (include/dc_backend.h:44-78) from the engine's stats.
     * The reference's counts are int; this engine's are 64-bit (they are truncated here). */
    static void fill_stats(const dcb_stats& s, DualContouringStats& out) {
        out.backend = "b200";
        out.nx = s.nx; out.ny = s.ny; out.nz = s.nz;
        out.total_cells = (int)s.total_cells;
        out.active_cells = (int)s.active_cells;
        out.total_bricks = (int)s.total_bricks;
        out.active_bricks = (int)s.active_bricks;
        out.upload_ms = s.upload_ms;
        out.marking_ms = s.marking_ms;
        out.compaction_ms = s.compaction_ms;
        out.active_brick_marking_ms = s.active_brick_marking_ms;
        out.active_brick_compaction_ms = s.active_brick_compaction_ms;
        out.active_cell_marking_ms = s.active_cell_marking_ms;
        out.active_cell_compaction_ms = s.active_cell_compaction_ms;
        out.qef_ms = s.qef_ms;
        out.face_emission_ms = s.face_emission_ms;
        out.face_count_ms = s.face_count_ms;
        out.face_prefix_sum_ms = s.face_prefix_sum_ms;
        out.face_fill_ms = s.face_fill_ms;
        out.download_ms = s.download_ms;
        out.total_ms = s.total_ms;
        out.vertex_count = (int)s.vertex_count;
        out.face_count = (int)s.face_count;
        out.qef_fallback_count = (int)s.qef_fallback_count;
        out.clamp_count = (int)s.clamp_count;
        out.invalid_count = (int)s.invalid_count;
        out.ambiguous_cells = (int)s.ambiguous_cells;
        out.multi_vertex_cells = (int)s.multi_vertex_cells;
        out.one_vertex_cells = (int)s.one_vertex_cells;
        out.two_vertex_cells = (int)s.two_vertex_cells;
        out.split_rejection_count = (int)s.split_rejection_count;
        out.bad_qef_count = (int)s.bad_qef_count;
        out.faces_skipped_due_to_missing_cluster = (int)s.faces_skipped;
    }

private:
    dcb_handle h_ = nullptr;
    dcb_opts o_{};

    void check(int st) {
        if (st != DCB_OK)
            throw std::runtime_error(std::string(dcb_status_string(st)) + ": " + (h_ ? dcb_last_error(h_) : ""));
    }
};
