// ref_b200_drive.cpp — TEST INFRASTRUCTURE ONLY: compiles include/dc_b200.h's
// B200DualContouringBackend against the reference's own include/dc_backend.h and dc_cuda.h
// (oracle/Makefile `ref` target, output in oracle/_ref/) and drives it the way the reference's
// callers do (dc_cli.cpp:315-332: construct the backend, extract a DenseSdfGrid), so the tests
// can check that the class compiles as a drop-in and that both of its entry points return the
// oracle's mesh.
//
//   ref_b200_drive <grid.sdf> <out.bin> [method]
//
// grid.sdf is the reference CLI's .sdf layout (dc_cli.cpp:31-47). out.bin receives, for
// extract() and then extract_device(): int64 vertex count, int64 face count, int64 ints per
// face, the vertices (float32 xyz), the faces (int32), then DualContouringStats' counts
// (int32: total_cells, active_cells, vertex_count, face_count, qef_fallback_count, clamp_count,
// bad_qef_count) and its times (float32: upload, marking, compaction, active_cell_marking,
// active_cell_compaction, qef, face_emission, face_count, face_prefix_sum, face_fill,
// download, total). Exit status 0 on success, 2 on a usage or file error, 3 when the backend
// throws (its message on stderr).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <cuda_runtime.h>
#include "dc_b200.h"

// DenseSdfGrid's key function lives in the reference's dc_backend.cpp (which needs Eigen and
// libigl for its CPU backend); this program never samples a grid, so a stand-in provides the
// vtable.
float DenseSdfGrid::sample(float, float, float) const { return 0.f; }

static void put(FILE* f, const DualContouringMesh& m, const DualContouringStats& st, int64_t vpf) {
    const int64_t nv = (int64_t)m.vertices.size() / 3, nf = vpf ? (int64_t)m.faces.size() / vpf : 0;
    std::fwrite(&nv, 8, 1, f);
    std::fwrite(&nf, 8, 1, f);
    std::fwrite(&vpf, 8, 1, f);
    if (nv) std::fwrite(m.vertices.data(), sizeof(float), m.vertices.size(), f);
    if (nf) std::fwrite(m.faces.data(), sizeof(int), m.faces.size(), f);
    const int32_t counts[7] = {st.total_cells, st.active_cells, st.vertex_count, st.face_count,
                               st.qef_fallback_count, st.clamp_count, st.bad_qef_count};
    const float times[12] = {st.upload_ms, st.marking_ms, st.compaction_ms, st.active_cell_marking_ms,
                             st.active_cell_compaction_ms, st.qef_ms, st.face_emission_ms, st.face_count_ms,
                             st.face_prefix_sum_ms, st.face_fill_ms, st.download_ms, st.total_ms};
    std::fwrite(counts, sizeof(counts), 1, f);
    std::fwrite(times, sizeof(times), 1, f);
}

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s <grid.sdf> <out.bin> [method]\n", argv[0]);
        return 2;
    }
    const int method = argc > 3 ? std::atoi(argv[3]) : DCB_METHOD_DUAL_CONTOURING;
    dcb_grid hdr{};
    if (dcb_read_sdf(argv[1], &hdr, nullptr, 0) != DCB_OK) { std::fprintf(stderr, "cannot read %s\n", argv[1]); return 2; }
    DenseSdfGrid grid;
    grid.nx = hdr.nx; grid.ny = hdr.ny; grid.nz = hdr.nz;
    grid.vx = hdr.vx; grid.vy = hdr.vy; grid.vz = hdr.vz;
    grid.ox = hdr.ox; grid.oy = hdr.oy; grid.oz = hdr.oz;
    grid.values.resize((size_t)hdr.nx * hdr.ny * hdr.nz);
    if (dcb_read_sdf(argv[1], &hdr, grid.values.data(), (int64_t)grid.values.size()) != DCB_OK) {
        std::fprintf(stderr, "cannot read %s\n", argv[1]);
        return 2;
    }
    FILE* f = std::fopen(argv[2], "wb");
    if (!f) { std::fprintf(stderr, "cannot write %s\n", argv[2]); return 2; }
    try {
        B200DualContouringBackend backend(0, method);
        const int64_t vpf = backend.options().emit_triangles ? 3 : 4;
        // IDualContouringBackend::extract through the interface, as dc_cli calls it
        IDualContouringBackend& be = backend;
        DualContouringStats st;
        const DualContouringMesh m = be.extract(grid, st);
        put(f, m, st, vpf);
        // extract_device on a device copy the caller owns (borrowed, not freed by the backend)
        float* d = nullptr;
        if (cudaMalloc(&d, sizeof(float) * grid.values.size()) != cudaSuccess ||
            cudaMemcpy(d, grid.values.data(), sizeof(float) * grid.values.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            throw std::runtime_error("device copy of the grid failed");
        DenseSdfGridDevice dg{grid.nx, grid.ny, grid.nz, grid.vx, grid.vy, grid.vz, grid.ox, grid.oy, grid.oz, d};
        DualContouringStats st2;
        const DualContouringMesh m2 = backend.extract_device(dg, st2);
        cudaFree(d);
        put(f, m2, st2, vpf);
    } catch (const std::exception& e) {
        std::fclose(f);
        std::fprintf(stderr, "B200DualContouringBackend: %s\n", e.what());
        return 3;
    }
    std::fclose(f);
    return 0;
}
