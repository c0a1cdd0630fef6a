// ref_cpu_harness.cpp — TEST INFRASTRUCTURE ONLY: the reference's own CPU dual contouring
// backend (CpuDualContouringBackend::extract, src/cpp/dc_backend.cpp:51-125, through
// contouring() and Cell / hermite_update, src/cpp/contouring.cpp, Cell.cpp, hermite_update.cpp),
// compiled from its sources where they lie by oracle/Makefile's `ref` target, with the Eigen,
// libigl, Polyscope and GLM headers it includes replaced by the stand-ins of oracle/ref_eigen/
// (Eigen's JacobiSVD restated as a one-sided Jacobi SVD; the viewer and the refinement's mesh
// queries are never reached on this path). The tests use it to pin the FP64 restatement
// oracle/dc_oracle.cpp, and through it the engine, to the reference's own code.
//
//   ref_cpu_dc <grid.sdf> <out.bin>
//
// grid.sdf is the reference CLI's .sdf layout (dc_cli.cpp:31-47). out.bin: int64 vertex count,
// int64 face count, int64 ints per face, the vertices (float32 xyz, as the backend returns
// them), the faces (int32), int64 stats.active_cells.
#include <cstdint>
#include <cstdio>
#include <vector>
#include "dc_backend.h"

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s <grid.sdf> <out.bin>\n", argv[0]);
        return 2;
    }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int n[3];
    float h[6];
    if (std::fread(n, sizeof(int), 3, f) != 3 || std::fread(h, sizeof(float), 6, f) != 6) { std::fclose(f); return 2; }
    DenseSdfGrid grid;
    grid.nx = n[0]; grid.ny = n[1]; grid.nz = n[2];
    grid.vx = h[0]; grid.vy = h[1]; grid.vz = h[2];
    grid.ox = h[3]; grid.oy = h[4]; grid.oz = h[5];
    grid.values.resize((size_t)n[0] * n[1] * n[2]);
    const size_t got = std::fread(grid.values.data(), sizeof(float), grid.values.size(), f);
    std::fclose(f);
    if (got != grid.values.size()) return 2;
    CpuDualContouringBackend backend;
    DualContouringStats stats;
    const DualContouringMesh mesh = backend.extract(grid, stats);
    FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 2;
    const int64_t nv = (int64_t)mesh.vertices.size() / 3, nf = (int64_t)mesh.faces.size() / 4, vpf = 4;
    const int64_t active = stats.active_cells;
    std::fwrite(&nv, 8, 1, o);
    std::fwrite(&nf, 8, 1, o);
    std::fwrite(&vpf, 8, 1, o);
    if (nv) std::fwrite(mesh.vertices.data(), sizeof(float), mesh.vertices.size(), o);
    if (nf) std::fwrite(mesh.faces.data(), sizeof(int), mesh.faces.size(), o);
    std::fwrite(&active, 8, 1, o);
    std::fclose(o);
    return 0;
}
