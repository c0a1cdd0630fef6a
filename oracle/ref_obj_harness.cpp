// ref_obj_harness.cpp — TEST INFRASTRUCTURE ONLY: runs the reference CLI's own OBJ -> SDF
// ingestion, read_obj_to_sdf (src/cpp/dc_cli.cpp:121-203), on a file and records what it hands
// to the mesh -> SDF conversion: the parsed vertices and triangles and the padded grid. The
// CLI source is compiled into this translation unit where it lies (its function is file-static;
// its main is renamed and never called); compute_mesh_sdf_cuda is replaced by the recorder
// below. Built by oracle/Makefile's `ref` target into oracle/_ref/ref_obj_to_sdf, with
// src/cpp/dc_backend.cpp (headers of ref_stubs/ first, as for ref_post_harness.cpp).
//
//   ref_obj_to_sdf obj2sdf <file.obj> <res> <record.bin>
//     record: int64 nv, int64 nt, float32 vertices[3 nv], int32 triangles[3 nt],
//             int32 nx, ny, nz, float32 ox, oy, oz, vx, vy, vz
// and the CLI's two other file functions (dc_cli.cpp:17-47), for the same kind of pin:
//   ref_obj_to_sdf write_obj <mesh.bin> <out.obj>   mesh: int64 nv, nf, float32 V[3 nv], int32 F[4 nf]
//   ref_obj_to_sdf read_sdf <in.sdf> <record.bin>   record: int32 nx, ny, nz, float32 vx, vy, vz,
//                                                   ox, oy, oz, values
// and its analytic test grids (dc_cli.cpp:49-118), written in the .sdf layout:
//   ref_obj_to_sdf generate <sphere|box|plane> <res> <out.sdf>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#define DC_ENABLE_CUDA 1
#define main reference_cli_main
#include "dc_cli.cpp"
#undef main

// dc_backend.cpp is linked for DenseSdfGrid's virtual sample(); the two functions it calls
// from the contouring library (declared by ref_stubs/) are never reached.
#include "Cell.h"
#include "contouring.h"
void contouring(const Eigen::VectorXd&, const Eigen::MatrixXd&, int, int, int, double, Eigen::MatrixXd&,
                Eigen::MatrixXi&, const ContouringOptions&) {
    std::abort();
}
std::vector<Cell>* getGeneratedCells() { return nullptr; }

static FILE* g_record = nullptr;

DenseSdfGrid compute_mesh_sdf_cuda(const float* vertices, int num_vertices, const int* faces, int num_faces, int nx,
                                   int ny, int nz, float ox, float oy, float oz, float vx, float vy, float vz, float*,
                                   bool, int) {
    const int64_t counts[2] = {num_vertices, num_faces};
    const int32_t dims[3] = {nx, ny, nz};
    const float geo[6] = {ox, oy, oz, vx, vy, vz};
    std::fwrite(counts, sizeof(int64_t), 2, g_record);
    std::fwrite(vertices, sizeof(float), 3 * (size_t)num_vertices, g_record);
    std::fwrite(faces, sizeof(int32_t), 3 * (size_t)num_faces, g_record);
    std::fwrite(dims, sizeof(int32_t), 3, g_record);
    std::fwrite(geo, sizeof(float), 6, g_record);
    DenseSdfGrid g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.ox = ox; g.oy = oy; g.oz = oz;
    g.vx = vx; g.vy = vy; g.vz = vz;
    return g;
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    const std::string mode = argv[1];
    if (mode == "obj2sdf" && argc == 5) {
        g_record = std::fopen(argv[4], "wb");
        if (!g_record) return 2;
        DenseSdfGrid grid;
        const bool ok = read_obj_to_sdf(argv[2], std::atoi(argv[3]), grid);
        std::fclose(g_record);
        return ok ? 0 : 1;
    }
    if (mode == "write_obj" && argc == 4) {
        FILE* f = std::fopen(argv[2], "rb");
        if (!f) return 2;
        int64_t n[2];
        DualContouringMesh mesh;
        bool ok = std::fread(n, sizeof(int64_t), 2, f) == 2;
        if (ok) {
            mesh.vertices.resize(3 * (size_t)n[0]);
            mesh.faces.resize(4 * (size_t)n[1]);
            ok = std::fread(mesh.vertices.data(), sizeof(float), mesh.vertices.size(), f) == mesh.vertices.size() &&
                 std::fread(mesh.faces.data(), sizeof(int32_t), mesh.faces.size(), f) == mesh.faces.size();
        }
        std::fclose(f);
        if (!ok) return 2;
        write_obj(argv[3], mesh);
        return 0;
    }
    if (mode == "read_sdf" && argc == 4) {
        DenseSdfGrid grid;
        if (!read_sdf(argv[2], grid)) return 1;
        FILE* f = std::fopen(argv[3], "wb");
        if (!f) return 2;
        const int32_t dims[3] = {grid.nx, grid.ny, grid.nz};
        const float geo[6] = {grid.vx, grid.vy, grid.vz, grid.ox, grid.oy, grid.oz};
        std::fwrite(dims, sizeof(int32_t), 3, f);
        std::fwrite(geo, sizeof(float), 6, f);
        std::fwrite(grid.values.data(), sizeof(float), grid.values.size(), f);
        std::fclose(f);
        return 0;
    }
    if (mode == "generate" && argc == 5) {
        DenseSdfGrid grid;
        const std::string shape = argv[2];
        const int res = std::atoi(argv[3]);
        if (res < 2) return 2;
        if (shape == "sphere") generate_sphere(grid, res);
        else if (shape == "box") generate_box(grid, res);
        else if (shape == "plane") generate_plane(grid, res);
        else return 2;
        FILE* f = std::fopen(argv[4], "wb");
        if (!f) return 2;
        const int32_t dims[3] = {grid.nx, grid.ny, grid.nz};
        const float geo[6] = {grid.vx, grid.vy, grid.vz, grid.ox, grid.oy, grid.oz};
        std::fwrite(dims, sizeof(int32_t), 3, f);
        std::fwrite(geo, sizeof(float), 6, f);
        std::fwrite(grid.values.data(), sizeof(float), grid.values.size(), f);
        std::fclose(f);
        return 0;
    }
    return 2;
}
