// ref_cuda_harness.cu — TEST INFRASTRUCTURE ONLY: a C entry point around the reference's own
// CUDA dense backend (CudaDualContouringBackend::extract_device, src/cuda/dc_cuda.cu:652-847,
// compiled from the reference's source by oracle/Makefile's `ref` target into oracle/_ref/,
// as shipped and, for parity checks, without FMA contraction).
// It serves two purposes. (1) A same-GPU speed bar for bench.py's refcuda512 workload.
// (2) A topology pin: the reference's dense kernels mark a cell active on strict signs of its
// corners exactly as the CPU backend does (mark_active_cells_kernel, dc_cuda.cu:241-281 vs
// Cell.cpp:57-77), number vertices by ascending cell index (thrust::copy_if, :701-712) and
// emit a quad for every interior edge with a strict sign change whose four cells are active,
// from the same four cells (count/emit_faces_kernel, :425-605 vs contouring.cpp:607-729), so
// refdc_extract_mesh's vertex count, the cell each vertex is clamped into and the unordered
// set of quads must equal the CPU semantics'. Its vertex positions and quad order and
// winding are not CPU semantics (no normal averaging, clamping into the cell, edge-major
// order) and are not compared.
//
// The reference indexes cells and grid edges with 32-bit ints; this entry point refuses
// grids whose interior-edge count does not fit, where that code would index out of range.
#include <cstdint>
#include <cuda_runtime.h>
#include "dc_cuda.h"

// total_ms: the backend's own host-clock time of the call (allocation, kernels, download);
// stage_ms: the sum of its own CUDA-event stage times (mark, compaction, QEF, faces).
extern "C" int refdc_extract_device(int nx, int ny, int nz, float vx, float vy, float vz, float ox, float oy,
                                    float oz, const float* d_values, double* total_ms, double* stage_ms,
                                    int64_t* vertex_count, int64_t* face_count) {
    if (nx < 3 || ny < 3 || nz < 3 || !d_values) return -1;
    const long long cx = nx - 1, cy = ny - 1, cz = nz - 1;
    const long long edges = cx * (cy - 1) * (cz - 1) + (cx - 1) * cy * (cz - 1) + (cx - 1) * (cy - 1) * cz;
    const long long points = (long long)nx * ny * nz;
    if (edges >= 0x7fffffffLL || points >= 0x7fffffffLL) return -2;
    DenseSdfGridDevice g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.vx = vx; g.vy = vy; g.vz = vz;
    g.ox = ox; g.oy = oy; g.oz = oz;
    g.d_values = d_values;
    CudaDualContouringBackend be;
    DualContouringStats st;
    DualContouringMesh m = be.extract_device(g, st);
    if (total_ms) *total_ms = st.total_ms;
    if (stage_ms) *stage_ms = (double)st.marking_ms + st.compaction_ms + st.qef_ms + st.face_emission_ms;
    if (vertex_count) *vertex_count = (int64_t)(m.vertices.size() / 3);
    if (face_count) *face_count = (int64_t)(m.faces.size() / 4);
    return 0;
}

// The same call returning the mesh: *vertex_count and *face_count are always set; vertices
// (3 floats each) and faces (4 ints each, the backend's own order) are copied to the host
// arrays when they hold vertex_cap / face_cap entries, else -3 is returned.
extern "C" int refdc_extract_mesh(int nx, int ny, int nz, float vx, float vy, float vz, float ox, float oy,
                                  float oz, const float* d_values, float* vertices, int64_t vertex_cap,
                                  int32_t* faces, int64_t face_cap, int64_t* vertex_count, int64_t* face_count) {
    if (nx < 3 || ny < 3 || nz < 3 || !d_values || !vertex_count || !face_count) return -1;
    const long long cx = nx - 1, cy = ny - 1, cz = nz - 1;
    const long long edges = cx * (cy - 1) * (cz - 1) + (cx - 1) * cy * (cz - 1) + (cx - 1) * (cy - 1) * cz;
    const long long points = (long long)nx * ny * nz;
    if (edges >= 0x7fffffffLL || points >= 0x7fffffffLL) return -2;
    DenseSdfGridDevice g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.vx = vx; g.vy = vy; g.vz = vz;
    g.ox = ox; g.oy = oy; g.oz = oz;
    g.d_values = d_values;
    CudaDualContouringBackend be;
    DualContouringStats st;
    DualContouringMesh m = be.extract_device(g, st);
    const int64_t nv = (int64_t)(m.vertices.size() / 3), nf = (int64_t)(m.faces.size() / 4);
    *vertex_count = nv;
    *face_count = nf;
    if (nv > vertex_cap || nf > face_cap || (nv && !vertices) || (nf && !faces)) return -3;
    for (int64_t q = 0; q < 3 * nv; ++q) vertices[q] = m.vertices[(size_t)q];
    for (int64_t q = 0; q < 4 * nf; ++q) faces[q] = m.faces[(size_t)q];
    return 0;
}

// The reference's own mesh -> SDF conversion (compute_mesh_sdf_device_cuda,
// src/cuda/mesh_to_sdf_cuda.cu:740-1009) on host vertices and faces; *ms receives its own
// timer (upload, allocation, conversion). When out_host is given, the values are copied there
// (nx*ny*nz floats). The device grid is freed before returning. Grids whose point count does
// not fit the reference's 32-bit indices are refused.
#include "mesh_to_sdf.h"

// DenseSdfGrid's key function lives in the reference's dc_backend.cpp, which needs Eigen and
// libigl; the conversion above only constructs a DenseSdfGrid in its host variant and never
// samples it, so a stand-in definition provides the vtable.
float DenseSdfGrid::sample(float, float, float) const { return 0.f; }

extern "C" int refsdf_compute(const float* vertices, int num_vertices, const int* faces, int num_faces, int nx,
                              int ny, int nz, float ox, float oy, float oz, float vx, float vy, float vz,
                              float* ms, float* out_host) {
    if (nx < 2 || ny < 2 || nz < 2 || !vertices || !faces) return -1;
    if ((long long)nx * ny * nz >= 0x7fffffffLL) return -2;
    float t = 0.f;
    DenseSdfGridDevice g = compute_mesh_sdf_device_cuda(vertices, num_vertices, faces, num_faces, nx, ny, nz, ox, oy,
                                                        oz, vx, vy, vz, &t, false, 256);
    if (ms) *ms = t;
    if (out_host)
        cudaMemcpy(out_host, g.d_values, sizeof(float) * (size_t)nx * ny * nz, cudaMemcpyDeviceToHost);
    free_mesh_sdf_device_cuda(g);
    return 0;
}

// The same with the reference's voxelize_first / voxel_res arguments (mesh_to_sdf_cuda.cu:764-832).
extern "C" int refsdf_compute_ex(const float* vertices, int num_vertices, const int* faces, int num_faces, int nx,
                                 int ny, int nz, float ox, float oy, float oz, float vx, float vy, float vz,
                                 int voxelize_first, int voxel_res, float* ms, float* out_host) {
    if (nx < 2 || ny < 2 || nz < 2 || !vertices || !faces) return -1;
    if ((long long)nx * ny * nz >= 0x7fffffffLL) return -2;
    float t = 0.f;
    DenseSdfGridDevice g = compute_mesh_sdf_device_cuda(vertices, num_vertices, faces, num_faces, nx, ny, nz, ox, oy,
                                                        oz, vx, vy, vz, &t, voxelize_first != 0, voxel_res);
    if (ms) *ms = t;
    if (out_host)
        cudaMemcpy(out_host, g.d_values, sizeof(float) * (size_t)nx * ny * nz, cudaMemcpyDeviceToHost);
    free_mesh_sdf_device_cuda(g);
    return 0;
}
