// ref_sparse_harness.cu — TEST INFRASTRUCTURE ONLY: C entry points around the reference's own
// sparse CUDA backends (CudaSparseDualContouringBackend::extract_device and its multi-vertex
// variant, src/cuda/dc_cuda_sparse.cu:1171-1415), compiled from the reference's source by
// oracle/Makefile's `ref` target into oracle/_ref/ twice: with nvcc's default flags (the
// backend as shipped: the same-GPU speed bar) and with --fmad=false (its float expressions
// rounded as written: the bit-exact parity pin of the float restatement and of the engine).
//
// The reference indexes points and cells with 32-bit ints; grids whose point count does not
// fit are refused here. It prints a memory estimate to stdout on every call.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>
#include "dc_cuda.h"

namespace {
struct RefSparseResult {
    std::vector<float> V;
    std::vector<int> F;
    int64_t stats[16];
    double times[4];   // total_ms, marking + compaction, qef, face emission (its own timers)
};
}  // namespace

// Runs the reference's sparse backend (multi_vertex_cells = mvdc) on a device grid. Returns a
// handle for refsparse_copy / refsparse_free, or null when the grid is refused.
extern "C" void* refsparse_run(int nx, int ny, int nz, float vx, float vy, float vz, float ox, float oy, float oz,
                               const float* d_values, int brick_size, int normal_mode, int mvdc) {
    if (nx < 2 || ny < 2 || nz < 2 || !d_values || brick_size < 1) return nullptr;
    if ((long long)nx * ny * nz >= 0x7fffffffLL) return nullptr;
    DenseSdfGridDevice g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.vx = vx; g.vy = vy; g.vz = vz;
    g.ox = ox; g.oy = oy; g.oz = oz;
    g.d_values = d_values;
    CudaSparseDualContouringBackend be(brick_size, (NormalComputationMode)normal_mode, 0, mvdc != 0);
    DualContouringStats st;
    DualContouringMesh m = be.extract_device(g, st);
    RefSparseResult* R = new RefSparseResult();
    R->V = m.vertices;
    R->F = m.faces;
    const int64_t s[16] = {st.total_bricks, st.active_bricks, st.active_cells, st.qef_fallback_count,
                           st.clamp_count, st.invalid_count, st.ambiguous_cells, st.multi_vertex_cells,
                           st.one_vertex_cells, st.two_vertex_cells, st.split_rejection_count,
                           st.faces_skipped_due_to_missing_cluster, st.vertex_count, st.face_count, 0, 0};
    std::memcpy(R->stats, s, sizeof(s));
    R->times[0] = st.total_ms;
    R->times[1] = (double)st.marking_ms + st.compaction_ms;
    R->times[2] = st.qef_ms;
    R->times[3] = st.face_emission_ms;
    return R;
}

extern "C" int64_t refsparse_num_vertices(void* h) { return h ? (int64_t)((RefSparseResult*)h)->V.size() / 3 : 0; }
extern "C" int64_t refsparse_num_faces(void* h) { return h ? (int64_t)((RefSparseResult*)h)->F.size() / 4 : 0; }

// stats: the 12 counters of the float restatement's order, then vertex and face counts.
extern "C" void refsparse_copy(void* h, float* V, int32_t* F, int64_t* stats, double* times) {
    if (!h) return;
    RefSparseResult* R = (RefSparseResult*)h;
    if (V) std::memcpy(V, R->V.data(), R->V.size() * sizeof(float));
    if (F) std::memcpy(F, R->F.data(), R->F.size() * sizeof(int32_t));
    if (stats) std::memcpy(stats, R->stats, sizeof(R->stats));
    if (times) std::memcpy(times, R->times, sizeof(R->times));
}

extern "C" void refsparse_free(void* h) { delete (RefSparseResult*)h; }
