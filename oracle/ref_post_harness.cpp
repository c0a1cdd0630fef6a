// ref_post_harness.cpp — TEST INFRASTRUCTURE ONLY: C entry points around the reference's own
// postprocess_mesh (src/cpp/dc_backend.cpp:127-558), compiled from that file where it lies by
// oracle/Makefile's `ref` target into oracle/_ref/libref_post.so. The file's other function
// (CpuDualContouringBackend::extract) needs Eigen and the contouring library, which are not
// here; the headers under ref_stubs/ declare just enough for it to compile, and the two
// functions it calls are defined below as stubs that are never reached.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "dc_backend.h"
#include "contouring.h"
#include "Cell.h"

void contouring(const Eigen::VectorXd&, const Eigen::MatrixXd&, int, int, int, double, Eigen::MatrixXd&,
                Eigen::MatrixXi&, const ContouringOptions&) {
    std::abort();
}
std::vector<Cell>* getGeneratedCells() { return nullptr; }

// Quads in (nf x 4 indices), as the reference's DualContouringMesh holds them.
extern "C" void* refpost_run(const float* V, int64_t nv, const int32_t* F, int64_t nf, int close_holes,
                             int remove_floaters) {
    DualContouringMesh m;
    m.vertices.assign(V, V + 3 * nv);
    m.faces.assign(F, F + 4 * nf);
    return new DualContouringMesh(postprocess_mesh(m, close_holes != 0, remove_floaters != 0));
}
extern "C" int64_t refpost_num_vertices(void* h) {
    return h ? (int64_t)((DualContouringMesh*)h)->vertices.size() / 3 : 0;
}
extern "C" int64_t refpost_num_faces(void* h) { return h ? (int64_t)((DualContouringMesh*)h)->faces.size() / 4 : 0; }
extern "C" void refpost_copy(void* h, float* V, int32_t* F) {
    if (!h) return;
    DualContouringMesh* m = (DualContouringMesh*)h;
    if (V) std::memcpy(V, m->vertices.data(), m->vertices.size() * sizeof(float));
    if (F) std::memcpy(F, m->faces.data(), m->faces.size() * sizeof(int32_t));
}
extern "C" void refpost_free(void* h) { delete (DualContouringMesh*)h; }
