// dcb_io.cpp — the file formats either side of the extraction in the reference's CLI
// (src/cpp/dc_cli.cpp:17-47): the binary `.sdf` grid (int32 nx, ny, nz; float32 vx, vy, vz,
// ox, oy, oz; then nx*ny*nz float32 values, x fastest) and the OBJ mesh ("v x y z" with the
// C++ stream's default 6 significant digits, "f" with 1-based indices).
//
// The OBJ text is formatted in parallel slices (one buffer per thread, written in order), so
// a 10-million-vertex mesh does not serialise on one formatting loop.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>
#include "../../include/dcb.h"

namespace {

// "%g" with precision 6 is the formatting of `std::ostream << float` with default flags.
void format_range(std::string& out, const float* V, int64_t v0, int64_t v1, const int32_t* F, int64_t f0, int64_t f1,
                  int vpf) {
    char buf[128];
    out.reserve((size_t)((v1 - v0) * 36 + (f1 - f0) * 40));
    for (int64_t i = v0; i < v1; ++i) {
        const int n = std::snprintf(buf, sizeof(buf), "v %g %g %g\n", (double)V[3 * i], (double)V[3 * i + 1],
                                    (double)V[3 * i + 2]);
        out.append(buf, (size_t)n);
    }
    for (int64_t i = f0; i < f1; ++i) {
        int n = 0;
        if (vpf == 4)
            n = std::snprintf(buf, sizeof(buf), "f %d %d %d %d\n", F[4 * i] + 1, F[4 * i + 1] + 1, F[4 * i + 2] + 1,
                              F[4 * i + 3] + 1);
        else
            n = std::snprintf(buf, sizeof(buf), "f %d %d %d\n", F[3 * i] + 1, F[3 * i + 1] + 1, F[3 * i + 2] + 1);
        out.append(buf, (size_t)n);
    }
}

}  // namespace

extern "C" {

int dcb_write_obj(const char* path, const float* vertices, int64_t num_vertices, const int32_t* faces,
                  int64_t num_faces, int verts_per_face, int threads) {
    if (!path || num_vertices < 0 || num_faces < 0 || (num_vertices && !vertices) || (num_faces && !faces) ||
        (verts_per_face != 3 && verts_per_face != 4))
        return DCB_ERR_INVALID_ARGUMENT;
    int nth = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
    if (nth < 1) nth = 1;
    const int64_t work = num_vertices + num_faces;
    if (work < 65536) nth = 1;
    std::vector<std::string> parts((size_t)nth);
    std::vector<std::thread> pool;
    for (int t = 0; t < nth; ++t) {
        // slice t of the concatenated vertex and face lines
        const int64_t a = work * t / nth, b = work * (t + 1) / nth;
        const int64_t v0 = std::min(a, num_vertices), v1 = std::min(b, num_vertices);
        const int64_t f0 = std::max<int64_t>(a - num_vertices, 0), f1 = std::max<int64_t>(b - num_vertices, 0);
        if (nth == 1) format_range(parts[0], vertices, v0, v1, faces, f0, f1, verts_per_face);
        else pool.emplace_back(format_range, std::ref(parts[(size_t)t]), vertices, v0, v1, faces, f0, f1, verts_per_face);
    }
    for (auto& th : pool) th.join();
    FILE* f = std::fopen(path, "wb");
    if (!f) return DCB_ERR_INVALID_ARGUMENT;
    bool ok = true;
    for (const auto& p : parts) ok = ok && std::fwrite(p.data(), 1, p.size(), f) == p.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? DCB_OK : DCB_ERR_INTERNAL;
}

int dcb_read_sdf(const char* path, dcb_grid* header, float* values, int64_t capacity) {
    if (!path || !header) return DCB_ERR_INVALID_ARGUMENT;
    FILE* f = std::fopen(path, "rb");
    if (!f) return DCB_ERR_INVALID_ARGUMENT;
    int32_t dims[3];
    float sp[6];
    int rc = DCB_OK;
    if (std::fread(dims, sizeof(int32_t), 3, f) != 3 || std::fread(sp, sizeof(float), 6, f) != 6) {
        rc = DCB_ERR_INVALID_ARGUMENT;
    } else {
        header->nx = dims[0]; header->ny = dims[1]; header->nz = dims[2];
        header->vx = sp[0]; header->vy = sp[1]; header->vz = sp[2];
        header->ox = sp[3]; header->oy = sp[4]; header->oz = sp[5];
        header->values = nullptr;
        if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1) {
            rc = DCB_ERR_INVALID_ARGUMENT;
        } else if (values) {
            const int64_t n = (int64_t)dims[0] * dims[1] * dims[2];
            if (capacity < n) rc = DCB_ERR_TOO_LARGE;
            else if ((int64_t)std::fread(values, sizeof(float), (size_t)n, f) != n) rc = DCB_ERR_INVALID_ARGUMENT;
            else header->values = values;
        }
    }
    std::fclose(f);
    return rc;
}

int dcb_write_sdf(const char* path, const dcb_grid* grid) {
    if (!path || !grid || !grid->values || grid->nx < 1 || grid->ny < 1 || grid->nz < 1) return DCB_ERR_INVALID_ARGUMENT;
    FILE* f = std::fopen(path, "wb");
    if (!f) return DCB_ERR_INVALID_ARGUMENT;
    const int32_t dims[3] = {grid->nx, grid->ny, grid->nz};
    const float sp[6] = {grid->vx, grid->vy, grid->vz, grid->ox, grid->oy, grid->oz};
    const size_t n = (size_t)grid->nx * grid->ny * grid->nz;
    bool ok = std::fwrite(dims, sizeof(int32_t), 3, f) == 3 && std::fwrite(sp, sizeof(float), 6, f) == 6 &&
              std::fwrite(grid->values, sizeof(float), n, f) == n;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? DCB_OK : DCB_ERR_INTERNAL;
}

}  // extern "C"
