// dcb_io.cpp — the file formats either side of the extraction in the reference's CLI
// (src/cpp/dc_cli.cpp:17-47): the binary `.sdf` grid (int32 nx, ny, nz; float32 vx, vy, vz,
// ox, oy, oz; then nx*ny*nz float32 values, x fastest) and the OBJ mesh ("v x y z" with the
// C++ stream's default 6 significant digits, "f" with 1-based indices).
//
// The OBJ text is formatted in parallel slices (one buffer per thread, written in order), so
// a 10-million-vertex mesh does not serialise on one formatting loop.
//
// OBJ input follows the CLI's read_obj_to_sdf (dc_cli.cpp:121-203): "v " lines with three
// floats, "f " lines whose tokens (split at blanks and tabs) give 1-based or negative
// (relative) vertex indices by their leading integer ("7/2/5" is vertex 7), polygons fanned
// into triangles from their first vertex; the grid around the mesh is its bounding box grown
// by 8% of the box diagonal on every side, in the reference's float arithmetic.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
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

struct ObjData {
    std::vector<float> V;
    std::vector<int32_t> T;     // triangles
};

// Parses the whole file; false when it cannot be read. Indices are not range-checked here.
bool parse_obj(const char* path, ObjData& D) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    std::string text;
    char chunk[1 << 16];
    size_t got;
    while ((got = std::fread(chunk, 1, sizeof(chunk), f)) > 0) text.append(chunk, got);
    std::fclose(f);
    std::string line;
    std::vector<int32_t> poly;
    size_t at = 0;
    while (at < text.size()) {
        size_t end = text.find('\n', at);
        if (end == std::string::npos) end = text.size();
        line.assign(text, at, end - at);
        at = end + 1;
        if (line.size() < 2 || line[1] != ' ') continue;
        if (line[0] == 'v') {
            // three floats, each after optional white space; the line counts only if all parse
            const char* p = line.c_str() + 2;
            char* e = nullptr;
            float xyz[3];
            int k = 0;
            for (; k < 3; ++k) {
                xyz[k] = std::strtof(p, &e);
                if (e == p) break;
                p = e;
            }
            if (k == 3) D.V.insert(D.V.end(), xyz, xyz + 3);
        } else if (line[0] == 'f') {
            poly.clear();
            const char* p = line.c_str() + 2;
            while (*p) {
                while (*p == ' ' || *p == '\t') ++p;
                if (!*p) break;
                int idx = (int)std::strtol(p, nullptr, 10);
                if (idx != 0) {
                    if (idx < 0) idx = (int)(D.V.size() / 3) + idx + 1;
                    poly.push_back(idx - 1);
                }
                while (*p && *p != ' ' && *p != '\t') ++p;
            }
            for (size_t k = 1; k + 1 < poly.size(); ++k) {
                D.T.push_back(poly[0]);
                D.T.push_back(poly[k]);
                D.T.push_back(poly[k + 1]);
            }
        }
    }
    return true;
}

}  // namespace

extern "C" {

int dcb_read_obj(const char* path, float* vertices, int64_t vertex_capacity, int32_t* triangles,
                 int64_t triangle_capacity, int64_t* num_vertices, int64_t* num_triangles) {
    if (!path || !num_vertices || !num_triangles) return DCB_ERR_INVALID_ARGUMENT;
    ObjData D;
    if (!parse_obj(path, D)) return DCB_ERR_INVALID_ARGUMENT;
    const int64_t nv = (int64_t)D.V.size() / 3, nt = (int64_t)D.T.size() / 3;
    *num_vertices = nv;
    *num_triangles = nt;
    if (nv == 0 || nt == 0) return DCB_ERR_INVALID_ARGUMENT;   // read_obj_to_sdf fails on such files
    for (int32_t v : D.T)
        if (v < 0 || v >= nv) return DCB_ERR_INVALID_ARGUMENT;
    if (!vertices && !triangles) return DCB_OK;                  // counts only
    if (!vertices || !triangles || vertex_capacity < nv || triangle_capacity < nt) return DCB_ERR_TOO_LARGE;
    std::memcpy(vertices, D.V.data(), sizeof(float) * D.V.size());
    std::memcpy(triangles, D.T.data(), sizeof(int32_t) * D.T.size());
    return DCB_OK;
}

int dcb_obj_grid(const float* vertices, int64_t num_vertices, int res, dcb_grid* grid) {
    if (!vertices || num_vertices < 1 || res < 2 || !grid) return DCB_ERR_INVALID_ARGUMENT;
    float lo[3] = {vertices[0], vertices[1], vertices[2]}, hi[3] = {vertices[0], vertices[1], vertices[2]};
    for (int64_t i = 0; i < num_vertices; ++i)
        for (int a = 0; a < 3; ++a) {
            const float x = vertices[3 * i + a];
            if (x < lo[a]) lo[a] = x;
            if (x > hi[a]) hi[a] = x;
        }
    const float diag = std::sqrt((hi[0] - lo[0]) * (hi[0] - lo[0]) + (hi[1] - lo[1]) * (hi[1] - lo[1]) +
                                 (hi[2] - lo[2]) * (hi[2] - lo[2]));
    const float pad = diag > 0.0f ? diag * 0.08f : 0.1f;
    for (int a = 0; a < 3; ++a) { lo[a] -= pad; hi[a] += pad; }
    grid->nx = grid->ny = grid->nz = res;
    grid->ox = lo[0]; grid->oy = lo[1]; grid->oz = lo[2];
    grid->vx = (hi[0] - lo[0]) / (res - 1);
    grid->vy = (hi[1] - lo[1]) / (res - 1);
    grid->vz = (hi[2] - lo[2]) / (res - 1);
    grid->values = nullptr;
    return DCB_OK;
}

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
