// mts_oracle.cpp — CPU restatement of the reference's mesh -> SDF conversion
// (TEST INFRASTRUCTURE ONLY: used by tests/ and bench.py's CPU legs as the checker and the
// CPU baseline, never by the engine).
//
// It follows compute_mesh_sdf_device_cuda without voxelisation
// (src/cuda/mesh_to_sdf_cuda.cu:740-1009, the `else` branch at :862-951):
//   bins            gx = max(1, nx/8) ..., bin size (n*v)/g, margin 2*max(v); every triangle
//                   goes into each bin its margin-grown bounding box overlaps
//                   (compute_bin_counts_kernel / populate_bins_kernel, :99-224)
//   active bins     a bin with a non-empty bin among its 27 neighbours (:192-224)
//   band values     evaluate_sdf_grid_kernel (:226-360): closest point over the triangles of
//                   the centre bin, then of its 26 neighbours, with the exact point-triangle
//                   case analysis (point_to_triangle_distance_sq, :40-97), ties within 1e-5
//                   relative sum their area-weighted (or angle-weighted near a vertex)
//                   normals, the sign from the summed normal, values beyond 2.5 bins cut
//   sign fill       init_exterior_border / propagate_exterior_signs /
//                   resolve_interior_cavities (:362-428)
//   eikonal         4 Jacobi passes of eikonal_relaxation_kernel (:430-456)
// With voxelize_first (mts_compute_voxelized; the `if` branch at :764-832): a voxel_res^3
// solid — every voxel corner within 0.866 * (largest voxel side) of a triangle is shell
// (rasterize_triangles_to_voxels_kernel, :458-501), the shell dilated by one voxel
// (dilate_voxel_shell_kernel, :503-526), the exterior flooded from the border through the
// other voxels to its fixpoint (:528-575; the reference stops after 3*voxel_res in-place
// passes), the rest solid — gives the points beyond the band -10 inside, +10 outside
// (apply_solid_voxel_sign_mask_kernel, :660-690), with no flood and no relaxation of the grid.
// All arithmetic is float, evaluated as the source writes it (no contraction: compile with
// -ffp-contract=off). Definitions where the reference's GPU execution is not deterministic:
//   * the triangles of a bin are visited in ascending triangle index (the reference fills
//     bins with atomics, so its visiting order, and with it the tie handling, varies);
//   * the exterior flood runs to its fixpoint (the reference stops after 40 in-place passes
//     whose reach per pass depends on thread scheduling);
//   * the vertex angle weight is acos evaluated in double and rounded to float (the
//     reference calls acosf).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {

int nthreads(int threads) { return threads > 0 ? threads : omp_get_max_threads(); }

struct F3 {
    float x, y, z;
};
inline F3 mk(float x, float y, float z) { return F3{x, y, z}; }
inline F3 add(F3 a, F3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline F3 sub(F3 a, F3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline F3 scl(float s, F3 a) { return mk(s * a.x, s * a.y, s * a.z); }
inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 cross(F3 a, F3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }

const float kFar = FLT_MAX;

// Closest point on triangle abc to p and its squared distance (Ericson, Real-Time Collision
// Detection 5.1.5: Voronoi regions of vertices, edges and face; mesh_to_sdf_cuda.cu:40-97).
float point_triangle(F3 p, F3 a, F3 b, F3 c, F3& out) {
    const F3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) { out = a; return dot(ap, ap); }
    const F3 bp = sub(p, b);
    const float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) { out = b; return dot(bp, bp); }
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        const float v = d1 / (d1 - d3);
        out = add(a, scl(v, ab));
        const F3 e = sub(p, out);
        return dot(e, e);
    }
    const F3 cp = sub(p, c);
    const float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) { out = c; return dot(cp, cp); }
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        const float w = d2 / (d2 - d6);
        out = add(a, scl(w, ac));
        const F3 e = sub(p, out);
        return dot(e, e);
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        out = add(b, scl(w, sub(c, b)));
        const F3 e = sub(p, out);
        return dot(e, e);
    }
    const float denom = 1.0f / (va + vb + vc);
    const float v = vb * denom, w = vc * denom;
    out = add(add(a, scl(v, ab)), scl(w, ac));
    const F3 e = sub(p, out);
    return dot(e, e);
}

float angle_at(F3 e1, F3 e2, float fallback) {
    const float l1 = std::sqrt(dot(e1, e1)), l2 = std::sqrt(dot(e2, e2));
    if (l1 > 1e-6f && l2 > 1e-6f) {
        const float c = std::fmax(-1.0f, std::fmin(1.0f, dot(e1, e2) / (l1 * l2)));
        return (float)std::acos((double)c);
    }
    return fallback;
}

struct Mesh {
    const float* V;
    const int* F;
    int64_t nf;
    F3 vtx(int f, int q) const {
        const int i = F[3 * (size_t)f + q];
        return mk(V[3 * (size_t)i], V[3 * (size_t)i + 1], V[3 * (size_t)i + 2]);
    }
};

struct Bins {
    int gx, gy, gz;
    float bdx, bdy, bdz, margin, min_box;
    std::vector<int> offsets;   // num_bins + 1
    std::vector<int> tris;
    std::vector<uint8_t> active;
};

inline int bin_coord(float x, float o, float bd, int g) {
    return std::max(0, std::min(g - 1, (int)std::floor((x - o) / bd)));
}

void build_bins(const Mesh& m, int nx, int ny, int nz, float ox, float oy, float oz, float vx, float vy, float vz,
                Bins& B) {
    B.gx = std::max(1, nx / 8);
    B.gy = std::max(1, ny / 8);
    B.gz = std::max(1, nz / 8);
    B.bdx = ((float)nx * vx) / (float)B.gx;
    B.bdy = ((float)ny * vy) / (float)B.gy;
    B.bdz = ((float)nz * vz) / (float)B.gz;
    B.margin = 2.0f * std::fmax(vx, std::fmax(vy, vz));
    B.min_box = std::fmin(B.bdx, std::fmin(B.bdy, B.bdz));
    const int64_t nb = (int64_t)B.gx * B.gy * B.gz;
    std::vector<int> cnt(nb + 1, 0);
    auto ranges = [&](int f, int* r) {
        const F3 a = m.vtx(f, 0), b = m.vtx(f, 1), c = m.vtx(f, 2);
        const float mnx = std::fmin(a.x, std::fmin(b.x, c.x)) - B.margin;
        const float mny = std::fmin(a.y, std::fmin(b.y, c.y)) - B.margin;
        const float mnz = std::fmin(a.z, std::fmin(b.z, c.z)) - B.margin;
        const float mxx = std::fmax(a.x, std::fmax(b.x, c.x)) + B.margin;
        const float mxy = std::fmax(a.y, std::fmax(b.y, c.y)) + B.margin;
        const float mxz = std::fmax(a.z, std::fmax(b.z, c.z)) + B.margin;
        r[0] = bin_coord(mnx, ox, B.bdx, B.gx); r[1] = bin_coord(mxx, ox, B.bdx, B.gx);
        r[2] = bin_coord(mny, oy, B.bdy, B.gy); r[3] = bin_coord(mxy, oy, B.bdy, B.gy);
        r[4] = bin_coord(mnz, oz, B.bdz, B.gz); r[5] = bin_coord(mxz, oz, B.bdz, B.gz);
    };
    for (int64_t f = 0; f < m.nf; ++f) {
        int r[6];
        ranges((int)f, r);
        for (int bz = r[4]; bz <= r[5]; ++bz)
            for (int by = r[2]; by <= r[3]; ++by)
                for (int bx = r[0]; bx <= r[1]; ++bx) cnt[bx + (int64_t)B.gx * (by + (int64_t)B.gy * bz)]++;
    }
    B.offsets.assign(nb + 1, 0);
    for (int64_t b = 0; b < nb; ++b) B.offsets[b + 1] = B.offsets[b] + cnt[b];
    B.tris.assign(B.offsets[nb], 0);
    std::vector<int> fill(nb, 0);
    for (int64_t f = 0; f < m.nf; ++f) {   // ascending triangle index within every bin
        int r[6];
        ranges((int)f, r);
        for (int bz = r[4]; bz <= r[5]; ++bz)
            for (int by = r[2]; by <= r[3]; ++by)
                for (int bx = r[0]; bx <= r[1]; ++bx) {
                    const int64_t b = bx + (int64_t)B.gx * (by + (int64_t)B.gy * bz);
                    B.tris[B.offsets[b] + fill[b]++] = (int)f;
                }
    }
    B.active.assign(nb, 0);
    for (int bz = 0; bz < B.gz; ++bz)
        for (int by = 0; by < B.gy; ++by)
            for (int bx = 0; bx < B.gx; ++bx) {
                bool act = false;
                for (int dz = -1; dz <= 1 && !act; ++dz)
                    for (int dy = -1; dy <= 1 && !act; ++dy)
                        for (int dx = -1; dx <= 1 && !act; ++dx) {
                            const int x = bx + dx, y = by + dy, z = bz + dz;
                            if (x < 0 || x >= B.gx || y < 0 || y >= B.gy || z < 0 || z >= B.gz) continue;
                            const int64_t n = x + (int64_t)B.gx * (y + (int64_t)B.gy * z);
                            if (B.offsets[n + 1] > B.offsets[n]) act = true;
                        }
                B.active[bx + (int64_t)B.gx * (by + (int64_t)B.gy * bz)] = act ? 1 : 0;
            }
}

// evaluate_sdf_grid_kernel for one grid point (mesh_to_sdf_cuda.cu:226-360).
float band_value(const Mesh& m, const Bins& B, int nx, int ny, float ox, float oy, float oz, float vx, float vy,
                 float vz, int64_t idx) {
    const int ix = (int)(idx % nx), iy = (int)((idx / nx) % ny), iz = (int)(idx / ((int64_t)nx * ny));
    const F3 p = mk(ox + (float)ix * vx, oy + (float)iy * vy, oz + (float)iz * vz);
    const int cbx = bin_coord(p.x, ox, B.bdx, B.gx), cby = bin_coord(p.y, oy, B.bdy, B.gy),
              cbz = bin_coord(p.z, oz, B.bdz, B.gz);
    if (!B.active[cbx + (int64_t)B.gx * (cby + (int64_t)B.gy * cbz)]) return kFar;
    float best = kFar;
    F3 best_p = mk(0.f, 0.f, 0.f), best_n = mk(0.f, 1.f, 0.f);
    const float veps = 1e-6f * B.min_box * B.min_box;
    for (int radius = 0; radius <= 1; ++radius) {
        for (int bz = std::max(0, cbz - radius); bz <= std::min(B.gz - 1, cbz + radius); ++bz)
            for (int by = std::max(0, cby - radius); by <= std::min(B.gy - 1, cby + radius); ++by)
                for (int bx = std::max(0, cbx - radius); bx <= std::min(B.gx - 1, cbx + radius); ++bx) {
                    if (std::abs(bx - cbx) < radius && std::abs(by - cby) < radius && std::abs(bz - cbz) < radius)
                        continue;
                    const int64_t b = bx + (int64_t)B.gx * (by + (int64_t)B.gy * bz);
                    for (int t = B.offsets[b]; t < B.offsets[b + 1]; ++t) {
                        const int f = B.tris[t];
                        const F3 v0 = m.vtx(f, 0), v1 = m.vtx(f, 1), v2 = m.vtx(f, 2);
                        F3 c;
                        const float d = point_triangle(p, v0, v1, v2, c);
                        F3 n = cross(sub(v1, v0), sub(v2, v0));
                        const float a2 = std::sqrt(dot(n, n));
                        if (!(a2 > 1e-12f)) continue;
                        n = mk(n.x / a2, n.y / a2, n.z / a2);
                        float w = a2;
                        const F3 c0 = sub(c, v0), c1 = sub(c, v1), c2 = sub(c, v2);
                        if (dot(c0, c0) < veps) w = angle_at(sub(v1, v0), sub(v2, v0), w);
                        else if (dot(c1, c1) < veps) w = angle_at(sub(v0, v1), sub(v2, v1), w);
                        else if (dot(c2, c2) < veps) w = angle_at(sub(v0, v2), sub(v1, v2), w);
                        const float tol = 1e-5f * (best + 1e-8f);
                        if (d < best - tol) {
                            best = d;
                            best_p = c;
                            best_n = mk(w * n.x, w * n.y, w * n.z);
                        } else if (std::fabs(d - best) <= tol) {
                            best_n = mk(best_n.x + w * n.x, best_n.y + w * n.y, best_n.z + w * n.z);
                        }
                    }
                }
        const float rr = (float)radius * B.min_box;
        if (best < rr * rr && radius > 0) break;
    }
    if (best == kFar) return kFar;
    float dist = std::sqrt(best);
    const float nl = std::sqrt(dot(best_n, best_n));
    if (nl > 1e-12f) best_n = mk(best_n.x / nl, best_n.y / nl, best_n.z / nl);
    if (dot(sub(p, best_p), best_n) < 0.0f) dist = -dist;
    if (dist > 2.5f * B.min_box || dist < -2.5f * B.min_box) return kFar;
    return dist;
}

}  // namespace

extern "C" {

typedef struct {
    int64_t num_bins;
    int64_t bin_entries;
    int64_t band_points;       // finite after the band evaluation
    int64_t exterior_filled;   // far points reached by the exterior flood
} mts_stats;

// Band values only, at the listed linear point indices (evaluate_sdf_grid_kernel).
int mts_band_values(const float* V, int64_t nv, const int* F, int64_t nf, int nx, int ny, int nz, float ox, float oy,
                    float oz, float vx, float vy, float vz, const int64_t* idx, int64_t n, int threads, float* out) {
    (void)nv;
    if (nx < 1 || ny < 1 || nz < 1 || !V || !F || !idx || !out) return -1;
    Mesh m{V, F, nf};
    Bins B;
    build_bins(m, nx, ny, nz, ox, oy, oz, vx, vy, vz, B);
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads(threads))
    for (int64_t q = 0; q < n; ++q) out[q] = band_value(m, B, nx, ny, ox, oy, oz, vx, vy, vz, idx[q]);
    return 0;
}

// The whole conversion into out[nx*ny*nz].
int mts_compute(const float* V, int64_t nv, const int* F, int64_t nf, int nx, int ny, int nz, float ox, float oy,
                float oz, float vx, float vy, float vz, int threads, float* out, mts_stats* st) {
    (void)nv;
    if (nx < 1 || ny < 1 || nz < 1 || !V || !F || !out) return -1;
    Mesh m{V, F, nf};
    Bins B;
    build_bins(m, nx, ny, nz, ox, oy, oz, vx, vy, vz, B);
    const int64_t N = (int64_t)nx * ny * nz;
    const int64_t plane = (int64_t)nx * ny;
#pragma omp parallel for schedule(dynamic, 4096) num_threads(nthreads(threads))
    for (int64_t q = 0; q < N; ++q) out[q] = band_value(m, B, nx, ny, ox, oy, oz, vx, vy, vz, q);
    int64_t band = 0;
    for (int64_t q = 0; q < N; ++q) band += out[q] != kFar;

    // exterior: border points that are far or positive, and positive band points; then
    // flood through far points to the fixpoint.
    std::vector<uint8_t> ext(N, 0);
    std::vector<int64_t> stack;
    for (int64_t q = 0; q < N; ++q) {
        const int ix = (int)(q % nx), iy = (int)((q / nx) % ny), iz = (int)(q / plane);
        const bool border = ix == 0 || ix == nx - 1 || iy == 0 || iy == ny - 1 || iz == 0 || iz == nz - 1;
        if (border) {
            if (out[q] == kFar || out[q] > 0.0f) {
                if (out[q] == kFar) out[q] = 10.0f;
                ext[q] = 1;
            }
        } else if (out[q] != kFar && out[q] > 0.0f) {
            ext[q] = 1;
        }
        if (ext[q]) stack.push_back(q);
    }
    int64_t filled = 0;
    while (!stack.empty()) {
        const int64_t q = stack.back();
        stack.pop_back();
        const int ix = (int)(q % nx), iy = (int)((q / nx) % ny), iz = (int)(q / plane);
        const int64_t nb[6] = {ix > 0 ? q - 1 : -1, ix < nx - 1 ? q + 1 : -1, iy > 0 ? q - nx : -1,
                               iy < ny - 1 ? q + nx : -1, iz > 0 ? q - plane : -1, iz < nz - 1 ? q + plane : -1};
        for (int t = 0; t < 6; ++t) {
            const int64_t r = nb[t];
            if (r < 0 || ext[r] || out[r] != kFar) continue;
            out[r] = 10.0f;
            ext[r] = 1;
            ++filled;
            stack.push_back(r);
        }
    }
    for (int64_t q = 0; q < N; ++q)
        if (out[q] == kFar) out[q] = ext[q] ? 10.0f : -10.0f;

    // 4 Jacobi passes of the eikonal relaxation.
    std::vector<float> tmp(N);
    const float keep = std::fmin(vx, std::fmin(vy, vz)) * 1.5f;
    for (int it = 0; it < 4; ++it) {
        const float* in = (it % 2 == 0) ? out : tmp.data();
        float* dst = (it % 2 == 0) ? tmp.data() : out;
#pragma omp parallel for schedule(static) num_threads(nthreads(threads))
        for (int64_t q = 0; q < N; ++q) {
            const float val = in[q];
            if (std::fabs(val) <= keep) { dst[q] = val; continue; }
            const int ix = (int)(q % nx), iy = (int)((q / nx) % ny), iz = (int)(q / plane);
            float a = std::fabs(val);
            const float s = val < 0.0f ? -1.0f : 1.0f;
            if (ix > 0) a = std::fmin(a, std::fabs(in[q - 1]) + vx);
            if (ix < nx - 1) a = std::fmin(a, std::fabs(in[q + 1]) + vx);
            if (iy > 0) a = std::fmin(a, std::fabs(in[q - nx]) + vy);
            if (iy < ny - 1) a = std::fmin(a, std::fabs(in[q + nx]) + vy);
            if (iz > 0) a = std::fmin(a, std::fabs(in[q - plane]) + vz);
            if (iz < nz - 1) a = std::fmin(a, std::fabs(in[q + plane]) + vz);
            dst[q] = s * a;
        }
    }
    if (st) {
        st->num_bins = (int64_t)B.gx * B.gy * B.gz;
        st->bin_entries = (int64_t)B.tris.size();
        st->band_points = band;
        st->exterior_filled = filled;
    }
    return 0;
}


// The conversion with voxelize_first (see the header); solid (optional, voxel_res^3 bytes,
// clamped resolution) receives the voxel solid.
int mts_compute_voxelized(const float* V, int64_t nv, const int* F, int64_t nf, int nx, int ny, int nz, float ox,
                          float oy, float oz, float vx, float vy, float vz, int voxel_res, int threads, float* out,
                          mts_stats* st, uint8_t* solid) {
    (void)nv;
    if (nx < 1 || ny < 1 || nz < 1 || !V || !F || !out) return -1;
    Mesh m{V, F, nf};
    const int vr = std::max(32, std::min(2048, voxel_res));
    const float vox_x = ((float)nx * vx) / (float)vr, vox_y = ((float)ny * vy) / (float)vr;
    const float vox_z = ((float)nz * vz) / (float)vr;
    const int64_t NV = (int64_t)vr * vr * vr;
    std::vector<uint8_t> shell(NV, 0);
    const float mvd = std::fmax(vox_x, std::fmax(vox_y, vox_z)) * 0.8660254f;
    const float lim = mvd * mvd;
    for (int64_t f = 0; f < nf; ++f) {
        const F3 a = m.vtx((int)f, 0), b = m.vtx((int)f, 1), c = m.vtx((int)f, 2);
        const float mnx = std::fmin(a.x, std::fmin(b.x, c.x)), mny = std::fmin(a.y, std::fmin(b.y, c.y));
        const float mnz = std::fmin(a.z, std::fmin(b.z, c.z)), mxx = std::fmax(a.x, std::fmax(b.x, c.x));
        const float mxy = std::fmax(a.y, std::fmax(b.y, c.y)), mxz = std::fmax(a.z, std::fmax(b.z, c.z));
        const int x0 = bin_coord(mnx, ox, vox_x, vr), x1 = bin_coord(mxx, ox, vox_x, vr);
        const int y0 = bin_coord(mny, oy, vox_y, vr), y1 = bin_coord(mxy, oy, vox_y, vr);
        const int z0 = bin_coord(mnz, oz, vox_z, vr), z1 = bin_coord(mxz, oz, vox_z, vr);
        for (int bz = z0; bz <= z1; ++bz)
            for (int by = y0; by <= y1; ++by)
                for (int bx = x0; bx <= x1; ++bx) {
                    F3 closest;
                    const F3 q = mk(ox + (float)bx * vox_x, oy + (float)by * vox_y, oz + (float)bz * vox_z);
                    if (point_triangle(q, a, b, c, closest) <= lim) shell[bx + (int64_t)vr * (by + (int64_t)vr * bz)] = 1;
                }
    }
    std::vector<uint8_t> dil(NV, 0);
#pragma omp parallel for schedule(static) num_threads(nthreads(threads))
    for (int64_t q = 0; q < NV; ++q) {
        const int ix = (int)(q % vr), iy = (int)((q / vr) % vr), iz = (int)(q / ((int64_t)vr * vr));
        uint8_t d = 0;
        for (int z = std::max(0, iz - 1); z <= std::min(vr - 1, iz + 1) && !d; ++z)
            for (int y = std::max(0, iy - 1); y <= std::min(vr - 1, iy + 1) && !d; ++y)
                for (int x = std::max(0, ix - 1); x <= std::min(vr - 1, ix + 1); ++x)
                    if (shell[x + (int64_t)vr * (y + (int64_t)vr * z)]) { d = 1; break; }
        dil[q] = d;
    }
    std::vector<uint8_t> ext(NV, 0);
    std::vector<int64_t> stack;
    for (int64_t q = 0; q < NV; ++q) {
        const int ix = (int)(q % vr), iy = (int)((q / vr) % vr), iz = (int)(q / ((int64_t)vr * vr));
        const bool border = ix == 0 || ix == vr - 1 || iy == 0 || iy == vr - 1 || iz == 0 || iz == vr - 1;
        if (border && !dil[q]) { ext[q] = 1; stack.push_back(q); }
    }
    const int64_t vplane = (int64_t)vr * vr;
    while (!stack.empty()) {
        const int64_t q = stack.back();
        stack.pop_back();
        const int ix = (int)(q % vr), iy = (int)((q / vr) % vr), iz = (int)(q / vplane);
        const int64_t nb[6] = {ix > 0 ? q - 1 : -1, ix < vr - 1 ? q + 1 : -1, iy > 0 ? q - vr : -1,
                               iy < vr - 1 ? q + vr : -1, iz > 0 ? q - vplane : -1, iz < vr - 1 ? q + vplane : -1};
        for (int t = 0; t < 6; ++t) {
            const int64_t r = nb[t];
            if (r < 0 || ext[r] || dil[r]) continue;
            ext[r] = 1;
            stack.push_back(r);
        }
    }
    if (solid)
        for (int64_t q = 0; q < NV; ++q) solid[q] = ext[q] ? 0 : 1;
    Bins B;
    build_bins(m, nx, ny, nz, ox, oy, oz, vx, vy, vz, B);
    const int64_t N = (int64_t)nx * ny * nz;
    const int64_t plane = (int64_t)nx * ny;
#pragma omp parallel for schedule(dynamic, 4096) num_threads(nthreads(threads))
    for (int64_t q = 0; q < N; ++q) out[q] = band_value(m, B, nx, ny, ox, oy, oz, vx, vy, vz, q);
    int64_t band = 0, outside = 0;
    for (int64_t q = 0; q < N; ++q) {
        if (out[q] != kFar) { ++band; continue; }
        const int ix = (int)(q % nx), iy = (int)((q / nx) % ny), iz = (int)(q / plane);
        const int bx = bin_coord(ox + (float)ix * vx, ox, vox_x, vr);
        const int by = bin_coord(oy + (float)iy * vy, oy, vox_y, vr);
        const int bz = bin_coord(oz + (float)iz * vz, oz, vox_z, vr);
        const bool exterior = ext[bx + (int64_t)vr * (by + (int64_t)vr * bz)] != 0;
        out[q] = exterior ? 10.0f : -10.0f;
        outside += exterior ? 1 : 0;
    }
    if (st) {
        st->num_bins = (int64_t)B.gx * B.gy * B.gz;
        st->bin_entries = (int64_t)B.tris.size();
        st->band_points = band;
        st->exterior_filled = outside;
    }
    return 0;
}

}  // extern "C"
