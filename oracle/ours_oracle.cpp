/*
 * ours_oracle.cpp — TEST INFRASTRUCTURE ONLY (the oracle; never shipped, never measured as
 * the product). Only tests/ may load it.
 *
 * FP64 C++ restatement of the reference's outer/inner vertex refinement, ContouringMethod::Ours
 * (src/cpp/contouring.cpp:1255-1328), run after the restated dual contouring of dc_oracle.cpp
 * (included below):
 *   start                     second average_hermite_normals after Cell::update
 *                             (contouring.cpp:1233-1241), vertex = Hermite centroid (:1258-1263)
 *   triangulate_v1            contouring.cpp:88-113
 *   assign_spheres_to_cells   contouring.cpp:807-933, cell_diagonal :788-804
 *   face intersections        compute_face_cell_intersections contouring.cpp:1081-1183
 *   Hermite update            update_hermite_points_and_normals hermite_update.cpp:441-607
 *                             (edges of process_edge :171-332)
 *   inner loop                contouring.cpp:1288-1309: refine_vertex_from_face_intersections
 *                             vertex_refinement.cpp:201-280 (closest points :110-198,
 *                             barycentric :36-66), Cell::minimize_qef Cell.cpp:364-473,
 *                             solve_quadratic_system :324-361
 *   re-extraction             extract_mesh_from_cells contouring.cpp:486-741
 * Three things the reference leaves to chance are fixed here (and in the engine) the same way:
 *   - the random fill of the sphere batch (std::random_device + std::shuffle,
 *     contouring.cpp:845-850) takes the candidates with the smallest seeded 64-bit keys;
 *   - spheres of equal radius (std::sort, :925-931) are ordered by grid index;
 *   - closest points on the mesh (libigl AABB, :869) take, among equally close triangles, the
 *     one of smallest index (brute force here, a BVH in the engine), and on a cell's local
 *     fan (vertex_refinement.cpp:132-141) the first in fan order.
 * libigl's point-triangle distance is restated by Ericson's closest-point case analysis
 * (Real-Time Collision Detection §5.1.5), the SVDs by the cyclic Jacobi eigen-decomposition.
 */
#include "dc_oracle.cpp"

#include <algorithm>
#include <cfloat>

namespace {

struct OursOpts {
    int outer_iters, inner_iters;
    double mu, dc_weight, sphere_weight, svd_threshold;
    int hermite_update, batch_size;
    double wpos, wface, wnormal;
    uint64_t seed;
};

const int kFaceCorners[6][4] = {{1, 5, 6, 2}, {0, 3, 7, 4}, {2, 6, 7, 3}, {0, 4, 5, 1}, {4, 7, 6, 5}, {0, 1, 2, 3}};

int edge_of_corners(int c1, int c2) {
    for (int e = 0; e < 12; ++e) {
        int a = kEdge[e][0], b = kEdge[e][1];
        if ((c1 == a && c2 == b) || (c1 == b && c2 == a)) return e;
    }
    return -1;
}

inline double norm3(const double* a) { return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

uint64_t mix64(uint64_t x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

void seg_closest(const double* p, const double* a, const double* b, double* out) {
    double ab[3], ap[3];
    for (int d = 0; d < 3; ++d) { ab[d] = b[d] - a[d]; ap[d] = p[d] - a[d]; }
    double l2 = dot3(ab, ab);
    double t = l2 > 0.0 ? dot3(ap, ab) / l2 : 0.0;
    t = std::min(1.0, std::max(0.0, t));
    for (int d = 0; d < 3; ++d) out[d] = a[d] + t * ab[d];
}

void tri_closest(const double* p, const double* a, const double* b, const double* c, double* out) {
    double ab[3], ac[3], ap[3], bp[3], cp[3];
    for (int d = 0; d < 3; ++d) { ab[d] = b[d] - a[d]; ac[d] = c[d] - a[d]; ap[d] = p[d] - a[d]; }
    double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) { for (int d = 0; d < 3; ++d) out[d] = a[d]; return; }
    for (int d = 0; d < 3; ++d) bp[d] = p[d] - b[d];
    double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) { for (int d = 0; d < 3; ++d) out[d] = b[d]; return; }
    double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        double v = d1 / (d1 - d3);
        for (int d = 0; d < 3; ++d) out[d] = a[d] + v * ab[d];
        return;
    }
    for (int d = 0; d < 3; ++d) cp[d] = p[d] - c[d];
    double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) { for (int d = 0; d < 3; ++d) out[d] = c[d]; return; }
    double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        double w = d2 / (d2 - d6);
        for (int d = 0; d < 3; ++d) out[d] = a[d] + w * ac[d];
        return;
    }
    double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        for (int d = 0; d < 3; ++d) out[d] = b[d] + w * (c[d] - b[d]);
        return;
    }
    double sum = va + vb + vc;
    if (sum != 0.0 && std::isfinite(sum)) {
        double denom = 1.0 / sum;
        double v = vb * denom, w = vc * denom;
        for (int d = 0; d < 3; ++d) out[d] = a[d] + ab[d] * v + ac[d] * w;
        if (std::isfinite(out[0]) && std::isfinite(out[1]) && std::isfinite(out[2])) return;
    }
    double q[3], best = DBL_MAX;
    const double* E[3][2] = {{a, b}, {b, c}, {c, a}};
    for (int s = 0; s < 3; ++s) {
        seg_closest(p, E[s][0], E[s][1], q);
        double dd[3] = {q[0] - p[0], q[1] - p[1], q[2] - p[2]};
        double d2q = dot3(dd, dd);
        if (d2q < best) { best = d2q; out[0] = q[0]; out[1] = q[1]; out[2] = q[2]; }
    }
}

void barycentric(const double* P, const double* V0, const double* V1, const double* V2, double out[3]) {
    double e1[3], e2[3], ep[3];
    for (int d = 0; d < 3; ++d) { e1[d] = V1[d] - V0[d]; e2[d] = V2[d] - V0[d]; ep[d] = P[d] - V0[d]; }
    double d11 = dot3(e1, e1), d12 = dot3(e1, e2), d22 = dot3(e2, e2);
    double dP1 = dot3(ep, e1), dP2 = dot3(ep, e2);
    double denom = d11 * d22 - d12 * d12;
    if (std::abs(denom) < 1e-12) { out[0] = 1.0; out[1] = 0.0; out[2] = 0.0; return; }
    double beta = (d22 * dP1 - d12 * dP2) / denom;
    double gamma = (d11 * dP2 - d12 * dP1) / denom;
    out[0] = 1.0 - beta - gamma; out[1] = beta; out[2] = gamma;
}

struct OCell {
    double v[3];
    double fi[6][3];
    int fmask = 0;
    std::vector<int64_t> spheres;
};

// The grid edges process_edge accepts (hermite_update.cpp:171-332) with their four cells in
// its order (owner, +dir1, +dir2, both) and each cell's local edge index.
struct EdgeQuad { int64_t r[4]; int e[4]; };

std::vector<EdgeQuad> averaged_edges(const Grid& g, const std::vector<int64_t>& cells, const std::vector<int32_t>& vid,
                                     const std::vector<Hermite>& H) {
    std::vector<EdgeQuad> out;
    const int nx = g.nx, ny = g.ny, nz = g.nz, cx = nx - 1, cy = ny - 1;
    auto inside = [&](int a, int b, int c) { return a > 0 && a < nx - 1 && b > 0 && b < ny - 1 && c > 0 && c < nz - 1; };
    for (size_t r = 0; r < cells.size(); ++r) {
        int64_t c = cells[r];
        int i = (int)(c % cx), j = (int)((c / cx) % cy), k = (int)(c / ((int64_t)cx * cy));
        const int ends[3][3] = {{i + 1, j, k}, {i, j + 1, k}, {i, j, k + 1}};
        for (int ax = 0; ax < 3; ++ax) {
            int i1 = ends[ax][0], j1 = ends[ax][1], k1 = ends[ax][2];
            if (i1 > nx - 1 || j1 > ny - 1 || k1 > nz - 1) continue;
            if (!inside(i, j, k) && !inside(i1, j1, k1)) continue;
            int e0 = edge_idx_from_points(i, j, k, i, j, k, i1, j1, k1);
            if (!(H[r].mask & (1u << e0))) continue;
            const int* d1 = kDirs[kEdgeFaces[e0][0]];
            const int* d2 = kDirs[kEdgeFaces[e0][1]];
            int nb[3][3] = {{i + d1[0], j + d1[1], k + d1[2]},
                            {i + d2[0], j + d2[1], k + d2[2]},
                            {i + d1[0] + d2[0], j + d1[1] + d2[1], k + d1[2] + d2[2]}};
            EdgeQuad q;
            q.r[0] = (int64_t)r; q.e[0] = e0;
            bool ok = true;
            for (int t = 0; t < 3 && ok; ++t) {
                int64_t cc = g.cidx(nb[t][0], nb[t][1], nb[t][2]);
                if (vid[cc] < 0) { ok = false; break; }
                q.r[t + 1] = vid[cc];
                q.e[t + 1] = edge_idx_from_points(nb[t][0], nb[t][1], nb[t][2], i, j, k, i1, j1, k1);
            }
            if (ok) out.push_back(q);
        }
    }
    return out;
}

}  // namespace

extern "C" {

typedef struct {
    int outer_iters, inner_iters;
    double mu, dc_weight, sphere_weight, svd_threshold;
    int hermite_update, batch_size;
    double new_hermite_pos_weight, new_face_pos_weight, new_hermite_normal_weight;
    uint64_t seed;
} dco_ours_opts;

/*
 * The refinement on a dense float grid (origin + i * spacing positions). Returns a handle for
 * dco_num_vertices / dco_num_faces / dco_copy / dco_free (V: refined FP64 vertices, F: quads
 * wound with them, cells: the active cells) or NULL on invalid input.
 */
void* dco_ours(int nx, int ny, int nz, float vx, float vy, float vz, float ox, float oy, float oz,
               const float* values, const dco_ours_opts* o, int threads, dco_stats* st) {
    if (!o || nx < 2 || ny < 2 || nz < 2 || !values) return nullptr;
#ifdef _OPENMP
    const int nth = threads > 0 ? threads : omp_get_max_threads();
#else
    const int nth = 1; (void)threads;
#endif
    std::vector<Hermite> H;
    // Cell::update's solve uses 0.01 whatever the options say (Cell.cpp:314)
    Result* R = (Result*)extract_impl(nx, ny, nz, vx, vy, vz, ox, oy, oz, nullptr, nullptr, nullptr, values, 0.01,
                                      threads, st, &H);
    if (!R) return nullptr;
    Grid g;
    g.nx = nx; g.ny = ny; g.nz = nz; g.vx = vx; g.vy = vy; g.vz = vz; g.ox = ox; g.oy = oy; g.oz = oz;
    g.v = values;
    g.gx.resize(nx); g.gy.resize(ny); g.gz.resize(nz);
    for (int i = 0; i < nx; ++i) { float f = (float)i; float pr = f * vx; float s = ox + pr; g.gx[i] = (double)s; }
    for (int j = 0; j < ny; ++j) { float f = (float)j; float pr = f * vy; float s = oy + pr; g.gy[j] = (double)s; }
    for (int k = 0; k < nz; ++k) { float f = (float)k; float pr = f * vz; float s = oz + pr; g.gz[k] = (double)s; }
    const int cx = nx - 1, cy = ny - 1, cz = nz - 1;
    const int64_t ncell = (int64_t)cx * cy * cz, npts = (int64_t)nx * ny * nz;
    const int64_t nv = (int64_t)R->cells.size();
    std::vector<int32_t> vid(ncell, -1);
    for (int64_t r = 0; r < nv; ++r) vid[R->cells[r]] = (int32_t)r;

    // second average_hermite_normals (contouring.cpp:1241)
    const std::vector<EdgeQuad> edges = averaged_edges(g, R->cells, vid, H);
    for (const EdgeQuad& q : edges) {
        double acc[3] = {0, 0, 0};
        for (int t = 0; t < 4; ++t) {
            const double* hn = H[q.r[t]].n[q.e[t]];
            if (std::sqrt(sqnorm3(hn)) > 0) { acc[0] += hn[0]; acc[1] += hn[1]; acc[2] += hn[2]; }
        }
        normalize3(acc);
        for (int t = 0; t < 4; ++t) std::memcpy(H[q.r[t]].n[q.e[t]], acc, sizeof acc);
    }
    // vertex = centroid of the Hermite points (contouring.cpp:1258-1263)
    std::vector<OCell> C(nv);
    for (int64_t r = 0; r < nv; ++r) {
        double c[3] = {0, 0, 0};
        int m = 0;
        for (int e = 0; e < 12; ++e) {
            if (!(H[r].mask & (1u << e))) continue;
            for (int d = 0; d < 3; ++d) c[d] += H[r].p[e][d];
            ++m;
        }
        for (int d = 0; d < 3; ++d) C[r].v[d] = m ? c[d] / double(m) : 0.0;
    }
    // cell_diagonal (contouring.cpp:788-804)
    const double gmin[3] = {std::min(g.gx[0], g.gx[nx - 1]), std::min(g.gy[0], g.gy[ny - 1]), std::min(g.gz[0], g.gz[nz - 1])};
    const double gmax[3] = {std::max(g.gx[0], g.gx[nx - 1]), std::max(g.gy[0], g.gy[ny - 1]), std::max(g.gz[0], g.gz[nz - 1])};
    const double gd[3] = {(gmax[0] - gmin[0]) / (double)(nx - 1), (gmax[1] - gmin[1]) / (double)(ny - 1),
                          (gmax[2] - gmin[2]) / (double)(nz - 1)};
    const double cell_diag = std::min({gd[0], gd[1], gd[2]}) * std::sqrt(3.0);
    // sphere batch: every point with |S| < 3 * cell diagonal, filled up to batch_size
    std::vector<int64_t> band, rest;
    for (int64_t p = 0; p < npts; ++p) {
        if (std::abs((double)values[p]) < 3.0 * cell_diag) band.push_back(p);
        else rest.push_back(p);
    }
    const int64_t bounded = std::min<int64_t>(o->batch_size, npts);
    const int64_t nfill = (int64_t)band.size() < bounded ? std::min<int64_t>(bounded - (int64_t)band.size(), (int64_t)rest.size()) : 0;

    std::vector<double> Vm = R->V;          // the extraction's mesh for the first iteration
    std::vector<int32_t> F = R->F;
    auto point = [&](int64_t p, double* c) {
        int i = (int)(p % nx), j = (int)((p / nx) % ny), k = (int)(p / ((int64_t)nx * ny));
        c[0] = g.gx[i]; c[1] = g.gy[j]; c[2] = g.gz[k];
    };
    const int dirs[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

    for (int it = 0; it < o->outer_iters; ++it) {
        // triangulate_v1 with orient_triangles_for_quad (contouring.cpp:40-113)
        const int64_t nq = (int64_t)F.size() / 4;
        std::vector<double> T(9 * 2 * nq);
        for (int64_t q = 0; q < nq; ++q) {
            const int32_t* f = &F[4 * q];
            int32_t id[2][3] = {{f[0], f[1], f[2]}, {f[0], f[2], f[3]}};
            const double* pa = &Vm[3 * (int64_t)f[0]];
            const double* pb = &Vm[3 * (int64_t)f[1]];
            const double* pc = &Vm[3 * (int64_t)f[2]];
            const double* pd = &Vm[3 * (int64_t)f[3]];
            double u[3], w[3], qn[3];
            for (int d = 0; d < 3; ++d) { u[d] = pb[d] - pa[d]; w[d] = pd[d] - pa[d]; }
            cross3(u, w, qn);
            if (sqnorm3(qn) < 1e-24) { for (int d = 0; d < 3; ++d) u[d] = pc[d] - pa[d]; cross3(u, w, qn); }
            if (!(sqnorm3(qn) < 1e-24)) {
                for (int h = 0; h < 2; ++h) {
                    const double* p1 = &Vm[3 * (int64_t)id[h][0]];
                    const double* p2 = &Vm[3 * (int64_t)id[h][1]];
                    const double* p3 = &Vm[3 * (int64_t)id[h][2]];
                    double x[3], y[3], tn[3];
                    for (int d = 0; d < 3; ++d) { x[d] = p2[d] - p1[d]; y[d] = p3[d] - p1[d]; }
                    cross3(x, y, tn);
                    if (dot3(tn, qn) < 0.0) std::swap(id[h][1], id[h][2]);
                }
            }
            for (int h = 0; h < 2; ++h)
                for (int v = 0; v < 3; ++v)
                    for (int d = 0; d < 3; ++d) T[9 * (2 * q + h) + 3 * v + d] = Vm[3 * (int64_t)id[h][v] + d];
        }
        std::vector<int64_t> sel = band;
        if (nfill > 0) {
            std::vector<std::pair<uint64_t, int64_t>> keyed(rest.size());
            for (size_t t = 0; t < rest.size(); ++t)
                keyed[t] = {mix64(o->seed ^ mix64(((uint64_t)it << 40) ^ (uint64_t)rest[t])), rest[t]};
            std::sort(keyed.begin(), keyed.end());
            for (int64_t t = 0; t < nfill; ++t) sel.push_back(keyed[t].second);
        }
        // closest points on the mesh, spheres into the cells holding them
        std::vector<int32_t> target(sel.size(), -1);
#pragma omp parallel for num_threads(nth) schedule(dynamic, 64)
        for (int64_t s = 0; s < (int64_t)sel.size(); ++s) {
            double c[3], best = DBL_MAX, bc[3] = {0, 0, 0};
            point(sel[s], c);
            for (int64_t t = 0; t < 2 * nq; ++t) {
                double q[3];
                tri_closest(c, &T[9 * t], &T[9 * t + 3], &T[9 * t + 6], q);
                double dd[3] = {q[0] - c[0], q[1] - c[1], q[2] - c[2]};
                double d2 = dot3(dd, dd);
                if (d2 < best) { best = d2; bc[0] = q[0]; bc[1] = q[1]; bc[2] = q[2]; }
            }
            const double radius = std::abs((double)values[sel[s]]);
            if (!(best < DBL_MAX) || std::sqrt(best) - radius >= cell_diag) continue;
            int ci[3];
            const int cmax[3] = {nx - 2, ny - 2, nz - 2};
            for (int d = 0; d < 3; ++d) {
                double f = std::floor((bc[d] - gmin[d]) / gd[d]);
                int v = f < -1e9 ? -1000000000 : (f > 1e9 ? 1000000000 : (int)f);
                ci[d] = std::max(0, std::min(v, cmax[d]));
            }
            target[s] = vid[g.cidx(ci[0], ci[1], ci[2])];
        }
        for (auto& c : C) c.spheres.clear();
        for (size_t s = 0; s < sel.size(); ++s)
            if (target[s] >= 0) C[target[s]].spheres.push_back(sel[s]);
        for (auto& c : C)
            std::sort(c.spheres.begin(), c.spheres.end(), [&](int64_t a, int64_t b) {
                float ra = std::fabs(values[a]), rb = std::fabs(values[b]);
                return ra < rb || (ra == rb && a < b);
            });
        // face intersections (reads the neighbours' vertices of this iteration)
        for (int64_t r = 0; r < nv; ++r) {
            int64_t cid = R->cells[r];
            int i = (int)(cid % cx), j = (int)((cid / cx) % cy), k = (int)(cid / ((int64_t)cx * cy));
            OCell& S = C[r];
            const double mn[3] = {g.gx[i], g.gy[j], g.gz[k]};
            const double mx[3] = {g.gx[i + 1], g.gy[j + 1], g.gz[k + 1]};
            for (int d = 0; d < 6; ++d) {
                int ni = i + dirs[d][0], nj = j + dirs[d][1], nk = k + dirs[d][2];
                if (ni < 0 || ni >= cx || nj < 0 || nj >= cy || nk < 0 || nk >= cz) continue;
                int32_t nr = vid[g.cidx(ni, nj, nk)];
                if (nr < 0) continue;
                double seg[3];
                for (int a = 0; a < 3; ++a) seg[a] = C[nr].v[a] - S.v[a];
                int ax = d >> 1;
                double plane = (d & 1) ? mn[ax] : mx[ax];
                double num = plane - S.v[ax], den = seg[ax];
                if (std::abs(den) < 1e-9) continue;
                double t = num / den;
                if (t >= -1e-6 && t <= 1.0 + 1e-6) {
                    double x[3];
                    for (int a = 0; a < 3; ++a) x[a] = S.v[a] + t * seg[a];
                    if (!(S.fmask & (1 << d))) {
                        std::memcpy(S.fi[d], x, sizeof x);
                        S.fmask |= 1 << d;
                    } else {
                        for (int a = 0; a < 3; ++a) S.fi[d][a] = x[a] * o->new_face_pos_weight + S.fi[d][a] * (1.0 - o->new_face_pos_weight);
                    }
                }
            }
        }
        // Hermite update from the second outer iteration on
        if (o->hermite_update && it > 0) {
            for (const EdgeQuad& q : edges) {
                double V4[4][3], cen[3] = {0, 0, 0};
                for (int t = 0; t < 4; ++t)
                    for (int d = 0; d < 3; ++d) { V4[t][d] = C[q.r[t]].v[d]; cen[d] += V4[t][d]; }
                for (int d = 0; d < 3; ++d) cen[d] /= 4.0;
                double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, U[3][3];
                for (int t = 0; t < 4; ++t) {
                    double x[3];
                    for (int d = 0; d < 3; ++d) x[d] = V4[t][d] - cen[d];
                    for (int a = 0; a < 3; ++a)
                        for (int b = 0; b < 3; ++b) M[a][b] += x[a] * x[b];
                }
                jacobi_eig3(M, U);
                int qmin = 0;
                for (int t = 1; t < 3; ++t) if (M[t][t] <= M[qmin][qmin]) qmin = t;
                double nrm[3] = {U[0][qmin], U[1][qmin], U[2][qmin]};
                normalize3(nrm);
                const int64_t cid = R->cells[q.r[0]];
                const int i = (int)(cid % cx), j = (int)((cid / cx) % cy), k = (int)(cid / ((int64_t)cx * cy));
                const int ca = kEdge[q.e[0]][0], cb = kEdge[q.e[0]][1];
                const double pA[3] = {g.gx[i + kOff[ca][0]], g.gy[j + kOff[ca][1]], g.gz[k + kOff[ca][2]]};
                const double pB[3] = {g.gx[i + kOff[cb][0]], g.gy[j + kOff[cb][1]], g.gz[k + kOff[cb][2]]};
                const double sA = g.S(i + kOff[ca][0], j + kOff[ca][1], k + kOff[ca][2]);
                double dir[3];
                for (int d = 0; d < 3; ++d) dir[d] = pB[d] - pA[d];
                const double len = norm3(dir);
                if (len > 0.0) for (int d = 0; d < 3; ++d) dir[d] /= len;
                double out[3];
                for (int d = 0; d < 3; ++d) out[d] = dir[d] * (sA < 0 ? -1.0 : 1.0);
                if (dot3(nrm, out) > 0) for (int d = 0; d < 3; ++d) nrm[d] = -nrm[d];
                if (norm3(nrm) > 0) {
                    for (int t = 0; t < 4; ++t) {
                        double* hn = H[q.r[t]].n[q.e[t]];
                        double u[3];
                        for (int d = 0; d < 3; ++d) u[d] = (1.0 - o->new_hermite_normal_weight) * hn[d] + o->new_hermite_normal_weight * nrm[d];
                        normalize3(u);
                        std::memcpy(hn, u, sizeof u);
                    }
                }
                const double denom = dot3(nrm, dir);
                if (std::abs(denom) > 1e-6) {
                    double w[3];
                    for (int d = 0; d < 3; ++d) w[d] = cen[d] - pA[d];
                    double tt = dot3(nrm, w) / denom;
                    if (tt < 0 || tt > len) continue;
                    tt = std::max(0.0, std::min(tt, len));
                    double x[3];
                    for (int d = 0; d < 3; ++d) x[d] = pA[d] + tt * dir[d];
                    for (int t = 0; t < 4; ++t) {
                        double* hp = H[q.r[t]].p[q.e[t]];
                        for (int d = 0; d < 3; ++d) hp[d] = (1.0 - o->new_hermite_pos_weight) * hp[d] + o->new_hermite_pos_weight * x[d];
                    }
                }
            }
        }
        // inner loops
        const double ssw = std::sqrt(o->sphere_weight), smu = std::sqrt(o->mu);
#pragma omp parallel for num_threads(nth) schedule(dynamic, 64)
        for (int64_t r = 0; r < nv; ++r) {
            OCell& S = C[r];
            const Hermite& h = H[r];
            if (!S.fmask || S.spheres.empty() || !h.mask) continue;
            std::vector<std::pair<int, int>> fan;          // (edge, face)
            for (int d = 0; d < 6; ++d) {
                if (!(S.fmask & (1 << d))) continue;
                for (int u = 0; u < 4; ++u) {
                    int e = edge_of_corners(kFaceCorners[d][u], kFaceCorners[d][(u + 1) & 3]);
                    if (e >= 0 && (h.mask & (1u << e))) fan.push_back({e, d});
                }
            }
            if (fan.empty()) continue;
            double H0[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, h0[3] = {0, 0, 0}, cen[3] = {0, 0, 0};
            int m = 0;
            for (int e = 0; e < 12; ++e) {
                if (!(h.mask & (1u << e))) continue;
                double sn[3];
                for (int d = 0; d < 3; ++d) sn[d] = o->dc_weight * h.n[e][d];
                double b = dot3(sn, h.p[e]);
                for (int a = 0; a < 3; ++a) {
                    for (int c = 0; c < 3; ++c) H0[a][c] += sn[a] * sn[c];
                    h0[a] += sn[a] * b;
                }
                for (int d = 0; d < 3; ++d) cen[d] += h.p[e][d];
                ++m;
            }
            for (int d = 0; d < 3; ++d) cen[d] /= double(m);
            double v[3] = {S.v[0], S.v[1], S.v[2]};
            const size_t nsph = S.spheres.size(), cs = (nsph + 31) / 32;
            for (int iter = 0; iter < o->inner_iters; ++iter) {
                const double prev[3] = {v[0], v[1], v[2]};
                double A[3][3], b[3];
                for (int a = 0; a < 3; ++a) { b[a] = h0[a]; for (int c = 0; c < 3; ++c) A[a][c] = H0[a][c]; }
                // sphere rows summed in 32 chunks of consecutive spheres, each from zero,
                // added in chunk order (the engine's order, for a thread or a warp per cell)
                for (size_t l = 0; l < 32; ++l) {
                    const size_t lo = l * cs, hi = std::min(nsph, lo + cs);
                    if (lo >= hi) break;
                    double PA[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, Pb[3] = {0, 0, 0};
                    for (size_t si = lo; si < hi; ++si) {
                    const int64_t gidx = S.spheres[si];
                    double c[3];
                    point(gidx, c);
                    const double sval = (double)values[gidx];
                    const double rs = std::abs(sval);
                    double best = DBL_MAX, tm[3] = {0, 0, 0};
                    size_t bf = 0;
                    for (size_t f = 0; f < fan.size(); ++f) {
                        double q[3];
                        tri_closest(c, prev, h.p[fan[f].first], S.fi[fan[f].second], q);
                        double dd[3] = {q[0] - c[0], q[1] - c[1], q[2] - c[2]};
                        double d2 = dot3(dd, dd);
                        if (d2 < best) { best = d2; bf = f; tm[0] = q[0]; tm[1] = q[1]; tm[2] = q[2]; }
                    }
                    const double* Hp = h.p[fan[bf].first];
                    const double* Fp = S.fi[fan[bf].second];
                    double ct[3];
                    for (int a = 0; a < 3; ++a) ct[a] = tm[a] - c[a];
                    const double rho0 = norm3(ct);
                    double qs[3];
                    if (rho0 < 1e-9) for (int a = 0; a < 3; ++a) qs[a] = c[a];
                    else for (int a = 0; a < 3; ++a) qs[a] = c[a] + (ct[a] / rho0) * rs;
                    double bc[3];
                    barycentric(tm, prev, Hp, Fp, bc);
                    double alpha = bc[0], beta = bc[1], gamma = bc[2];
                    if (std::abs(alpha) < 1e-6) { alpha = 1.0; beta = 0.0; gamma = 0.0; }
                    double tt[3], ctt[3];
                    for (int a = 0; a < 3; ++a) { tt[a] = alpha * prev[a] + beta * Hp[a] + gamma * Fp[a]; ctt[a] = tt[a] - c[a]; }
                    const double rho = norm3(ctt);
                    double qc[3];
                    for (int a = 0; a < 3; ++a) qc[a] = qs[a] - c[a];
                    const double radius = norm3(qc);
                    if (rho > radius && sval < 0.0) continue;
                    double q[3];
                    if (rho < 1e-9) for (int a = 0; a < 3; ++a) q[a] = c[a];
                    else for (int a = 0; a < 3; ++a) q[a] = c[a] + (ctt[a] / rho) * radius;
                    double dv[3], row[3];
                    for (int a = 0; a < 3; ++a) dv[a] = q[a] - c[a];
                    for (int a = 0; a < 3; ++a) row[a] = alpha * ssw * dv[a];
                    const double rb = ssw * ((dot3(q, dv) - beta * dot3(Hp, dv)) - gamma * dot3(Fp, dv));
                    for (int a = 0; a < 3; ++a) {
                        for (int c2 = 0; c2 < 3; ++c2) PA[a][c2] += row[a] * row[c2];
                        Pb[a] += row[a] * rb;
                    }
                    }
                    for (int a = 0; a < 3; ++a) {
                        for (int c2 = 0; c2 < 3; ++c2) A[a][c2] += PA[a][c2];
                        b[a] += Pb[a];
                    }
                }
                for (int a = 0; a < 3; ++a) { A[a][a] += smu * smu; b[a] += smu * (smu * prev[a]); }
                double E[3][3], U[3][3];
                std::memcpy(E, A, sizeof E);
                jacobi_eig3(E, U);
                double rhs[3];
                for (int a = 0; a < 3; ++a) rhs[a] = b[a] - (A[a][0] * cen[0] + A[a][1] * cen[1] + A[a][2] * cen[2]);
                double x[3] = {cen[0], cen[1], cen[2]};
                for (int q = 0; q < 3; ++q) {
                    double sv = std::abs(E[q][q]);
                    if (sv > o->svd_threshold) {
                        double coef = (U[0][q] * rhs[0] + U[1][q] * rhs[1] + U[2][q] * rhs[2]) / sv;
                        for (int a = 0; a < 3; ++a) x[a] += U[a][q] * coef;
                    }
                }
                std::memcpy(v, x, sizeof v);
                double dm[3] = {v[0] - prev[0], v[1] - prev[1], v[2] - prev[2]};
                if (norm3(dm) < 1e-6) break;
            }
            std::memcpy(S.v, v, sizeof v);
        }
        // re-extraction with the cells' vertices
        for (int64_t r = 0; r < nv; ++r) std::memcpy(&Vm[3 * r], C[r].v, sizeof C[r].v);
        F.clear();
        emit_quads(g, vid, Vm.data(), nth, F);
    }
    if (o->outer_iters == 0) {
        for (int64_t r = 0; r < nv; ++r) std::memcpy(&Vm[3 * r], C[r].v, sizeof C[r].v);
        F.clear();
        emit_quads(g, vid, Vm.data(), nth, F);
    }
    R->V = Vm;
    R->F = F;
    if (st) st->face_count = (int64_t)F.size() / 4;
    return R;
}

}  // extern "C"
