/*
 * dc_oracle.cpp — TEST INFRASTRUCTURE ONLY (the oracle; never shipped, never measured
 * as the product). Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
 * reference legs may load it.
 *
 * A plain C++17, FP64 restatement of the reference's CPU dual-contouring backend,
 * i.e. CpuDualContouringBackend::extract (src/cpp/dc_backend.cpp:51-125) with
 * ContouringOptions::method forced to DualContouring (dc_backend.cpp:70-77), which runs
 * contouring() (src/cpp/contouring.cpp:1199-1250):
 *
 *   generate_cells            contouring.cpp:210-271   (sign test Cell.cpp:57-77,
 *                                                       fill_hermite_data Cell.cpp:162-212,
 *                                                       lerp_t Cell.cpp:49-52,
 *                                                       trilinear gradient Cell.cpp:80-155)
 *   average_hermite_normals   hermite_update.cpp:334-438 via process_edge :171-332
 *   Cell::update              Cell.cpp:284-320 -> solve_quadratic_system :324-361
 *   extract_mesh_from_cells   contouring.cpp:486-741 (gradientAt :141-207)
 *
 * The reference needs Eigen (JacobiSVD) and libigl v2.6.0, neither of which exists in
 * this environment, so it cannot be compiled here. JacobiSVD of the symmetric PSD 3x3
 * matrix A^T A is restated as a cyclic Jacobi eigen-decomposition (Golub & Van Loan,
 * "Matrix Computations", 4th ed., section 8.5): for a symmetric PSD matrix the singular
 * values are the eigenvalues and U = V, so pinv = sum_{lambda_i > thr} v_i v_i^T / lambda_i,
 * which is the reference's V * diag(S_inv) * U^T.
 *
 * Arithmetic follows the reference statement by statement in double precision.
 * Grid positions are computed in float exactly as dc_backend.cpp:63-65 does
 * (grid.ox + i * grid.vx with int->float conversion) and then widened to double.
 * Build with -ffp-contract=off so no fused multiply-add changes a rounding.
 * Known unverifiable detail: Eigen's internal summation order inside norm()/dot() and
 * inside the small A^T A product; sums here run left to right.
 */
#include <cstdint>
#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>
#include <chrono>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Corner order of Cell.h:9-20 / contouring.cpp:232-241.
const int kOff[8][3] = {{0,0,0},{1,0,0},{1,1,0},{0,1,0},{0,0,1},{1,0,1},{1,1,1},{0,1,1}};
// EDGE_PAIRS, Cell.h:26-30.
const int kEdge[12][2] = {{0,1},{1,2},{2,3},{3,0},{4,5},{5,6},{6,7},{7,4},{0,4},{1,5},{2,6},{3,7}};
// get_face_normals_from_edge_idx, Cell.cpp:26-45 (0:+X,1:-X,2:+Y,3:-Y,4:+Z,5:-Z).
const int kEdgeFaces[12][2] = {{3,5},{0,5},{2,5},{1,5},{3,4},{0,4},{2,4},{1,4},{1,3},{0,3},{0,2},{1,2}};
const int kDirs[6][3] = {{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},{0,0,1},{0,0,-1}};

struct Grid {
    int nx, ny, nz;
    float vx, vy, vz, ox, oy, oz;
    const float* v;
    std::vector<double> gx, gy, gz;   // GV columns (separable), float-computed
    int64_t pidx(int i, int j, int k) const { return i + (int64_t)nx * (j + (int64_t)ny * k); }
    double S(int i, int j, int k) const { return (double)v[pidx(i, j, k)]; }
    int cx() const { return nx - 1; }
    int cy() const { return ny - 1; }
    int cz() const { return nz - 1; }
    int64_t cidx(int i, int j, int k) const { return i + (int64_t)(nx - 1) * (j + (int64_t)(ny - 1) * k); }
};

inline double sqnorm3(const double* a) { return a[0] * a[0] + a[1] * a[1] + a[2] * a[2]; }
inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline void cross3(const double* a, const double* b, double* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
// Eigen 3.4 normalize(): divide by sqrt(squaredNorm) only when it is > 0.
inline void normalize3(double* a) {
    double z = sqnorm3(a);
    if (z > 0.0) { double s = std::sqrt(z); a[0] /= s; a[1] /= s; a[2] /= s; }
}

// gradientAtPointUsingTrilinear, Cell.cpp:80-155.
void trilinear_gradient(const double cs[8], const double cp[8][3], const double p[3], double g[3]) {
    const double S000 = cs[0], S100 = cs[1], S110 = cs[2], S010 = cs[3];
    const double S001 = cs[4], S101 = cs[5], S111 = cs[6], S011 = cs[7];
    const double x0 = cp[0][0], x1 = cp[1][0];
    const double y0 = cp[0][1], y1 = cp[3][1];
    const double z0 = cp[0][2], z1 = cp[4][2];
    const double dx = x1 - x0, dy = y1 - y0, dz = z1 - z0;
    const double eps = 1e-12;
    double u = 0.5, v = 0.5, w = 0.5;
    if (std::abs(dx) > eps) u = (p[0] - x0) / dx;
    if (std::abs(dy) > eps) v = (p[1] - y0) / dy;
    if (std::abs(dz) > eps) w = (p[2] - z0) / dz;
    u = std::max(0.0, std::min(1.0, u));
    v = std::max(0.0, std::min(1.0, v));
    w = std::max(0.0, std::min(1.0, w));
    const double omu = 1.0 - u, omv = 1.0 - v, omw = 1.0 - w;
    double df_du = (S100 - S000) * omv * omw + (S110 - S010) * v * omw
                 + (S101 - S001) * omv * w + (S111 - S011) * v * w;
    double df_dv = (S010 - S000) * omu * omw + (S110 - S100) * u * omw
                 + (S011 - S001) * omu * w + (S111 - S101) * u * w;
    double df_dw = (S001 - S000) * omu * omv + (S101 - S100) * u * omv
                 + (S011 - S010) * omu * v + (S111 - S110) * u * v;
    g[0] = g[1] = g[2] = 0.0;
    if (std::abs(dx) > eps) g[0] = df_du / dx;
    if (std::abs(dy) > eps) g[1] = df_dv / dy;
    if (std::abs(dz) > eps) g[2] = df_dw / dz;
}

// Hermite data of one cell: Cell ctor (Cell.cpp:57-77) + fill_hermite_data (Cell.cpp:162-212).
struct Hermite {
    uint16_t mask = 0;
    double p[12][3];
    double n[12][3];
};

void fill_hermite(const Grid& g, int i, int j, int k, Hermite& h) {
    double cs[8], cp[8][3];
    for (int c = 0; c < 8; ++c) {
        int gi = i + kOff[c][0], gj = j + kOff[c][1], gk = k + kOff[c][2];
        cs[c] = g.S(gi, gj, gk);
        cp[c][0] = g.gx[gi]; cp[c][1] = g.gy[gj]; cp[c][2] = g.gz[gk];
    }
    h.mask = 0;
    for (int e = 0; e < 12; ++e) {
        int a = kEdge[e][0], b = kEdge[e][1];
        double fa = cs[a], fb = cs[b];
        if (fa * fb > 0.0) continue;                       // Cell.cpp:185
        double t = (fa - 0.0) / (fa - fb + 1e-16);         // lerp_t, Cell.cpp:49-52
        double p[3];
        for (int d = 0; d < 3; ++d) p[d] = (1.0 - t) * cp[a][d] + t * cp[b][d];
        double n[3];
        trilinear_gradient(cs, cp, p, n);
        if (std::sqrt(sqnorm3(n)) > 0.0) normalize3(n);
        std::memcpy(h.p[e], p, sizeof p);
        std::memcpy(h.n[e], n, sizeof n);
        h.mask |= (uint16_t)(1u << e);
    }
}

// get_corner_offsets + get_edge_idx_from_grid_vertices, hermite_update.cpp:34-91.
int edge_idx_from_points(int ci, int cj, int ck, int i0, int j0, int k0, int i1, int j1, int k1) {
    int di0 = i0 - ci, dj0 = j0 - cj, dk0 = k0 - ck;
    int di1 = i1 - ci, dj1 = j1 - cj, dk1 = k1 - ck;
    for (int e = 0; e < 12; ++e) {
        const int* A = kOff[kEdge[e][0]];
        const int* B = kOff[kEdge[e][1]];
        bool fwd = di0 == A[0] && dj0 == A[1] && dk0 == A[2] && di1 == B[0] && dj1 == B[1] && dk1 == B[2];
        bool bwd = di0 == B[0] && dj0 == B[1] && dk0 == B[2] && di1 == A[0] && dj1 == A[1] && dk1 == A[2];
        if (fwd || bwd) return e;
    }
    return -1;
}

// Cyclic Jacobi eigen-decomposition of a symmetric 3x3 matrix (Golub & Van Loan 8.5).
// On return a[][] holds eigenvalues on its diagonal and V's columns are eigenvectors.
// Stops when the off-diagonal mass is below 1e-30 of the diagonal's (off-diagonals ~1e-15
// relative, the level of Eigen's 2*eps per-pair test): a stricter bound sits under the
// rounding noise a rotation leaves in a rank-1 matrix, which then never converges.
void jacobi_eig3(double a[3][3], double V[3][3]) {
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) V[r][c] = (r == c) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        double diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (off <= 1e-30 * diag || off == 0.0) break;
        for (int p = 0; p < 2; ++p) {
            for (int q = p + 1; q < 3; ++q) {
                double apq = a[p][q];
                if (apq == 0.0) continue;
                double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
                double t = (theta >= 0.0 ? 1.0 : -1.0) / (std::abs(theta) + std::sqrt(theta * theta + 1.0));
                double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int r = 0; r < 3; ++r) {           // A <- A J
                    double arp = a[r][p], arq = a[r][q];
                    a[r][p] = c * arp - s * arq;
                    a[r][q] = s * arp + c * arq;
                }
                for (int r = 0; r < 3; ++r) {           // A <- J^T A
                    double apr = a[p][r], aqr = a[q][r];
                    a[p][r] = c * apr - s * aqr;
                    a[q][r] = s * apr + c * aqr;
                }
                for (int r = 0; r < 3; ++r) {           // V <- V J
                    double vrp = V[r][p], vrq = V[r][q];
                    V[r][p] = c * vrp - s * vrq;
                    V[r][q] = s * vrp + c * vrq;
                }
            }
        }
    }
}

// Cell::update (Cell.cpp:284-320) + solve_quadratic_system (Cell.cpp:324-361)
// + getCentroid (Cell.cpp:586-600). Returns the vertex and the eigenvalues (descending).
void solve_qef(const Hermite& h, double thr, double out[3], double eig[3]) {
    double ATA[3][3] = {{0,0,0},{0,0,0},{0,0,0}}, ATb[3] = {0,0,0}, c[3] = {0,0,0};
    int m = 0;
    for (int e = 0; e < 12; ++e) {                     // std::map iteration = ascending edge id
        if (!(h.mask & (1u << e))) continue;
        double n[3] = {h.n[e][0], h.n[e][1], h.n[e][2]};
        if (std::sqrt(sqnorm3(n)) > 0.0) normalize3(n);
        double b = dot3(n, h.p[e]);
        for (int r = 0; r < 3; ++r) {
            for (int s = 0; s < 3; ++s) ATA[r][s] += n[r] * n[s];
            ATb[r] += n[r] * b;
        }
        for (int d = 0; d < 3; ++d) c[d] += h.p[e][d];
        ++m;
    }
    for (int d = 0; d < 3; ++d) c[d] /= double(m);
    double a[3][3], V[3][3];
    std::memcpy(a, ATA, sizeof a);
    jacobi_eig3(a, V);
    double lam[3] = {a[0][0], a[1][1], a[2][2]};
    double rhs[3];
    for (int r = 0; r < 3; ++r) rhs[r] = ATb[r] - (ATA[r][0] * c[0] + ATA[r][1] * c[1] + ATA[r][2] * c[2]);
    double x[3] = {c[0], c[1], c[2]};
    for (int i = 0; i < 3; ++i) {
        double sv = std::abs(lam[i]);                  // singular value of a PSD matrix
        if (sv > thr) {
            double proj = V[0][i] * rhs[0] + V[1][i] * rhs[1] + V[2][i] * rhs[2];
            double coef = proj / sv;
            for (int d = 0; d < 3; ++d) x[d] += V[d][i] * coef;
        }
    }
    out[0] = x[0]; out[1] = x[1]; out[2] = x[2];
    double s[3] = {std::abs(lam[0]), std::abs(lam[1]), std::abs(lam[2])};
    std::sort(s, s + 3, [](double p, double q) { return p > q; });
    eig[0] = s[0]; eig[1] = s[1]; eig[2] = s[2];
}

// gradientAt, contouring.cpp:141-207 (central differences with clamped neighbours).
void grid_gradient(const Grid& g, int i, int j, int k, double out[3]) {
    auto cl = [](int v, int lo, int hi) { return std::max(lo, std::min(hi, v)); };
    int im = cl(i - 1, 0, g.nx - 1), ip = cl(i + 1, 0, g.nx - 1);
    int jm = cl(j - 1, 0, g.ny - 1), jp = cl(j + 1, 0, g.ny - 1);
    int km = cl(k - 1, 0, g.nz - 1), kp = cl(k + 1, 0, g.nz - 1);
    out[0] = out[1] = out[2] = 0.0;
    double dx = g.gx[ip] - g.gx[im];
    if (std::abs(dx) > 1e-12) out[0] = (g.S(ip, j, k) - g.S(im, j, k)) / dx;
    double dy = g.gy[jp] - g.gy[jm];
    if (std::abs(dy) > 1e-12) out[1] = (g.S(i, jp, k) - g.S(i, jm, k)) / dy;
    double dz = g.gz[kp] - g.gz[km];
    if (std::abs(dz) > 1e-12) out[2] = (g.S(i, j, kp) - g.S(i, j, km)) / dz;
    double nrm = std::sqrt(sqnorm3(out));
    if (nrm > 0.0) { out[0] /= nrm; out[1] /= nrm; out[2] /= nrm; }
}

struct Result {
    std::vector<double> V;        // 3 per vertex, FP64
    std::vector<int32_t> F;       // 4 per quad
    std::vector<int64_t> cells;   // linear cell index per vertex
    std::vector<double> eig;      // 3 per vertex (descending eigenvalues of A^T A)
    std::vector<int32_t> nrows;   // Hermite samples per vertex
    double ms = 0.0;
};

}  // namespace

// extract_mesh_from_cells quads (contouring.cpp:607-729) from vertices V: X edges, then Y, then
// Z; i outermost, k innermost. Each i-slice is produced independently and concatenated.
static void emit_quads(const Grid& g, const std::vector<int32_t>& vid, const double* V, int nth,
                       std::vector<int32_t>& F) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int cx = nx - 1, cy = ny - 1, cz = nz - 1;
    (void)nth; (void)ny; (void)nz;
    auto vcell = [&](int a, int b, int c) -> int32_t {
        if (a < 0 || a >= cx || b < 0 || b >= cy || c < 0 || c >= cz) return -1;
        return vid[g.cidx(a, b, c)];
    };
    auto emit = [&](std::vector<int32_t>& out, int i0, int j0, int k0, int i1, int j1, int k1,
                    int32_t c0, int32_t c1, int32_t c2, int32_t c3) {
        double g0[3], g1[3];
        grid_gradient(g, i0, j0, k0, g0);
        grid_gradient(g, i1, j1, k1, g1);
        double gn[3] = {g0[0] + g1[0], g0[1] + g1[1], g0[2] + g1[2]};
        const double* pa = &V[3 * (int64_t)c0];
        const double* pb = &V[3 * (int64_t)c1];
        const double* pc = &V[3 * (int64_t)c2];
        const double* pd = &V[3 * (int64_t)c3];
        double ba[3] = {pb[0] - pa[0], pb[1] - pa[1], pb[2] - pa[2]};
        double da[3] = {pd[0] - pa[0], pd[1] - pa[1], pd[2] - pa[2]};
        double qn[3];
        cross3(ba, da, qn);
        if (sqnorm3(qn) < 1e-24) {
            double ca[3] = {pc[0] - pa[0], pc[1] - pa[1], pc[2] - pa[2]};
            cross3(ca, da, qn);
        }
        if (sqnorm3(gn) > 0 && sqnorm3(qn) > 0) {
            if (dot3(qn, gn) < 0.0) std::swap(c1, c3);
        }
        out.push_back(c0); out.push_back(c1); out.push_back(c2); out.push_back(c3);
    };
    auto sc = [&](int i0, int j0, int k0, int i1, int j1, int k1) {
        double s0 = g.S(i0, j0, k0), s1 = g.S(i1, j1, k1);
        return s0 * s1 < 0.0;
    };
    for (int axis = 0; axis < 3; ++axis) {
        int ilo = axis == 0 ? 0 : 1;
        std::vector<std::vector<int32_t>> parts(cx);
#pragma omp parallel for num_threads(nth) schedule(dynamic, 1)
        for (int i = ilo; i < cx; ++i) {
            auto& out = parts[i];
            if (axis == 0) {
                for (int j = 1; j < cy; ++j)
                    for (int k = 1; k < cz; ++k) {
                        if (!sc(i, j, k, i + 1, j, k)) continue;
                        int32_t c0 = vcell(i, j - 1, k - 1), c1 = vcell(i, j, k - 1);
                        int32_t c2 = vcell(i, j, k), c3 = vcell(i, j - 1, k);
                        if (c0 < 0 || c1 < 0 || c2 < 0 || c3 < 0) continue;
                        emit(out, i, j, k, i + 1, j, k, c0, c1, c2, c3);
                    }
            } else if (axis == 1) {
                for (int j = 0; j < cy; ++j)
                    for (int k = 1; k < cz; ++k) {
                        if (!sc(i, j, k, i, j + 1, k)) continue;
                        int32_t c0 = vcell(i - 1, j, k - 1), c1 = vcell(i, j, k - 1);
                        int32_t c2 = vcell(i, j, k), c3 = vcell(i - 1, j, k);
                        if (c0 < 0 || c1 < 0 || c2 < 0 || c3 < 0) continue;
                        emit(out, i, j, k, i, j + 1, k, c0, c1, c2, c3);
                    }
            } else {
                for (int j = 1; j < cy; ++j)
                    for (int k = 0; k < cz; ++k) {
                        if (!sc(i, j, k, i, j, k + 1)) continue;
                        int32_t c0 = vcell(i - 1, j - 1, k), c1 = vcell(i, j - 1, k);
                        int32_t c2 = vcell(i, j, k), c3 = vcell(i - 1, j, k);
                        if (c0 < 0 || c1 < 0 || c2 < 0 || c3 < 0) continue;
                        emit(out, i, j, k, i, j, k + 1, c0, c1, c2, c3);
                    }
            }
        }
        for (auto& p : parts) F.insert(F.end(), p.begin(), p.end());
    }

}

extern "C" {

typedef struct {
    int64_t total_cells;
    int64_t active_cells;
    int64_t vertex_count;
    int64_t face_count;
    double total_ms;
} dco_stats;

/*
 * Run the restated CPU backend on a dense x-fastest float grid.
 * threads <= 0 uses every OpenMP thread; 1 reproduces the reference's single thread.
 * Returns an opaque handle (free with dco_free) or NULL on invalid input.
 */
static void* extract_impl(int nx, int ny, int nz, float vx, float vy, float vz,
                          float ox, float oy, float oz, const double* px, const double* py,
                          const double* pz, const float* values, double svd_threshold,
                          int threads, dco_stats* st, std::vector<Hermite>* keep_hermite = nullptr);

void* dco_extract(int nx, int ny, int nz, float vx, float vy, float vz,
                  float ox, float oy, float oz, const float* values,
                  double svd_threshold, int threads, dco_stats* st) {
    return extract_impl(nx, ny, nz, vx, vy, vz, ox, oy, oz, nullptr, nullptr, nullptr, values,
                        svd_threshold, threads, st);
}

/*
 * Same, with explicit grid-point coordinates per axis (px[nx], py[ny], pz[nz]) instead of
 * origin + i * spacing. Used to run the restatement on a window of a larger grid with the
 * larger grid's own float positions.
 */
void* dco_extract_pos(int nx, int ny, int nz, const double* px, const double* py, const double* pz,
                      const float* values, double svd_threshold, int threads, dco_stats* st) {
    if (!px || !py || !pz) return nullptr;
    return extract_impl(nx, ny, nz, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, px, py, pz, values, svd_threshold,
                        threads, st);
}

}  // extern "C"

static void* extract_impl(int nx, int ny, int nz, float vx, float vy, float vz,
                          float ox, float oy, float oz, const double* px, const double* py,
                          const double* pz, const float* values, double svd_threshold,
                          int threads, dco_stats* st, std::vector<Hermite>* keep_hermite) {
    if (nx < 2 || ny < 2 || nz < 2 || !values) return nullptr;
    auto t0 = std::chrono::high_resolution_clock::now();
#ifdef _OPENMP
    int nth = threads > 0 ? threads : omp_get_max_threads();
#else
    int nth = 1; (void)threads;
#endif
    Grid g;
    g.nx = nx; g.ny = ny; g.nz = nz; g.vx = vx; g.vy = vy; g.vz = vz; g.ox = ox; g.oy = oy; g.oz = oz;
    g.v = values;
    // dc_backend.cpp:63-65: float arithmetic, then stored into a double matrix.
    g.gx.resize(nx); g.gy.resize(ny); g.gz.resize(nz);
    for (int i = 0; i < nx; ++i) { float f = (float)i; float pr = f * vx; float s = ox + pr; g.gx[i] = px ? px[i] : (double)s; }
    for (int j = 0; j < ny; ++j) { float f = (float)j; float pr = f * vy; float s = oy + pr; g.gy[j] = py ? py[j] : (double)s; }
    for (int k = 0; k < nz; ++k) { float f = (float)k; float pr = f * vz; float s = oz + pr; g.gz[k] = pz ? pz[k] : (double)s; }

    const int cx = nx - 1, cy = ny - 1, cz = nz - 1;
    const int64_t ncell = (int64_t)cx * cy * cz;

    // 1) sign test of every cell (Cell.cpp:68-76); vertex numbering in k,j,i order
    //    (contouring.cpp:513-524).
    std::vector<uint8_t> active(ncell, 0);
#pragma omp parallel for num_threads(nth) schedule(static)
    for (int k = 0; k < cz; ++k)
        for (int j = 0; j < cy; ++j)
            for (int i = 0; i < cx; ++i) {
                bool neg = false, pos = false;
                for (int c = 0; c < 8; ++c) {
                    double s = g.S(i + kOff[c][0], j + kOff[c][1], k + kOff[c][2]);
                    if (s < 0) neg = true;
                    if (s > 0) pos = true;
                }
                active[g.cidx(i, j, k)] = (neg && pos) ? 1 : 0;
            }
    std::vector<int32_t> vid(ncell, -1);
    Result* R = new Result();
    int64_t nv = 0;
    for (int64_t c = 0; c < ncell; ++c)
        if (active[c]) { vid[c] = (int32_t)nv; R->cells.push_back(c); ++nv; }

    // 2) Hermite data of active cells.
    std::vector<Hermite> H(nv);
#pragma omp parallel for num_threads(nth) schedule(dynamic, 256)
    for (int64_t r = 0; r < nv; ++r) {
        int64_t c = R->cells[r];
        int i = (int)(c % cx), j = (int)((c / cx) % cy), k = (int)(c / ((int64_t)cx * cy));
        fill_hermite(g, i, j, k, H[r]);
    }

    // 3) average_hermite_normals (hermite_update.cpp:334-438). Each cell-local edge belongs
    //    to exactly one grid edge, so averages are computed from the trilinear normals and
    //    written back afterwards; grid-edge iteration order therefore does not matter.
    //    Only grid edges whose min-corner cell has a Hermite sample pass process_edge
    //    (hermite_update.cpp:238-243), so the loop runs over active owner cells.
    struct Avg { int64_t r[4]; int e[4]; double n[3]; };
    std::vector<std::vector<Avg>> avg_parts(nth);
    auto inside = [&](int a, int b, int c) {
        return a > 0 && a < nx - 1 && b > 0 && b < ny - 1 && c > 0 && c < nz - 1;
    };
#pragma omp parallel for num_threads(nth) schedule(dynamic, 256)
    for (int64_t r = 0; r < nv; ++r) {
#ifdef _OPENMP
        auto& out = avg_parts[omp_get_thread_num()];
#else
        auto& out = avg_parts[0];
#endif
        int64_t c = R->cells[r];
        int i = (int)(c % cx), j = (int)((c / cx) % cy), k = (int)(c / ((int64_t)cx * cy));
        const int ends[3][3] = {{i + 1, j, k}, {i, j + 1, k}, {i, j, k + 1}};
        for (int ax = 0; ax < 3; ++ax) {
            int i1 = ends[ax][0], j1 = ends[ax][1], k1 = ends[ax][2];
            if (i1 > nx - 1 || j1 > ny - 1 || k1 > nz - 1) continue;
            if (!inside(i, j, k) && !inside(i1, j1, k1)) continue;       // :196-215
            int e0 = edge_idx_from_points(i, j, k, i, j, k, i1, j1, k1);
            if (!(H[r].mask & (1u << e0))) continue;                    // :238-243
            const int* d1 = kDirs[kEdgeFaces[e0][0]];
            const int* d2 = kDirs[kEdgeFaces[e0][1]];
            int nb[3][3] = {{i + d1[0], j + d1[1], k + d1[2]},
                            {i + d2[0], j + d2[1], k + d2[2]},
                            {i + d1[0] + d2[0], j + d1[1] + d2[1], k + d1[2] + d2[2]}};
            Avg a;
            a.r[0] = r; a.e[0] = e0;
            bool ok = true;
            for (int q = 0; q < 3 && ok; ++q) {
                int64_t cc = g.cidx(nb[q][0], nb[q][1], nb[q][2]);
                if (vid[cc] < 0) { ok = false; break; }                  // :298-303
                a.r[q + 1] = vid[cc];
                a.e[q + 1] = edge_idx_from_points(nb[q][0], nb[q][1], nb[q][2], i, j, k, i1, j1, k1);
            }
            if (!ok) continue;
            double acc[3] = {0, 0, 0};
            for (int q = 0; q < 4; ++q) {                                 // :415-426
                const double* hn = H[a.r[q]].n[a.e[q]];
                if (std::sqrt(sqnorm3(hn)) > 0) { acc[0] += hn[0]; acc[1] += hn[1]; acc[2] += hn[2]; }
            }
            normalize3(acc);                                              // :427
            a.n[0] = acc[0]; a.n[1] = acc[1]; a.n[2] = acc[2];
            out.push_back(a);
        }
    }
    for (auto& part : avg_parts)
        for (auto& a : part)
            for (int q = 0; q < 4; ++q) std::memcpy(H[a.r[q]].n[a.e[q]], a.n, sizeof a.n);

    // 4) QEF per active cell.
    R->V.resize(3 * nv);
    R->eig.resize(3 * nv);
    R->nrows.resize(nv);
#pragma omp parallel for num_threads(nth) schedule(dynamic, 256)
    for (int64_t r = 0; r < nv; ++r) {
        solve_qef(H[r], svd_threshold, &R->V[3 * r], &R->eig[3 * r]);
        int m = 0;
        for (int e = 0; e < 12; ++e) m += (H[r].mask >> e) & 1;
        R->nrows[r] = m;
    }
    if (keep_hermite) *keep_hermite = std::move(H);
    else { H.clear(); H.shrink_to_fit(); }

    // 5) extract_mesh_from_cells quads (contouring.cpp:607-729).
    emit_quads(g, vid, R->V.data(), nth, R->F);

    auto t1 = std::chrono::high_resolution_clock::now();
    R->ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    if (st) {
        st->total_cells = ncell;
        st->active_cells = nv;
        st->vertex_count = nv;
        st->face_count = (int64_t)R->F.size() / 4;
        st->total_ms = R->ms;
    }
    return R;
}

extern "C" {

int64_t dco_num_vertices(void* h) { return h ? (int64_t)((Result*)h)->cells.size() : 0; }
int64_t dco_num_faces(void* h) { return h ? (int64_t)((Result*)h)->F.size() / 4 : 0; }

/* Copy results out; any pointer may be NULL. */
void dco_copy(void* h, double* V, int32_t* F, int64_t* cells, double* eig, int32_t* nrows) {
    if (!h) return;
    Result* R = (Result*)h;
    if (V) std::memcpy(V, R->V.data(), R->V.size() * sizeof(double));
    if (F) std::memcpy(F, R->F.data(), R->F.size() * sizeof(int32_t));
    if (cells) std::memcpy(cells, R->cells.data(), R->cells.size() * sizeof(int64_t));
    if (eig) std::memcpy(eig, R->eig.data(), R->eig.size() * sizeof(double));
    if (nrows) std::memcpy(nrows, R->nrows.data(), R->nrows.size() * sizeof(int32_t));
}

void dco_free(void* h) { delete (Result*)h; }

}  // extern "C"
