// sparse_oracle.cpp — TEST INFRASTRUCTURE ONLY: a float CPU restatement of the reference's
// sparse (brick) dual-contouring backend and its multi-vertex variant
// (CudaSparseDualContouringBackend / CudaSparseMvdcDualContouringBackend,
// src/cuda/dc_cuda_sparse.cu:271-1415, include/dc_cuda.h:37-66). Only tests/ and the bench's
// CPU leg use it, as the checker.
//
// The reference runs this path in float on the GPU. Every float operation here is written in
// the reference's order and rounded once (built with -ffp-contract=off), so the result equals
// the reference compiled without FMA contraction bit for bit; the tests check that on the GPU.
//
// Pipeline (one thread per item in the reference; sequential or OpenMP here, same results):
//   bricks   brick (bx,by,bz) of brick_size^3 cells is active iff its points
//            [b*s, min(b*s + s + 1, n)) per axis hold a value < 0 and a value > 0 (:271-308)
//   cells    a cell of an active brick is active iff it has a corner < 0 and one > 0, or any
//            corner with |v| <= 0.45*vx (:321-377); vertices follow ascending linear cell
//            order (the copy_if compaction, :1263-1276)
//   samples  per cell edge (EDGE_PAIRS order): a crossing (fa*fb <= 0 in float) or a thin
//            edge (same sign, both |v| <= 0.45*vx, central-difference gradients at the ends
//            with dot < -0.3, :310-319) gives Hermite samples (:676-752)
//   vertices one QEF per cell, or for the multi-vertex variant two when the most opposed
//            pair of sample normals has dot < -0.3 and both halves hold >= 2 samples
//            (:445-620, :753-826); max-pivot float Jacobi, pinv truncating at 0.01, centroid
//            fallback, clamp into the cell (:181-269, :380-443)
//   faces    per active cell its min-corner X, Y, Z edges with a strict crossing (float
//            product < 0) or a thin edge, all four cells with a vertex (multi-vertex cells
//            pick the vertex whose normal best matches the gradient sum, rejecting
//            dot < -0.5), winding by the gradient sum, a thin edge adding the reversed quad
//            (:829-1102); faces in active-cell order, X then Y then Z.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct F3 {
    float x, y, z;
};
inline F3 mk(float x, float y, float z) { return F3{x, y, z}; }
inline F3 add(F3 a, F3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline F3 sub(F3 a, F3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline F3 scale(float s, F3 b) { return mk(s * b.x, s * b.y, s * b.z); }
inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 cross(F3 a, F3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline bool bad(F3 v) { return std::isnan(v.x) || std::isnan(v.y) || std::isnan(v.z) || std::isinf(v.x) || std::isinf(v.y) || std::isinf(v.z); }

const int kCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
const int kEdge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

enum { kFallback, kClamp, kInvalid, kNCounters };

struct Grid {
    int nx, ny, nz;
    float vx, vy, vz, ox, oy, oz;
    const float* v;
    int normal_mode;
    float at(int i, int j, int k) const { return v[(int64_t)i + (int64_t)nx * ((int64_t)j + (int64_t)ny * k)]; }
    // central differences with clamped neighbours (:155-179)
    F3 grad(int i, int j, int k) const {
        const int im = i > 0 ? i - 1 : 0, ip = i < nx - 1 ? i + 1 : nx - 1;
        const int jm = j > 0 ? j - 1 : 0, jp = j < ny - 1 ? j + 1 : ny - 1;
        const int km = k > 0 ? k - 1 : 0, kp = k < nz - 1 ? k + 1 : nz - 1;
        F3 g = mk(0.f, 0.f, 0.f);
        const float dx = (float)(ip - im) * vx, dy = (float)(jp - jm) * vy, dz = (float)(kp - km) * vz;
        if (dx > 1e-12f) g.x = (at(ip, j, k) - at(im, j, k)) / dx;
        if (dy > 1e-12f) g.y = (at(i, jp, k) - at(i, jm, k)) / dy;
        if (dz > 1e-12f) g.z = (at(i, j, kp) - at(i, j, km)) / dz;
        return g;
    }
    // :310-319
    bool thin(float fa, float fb, int ai, int aj, int ak, int bi, int bj, int bk) const {
        if (fa * fb <= 0.0f) return false;
        if (std::fabs(fa) > 0.45f * vx || std::fabs(fb) > 0.45f * vx) return false;
        return dot(grad(ai, aj, ak), grad(bi, bj, bk)) < -0.3f;
    }
};

// Trilinear gradient of the cell at p (:91-153).
F3 trilinear(const float s[8], const F3 cp[8], F3 p) {
    const float S000 = s[0], S100 = s[1], S110 = s[2], S010 = s[3];
    const float S001 = s[4], S101 = s[5], S111 = s[6], S011 = s[7];
    const float x0 = cp[0].x, x1 = cp[1].x, y0 = cp[0].y, y1 = cp[3].y, z0 = cp[0].z, z1 = cp[4].z;
    const float dx = x1 - x0, dy = y1 - y0, dz = z1 - z0;
    float u = 0.5f, v = 0.5f, w = 0.5f;
    if (std::fabs(dx) > 1e-12f) u = (p.x - x0) / dx;
    if (std::fabs(dy) > 1e-12f) v = (p.y - y0) / dy;
    if (std::fabs(dz) > 1e-12f) w = (p.z - z0) / dz;
    u = std::fmax(0.0f, std::fmin(1.0f, u));
    v = std::fmax(0.0f, std::fmin(1.0f, v));
    w = std::fmax(0.0f, std::fmin(1.0f, w));
    const float omu = 1.0f - u, omv = 1.0f - v, omw = 1.0f - w;
    const float du = (S100 - S000) * omv * omw + (S110 - S010) * v * omw + (S101 - S001) * omv * w + (S111 - S011) * v * w;
    const float dv = (S010 - S000) * omu * omw + (S110 - S100) * u * omw + (S011 - S001) * omu * w + (S111 - S101) * u * w;
    const float dw = (S001 - S000) * omu * omv + (S101 - S100) * u * omv + (S011 - S010) * omu * v + (S111 - S110) * u * v;
    F3 g = mk(0.f, 0.f, 0.f);
    if (std::fabs(dx) > 1e-12f) g.x = du / dx;
    if (std::fabs(dy) > 1e-12f) g.y = dv / dy;
    if (std::fabs(dz) > 1e-12f) g.z = dw / dz;
    return g;
}

// Max-pivot Jacobi on the 3x3 normal matrix, at most 15 rotations, pinv of the diagonal
// above thr (:181-269). Returns y = V S^+ V^T d; singular when nothing is retained.
void jacobi_solve(const float B[9], const float d[3], float thr, float y[3], bool& singular) {
    float V[9] = {1.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f};
    float A[9];
    for (int i = 0; i < 9; ++i) A[i] = B[i];
    for (int it = 0; it < 15; ++it) {
        int p = 0, q = 1;
        float mv = std::fabs(A[1]);
        if (std::fabs(A[2]) > mv) { p = 0; q = 2; mv = std::fabs(A[2]); }
        if (std::fabs(A[5]) > mv) { p = 1; q = 2; mv = std::fabs(A[5]); }
        if (mv < 1e-7f) break;
        const float ap = A[p * 3 + p], aq = A[q * 3 + q], apq = A[p * 3 + q];
        const float phi = 0.5f * (aq - ap) / apq;
        float t = 1.0f / (std::fabs(phi) + std::sqrt(phi * phi + 1.0f));
        if (phi < 0.0f) t = -t;
        const float c = 1.0f / std::sqrt(t * t + 1.0f), s = t * c;
        for (int i = 0; i < 3; ++i) {
            if (i == p || i == q) continue;
            const float aip = A[i * 3 + p], aiq = A[i * 3 + q];
            A[i * 3 + p] = A[p * 3 + i] = c * aip - s * aiq;
            A[i * 3 + q] = A[q * 3 + i] = s * aip + c * aiq;
        }
        A[p * 3 + p] = ap - t * apq;
        A[q * 3 + q] = aq + t * apq;
        A[p * 3 + q] = A[q * 3 + p] = 0.0f;
        for (int i = 0; i < 3; ++i) {
            const float vip = V[i * 3 + p], viq = V[i * 3 + q];
            V[i * 3 + p] = c * vip - s * viq;
            V[i * 3 + q] = s * vip + c * viq;
        }
    }
    const float S[3] = {A[0], A[4], A[8]};
    float Si[3];
    int ok = 0;
    for (int i = 0; i < 3; ++i) {
        if (S[i] > thr) { Si[i] = 1.0f / S[i]; ++ok; } else Si[i] = 0.0f;
    }
    singular = ok == 0;
    float tmp[3];
    tmp[0] = V[0] * d[0] + V[3] * d[1] + V[6] * d[2];
    tmp[1] = V[1] * d[0] + V[4] * d[1] + V[7] * d[2];
    tmp[2] = V[2] * d[0] + V[5] * d[1] + V[8] * d[2];
    tmp[0] *= Si[0]; tmp[1] *= Si[1]; tmp[2] *= Si[2];
    y[0] = V[0] * tmp[0] + V[1] * tmp[1] + V[2] * tmp[2];
    y[1] = V[3] * tmp[0] + V[4] * tmp[1] + V[5] * tmp[2];
    y[2] = V[6] * tmp[0] + V[7] * tmp[1] + V[8] * tmp[2];
}

// One cluster's vertex (:380-443); cnt receives the fallback / invalid / clamp events.
F3 solve_cluster(const F3* pts, const F3* nrm, int m, F3 cmin, F3 cmax, const Grid& g, int64_t* cnt) {
    const F3 half = scale(0.5f, mk(g.vx, g.vy, g.vz));
    if (m == 0) return add(cmin, half);
    F3 c = mk(0.f, 0.f, 0.f);
    for (int i = 0; i < m; ++i) c = add(c, pts[i]);
    c = scale(1.0f / (float)m, c);
    float B[9] = {0.f}, d[3] = {0.f};
    for (int i = 0; i < m; ++i) {
        const F3 n = nrm[i];
        const float dv = dot(n, sub(pts[i], c));
        B[0] += n.x * n.x; B[1] += n.x * n.y; B[2] += n.x * n.z;
        B[3] += n.y * n.x; B[4] += n.y * n.y; B[5] += n.y * n.z;
        B[6] += n.z * n.x; B[7] += n.z * n.y; B[8] += n.z * n.z;
        d[0] += n.x * dv; d[1] += n.y * dv; d[2] += n.z * dv;
    }
    float y[3] = {0.f, 0.f, 0.f};
    bool singular = false;
    jacobi_solve(B, d, 0.01f, y, singular);
    F3 v = add(c, mk(y[0], y[1], y[2]));
    if (singular || bad(v)) { ++cnt[kFallback]; v = c; }
    if (bad(v)) { ++cnt[kInvalid]; v = add(cmin, half); }
    if (v.x < cmin.x || v.x > cmax.x || v.y < cmin.y || v.y > cmax.y || v.z < cmin.z || v.z > cmax.z) {
        ++cnt[kClamp];
        v.x = std::fmax(cmin.x, std::fmin(cmax.x, v.x));
        v.y = std::fmax(cmin.y, std::fmin(cmax.y, v.y));
        v.z = std::fmax(cmin.z, std::fmin(cmax.z, v.z));
    }
    return v;
}

struct CellOut {
    int count = 1;             // vertices of the cell (1 or 2)
    F3 v[2], n[2];
    int64_t cnt[kNCounters] = {0, 0, 0};
    int ambiguous = 0, split_rejected = 0;
};

// Hermite samples of cell (i,j,k) (:663-752); returns m.
int cell_samples(const Grid& g, int i, int j, int k, F3* pts, F3* nrm, float s[8], F3 cp[8]) {
    for (int c = 0; c < 8; ++c) {
        const int ci = i + kCorner[c][0], cj = j + kCorner[c][1], ck = k + kCorner[c][2];
        s[c] = g.at(ci, cj, ck);
        cp[c] = mk(g.ox + (float)ci * g.vx, g.oy + (float)cj * g.vy, g.oz + (float)ck * g.vz);
    }
    int m = 0;
    for (int e = 0; e < 12; ++e) {
        const int a = kEdge[e][0], b = kEdge[e][1];
        const float fa = s[a], fb = s[b];
        const int ai = i + kCorner[a][0], aj = j + kCorner[a][1], ak = k + kCorner[a][2];
        const int bi = i + kCorner[b][0], bj = j + kCorner[b][1], bk = k + kCorner[b][2];
        const bool crossing = fa * fb <= 0.0f;
        const bool thin = !crossing && g.thin(fa, fb, ai, aj, ak, bi, bj, bk);
        if (!crossing && !thin) continue;
        float t = crossing ? fa / (fa - fb + 1e-12f) : std::fabs(fa) / (std::fabs(fa) + std::fabs(fb) + 1e-12f);
        t = std::fmax(0.0f, std::fmin(1.0f, t));
        const F3 p = add(scale(1.0f - t, cp[a]), scale(t, cp[b]));
        if (thin) {
            F3 ga = g.grad(ai, aj, ak), gb = g.grad(bi, bj, bk);
            const float la = std::sqrt(dot(ga, ga)), lb = std::sqrt(dot(gb, gb));
            if (la > 1e-6f) ga = scale(1.0f / la, ga);
            if (lb > 1e-6f) gb = scale(1.0f / lb, gb);
            if (m < 11) {
                pts[m] = p; nrm[m] = ga; ++m;
                pts[m] = p; nrm[m] = gb; ++m;
            }
        } else {
            F3 n;
            if (g.normal_mode == 1) {
                const F3 ga = g.grad(ai, aj, ak), gb = g.grad(bi, bj, bk);
                n = add(scale(1.0f - t, ga), scale(t, gb));
            } else {
                n = trilinear(s, cp, p);   // mode 0, and mode 2 without precomputed gradients
            }
            const float ln = std::sqrt(dot(n, n));
            if (ln > 1e-6f) n = scale(1.0f / ln, n);
            if (m < 12) { pts[m] = p; nrm[m] = n; ++m; }
        }
    }
    return m;
}

// Most opposed pair of sample normals (first minimum in (i, j>i) order).
void opposed_pair(const F3* nrm, int m, int& A, int& B, float& mind) {
    A = -1; B = -1; mind = 1.0f;
    for (int i = 0; i < m; ++i)
        for (int j = i + 1; j < m; ++j) {
            const float dt = dot(nrm[i], nrm[j]);
            if (dt < mind) { mind = dt; A = i; B = j; }
        }
}

F3 unit_or(F3 a, F3 fallback) {
    const float l = std::sqrt(dot(a, a));
    return l > 1e-6f ? scale(1.0f / l, a) : fallback;
}

void cell_vertices(const Grid& g, int i, int j, int k, bool mvdc, CellOut& o) {
    F3 pts[12], nrm[12], cp[8];
    float s[8];
    const int m = cell_samples(g, i, j, k, pts, nrm, s, cp);
    const F3 cmin = cp[0], cmax = cp[6];
    // vertex count (:445-620)
    int count = 1;
    if (mvdc && m >= 2) {
        int A, B;
        float mind;
        opposed_pair(nrm, m, A, B, mind);
        if (A >= 0 && B >= 0 && mind < -0.3f) {
            int ca = 0, cb = 0;
            for (int q = 0; q < m; ++q) (dot(nrm[q], nrm[A]) >= dot(nrm[q], nrm[B]) ? ca : cb)++;
            if (ca < 2 || cb < 2) o.split_rejected = 1;
            else { count = 2; o.ambiguous = 1; }
        }
    }
    o.count = count;
    // vertices (:753-826)
    if (count == 1 || m < 2) {
        o.v[0] = solve_cluster(pts, nrm, m, cmin, cmax, g, o.cnt);
        F3 avg = mk(0.f, 0.f, 0.f);
        for (int q = 0; q < m; ++q) avg = add(avg, nrm[q]);
        o.n[0] = unit_or(avg, mk(0.f, 1.f, 0.f));
        return;
    }
    int A, B;
    float mind;
    opposed_pair(nrm, m, A, B, mind);
    const F3 nA = nrm[A], nB = nrm[B];
    F3 p0[12], n0[12], p1[12], n1[12];
    int m0 = 0, m1 = 0;
    for (int q = 0; q < m; ++q) {
        if (dot(nrm[q], nA) >= dot(nrm[q], nB)) { p0[m0] = pts[q]; n0[m0] = nrm[q]; ++m0; }
        else { p1[m1] = pts[q]; n1[m1] = nrm[q]; ++m1; }
    }
    o.v[0] = solve_cluster(p0, n0, m0, cmin, cmax, g, o.cnt);
    o.v[1] = solve_cluster(p1, n1, m1, cmin, cmax, g, o.cnt);
    F3 a0 = mk(0.f, 0.f, 0.f), a1 = mk(0.f, 0.f, 0.f);
    for (int q = 0; q < m0; ++q) a0 = add(a0, n0[q]);
    for (int q = 0; q < m1; ++q) a1 = add(a1, n1[q]);
    o.n[0] = unit_or(a0, nA);
    o.n[1] = unit_or(a1, nB);
}

struct Result {
    std::vector<float> V, N;          // 3 per vertex
    std::vector<int32_t> F;           // 4 per face
    std::vector<int64_t> cells;       // linear index of every active cell (ascending)
    std::vector<int32_t> vstart;      // first vertex of every active cell
    int64_t stats[12] = {0};
};

}  // namespace

extern "C" {

/*
 * stats: [0] total bricks, [1] active bricks, [2] active cells, [3] QEF fallbacks to the
 * centroid, [4] out-of-cell clamps, [5] invalid vertices, [6] ambiguous (split) cells,
 * [7] multi-vertex cells, [8] one-vertex cells, [9] two-vertex cells, [10] split
 * rejections, [11] faces skipped for a missing vertex (multi-vertex variant only).
 * normal_mode: 0 trilinear (FiniteDifference), 1 EdgeGradient, 2 PrecomputedGradient
 * (which the reference calls without gradients, so it is the trilinear normal).
 */
void* sdo_extract(const float* values, int nx, int ny, int nz, float vx, float vy, float vz, float ox, float oy,
                  float oz, int brick_size, int mvdc, int normal_mode, int threads) {
    if (!values || nx < 2 || ny < 2 || nz < 2 || brick_size < 1) return nullptr;
#ifdef _OPENMP
    const int nth = threads > 0 ? threads : omp_get_max_threads();
#else
    const int nth = 1; (void)threads;
#endif
    Grid g{nx, ny, nz, vx, vy, vz, ox, oy, oz, values, normal_mode};
    const int cx = nx - 1, cy = ny - 1, cz = nz - 1;
    const int bs = brick_size;
    const int nbx = (cx + bs - 1) / bs, nby = (cy + bs - 1) / bs, nbz = (cz + bs - 1) / bs;
    const int64_t nbricks = (int64_t)nbx * nby * nbz;
    Result* R = new Result();
    R->stats[0] = nbricks;
    std::vector<uint8_t> brick(nbricks, 0);
#pragma omp parallel for schedule(dynamic, 64) num_threads(nth)
    for (int64_t b = 0; b < nbricks; ++b) {
        const int bx = (int)(b % nbx), by = (int)((b / nbx) % nby), bz = (int)(b / ((int64_t)nbx * nby));
        const int i0 = bx * bs, j0 = by * bs, k0 = bz * bs;
        const int i1 = std::min(i0 + bs + 1, nx), j1 = std::min(j0 + bs + 1, ny), k1 = std::min(k0 + bs + 1, nz);
        bool neg = false, pos = false;
        for (int k = k0; k < k1 && !(neg && pos); ++k)
            for (int j = j0; j < j1 && !(neg && pos); ++j)
                for (int i = i0; i < i1; ++i) {
                    const float v = g.at(i, j, k);
                    if (v < 0.0f) neg = true;
                    if (v > 0.0f) pos = true;
                }
        brick[b] = (neg && pos) ? 1 : 0;
    }
    for (int64_t b = 0; b < nbricks; ++b) R->stats[1] += brick[b];
    // active cells, ascending linear order (per z-plane lists, concatenated)
    const float close = 0.45f * vx;
    std::vector<std::vector<int64_t>> plane(cz);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nth)
    for (int k = 0; k < cz; ++k) {
        for (int j = 0; j < cy; ++j)
            for (int i = 0; i < cx; ++i) {
                if (!brick[(int64_t)(i / bs) + nbx * ((int64_t)(j / bs) + (int64_t)nby * (k / bs))]) continue;
                bool neg = false, pos = false, near = false;
                for (int c = 0; c < 8; ++c) {
                    const float v = g.at(i + kCorner[c][0], j + kCorner[c][1], k + kCorner[c][2]);
                    if (v < 0.0f) neg = true;
                    if (v > 0.0f) pos = true;
                    if (std::fabs(v) <= close) near = true;
                }
                if ((neg && pos) || near) plane[k].push_back((int64_t)i + (int64_t)cx * ((int64_t)j + (int64_t)cy * k));
            }
    }
    for (int k = 0; k < cz; ++k) R->cells.insert(R->cells.end(), plane[k].begin(), plane[k].end());
    const int64_t na = (int64_t)R->cells.size();
    R->stats[2] = na;
    std::vector<CellOut> out(na);
#pragma omp parallel for schedule(dynamic, 256) num_threads(nth)
    for (int64_t r = 0; r < na; ++r) {
        const int64_t c = R->cells[r];
        const int i = (int)(c % cx), j = (int)((c / cx) % cy), k = (int)(c / ((int64_t)cx * cy));
        cell_vertices(g, i, j, k, mvdc != 0, out[r]);
    }
    R->vstart.resize(na);
    int64_t nv = 0;
    for (int64_t r = 0; r < na; ++r) {
        R->vstart[r] = (int32_t)nv;
        nv += out[r].count;
        for (int q = 0; q < kNCounters; ++q) R->stats[3 + q] += out[r].cnt[q];
        if (mvdc) {
            R->stats[6] += out[r].ambiguous;
            R->stats[7] += out[r].count == 2;
            R->stats[8] += out[r].count == 1;
            R->stats[9] += out[r].count == 2;
            R->stats[10] += out[r].split_rejected;
        }
    }
    R->V.resize(3 * nv);
    R->N.resize(3 * nv);
    for (int64_t r = 0; r < na; ++r)
        for (int q = 0; q < out[r].count; ++q) {
            const int64_t v = R->vstart[r] + q;
            R->V[3 * v] = out[r].v[q].x; R->V[3 * v + 1] = out[r].v[q].y; R->V[3 * v + 2] = out[r].v[q].z;
            R->N[3 * v] = out[r].n[q].x; R->N[3 * v + 1] = out[r].n[q].y; R->N[3 * v + 2] = out[r].n[q].z;
        }
    // cell -> rank lookup
    auto rank_of = [&](int i, int j, int k) -> int64_t {
        const int64_t c = (int64_t)i + (int64_t)cx * ((int64_t)j + (int64_t)cy * k);
        auto it = std::lower_bound(R->cells.begin(), R->cells.end(), c);
        return (it != R->cells.end() && *it == c) ? (int64_t)(it - R->cells.begin()) : -1;
    };
    // vertex of a face cell (:829-851)
    auto pick = [&](int i, int j, int k, F3 gn) -> int64_t {
        const int64_t r = rank_of(i, j, k);
        if (r < 0) return -1;
        const int64_t st = R->vstart[r];
        if (!mvdc || out[r].count == 1) return st;
        const F3 n0 = mk(R->N[3 * st], R->N[3 * st + 1], R->N[3 * st + 2]);
        const F3 n1 = mk(R->N[3 * st + 3], R->N[3 * st + 4], R->N[3 * st + 5]);
        const float d0 = dot(gn, n0), d1 = dot(gn, n1);
        const int64_t best = d0 >= d1 ? st : st + 1;
        return std::fmax(d0, d1) < -0.5f ? -1 : best;
    };
    auto vtx = [&](int64_t v) { return mk(R->V[3 * v], R->V[3 * v + 1], R->V[3 * v + 2]); };
    std::vector<std::vector<int32_t>> faces(na);
    std::vector<int64_t> skipped(na, 0);
#pragma omp parallel for schedule(dynamic, 256) num_threads(nth)
    for (int64_t r = 0; r < na; ++r) {
        const int64_t c = R->cells[r];
        const int i = (int)(c % cx), j = (int)((c / cx) % cy), k = (int)(c / ((int64_t)cx * cy));
        for (int axis = 0; axis < 3; ++axis) {
            // X needs j,k >= 1; Y needs i,k >= 1; Z needs i,j >= 1 (:866, :887, :908)
            if (axis == 0 && !(j >= 1 && k >= 1 && i < nx - 1)) continue;
            if (axis == 1 && !(i >= 1 && k >= 1 && j < ny - 1)) continue;
            if (axis == 2 && !(i >= 1 && j >= 1 && k < nz - 1)) continue;
            const int i1 = i + (axis == 0), j1 = j + (axis == 1), k1 = k + (axis == 2);
            const float s0 = g.at(i, j, k), s1 = g.at(i1, j1, k1);
            const bool crossing = s0 * s1 < 0.0f;
            const bool thin = !crossing && g.thin(s0, s1, i, j, k, i1, j1, k1);
            if (!crossing && !thin) continue;
            const F3 gn = add(g.grad(i, j, k), g.grad(i1, j1, k1));
            int64_t v[4];
            if (axis == 0) { v[0] = pick(i, j - 1, k - 1, gn); v[1] = pick(i, j, k - 1, gn); v[2] = pick(i, j, k, gn); v[3] = pick(i, j - 1, k, gn); }
            else if (axis == 1) { v[0] = pick(i - 1, j, k - 1, gn); v[1] = pick(i, j, k - 1, gn); v[2] = pick(i, j, k, gn); v[3] = pick(i - 1, j, k, gn); }
            else { v[0] = pick(i - 1, j - 1, k, gn); v[1] = pick(i, j - 1, k, gn); v[2] = pick(i, j, k, gn); v[3] = pick(i - 1, j, k, gn); }
            if (v[0] < 0 || v[1] < 0 || v[2] < 0 || v[3] < 0) {
                if (mvdc) ++skipped[r];
                continue;
            }
            const F3 pa = vtx(v[0]), pb = vtx(v[1]), pc = vtx(v[2]), pd = vtx(v[3]);
            F3 qn = cross(sub(pb, pa), sub(pd, pa));
            if (dot(qn, qn) < 1e-12f) qn = cross(sub(pc, pa), sub(pd, pa));
            if (dot(gn, gn) > 0.0f && dot(qn, qn) > 0.0f && dot(qn, gn) < 0.0f) std::swap(v[1], v[3]);
            auto& f = faces[r];
            f.push_back((int32_t)v[0]); f.push_back((int32_t)v[1]); f.push_back((int32_t)v[2]); f.push_back((int32_t)v[3]);
            if (thin) {
                f.push_back((int32_t)v[0]); f.push_back((int32_t)v[3]); f.push_back((int32_t)v[2]); f.push_back((int32_t)v[1]);
            }
        }
    }
    for (int64_t r = 0; r < na; ++r) {
        R->F.insert(R->F.end(), faces[r].begin(), faces[r].end());
        if (!faces[r].empty()) R->stats[11] += skipped[r];   // the emit pass skips face-less cells (:954)
    }
    return R;
}

int64_t sdo_num_vertices(void* h) { return h ? (int64_t)((Result*)h)->V.size() / 3 : 0; }
int64_t sdo_num_faces(void* h) { return h ? (int64_t)((Result*)h)->F.size() / 4 : 0; }
int64_t sdo_num_cells(void* h) { return h ? (int64_t)((Result*)h)->cells.size() : 0; }

/* Copy results out; any pointer may be NULL. */
void sdo_copy(void* h, float* V, float* N, int32_t* F, int64_t* cells, int32_t* vstart, int64_t* stats) {
    if (!h) return;
    Result* R = (Result*)h;
    if (V) std::memcpy(V, R->V.data(), R->V.size() * sizeof(float));
    if (N) std::memcpy(N, R->N.data(), R->N.size() * sizeof(float));
    if (F) std::memcpy(F, R->F.data(), R->F.size() * sizeof(int32_t));
    if (cells) std::memcpy(cells, R->cells.data(), R->cells.size() * sizeof(int64_t));
    if (vstart) std::memcpy(vstart, R->vstart.data(), R->vstart.size() * sizeof(int32_t));
    if (stats) std::memcpy(stats, R->stats, sizeof(R->stats));
}

void sdo_free(void* h) { delete (Result*)h; }

}  // extern "C"
