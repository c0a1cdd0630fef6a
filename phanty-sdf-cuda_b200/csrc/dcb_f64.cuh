// dcb_f64.cuh — FP64 restatement of the reference CPU backend's per-cell arithmetic, shared by
// the FP64 vertex path, the adjoint and the refinement. Every translation unit that includes
// it is compiled with --fmad=false, so each double operation is rounded as written, like the
// reference's x86-64 build (Cell.cpp:57-361, hermite_update.cpp:171-438,
// contouring.cpp:141-207).
#pragma once
#include "dcb_kernels.cuh"

namespace dcb {
namespace f64 {

struct Cell64 {
    double cs[8];
    double cp[8][3];
};

__device__ __forceinline__ double sq3(const double* a) { return a[0] * a[0] + a[1] * a[1] + a[2] * a[2]; }
__device__ __forceinline__ void normalize3(double* a) {
    const double z = sq3(a);
    if (z > 0.0) { const double s = sqrt(z); a[0] /= s; a[1] /= s; a[2] /= s; }
}

__device__ inline void load_cell(const GridDesc& g, int i, int j, int k, Cell64& C) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int gi = i + corner_dx(c), gj = j + corner_dy(c), gk = k + corner_dz(c);
        C.cs[c] = (double)__ldg(g.v + pidx(g, gi, gj, gk));
        C.cp[c][0] = (double)pos_axis(g.ox, g.vx, gi);
        C.cp[c][1] = (double)pos_axis(g.oy, g.vy, gj);
        C.cp[c][2] = (double)pos_axis(g.oz, g.vz, gk);
    }
}

__device__ inline bool active(const Cell64& C) {
    bool neg = false, pos = false;
    for (int c = 0; c < 8; ++c) { if (C.cs[c] < 0) neg = true; if (C.cs[c] > 0) pos = true; }
    return neg && pos;
}

// gradientAtPointUsingTrilinear (Cell.cpp:80-155).
__device__ inline void tri_grad(const Cell64& C, const double p[3], double g[3]) {
    const double S000 = C.cs[0], S100 = C.cs[1], S110 = C.cs[2], S010 = C.cs[3];
    const double S001 = C.cs[4], S101 = C.cs[5], S111 = C.cs[6], S011 = C.cs[7];
    const double x0 = C.cp[0][0], x1 = C.cp[1][0];
    const double y0 = C.cp[0][1], y1 = C.cp[3][1];
    const double z0 = C.cp[0][2], z1 = C.cp[4][2];
    const double dx = x1 - x0, dy = y1 - y0, dz = z1 - z0;
    const double eps = 1e-12;
    double u = 0.5, v = 0.5, w = 0.5;
    if (fabs(dx) > eps) u = (p[0] - x0) / dx;
    if (fabs(dy) > eps) v = (p[1] - y0) / dy;
    if (fabs(dz) > eps) w = (p[2] - z0) / dz;
    u = fmax(0.0, fmin(1.0, u));
    v = fmax(0.0, fmin(1.0, v));
    w = fmax(0.0, fmin(1.0, w));
    const double omu = 1.0 - u, omv = 1.0 - v, omw = 1.0 - w;
    const double df_du = (S100 - S000) * omv * omw + (S110 - S010) * v * omw
                       + (S101 - S001) * omv * w + (S111 - S011) * v * w;
    const double df_dv = (S010 - S000) * omu * omw + (S110 - S100) * u * omw
                       + (S011 - S001) * omu * w + (S111 - S101) * u * w;
    const double df_dw = (S001 - S000) * omu * omv + (S101 - S100) * u * omv
                       + (S011 - S010) * omu * v + (S111 - S110) * u * v;
    g[0] = g[1] = g[2] = 0.0;
    if (fabs(dx) > eps) g[0] = df_du / dx;
    if (fabs(dy) > eps) g[1] = df_dv / dy;
    if (fabs(dz) > eps) g[2] = df_dw / dz;
}

// Hermite sample of local edge e of a cell (Cell.cpp:176-212). Returns false if no crossing.
__device__ inline bool hermite(const Cell64& C, int e, double p[3], double n[3]) {
    const int a = edge_a(e), b = edge_b(e);
    const double fa = C.cs[a], fb = C.cs[b];
    if (fa * fb > 0.0) return false;
    const double t = (fa - 0.0) / (fa - fb + 1e-16);
    for (int d = 0; d < 3; ++d) p[d] = (1.0 - t) * C.cp[a][d] + t * C.cp[b][d];
    tri_grad(C, p, n);
    if (sqrt(sq3(n)) > 0.0) normalize3(n);
    return true;
}

// The cell's local index of a grid edge along `axis` at local perpendicular coordinates
// (l1, l2) in {0,1}: the unique match get_edge_idx_from_grid_vertices finds, as a table.
__device__ __forceinline__ int local_edge(int axis, int l1, int l2) {
    const int q = l1 + 2 * l2;
    if (axis == 0) return 2 * q;                          // (y,z): 00->0 10->2 01->4 11->6
    if (axis == 1) return q == 0 ? 3 : q == 1 ? 1 : q == 2 ? 7 : 5;   // (x,z)
    return q == 0 ? 8 : q == 1 ? 9 : q == 2 ? 11 : 10;    // (x,y)
}

// Hermite sample of edge e of cell (i,j,k) with the 4-cell averaged normal when the edge
// qualifies (hermite_update.cpp:171-438).
__device__ inline bool edge_sample(const GridDesc& g, const Cell64& C, int i, int j, int k, int e, double p[3], double n[3]) {
    if (!hermite(C, e, p, n)) return false;
    const int a = edge_a(e), b = edge_b(e);
    const int Pa[3] = {i + corner_dx(a), j + corner_dy(a), k + corner_dz(a)};
    const int Pb[3] = {i + corner_dx(b), j + corner_dy(b), k + corner_dz(b)};
    int Pm[3], PM[3];
    for (int d = 0; d < 3; ++d) { Pm[d] = min(Pa[d], Pb[d]); PM[d] = max(Pa[d], Pb[d]); }
    const bool in0 = Pm[0] > 0 && Pm[0] < g.nx - 1 && Pm[1] > 0 && Pm[1] < g.ny - 1 && Pm[2] > 0 && Pm[2] < g.nz - 1;
    const bool in1 = PM[0] > 0 && PM[0] < g.nx - 1 && PM[1] > 0 && PM[1] < g.ny - 1 && PM[2] > 0 && PM[2] < g.nz - 1;
    if (!in0 && !in1) return true;
    const int axis = Pa[0] != Pb[0] ? 0 : (Pa[1] != Pb[1] ? 1 : 2);
    const int d1 = axis == 0 ? 1 : 0;
    const int d2 = axis == 2 ? 1 : 2;
    double nq[4][3];
    for (int q = 0; q < 4; ++q) {
        int cc[3] = {Pm[0], Pm[1], Pm[2]};
        if (q & 1) cc[d1] -= 1;
        if (q & 2) cc[d2] -= 1;
        if (cc[0] == i && cc[1] == j && cc[2] == k) {
            nq[q][0] = n[0]; nq[q][1] = n[1]; nq[q][2] = n[2];
            continue;
        }
        Cell64 X;
        load_cell(g, cc[0], cc[1], cc[2], X);
        if (!active(X)) return true;
        const int ex = local_edge(axis, Pm[d1] - cc[d1], Pm[d2] - cc[d2]);
        double px[3];
        if (ex < 0 || !hermite(X, ex, px, nq[q])) return true;
    }
    double acc[3] = {0.0, 0.0, 0.0};
    for (int q = 0; q < 4; ++q) {
        if (sqrt(sq3(nq[q])) > 0) { acc[0] += nq[q][0]; acc[1] += nq[q][1]; acc[2] += nq[q][2]; }
    }
    normalize3(acc);
    n[0] = acc[0]; n[1] = acc[1]; n[2] = acc[2];
    return true;
}

// Cyclic Jacobi, same sweep order and stopping rule as the CPU restatement.
__device__ inline void jacobi3(double a[3][3], double V[3][3]) {
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) V[r][c] = (r == c) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 64; ++sweep) {
        const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        const double diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (off <= 1e-30 * diag || off == 0.0) break;
        // unrolled: a and V stay in registers (the order of the rotations is unchanged)
#pragma unroll
        for (int p = 0; p < 2; ++p) {
#pragma unroll
            for (int q = p + 1; q < 3; ++q) {
                const double apq = a[p][q];
                if (apq == 0.0) continue;
                const double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int r = 0; r < 3; ++r) {
                    const double arp = a[r][p], arq = a[r][q];
                    a[r][p] = c * arp - s * arq;
                    a[r][q] = s * arp + c * arq;
                }
                for (int r = 0; r < 3; ++r) {
                    const double apr = a[p][r], aqr = a[q][r];
                    a[p][r] = c * apr - s * aqr;
                    a[q][r] = s * apr + c * aqr;
                }
                for (int r = 0; r < 3; ++r) {
                    const double vrp = V[r][p], vrq = V[r][q];
                    V[r][p] = c * vrp - s * vrq;
                    V[r][q] = s * vrp + c * vrq;
                }
            }
        }
    }
}

// Solve of Cell.cpp:318-361 for summed rows (A^T A, A^T b, sum of the m Hermite points):
// the Jacobi eigen-decomposition and the pseudo-inverse truncated at thr, about the centroid.
__device__ inline void solve_about_centroid(const double ATA[3][3], const double ATb[3], double c[3], int m,
                                            double thr, double out[3]) {
    for (int d = 0; d < 3; ++d) c[d] /= double(m);
    double A[3][3], V[3][3];
    for (int r = 0; r < 3; ++r) for (int s = 0; s < 3; ++s) A[r][s] = ATA[r][s];
    jacobi3(A, V);
    const double lam[3] = {A[0][0], A[1][1], A[2][2]};
    double rhs[3];
    for (int r = 0; r < 3; ++r) rhs[r] = ATb[r] - (ATA[r][0] * c[0] + ATA[r][1] * c[1] + ATA[r][2] * c[2]);
    double x[3] = {c[0], c[1], c[2]};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const double sv = fabs(lam[q]);
        if (sv > thr) {
            const double proj = V[0][q] * rhs[0] + V[1][q] * rhs[1] + V[2][q] * rhs[2];
            const double coef = proj / sv;
            for (int d = 0; d < 3; ++d) x[d] += V[d][q] * coef;
        }
    }
    out[0] = x[0]; out[1] = x[1]; out[2] = x[2];
}

// FP64 vertex of active cell (i,j,k), by one thread: Hermite samples with their averaged
// normals in edge order (the CPU's std::map order), A^T A, A^T b and the centroid summed in
// that order, then the Jacobi eigen-decomposition and the truncated pseudo-inverse about the
// centroid (Cell.cpp:284-361). A thread per cell keeps every lane busy on the serial solve.
__device__ inline void cell_vertex_thread(const GridDesc& g, int i, int j, int k, double thr, double out[3]) {
    Cell64 C;
    load_cell(g, i, j, k, C);
    double ATA[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, ATb[3] = {0, 0, 0}, c[3] = {0, 0, 0};
    int m = 0;
    for (int e = 0; e < 12; ++e) {
        double p[3], n[3];
        if (!edge_sample(g, C, i, j, k, e, p, n)) continue;
        // Cell::update row (Cell.cpp:298-311): normalise, b = n.p
        if (sqrt(sq3(n)) > 0.0) normalize3(n);
        const double bb = n[0] * p[0] + n[1] * p[1] + n[2] * p[2];
        for (int r = 0; r < 3; ++r) {
            for (int s = 0; s < 3; ++s) ATA[r][s] += n[r] * n[s];
            ATb[r] += n[r] * bb;
        }
        for (int d = 0; d < 3; ++d) c[d] += p[d];
        ++m;
    }
    solve_about_centroid(ATA, ATb, c, m, thr, out);
}

// gradientAt (contouring.cpp:141-207).
__device__ inline void grid_gradient(const GridDesc& g, int i, int j, int k, double out[3]) {
    const int im = max(i - 1, 0), ip = min(i + 1, g.nx - 1);
    const int jm = max(j - 1, 0), jp = min(j + 1, g.ny - 1);
    const int km = max(k - 1, 0), kp = min(k + 1, g.nz - 1);
    out[0] = out[1] = out[2] = 0.0;
    const double dx = (double)pos_axis(g.ox, g.vx, ip) - (double)pos_axis(g.ox, g.vx, im);
    if (fabs(dx) > 1e-12) out[0] = ((double)__ldg(g.v + pidx(g, ip, j, k)) - (double)__ldg(g.v + pidx(g, im, j, k))) / dx;
    const double dy = (double)pos_axis(g.oy, g.vy, jp) - (double)pos_axis(g.oy, g.vy, jm);
    if (fabs(dy) > 1e-12) out[1] = ((double)__ldg(g.v + pidx(g, i, jp, k)) - (double)__ldg(g.v + pidx(g, i, jm, k))) / dy;
    const double dz = (double)pos_axis(g.oz, g.vz, kp) - (double)pos_axis(g.oz, g.vz, km);
    if (fabs(dz) > 1e-12) out[2] = ((double)__ldg(g.v + pidx(g, i, j, kp)) - (double)__ldg(g.v + pidx(g, i, j, km))) / dz;
    const double nrm = sqrt(sq3(out));
    if (nrm > 0.0) { out[0] /= nrm; out[1] /= nrm; out[2] /= nrm; }
}

// The four cells of an averaged edge (hermite_update.cpp:171-332) in the CPU's sum order:
// q = 0 the cell at the edge's minimum endpoint, 1 = -d1, 2 = -d2, 3 = both.
__device__ inline bool edge_cells(const GridDesc& g, int i, int j, int k, int e, int cc[4][3], int ex[4]) {
    const int a = edge_a(e), b = edge_b(e);
    const int Pa[3] = {i + corner_dx(a), j + corner_dy(a), k + corner_dz(a)};
    const int Pb[3] = {i + corner_dx(b), j + corner_dy(b), k + corner_dz(b)};
    int Pm[3], PM[3];
    for (int d = 0; d < 3; ++d) { Pm[d] = min(Pa[d], Pb[d]); PM[d] = max(Pa[d], Pb[d]); }
    const bool in0 = Pm[0] > 0 && Pm[0] < g.nx - 1 && Pm[1] > 0 && Pm[1] < g.ny - 1 && Pm[2] > 0 && Pm[2] < g.nz - 1;
    const bool in1 = PM[0] > 0 && PM[0] < g.nx - 1 && PM[1] > 0 && PM[1] < g.ny - 1 && PM[2] > 0 && PM[2] < g.nz - 1;
    if (!in0 && !in1) return false;
    const int axis = Pa[0] != Pb[0] ? 0 : (Pa[1] != Pb[1] ? 1 : 2);
    const int d1 = axis == 0 ? 1 : 0;
    const int d2 = axis == 2 ? 1 : 2;
    for (int q = 0; q < 4; ++q) {
        cc[q][0] = Pm[0]; cc[q][1] = Pm[1]; cc[q][2] = Pm[2];
        if (q & 1) cc[q][d1] -= 1;
        if (q & 2) cc[q][d2] -= 1;
        ex[q] = local_edge(axis, Pm[d1] - cc[q][d1], Pm[d2] - cc[q][d2]);
    }
    return true;
}

}  // namespace f64
}  // namespace dcb
