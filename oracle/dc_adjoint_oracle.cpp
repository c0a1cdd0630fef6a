/*
 * dc_adjoint_oracle.cpp — TEST INFRASTRUCTURE ONLY (the oracle; never shipped, never measured
 * as the product). Only tests/ may load it.
 *
 * FP64 reference for the derivatives of the dual-contouring vertices with respect to the
 * grid values, by forward-mode automatic differentiation: the per-cell vertex of the
 * reference CPU backend is restated once as a template over its scalar type and run with
 * dual numbers that carry the 64 partial derivatives with respect to the values of the
 * cell's 4x4x4 stencil (grid points i-1..i+2, j-1..j+2, k-1..k+2). The Jacobian that comes
 * out is exact for the arithmetic as written, including the Jacobi iterations, so it checks
 * the engine's hand-derived implicit adjoint without sharing any of its algebra.
 *
 * The per-cell vertex restated (run with double it is the FP64 vertex, used for central
 * finite differences on a double-valued grid):
 *   Hermite samples      Cell.cpp:162-212 (lerp_t :49-52, trilinear gradient :80-155)
 *   4-cell averaging     hermite_update.cpp:171-438 (an edge strictly inside the grid whose
 *                        four cells are active with a sample on it takes the normalised sum
 *                        of their own normals)
 *   QEF                  Cell::update Cell.cpp:284-320, solve_quadratic_system :324-361,
 *                        getCentroid :586-600 (A^T A and A^T b in edge order, truncated
 *                        pseudo-inverse about the centroid)
 * The Jacobi eigen-decomposition is the cyclic one of oracle/dc_oracle.cpp, with two changes
 * that keep the derivatives exact and leave values unchanged to rounding: a rotation whose
 * pivot is tiny next to its diagonal gap uses the first-order angle t = a_pq/(a_qq - a_pp),
 * and sweeps continue until the off-diagonal derivatives have converged too.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int N = 64;

struct Dual {
    double v;
    double d[N];
};

inline Dual mk(double v) { Dual r; r.v = v; std::memset(r.d, 0, sizeof r.d); return r; }
inline Dual operator+(const Dual& a, const Dual& b) { Dual r; r.v = a.v + b.v; for (int q = 0; q < N; ++q) r.d[q] = a.d[q] + b.d[q]; return r; }
inline Dual operator-(const Dual& a, const Dual& b) { Dual r; r.v = a.v - b.v; for (int q = 0; q < N; ++q) r.d[q] = a.d[q] - b.d[q]; return r; }
inline Dual operator-(const Dual& a) { Dual r; r.v = -a.v; for (int q = 0; q < N; ++q) r.d[q] = -a.d[q]; return r; }
inline Dual operator*(const Dual& a, const Dual& b) { Dual r; r.v = a.v * b.v; for (int q = 0; q < N; ++q) r.d[q] = a.d[q] * b.v + a.v * b.d[q]; return r; }
inline Dual operator/(const Dual& a, const Dual& b) {
    Dual r; r.v = a.v / b.v;
    const double ib = 1.0 / b.v;
    for (int q = 0; q < N; ++q) r.d[q] = (a.d[q] - r.v * b.d[q]) * ib;
    return r;
}
inline Dual operator+(const Dual& a, double b) { Dual r = a; r.v += b; return r; }
inline Dual operator+(double a, const Dual& b) { return b + a; }
inline Dual operator-(const Dual& a, double b) { Dual r = a; r.v -= b; return r; }
inline Dual operator-(double a, const Dual& b) { Dual r = -b; r.v += a; return r; }
inline Dual operator*(const Dual& a, double b) { Dual r; r.v = a.v * b; for (int q = 0; q < N; ++q) r.d[q] = a.d[q] * b; return r; }
inline Dual operator*(double a, const Dual& b) { return b * a; }
inline Dual operator/(const Dual& a, double b) { Dual r; r.v = a.v / b; for (int q = 0; q < N; ++q) r.d[q] = a.d[q] / b; return r; }
inline Dual operator/(double a, const Dual& b) { return mk(a) / b; }
inline Dual dsqrt(const Dual& a) {
    Dual r; r.v = std::sqrt(a.v);
    const double k = r.v > 0.0 ? 0.5 / r.v : 0.0;
    for (int q = 0; q < N; ++q) r.d[q] = a.d[q] * k;
    return r;
}
inline Dual dabs(const Dual& a) { return a.v < 0.0 ? -a : a; }
inline double val(const Dual& a) { return a.v; }
inline double dnorm2(const Dual& a) { double s = 0.0; for (int q = 0; q < N; ++q) s += a.d[q] * a.d[q]; return s; }

inline double dsqrt(double a) { return std::sqrt(a); }
inline double dabs(double a) { return std::fabs(a); }
inline double val(double a) { return a; }
inline double dnorm2(double) { return 0.0; }

template <typename T> inline T make(double v);
template <> inline double make<double>(double v) { return v; }
template <> inline Dual make<Dual>(double v) { return mk(v); }

const int kOff[8][3] = {{0,0,0},{1,0,0},{1,1,0},{0,1,0},{0,0,1},{1,0,1},{1,1,1},{0,1,1}};
const int kEdge[12][2] = {{0,1},{1,2},{2,3},{3,0},{4,5},{5,6},{6,7},{7,4},{0,4},{1,5},{2,6},{3,7}};

struct GridD {
    int nx, ny, nz;
    const double* gx; const double* gy; const double* gz;
    const float* vf; const double* vd;
    double S(int i, int j, int k) const {
        const int64_t p = i + (int64_t)nx * (j + (int64_t)ny * k);
        return vd ? vd[p] : (double)vf[p];
    }
};

template <typename T> struct CellT {
    T cs[8];
    double cp[8][3];
};

// Corner values of cell (ci,cj,ck); with dual numbers each is seeded with its slot in the
// stencil of the centre cell (i,j,k).
template <typename T>
void load(const GridD& g, int ci, int cj, int ck, int i, int j, int k, CellT<T>& C);

template <> void load<double>(const GridD& g, int ci, int cj, int ck, int, int, int, CellT<double>& C) {
    for (int c = 0; c < 8; ++c) {
        const int gi = ci + kOff[c][0], gj = cj + kOff[c][1], gk = ck + kOff[c][2];
        C.cs[c] = g.S(gi, gj, gk);
        C.cp[c][0] = g.gx[gi]; C.cp[c][1] = g.gy[gj]; C.cp[c][2] = g.gz[gk];
    }
}
template <> void load<Dual>(const GridD& g, int ci, int cj, int ck, int i, int j, int k, CellT<Dual>& C) {
    for (int c = 0; c < 8; ++c) {
        const int gi = ci + kOff[c][0], gj = cj + kOff[c][1], gk = ck + kOff[c][2];
        C.cs[c] = mk(g.S(gi, gj, gk));
        const int slot = (gi - i + 1) + 4 * (gj - j + 1) + 16 * (gk - k + 1);
        C.cs[c].d[slot] = 1.0;
        C.cp[c][0] = g.gx[gi]; C.cp[c][1] = g.gy[gj]; C.cp[c][2] = g.gz[gk];
    }
}

template <typename T> bool is_active(const CellT<T>& C) {
    bool neg = false, pos = false;
    for (int c = 0; c < 8; ++c) { if (val(C.cs[c]) < 0) neg = true; if (val(C.cs[c]) > 0) pos = true; }
    return neg && pos;
}

template <typename T> T sq3(const T* a) { return a[0] * a[0] + a[1] * a[1] + a[2] * a[2]; }
template <typename T> void normalize3(T* a) {
    const T z = sq3(a);
    if (val(z) > 0.0) { const T s = dsqrt(z); a[0] = a[0] / s; a[1] = a[1] / s; a[2] = a[2] / s; }
}

// Cell.cpp:80-155.
template <typename T> void tri_grad(const CellT<T>& C, const T p[3], T g[3]) {
    const T &S000 = C.cs[0], &S100 = C.cs[1], &S110 = C.cs[2], &S010 = C.cs[3];
    const T &S001 = C.cs[4], &S101 = C.cs[5], &S111 = C.cs[6], &S011 = C.cs[7];
    const double x0 = C.cp[0][0], x1 = C.cp[1][0], y0 = C.cp[0][1], y1 = C.cp[3][1];
    const double z0 = C.cp[0][2], z1 = C.cp[4][2];
    const double dx = x1 - x0, dy = y1 - y0, dz = z1 - z0, eps = 1e-12;
    T u = make<T>(0.5), v = make<T>(0.5), w = make<T>(0.5);
    if (std::fabs(dx) > eps) u = (p[0] - x0) / dx;
    if (std::fabs(dy) > eps) v = (p[1] - y0) / dy;
    if (std::fabs(dz) > eps) w = (p[2] - z0) / dz;
    if (val(u) < 0.0) u = make<T>(0.0); else if (val(u) > 1.0) u = make<T>(1.0);
    if (val(v) < 0.0) v = make<T>(0.0); else if (val(v) > 1.0) v = make<T>(1.0);
    if (val(w) < 0.0) w = make<T>(0.0); else if (val(w) > 1.0) w = make<T>(1.0);
    const T omu = 1.0 - u, omv = 1.0 - v, omw = 1.0 - w;
    const T df_du = (S100 - S000) * omv * omw + (S110 - S010) * v * omw + (S101 - S001) * omv * w + (S111 - S011) * v * w;
    const T df_dv = (S010 - S000) * omu * omw + (S110 - S100) * u * omw + (S011 - S001) * omu * w + (S111 - S101) * u * w;
    const T df_dw = (S001 - S000) * omu * omv + (S101 - S100) * u * omv + (S011 - S010) * omu * v + (S111 - S110) * u * v;
    g[0] = g[1] = g[2] = make<T>(0.0);
    if (std::fabs(dx) > eps) g[0] = df_du / dx;
    if (std::fabs(dy) > eps) g[1] = df_dv / dy;
    if (std::fabs(dz) > eps) g[2] = df_dw / dz;
}

// Cell.cpp:176-212.
template <typename T> bool hermite(const CellT<T>& C, int e, T p[3], T n[3]) {
    const int a = kEdge[e][0], b = kEdge[e][1];
    const T &fa = C.cs[a], &fb = C.cs[b];
    if (val(fa) * val(fb) > 0.0) return false;
    const T t = (fa - 0.0) / (fa - fb + 1e-16);
    for (int d = 0; d < 3; ++d) p[d] = (1.0 - t) * C.cp[a][d] + t * C.cp[b][d];
    tri_grad(C, p, n);
    if (val(dsqrt(sq3(n))) > 0.0) normalize3(n);
    return true;
}

// Local edge of a cell for a grid edge along `axis` at perpendicular offsets (l1, l2).
int local_edge(int axis, int l1, int l2) {
    const int q = l1 + 2 * l2;
    if (axis == 0) return 2 * q;
    if (axis == 1) return q == 0 ? 3 : q == 1 ? 1 : q == 2 ? 7 : 5;
    return q == 0 ? 8 : q == 1 ? 9 : q == 2 ? 11 : 10;
}

template <typename T>
bool edge_sample(const GridD& g, const CellT<T>& C, int i, int j, int k, int e, T p[3], T n[3]) {
    if (!hermite(C, e, p, n)) return false;
    const int a = kEdge[e][0], b = kEdge[e][1];
    const int Pa[3] = {i + kOff[a][0], j + kOff[a][1], k + kOff[a][2]};
    const int Pb[3] = {i + kOff[b][0], j + kOff[b][1], k + kOff[b][2]};
    int Pm[3], PM[3];
    for (int d = 0; d < 3; ++d) { Pm[d] = Pa[d] < Pb[d] ? Pa[d] : Pb[d]; PM[d] = Pa[d] < Pb[d] ? Pb[d] : Pa[d]; }
    const bool in0 = Pm[0] > 0 && Pm[0] < g.nx - 1 && Pm[1] > 0 && Pm[1] < g.ny - 1 && Pm[2] > 0 && Pm[2] < g.nz - 1;
    const bool in1 = PM[0] > 0 && PM[0] < g.nx - 1 && PM[1] > 0 && PM[1] < g.ny - 1 && PM[2] > 0 && PM[2] < g.nz - 1;
    if (!in0 && !in1) return true;
    const int axis = Pa[0] != Pb[0] ? 0 : (Pa[1] != Pb[1] ? 1 : 2);
    const int d1 = axis == 0 ? 1 : 0, d2 = axis == 2 ? 1 : 2;
    T nq[4][3];
    for (int q = 0; q < 4; ++q) {
        int cc[3] = {Pm[0], Pm[1], Pm[2]};
        if (q & 1) cc[d1] -= 1;
        if (q & 2) cc[d2] -= 1;
        if (cc[0] == i && cc[1] == j && cc[2] == k) { for (int d = 0; d < 3; ++d) nq[q][d] = n[d]; continue; }
        CellT<T> X;
        load<T>(g, cc[0], cc[1], cc[2], i, j, k, X);
        if (!is_active(X)) return true;
        T px[3];
        if (!hermite(X, local_edge(axis, Pm[d1] - cc[d1], Pm[d2] - cc[d2]), px, nq[q])) return true;
    }
    T acc[3] = {make<T>(0.0), make<T>(0.0), make<T>(0.0)};
    for (int q = 0; q < 4; ++q)
        if (val(dsqrt(sq3(nq[q]))) > 0) for (int d = 0; d < 3; ++d) acc[d] = acc[d] + nq[q][d];
    normalize3(acc);
    for (int d = 0; d < 3; ++d) n[d] = acc[d];
    return true;
}

template <typename T> void jacobi(T a[3][3], T V[3][3]) {
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) V[r][c] = make<T>(r == c ? 1.0 : 0.0);
    for (int sweep = 0; sweep < 64; ++sweep) {
        const double off = val(a[0][1]) * val(a[0][1]) + val(a[0][2]) * val(a[0][2]) + val(a[1][2]) * val(a[1][2]);
        const double diag = val(a[0][0]) * val(a[0][0]) + val(a[1][1]) * val(a[1][1]) + val(a[2][2]) * val(a[2][2]);
        const double doff = dnorm2(a[0][1]) + dnorm2(a[0][2]) + dnorm2(a[1][2]);
        const double dall = doff + dnorm2(a[0][0]) + dnorm2(a[1][1]) + dnorm2(a[2][2]);
        if ((off <= 1e-30 * diag || off == 0.0) && doff <= 1e-30 * dall) break;
        for (int p = 0; p < 2; ++p) {
            for (int q = p + 1; q < 3; ++q) {
                const T apq = a[p][q];
                if (val(apq) == 0.0 && dnorm2(apq) == 0.0) continue;
                const T gap = a[q][q] - a[p][p];
                T t;
                if (std::fabs(val(apq)) < 1e-8 * std::fabs(val(gap))) {
                    t = apq / gap;                             // first order in a_pq
                } else if (val(apq) == 0.0) {
                    continue;                                  // degenerate pair: no direction
                } else {
                    const T theta = gap / (2.0 * apq);
                    const T at = dabs(theta);
                    t = (val(theta) >= 0.0 ? 1.0 : -1.0) / (at + dsqrt(theta * theta + 1.0));
                }
                const T c = 1.0 / dsqrt(t * t + 1.0), s = t * c;
                for (int r = 0; r < 3; ++r) {
                    const T arp = a[r][p], arq = a[r][q];
                    a[r][p] = c * arp - s * arq;
                    a[r][q] = s * arp + c * arq;
                }
                for (int r = 0; r < 3; ++r) {
                    const T apr = a[p][r], aqr = a[q][r];
                    a[p][r] = c * apr - s * aqr;
                    a[q][r] = s * apr + c * aqr;
                }
                for (int r = 0; r < 3; ++r) {
                    const T vrp = V[r][p], vrq = V[r][q];
                    V[r][p] = c * vrp - s * vrq;
                    V[r][q] = s * vrp + c * vrq;
                }
            }
        }
    }
}

// The vertex of active cell (i,j,k) and the number of eigenvalues its solve keeps; returns
// false if it has no Hermite sample.
template <typename T> bool cell_vertex(const GridD& g, int i, int j, int k, double thr, T out[3], int* kept = nullptr) {
    CellT<T> C;
    load<T>(g, i, j, k, i, j, k, C);
    T A[3][3], ATb[3], c[3];
    for (int r = 0; r < 3; ++r) { ATb[r] = make<T>(0.0); c[r] = make<T>(0.0); for (int s = 0; s < 3; ++s) A[r][s] = make<T>(0.0); }
    int m = 0;
    for (int e = 0; e < 12; ++e) {
        T p[3], n[3];
        if (!edge_sample(g, C, i, j, k, e, p, n)) continue;
        if (val(dsqrt(sq3(n))) > 0.0) normalize3(n);
        const T b = n[0] * p[0] + n[1] * p[1] + n[2] * p[2];
        for (int r = 0; r < 3; ++r) {
            for (int s = 0; s < 3; ++s) A[r][s] = A[r][s] + n[r] * n[s];
            ATb[r] = ATb[r] + n[r] * b;
        }
        for (int d = 0; d < 3; ++d) c[d] = c[d] + p[d];
        ++m;
    }
    if (m == 0) return false;
    for (int d = 0; d < 3; ++d) c[d] = c[d] / double(m);
    T E[3][3], V[3][3];
    for (int r = 0; r < 3; ++r) for (int s = 0; s < 3; ++s) E[r][s] = A[r][s];
    jacobi(E, V);
    T rhs[3];
    for (int r = 0; r < 3; ++r) rhs[r] = ATb[r] - (A[r][0] * c[0] + A[r][1] * c[1] + A[r][2] * c[2]);
    for (int d = 0; d < 3; ++d) out[d] = c[d];
    if (kept) *kept = 0;
    for (int q = 0; q < 3; ++q) {
        const T sv = dabs(E[q][q]);
        if (val(sv) > thr) {
            if (kept) ++*kept;
            const T coef = (V[0][q] * rhs[0] + V[1][q] * rhs[1] + V[2][q] * rhs[2]) / sv;
            for (int d = 0; d < 3; ++d) out[d] = out[d] + V[d][q] * coef;
        }
    }
    return true;
}

GridD make_grid(int nx, int ny, int nz, const double* px, const double* py, const double* pz,
                const float* vf, const double* vd) {
    GridD g;
    g.nx = nx; g.ny = ny; g.nz = nz; g.gx = px; g.gy = py; g.gz = pz; g.vf = vf; g.vd = vd;
    return g;
}

void unpack(const GridD& g, int64_t c, int& i, int& j, int& k) {
    const int64_t cx = g.nx - 1, cy = g.ny - 1;
    i = (int)(c % cx); j = (int)((c / cx) % cy); k = (int)(c / (cx * cy));
}

}  // namespace

extern "C" {

/*
 * FP64 vertices of the listed active cells (linear index i + cx*(j + cy*k)) of a grid with
 * float (vf) or double (vd) values and explicit grid-point coordinates px[nx], py[ny],
 * pz[nz]. out: 3 doubles per cell; kept (optional): the eigenvalues each solve keeps.
 * Returns 0, or -1 on invalid input.
 */
int dca_cell_vertices(int nx, int ny, int nz, const double* px, const double* py, const double* pz,
                      const float* vf, const double* vd, const int64_t* cells, int64_t n, double thr,
                      double* out, int* kept, int threads) {
    if (nx < 2 || ny < 2 || nz < 2 || (!vf && !vd) || !px || !py || !pz) return -1;
    const GridD g = make_grid(nx, ny, nz, px, py, pz, vf, vd);
#ifdef _OPENMP
    const int nth = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for num_threads(nth) schedule(dynamic, 64)
#endif
    for (int64_t r = 0; r < n; ++r) {
        int i, j, k;
        unpack(g, cells[r], i, j, k);
        double v[3] = {NAN, NAN, NAN};
        int kr = 0;
        cell_vertex<double>(g, i, j, k, thr, v, &kr);
        if (kept) kept[r] = kr;
        for (int d = 0; d < 3; ++d) out[3 * r + d] = v[d];
    }
    (void)threads;
    return 0;
}

/*
 * Jacobians of the listed cells' FP64 vertices with respect to the values of their 4x4x4
 * stencils: jac[r][d][s] = d vertex_d / d value(i-1+s%4, j-1+(s/4)%4, k-1+s/16). Also the
 * vertices (out, 3 per cell). Returns 0, or -1 on invalid input.
 */
int dca_cell_jacobians(int nx, int ny, int nz, const double* px, const double* py, const double* pz,
                       const float* vf, const double* vd, const int64_t* cells, int64_t n, double thr,
                       double* out, double* jac, int threads) {
    if (nx < 2 || ny < 2 || nz < 2 || (!vf && !vd) || !px || !py || !pz) return -1;
    const GridD g = make_grid(nx, ny, nz, px, py, pz, vf, vd);
#ifdef _OPENMP
    const int nth = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for num_threads(nth) schedule(dynamic, 16)
#endif
    for (int64_t r = 0; r < n; ++r) {
        int i, j, k;
        unpack(g, cells[r], i, j, k);
        Dual v[3] = {mk(NAN), mk(NAN), mk(NAN)};
        cell_vertex<Dual>(g, i, j, k, thr, v);
        for (int d = 0; d < 3; ++d) {
            out[3 * r + d] = v[d].v;
            for (int s = 0; s < N; ++s) jac[(r * 3 + d) * N + s] = v[d].d[s];
        }
    }
    (void)threads;
    return 0;
}

}  // extern "C"
