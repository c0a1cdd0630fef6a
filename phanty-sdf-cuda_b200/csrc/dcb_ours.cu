// dcb_ours.cu — the outer/inner vertex refinement ("Ours", contouring.cpp:1255-1328) on the GPU.
//
// Starting from a dual-contouring extraction (cells, vertices, quads), every outer iteration:
//   1. winds the quads with the current vertices and triangulates them (triangulate_v1 with
//      orient_triangles_for_quad, contouring.cpp:40-113),
//   2. builds a BVH over those triangles (Morton-sorted leaves, radix tree after Karras 2012,
//      boxes bottom-up) and finds for every selected grid point — all points with
//      |S| < 3 * cell diagonal, filled up to batch_size with seeded random others
//      (assign_spheres_to_cells, contouring.cpp:807-933) — its closest point on the mesh; a
//      sphere (centre = grid point, radius |S|) goes to the active cell holding that point
//      unless it floats more than a cell diagonal off the mesh; each cell's spheres are
//      ordered by radius,
//   3. intersects every cell's segments to its six face neighbours' vertices with the shared
//      faces and blends them into the cell's face points (compute_face_cell_intersections,
//      contouring.cpp:1081-1183),
//   4. from the second iteration on, fits a plane (PCA) to the four vertices around every
//      averaged Hermite edge and blends its normal and its crossing with the edge into the
//      four cells' Hermite data (update_hermite_points_and_normals, hermite_update.cpp:441-607),
//   5. runs each cell's inner loop: the local fan of triangles (vertex, Hermite point, face
//      point), every sphere's closest point on it and its barycentric coordinates
//      (vertex_refinement.cpp:110-280), and the regularised QEF with Hermite, sphere and
//      proximal rows (Cell::minimize_qef, Cell.cpp:364-473), until the vertex moves less
//      than 1e-6 (contouring.cpp:1288-1309).
// Everything is FP64 and compiled with --fmad=false, like the CPU restatement it is checked
// against. One thread per cell (steps 3-5), per quad (1), per grid point (2).
#include <cfloat>
#include "dcb_f64.cuh"
#include "dcb_sort.cuh"

namespace dcb {

namespace {

// Corners of the six faces (vertex_refinement.cpp:12-19), faces 0:+X 1:-X 2:+Y 3:-Y 4:+Z 5:-Z.
__constant__ int kFaceCorners[6][4] = {{1, 5, 6, 2}, {0, 3, 7, 4}, {2, 6, 7, 3}, {0, 4, 5, 1}, {4, 7, 6, 5}, {0, 1, 2, 3}};

__device__ __forceinline__ int edge_of_corners(int c1, int c2) {
    for (int e = 0; e < 12; ++e) {
        const int a = edge_a(e), b = edge_b(e);
        if ((c1 == a && c2 == b) || (c1 == b && c2 == a)) return e;
    }
    return -1;
}

__device__ __forceinline__ double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
__device__ __forceinline__ double norm3(const double* a) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }
__device__ __forceinline__ void cross3(const double* a, const double* b, double* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

__device__ __forceinline__ bool active_bit(const OursParams& P, int i, int j, int k) {
    const uint32_t w = __ldg(P.bits + ((long long)j + (long long)P.g.cy * k) * P.g.W + (i >> 5));
    return (w >> (i & 31)) & 1u;
}

__device__ __forceinline__ double gpos(const GridDesc& g, int axis, int i) {
    return axis == 0 ? (double)pos_axis(g.ox, g.vx, i) : axis == 1 ? (double)pos_axis(g.oy, g.vy, i)
                                                                   : (double)pos_axis(g.oz, g.vz, i);
}

__device__ __forceinline__ void point_of(const GridDesc& g, long long gidx, double c[3]) {
    const int i = (int)(gidx % g.nx);
    const int j = (int)((gidx / g.nx) % g.ny);
    const int k = (int)(gidx / ((long long)g.nx * g.ny));
    c[0] = gpos(g, 0, i); c[1] = gpos(g, 1, j); c[2] = gpos(g, 2, k);
}

// Closest point of triangle (a,b,c) to p (Ericson, Real-Time Collision Detection §5.1.5);
// degenerate triangles fall back to the closest of their three edges.
__device__ void seg_closest(const double* p, const double* a, const double* b, double* out) {
    double ab[3], ap[3];
    for (int d = 0; d < 3; ++d) { ab[d] = b[d] - a[d]; ap[d] = p[d] - a[d]; }
    const double l2 = dot3(ab, ab);
    double t = l2 > 0.0 ? dot3(ap, ab) / l2 : 0.0;
    t = fmin(1.0, fmax(0.0, t));
    for (int d = 0; d < 3; ++d) out[d] = a[d] + t * ab[d];
}

__device__ void tri_closest(const double* p, const double* a, const double* b, const double* c, double* out) {
    double ab[3], ac[3], ap[3], bp[3], cp[3];
    for (int d = 0; d < 3; ++d) { ab[d] = b[d] - a[d]; ac[d] = c[d] - a[d]; ap[d] = p[d] - a[d]; }
    const double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) { for (int d = 0; d < 3; ++d) out[d] = a[d]; return; }
    for (int d = 0; d < 3; ++d) bp[d] = p[d] - b[d];
    const double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) { for (int d = 0; d < 3; ++d) out[d] = b[d]; return; }
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        const double v = d1 / (d1 - d3);
        for (int d = 0; d < 3; ++d) out[d] = a[d] + v * ab[d];
        return;
    }
    for (int d = 0; d < 3; ++d) cp[d] = p[d] - c[d];
    const double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) { for (int d = 0; d < 3; ++d) out[d] = c[d]; return; }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        const double w = d2 / (d2 - d6);
        for (int d = 0; d < 3; ++d) out[d] = a[d] + w * ac[d];
        return;
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        for (int d = 0; d < 3; ++d) out[d] = b[d] + w * (c[d] - b[d]);
        return;
    }
    const double sum = va + vb + vc;
    if (sum != 0.0 && isfinite(sum)) {
        const double denom = 1.0 / sum;
        const double v = vb * denom, w = vc * denom;
        for (int d = 0; d < 3; ++d) out[d] = a[d] + ab[d] * v + ac[d] * w;
        if (isfinite(out[0]) && isfinite(out[1]) && isfinite(out[2])) return;
    }
    double q[3], best = DBL_MAX;
    const double* E[3][2] = {{a, b}, {b, c}, {c, a}};
    for (int s = 0; s < 3; ++s) {
        seg_closest(p, E[s][0], E[s][1], q);
        double dd[3] = {q[0] - p[0], q[1] - p[1], q[2] - p[2]};
        const double d2q = dot3(dd, dd);
        if (d2q < best) { best = d2q; out[0] = q[0]; out[1] = q[1]; out[2] = q[2]; }
    }
}

// compute_barycentric_coords (vertex_refinement.cpp:36-66).
__device__ void barycentric(const double* P, const double* V0, const double* V1, const double* V2, double out[3]) {
    double e1[3], e2[3], ep[3];
    for (int d = 0; d < 3; ++d) { e1[d] = V1[d] - V0[d]; e2[d] = V2[d] - V0[d]; ep[d] = P[d] - V0[d]; }
    const double d11 = dot3(e1, e1), d12 = dot3(e1, e2), d22 = dot3(e2, e2);
    const double dP1 = dot3(ep, e1), dP2 = dot3(ep, e2);
    const double denom = d11 * d22 - d12 * d12;
    if (fabs(denom) < 1e-12) { out[0] = 1.0; out[1] = 0.0; out[2] = 0.0; return; }
    const double beta = (d22 * dP1 - d12 * dP2) / denom;
    const double gamma = (d11 * dP2 - d12 * dP1) / denom;
    out[0] = 1.0 - beta - gamma; out[1] = beta; out[2] = gamma;
}

// Hermite sample of edge e with the 4-cell average, and whether the edge was averaged.
__device__ bool edge_sample_avg(const GridDesc& g, const f64::Cell64& C, int i, int j, int k, int e, double p[3],
                                double n[3], bool& avg) {
    avg = false;
    if (!f64::hermite(C, e, p, n)) return false;
    int cc[4][3], ex[4];
    const int a = edge_a(e), b = edge_b(e);
    const int Pa[3] = {i + corner_dx(a), j + corner_dy(a), k + corner_dz(a)};
    const int Pb[3] = {i + corner_dx(b), j + corner_dy(b), k + corner_dz(b)};
    int Pm[3], PM[3];
    for (int d = 0; d < 3; ++d) { Pm[d] = min(Pa[d], Pb[d]); PM[d] = max(Pa[d], Pb[d]); }
    const bool in0 = Pm[0] > 0 && Pm[0] < g.nx - 1 && Pm[1] > 0 && Pm[1] < g.ny - 1 && Pm[2] > 0 && Pm[2] < g.nz - 1;
    const bool in1 = PM[0] > 0 && PM[0] < g.nx - 1 && PM[1] > 0 && PM[1] < g.ny - 1 && PM[2] > 0 && PM[2] < g.nz - 1;
    if (!in0 && !in1) return true;
    const int axis = Pa[0] != Pb[0] ? 0 : (Pa[1] != Pb[1] ? 1 : 2);
    const int d1 = axis == 0 ? 1 : 0, d2 = axis == 2 ? 1 : 2;
    double nq[4][3];
    for (int q = 0; q < 4; ++q) {
        cc[q][0] = Pm[0]; cc[q][1] = Pm[1]; cc[q][2] = Pm[2];
        if (q & 1) cc[q][d1] -= 1;
        if (q & 2) cc[q][d2] -= 1;
        if (cc[q][0] == i && cc[q][1] == j && cc[q][2] == k) { for (int d = 0; d < 3; ++d) nq[q][d] = n[d]; continue; }
        f64::Cell64 X;
        f64::load_cell(g, cc[q][0], cc[q][1], cc[q][2], X);
        if (!f64::active(X)) return true;
        ex[q] = f64::local_edge(axis, Pm[d1] - cc[q][d1], Pm[d2] - cc[q][d2]);
        double px[3];
        if (!f64::hermite(X, ex[q], px, nq[q])) return true;
    }
    double acc[3] = {0.0, 0.0, 0.0};
    for (int q = 0; q < 4; ++q)
        if (sqrt(f64::sq3(nq[q])) > 0) { acc[0] += nq[q][0]; acc[1] += nq[q][1]; acc[2] += nq[q][2]; }
    f64::normalize3(acc);
    for (int d = 0; d < 3; ++d) n[d] = acc[d];
    avg = true;
    return true;
}

__device__ __forceinline__ unsigned long long expand_bits10(unsigned long long v) {
    v = (v * 0x00010001ull) & 0xFF0000FFull;
    v = (v * 0x00000101ull) & 0x0F00F00Full;
    v = (v * 0x00000011ull) & 0xC30C30C3ull;
    v = (v * 0x00000005ull) & 0x49249249ull;
    return v;
}

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

}  // namespace

// Cells with at least this many spheres run their inner loop on a warp (a chunk per lane).
constexpr unsigned int kWarpCellSpheres = 8;

// ---- setup -------------------------------------------------------------------------------

// Per cell: Hermite points and normals as the refinement starts (after Cell::update and the
// second average_hermite_normals, contouring.cpp:1233-1241), vertex = Hermite centroid
// (contouring.cpp:1258-1263), and the extraction's FP64 vertex for the first mesh.
__global__ void __launch_bounds__(128) k_ours_init(OursParams P) {
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < P.nv; r += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        unpack_cell(P.list[r], i, j, k);
        f64::Cell64 C;
        f64::load_cell(P.g, i, j, k, C);
        OursCell& S = P.cells[r];
        int hmask = 0, m = 0;
        double c[3] = {0.0, 0.0, 0.0};
        for (int e = 0; e < 12; ++e) {
            double p[3], n[3];
            bool avg;
            if (!edge_sample_avg(P.g, C, i, j, k, e, p, n, avg)) continue;
            if (avg) {
                // the second averaging sums the four (identical) averaged normals again
                double acc[3];
                for (int d = 0; d < 3; ++d) acc[d] = ((n[d] + n[d]) + n[d]) + n[d];
                if (sqrt(f64::sq3(n)) > 0) f64::normalize3(acc);
                else acc[0] = acc[1] = acc[2] = 0.0;
                for (int d = 0; d < 3; ++d) n[d] = acc[d];
            }
            for (int d = 0; d < 3; ++d) { S.hp[e][d] = p[d]; S.hn[e][d] = n[d]; c[d] += p[d]; }
            hmask |= 1 << e;
            ++m;
        }
        for (int d = 0; d < 3; ++d) S.v[d] = m ? c[d] / double(m) : 0.0;
        S.hmask = hmask;
        S.fmask = 0;
        double x[3];
        f64::cell_vertex_thread(P.g, i, j, k, 0.01, x);        // Cell::update's threshold (Cell.cpp:314)
        for (int d = 0; d < 3; ++d) P.Vm[3 * r + d] = x[d];
    }
}

// Per extracted quad: the canonical cell order of its grid edge (contouring.cpp:607-729; the
// extraction may have swapped c1 and c3) and the edge's gradient sum gradientAt(p0)+gradientAt(p1).
__global__ void __launch_bounds__(128) k_ours_quads(OursParams P) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < P.nq; q += (long long)gridDim.x * blockDim.x) {
        const int4 f = P.dc_faces[q];
        int a0, a1, a2, c0, c1, c2, b0, b1, b2;
        unpack_cell(P.list[f.x], a0, a1, a2);
        unpack_cell(P.list[f.z], c0, c1, c2);
        unpack_cell(P.list[f.y], b0, b1, b2);
        const int axis = a0 == c0 ? 0 : (a1 == c1 ? 1 : 2);
        // canonical c1 = c2 - e_z for x and y edges, c2 - e_y for z edges
        int w0 = c0, w1 = c1, w2 = c2;
        if (axis == 2) w1 -= 1; else w2 -= 1;
        const bool canon = b0 == w0 && b1 == w1 && b2 == w2;
        P.quads[q] = canon ? f : make_int4(f.x, f.w, f.z, f.y);
        double g0[3], g1[3];
        f64::grid_gradient(P.g, c0, c1, c2, g0);
        f64::grid_gradient(P.g, c0 + (axis == 0), c1 + (axis == 1), c2 + (axis == 2), g1);
        for (int d = 0; d < 3; ++d) P.gsum[3 * q + d] = g0[d] + g1[d];
    }
}

// Grid points with |S| < 3 * cell diagonal (the sphere batch) and the others (the random fill).
__global__ void __launch_bounds__(256) k_ours_select(OursParams P, long long npts, uint32_t* band, uint32_t* rest,
                                                     unsigned int* counts) {
    const int lane = threadIdx.x & 31;
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < npts;
         base += (long long)gridDim.x * blockDim.x) {
        const long long t = base + lane;
        bool in = false, ok = t < npts;
        if (ok) in = fabs((double)__ldg(P.g.v + t)) < 3.0 * P.cell_diag;
        for (int w = 0; w < 2; ++w) {
            const uint32_t m = __ballot_sync(0xffffffffu, ok && (w == 0 ? in : !in));
            if (!m) continue;
            unsigned int first = 0;
            if (lane == __ffs(m) - 1) first = atomicAdd(counts + w, (unsigned int)__popc(m));
            first = __shfl_sync(0xffffffffu, first, __ffs(m) - 1);
            if (ok && (w == 0 ? in : !in)) (w == 0 ? band : rest)[first + __popc(m & ((1u << lane) - 1u))] = (uint32_t)t;
        }
    }
}

__device__ __forceinline__ unsigned long long spread21(unsigned long long v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

// Morton keys of the selected grid points: the queries of a warp then cover a compact block.
__global__ void k_ours_point_keys(OursParams P, const uint32_t* sel, long long n, unsigned long long* keys) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long g = sel[t];
        const unsigned long long i = g % P.g.nx, j = (g / P.g.nx) % P.g.ny, k = g / ((long long)P.g.nx * P.g.ny);
        keys[t] = spread21(i) | (spread21(j) << 1) | (spread21(k) << 2);
    }
}

// Random keys of the fill candidates for one outer iteration (seeded).
__global__ void k_ours_fill_keys(const uint32_t* rest, long long n, unsigned long long seed, int it,
                                 unsigned long long* keys) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        keys[t] = splitmix64(seed ^ splitmix64(((unsigned long long)it << 40) ^ (unsigned long long)rest[t]));
}

// ---- the mesh's BVH ----------------------------------------------------------------------

// The quad of canonical cells wound by its grid edge's gradient (contouring.cpp:624-641).
__device__ __forceinline__ int4 wound_quad(const OursParams& P, long long q) {
    int4 f = P.quads[q];
    const double* pa = P.Vm + 3 * (long long)f.x;
    const double* pb = P.Vm + 3 * (long long)f.y;
    const double* pc = P.Vm + 3 * (long long)f.z;
    const double* pd = P.Vm + 3 * (long long)f.w;
    double u[3], w[3], n[3];
    for (int d = 0; d < 3; ++d) { u[d] = pb[d] - pa[d]; w[d] = pd[d] - pa[d]; }
    cross3(u, w, n);
    if (dot3(n, n) < 1e-24) { for (int d = 0; d < 3; ++d) u[d] = pc[d] - pa[d]; cross3(u, w, n); }
    const double* gs = P.gsum + 3 * q;
    if (dot3(gs, gs) > 0 && dot3(n, n) > 0 && dot3(n, gs) < 0.0) { const int t = f.y; f.y = f.w; f.w = t; }
    return f;
}

// triangulate_v1 + orient_triangles_for_quad (contouring.cpp:40-113) of a wound quad.
__device__ __forceinline__ void quad_triangles(const OursParams& P, int4 f, int t0[3], int t1[3]) {
    const double* qa = P.Vm + 3 * (long long)f.x;
    const double* qb = P.Vm + 3 * (long long)f.y;
    const double* qc = P.Vm + 3 * (long long)f.z;
    const double* qd = P.Vm + 3 * (long long)f.w;
    double u[3], w[3], qn[3];
    for (int d = 0; d < 3; ++d) { u[d] = qb[d] - qa[d]; w[d] = qd[d] - qa[d]; }
    cross3(u, w, qn);
    if (dot3(qn, qn) < 1e-24) { for (int d = 0; d < 3; ++d) u[d] = qc[d] - qa[d]; cross3(u, w, qn); }
    t0[0] = f.x; t0[1] = f.y; t0[2] = f.z;
    t1[0] = f.x; t1[1] = f.z; t1[2] = f.w;
    if (dot3(qn, qn) < 1e-24) return;                 // degenerate quad: left as it is
    int* tt[2] = {t0, t1};
    for (int h = 0; h < 2; ++h) {
        const double* p1 = P.Vm + 3 * (long long)tt[h][0];
        const double* p2 = P.Vm + 3 * (long long)tt[h][1];
        const double* p3 = P.Vm + 3 * (long long)tt[h][2];
        double x[3], y[3], tn[3];
        for (int d = 0; d < 3; ++d) { x[d] = p2[d] - p1[d]; y[d] = p3[d] - p1[d]; }
        cross3(x, y, tn);
        if (dot3(tn, qn) < 0.0) { const int s = tt[h][1]; tt[h][1] = tt[h][2]; tt[h][2] = s; }
    }
}

// The current mesh's triangles (the quads wound with the current vertices, then
// triangulate_v1) with their Morton keys (key << 32 | triangle).
__global__ void __launch_bounds__(128) k_ours_tris(OursParams P) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < P.nq; q += (long long)gridDim.x * blockDim.x) {
        int id[2][3];
        quad_triangles(P, wound_quad(P, q), id[0], id[1]);
        for (int h = 0; h < 2; ++h) {
            const long long t = 2 * q + h;
            double cen[3] = {0.0, 0.0, 0.0};
            for (int v = 0; v < 3; ++v)
                for (int d = 0; d < 3; ++d) {
                    const double x = P.Vm[3 * (long long)id[h][v] + d];
                    P.tri9[9 * t + 3 * v + d] = x;
                    cen[d] += x;
                }
            unsigned long long code = 0;
            for (int d = 0; d < 3; ++d) {
                double u = (cen[d] / 3.0 - P.lo[d]) / (P.hi[d] - P.lo[d]);
                u = fmin(1.0, fmax(0.0, u));
                const unsigned long long b = (unsigned long long)fmin(1023.0, u * 1024.0);
                code |= expand_bits10(b) << (2 - d);
            }
            P.tcode[t] = (uint32_t)code;
            P.tidx[t] = (uint32_t)t;
        }
    }
}

// Unique sorted keys (Morton code << 32 | triangle): the pairs were sorted stably by code, so
// equal codes keep ascending triangle order.
__global__ void k_bvh_keys(OursParams P) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < P.nt; i += (long long)gridDim.x * blockDim.x)
        P.mkeys_sorted[i] = ((unsigned long long)P.tcode_sorted[i] << 32) | P.tidx_sorted[i];
}

// Radix tree over the sorted keys (Karras, "Maximizing parallelism in the construction of
// BVHs, octrees, and k-d trees", HPG 2012). Children < 0 are leaves (~leaf).
__device__ __forceinline__ int key_delta(const unsigned long long* k, long long n, long long a, long long b) {
    if (b < 0 || b >= n) return -1;
    return __clzll(k[a] ^ k[b]);
}

__global__ void __launch_bounds__(128) k_bvh_tree(OursParams P) {
    const long long n = P.nt;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long* K = P.mkeys_sorted;
        const int d = (key_delta(K, n, i, i + 1) - key_delta(K, n, i, i - 1)) >= 0 ? 1 : -1;
        const int dmin = key_delta(K, n, i, i - d);
        long long lmax = 2;
        while (key_delta(K, n, i, i + lmax * d) > dmin) lmax *= 2;
        long long l = 0;
        for (long long t = lmax / 2; t >= 1; t /= 2)
            if (key_delta(K, n, i, i + (l + t) * d) > dmin) l += t;
        const long long j = i + l * d;
        const int dnode = key_delta(K, n, i, j);
        long long s = 0;
        for (long long div = 2;; div *= 2) {
            const long long t = (l + div - 1) / div;
            if (key_delta(K, n, i, i + (s + t) * d) > dnode) s += t;
            if (t <= 1) break;
        }
        const long long gamma = i + s * d + (d < 0 ? -1 : 0);
        const long long lo = i < j ? i : j, hi = i < j ? j : i;
        const int left = lo == gamma ? ~(int)gamma : (int)gamma;
        const int right = hi == gamma + 1 ? ~(int)(gamma + 1) : (int)(gamma + 1);
        P.child[i] = make_int2(left, right);
        if (left < 0) P.parent[n - 1 + ~left] = (int)i; else P.parent[left] = (int)i;
        if (right < 0) P.parent[n - 1 + ~right] = (int)i; else P.parent[right] = (int)i;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) P.parent[0] = -1;
}

// Boxes bottom-up: leaf boxes rounded outward to float; the second child to arrive at a node
// writes the union.
__global__ void __launch_bounds__(128) k_bvh_boxes(OursParams P) {
    const long long n = P.nt;
    for (long long L = (long long)blockIdx.x * blockDim.x + threadIdx.x; L < n; L += (long long)gridDim.x * blockDim.x) {
        const long long t = (long long)(P.mkeys_sorted[L] & 0xffffffffull);
        float lo[3], hi[3];
        for (int d = 0; d < 3; ++d) {
            double a = P.tri9[9 * t + d], b = P.tri9[9 * t + 3 + d], c = P.tri9[9 * t + 6 + d];
            lo[d] = __double2float_rd(fmin(a, fmin(b, c)));
            hi[d] = __double2float_ru(fmax(a, fmax(b, c)));
        }
        const long long node_l = n - 1 + L;
        P.bmin[node_l] = make_float4(lo[0], lo[1], lo[2], 0.f);
        P.bmax[node_l] = make_float4(hi[0], hi[1], hi[2], 0.f);
        __threadfence();
        int node = P.parent[node_l];
        while (node >= 0) {
            if (atomicAdd(P.flags + node, 1u) == 0) break;       // the other child is not done yet
            __threadfence();
            const int2 ch = P.child[node];
            const long long a = ch.x < 0 ? n - 1 + ~ch.x : ch.x, b = ch.y < 0 ? n - 1 + ~ch.y : ch.y;
            const float4 amin = __ldcg(P.bmin + a), amax = __ldcg(P.bmax + a);
            const float4 bmn = __ldcg(P.bmin + b), bmx = __ldcg(P.bmax + b);
            P.bmin[node] = make_float4(fminf(amin.x, bmn.x), fminf(amin.y, bmn.y), fminf(amin.z, bmn.z), 0.f);
            P.bmax[node] = make_float4(fmaxf(amax.x, bmx.x), fmaxf(amax.y, bmx.y), fmaxf(amax.z, bmx.z), 0.f);
            __threadfence();
            node = P.parent[node];
        }
    }
}

__device__ __forceinline__ double box_d2(const OursParams& P, long long node, const double* p) {
    const float4 a = __ldg(P.bmin + node), b = __ldg(P.bmax + node);
    const double lo[3] = {a.x, a.y, a.z}, hi[3] = {b.x, b.y, b.z};
    double s = 0.0;
    for (int d = 0; d < 3; ++d) {
        const double e = p[d] < lo[d] ? lo[d] - p[d] : (p[d] > hi[d] ? p[d] - hi[d] : 0.0);
        s += e * e;
    }
    return s;
}

// Closest point of the mesh to p (point_mesh_squared_distance, contouring.cpp:869): among
// equally close triangles the one of smallest index, so the answer does not depend on the
// traversal order (nodes as close as the best so far are still visited).
// seed: a triangle to test first (the previous outer iteration's answer for this point), or -1;
// the answer does not depend on it, only the number of nodes visited does.
__device__ double bvh_closest(const OursParams& P, const double* p, double* best_c, long long seed, int& out_t) {
    const long long n = P.nt;
    double best = DBL_MAX;
    long long best_t = 0x7fffffffffffffffLL;
    auto test = [&](long long t) {
        const double* T = P.tri9 + 9 * t;
        double q[3];
        tri_closest(p, T, T + 3, T + 6, q);
        double dd[3] = {q[0] - p[0], q[1] - p[1], q[2] - p[2]};
        const double d2 = dot3(dd, dd);
        if (d2 < best || (d2 == best && t < best_t)) {
            best = d2; best_t = t;
            best_c[0] = q[0]; best_c[1] = q[1]; best_c[2] = q[2];
        }
    };
    auto leaf = [&](long long L) { test((long long)(P.mkeys_sorted[L] & 0xffffffffull)); };
    if (seed >= 0 && seed < n) test(seed);
    if (n == 1) { leaf(0); out_t = (int)best_t; return best; }
    int stack[96];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const int node = stack[--sp];
        const int2 ch = P.child[node];
        const int c2[2] = {ch.x, ch.y};
        double dc[2];
        for (int u = 0; u < 2; ++u) dc[u] = box_d2(P, c2[u] < 0 ? n - 1 + ~c2[u] : c2[u], p);
        const int first = dc[1] < dc[0] ? 1 : 0;
        // leaves now, internal nodes onto the stack (the nearer one on top)
        for (int u = 0; u < 2; ++u) {
            const int w = u == 0 ? first : 1 - first;
            if (c2[w] < 0 && dc[w] <= best) leaf(~c2[w]);
        }
        for (int u = 1; u >= 0; --u) {
            const int w = u == 0 ? first : 1 - first;
            if (c2[w] >= 0 && dc[w] <= best) {
                if (sp < 96) stack[sp++] = c2[w];
                else set_error(P.err, kErrOverflow);
            }
        }
    }
    out_t = (int)best_t;
    return best;
}

// ---- sphere assignment ---------------------------------------------------------------------

__global__ void __launch_bounds__(128) k_ours_query(OursParams P) {
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < P.nsel; s += (long long)gridDim.x * blockDim.x) {
        const long long gidx = P.sel[s];
        double c[3], C[3];
        point_of(P.g, gidx, c);
        int t = -1;
        const double d2 = bvh_closest(P, c, C, P.prev_tri[gidx], t);
        P.prev_tri[gidx] = t;
        const double radius = fabs((double)__ldg(P.g.v + gidx));
        int rank = -1;
        if (d2 < DBL_MAX && sqrt(d2) - radius < P.cell_diag) {
            int ci[3];
            const int cmax[3] = {P.g.nx - 2, P.g.ny - 2, P.g.nz - 2};
            for (int d = 0; d < 3; ++d) {
                const double f = floor((C[d] - P.gmin[d]) / P.gd[d]);
                int v = f < -1e9 ? -1000000000 : (f > 1e9 ? 1000000000 : (int)f);
                ci[d] = max(0, min(v, cmax[d]));
            }
            if (active_bit(P, ci[0], ci[1], ci[2])) {
                rank = (int)cell_rank(P.bits, P.super, P.g, ci[0], ci[1], ci[2]);
                atomicAdd(P.cell_count + rank, 1u);
            }
        }
        P.sel_cell[s] = rank;
    }
}

__global__ void __launch_bounds__(128) k_ours_scatter(OursParams P) {
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < P.nsel; s += (long long)gridDim.x * blockDim.x) {
        const int rank = P.sel_cell[s];
        if (rank < 0) continue;
        const unsigned int at = P.cell_start[rank] + atomicAdd(P.cell_fill + rank, 1u);
        P.cell_spheres[at] = P.sel[s];
    }
}

// Each cell's spheres by radius (then grid index, for a deterministic order among equal radii).
__global__ void __launch_bounds__(128) k_ours_sort(OursParams P) {
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < P.nv; r += (long long)gridDim.x * blockDim.x) {
        const unsigned int n = P.cell_count[r];
        if (n >= kWarpCellSpheres) P.heavy[atomicAdd(P.heavy_count, 1u)] = (uint32_t)r;
        if (n < 2) continue;
        uint32_t* a = P.cell_spheres + P.cell_start[r];
        auto less = [&](uint32_t x, uint32_t y) {
            const float rx = fabsf(__ldg(P.g.v + x)), ry = fabsf(__ldg(P.g.v + y));
            return rx < ry || (rx == ry && x < y);
        };
        // Shell sort (Ciura gaps)
        const unsigned int gaps[8] = {701, 301, 132, 57, 23, 10, 4, 1};
        for (int gi = 0; gi < 8; ++gi) {
            const unsigned int gap = gaps[gi];
            for (unsigned int x = gap; x < n; ++x) {
                const uint32_t t = a[x];
                unsigned int y = x;
                while (y >= gap && less(t, a[y - gap])) { a[y] = a[y - gap]; y -= gap; }
                a[y] = t;
            }
        }
    }
}

// ---- per-cell steps --------------------------------------------------------------------------

// compute_face_cell_intersections (contouring.cpp:1081-1183).
__global__ void __launch_bounds__(128) k_ours_faces(OursParams P) {
    const int dirs[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < P.nv; r += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        unpack_cell(P.list[r], i, j, k);
        OursCell& S = P.cells[r];
        const double v[3] = {S.v[0], S.v[1], S.v[2]};
        const double mn[3] = {gpos(P.g, 0, i), gpos(P.g, 1, j), gpos(P.g, 2, k)};
        const double mx[3] = {gpos(P.g, 0, i + 1), gpos(P.g, 1, j + 1), gpos(P.g, 2, k + 1)};
        int fmask = S.fmask;
        for (int d = 0; d < 6; ++d) {
            const int ni = i + dirs[d][0], nj = j + dirs[d][1], nk = k + dirs[d][2];
            if (ni < 0 || ni >= P.g.cx || nj < 0 || nj >= P.g.cy || nk < 0 || nk >= P.g.cz) continue;
            if (!active_bit(P, ni, nj, nk)) continue;
            const OursCell& N = P.cells[cell_rank(P.bits, P.super, P.g, ni, nj, nk)];
            double seg[3];
            for (int a = 0; a < 3; ++a) seg[a] = N.v[a] - v[a];
            const int ax = d >> 1;
            const double plane = (d & 1) ? mn[ax] : mx[ax];
            const double num = plane - v[ax], den = seg[ax];
            if (fabs(den) < 1e-9) continue;
            const double t = num / den;
            if (t >= -1e-6 && t <= 1.0 + 1e-6) {
                double x[3];
                for (int a = 0; a < 3; ++a) x[a] = v[a] + t * seg[a];
                if (!(fmask & (1 << d))) {
                    for (int a = 0; a < 3; ++a) S.fi[d][a] = x[a];
                    fmask |= 1 << d;
                } else {
                    for (int a = 0; a < 3; ++a) S.fi[d][a] = x[a] * P.wface + S.fi[d][a] * (1.0 - P.wface);
                }
            }
        }
        S.fmask = fmask;
    }
}

// update_hermite_points_and_normals (hermite_update.cpp:441-607): one thread per (cell, edge);
// the cell at the edge's minimum endpoint handles an edge whose four cells have vertices.
__global__ void __launch_bounds__(128) k_ours_hermite(OursParams P) {
    const long long nrow = 12 * P.nv;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nrow; t += (long long)gridDim.x * blockDim.x) {
        const long long r = t / 12;
        const int e = (int)(t - 12 * r);
        if (e != 0 && e != 3 && e != 8) continue;          // edges leaving corner 0: the owner's
        int i, j, k;
        unpack_cell(P.list[r], i, j, k);
        const OursCell& S0 = P.cells[r];
        if (!(S0.hmask & (1 << e))) continue;
        int cc[4][3], ex[4];
        if (!f64::edge_cells(P.g, i, j, k, e, cc, ex)) continue;
        long long rk[4];
        bool all = true;
        for (int q = 0; q < 4 && all; ++q) {
            if (q == 0) { rk[0] = r; continue; }
            all = active_bit(P, cc[q][0], cc[q][1], cc[q][2]);
            if (all) rk[q] = cell_rank(P.bits, P.super, P.g, cc[q][0], cc[q][1], cc[q][2]);
        }
        if (!all) continue;
        ex[0] = e;
        // PCA of the four vertices: the normal is the direction of least variance
        double V[4][3], cen[3] = {0.0, 0.0, 0.0};
        for (int q = 0; q < 4; ++q)
            for (int d = 0; d < 3; ++d) { V[q][d] = P.cells[rk[q]].v[d]; cen[d] += V[q][d]; }
        for (int d = 0; d < 3; ++d) cen[d] /= 4.0;
        double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, U[3][3];
        for (int q = 0; q < 4; ++q) {
            double x[3];
            for (int d = 0; d < 3; ++d) x[d] = V[q][d] - cen[d];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) M[a][b] += x[a] * x[b];
        }
        f64::jacobi3(M, U);
        int qmin = 0;
        for (int q = 1; q < 3; ++q) if (M[q][q] <= M[qmin][qmin]) qmin = q;
        double nrm[3] = {U[0][qmin], U[1][qmin], U[2][qmin]};
        f64::normalize3(nrm);
        // orientation against the edge of the owner cell (EDGE_PAIRS order)
        const int ca = edge_a(e), cb = edge_b(e);
        const double pA[3] = {gpos(P.g, 0, i + corner_dx(ca)), gpos(P.g, 1, j + corner_dy(ca)), gpos(P.g, 2, k + corner_dz(ca))};
        const double pB[3] = {gpos(P.g, 0, i + corner_dx(cb)), gpos(P.g, 1, j + corner_dy(cb)), gpos(P.g, 2, k + corner_dz(cb))};
        const double sA = (double)__ldg(P.g.v + pidx(P.g, i + corner_dx(ca), j + corner_dy(ca), k + corner_dz(ca)));
        double dir[3];
        for (int d = 0; d < 3; ++d) dir[d] = pB[d] - pA[d];
        const double len = norm3(dir);
        if (len > 0.0) for (int d = 0; d < 3; ++d) dir[d] /= len;
        double out[3];
        for (int d = 0; d < 3; ++d) out[d] = dir[d] * (sA < 0 ? -1.0 : 1.0);
        if (dot3(nrm, out) > 0) for (int d = 0; d < 3; ++d) nrm[d] = -nrm[d];
        const bool has_n = norm3(nrm) > 0;
        for (int q = 0; q < 4; ++q) {
            OursCell& C = P.cells[rk[q]];
            if (!has_n) continue;
            double u[3];
            for (int d = 0; d < 3; ++d) u[d] = (1.0 - P.wnormal) * C.hn[ex[q]][d] + P.wnormal * nrm[d];
            f64::normalize3(u);
            for (int d = 0; d < 3; ++d) C.hn[ex[q]][d] = u[d];
        }
        const double denom = dot3(nrm, dir);
        if (fabs(denom) > 1e-6) {
            double w[3];
            for (int d = 0; d < 3; ++d) w[d] = cen[d] - pA[d];
            double tt = dot3(nrm, w) / denom;
            if (tt < 0 || tt > len) continue;
            tt = fmax(0.0, fmin(tt, len));
            double x[3];
            for (int d = 0; d < 3; ++d) x[d] = pA[d] + tt * dir[d];
            for (int q = 0; q < 4; ++q) {
                OursCell& C = P.cells[rk[q]];
                for (int d = 0; d < 3; ++d) C.hp[ex[q]][d] = (1.0 - P.wpos) * C.hp[ex[q]][d] + P.wpos * x[d];
            }
        }
    }
}

// One sphere's row of Cell::minimize_qef (Cell.cpp:400-446) for a cell whose vertex is prev:
// its closest point on the local fan (first minimum in fan order), the point on the sphere,
// the barycentric blend of (vertex, Hermite point, face point). False if the row is skipped.
__device__ bool sphere_row(const OursParams& P, const OursCell& S, const int* fan, int nfan, const double* prev,
                           uint32_t gidx, double ssw, double row[3], double& rb) {
    double c[3];
    point_of(P.g, gidx, c);
    const double sval = (double)__ldg(P.g.v + gidx);
    const double rs = fabs(sval);
    double best = DBL_MAX, tm[3] = {0, 0, 0};
    int bf = 0;
    for (int f = 0; f < nfan; ++f) {
        const int e = fan[f] & 15, d = fan[f] >> 4;
        double q[3];
        tri_closest(c, prev, S.hp[e], S.fi[d], q);
        double dd[3] = {q[0] - c[0], q[1] - c[1], q[2] - c[2]};
        const double d2 = dot3(dd, dd);
        if (d2 < best) { best = d2; bf = f; tm[0] = q[0]; tm[1] = q[1]; tm[2] = q[2]; }
    }
    const int e = fan[bf] & 15, d = fan[bf] >> 4;
    const double* Hp = S.hp[e];
    const double* Fp = S.fi[d];
    double ct[3];
    for (int a = 0; a < 3; ++a) ct[a] = tm[a] - c[a];
    const double rho0 = norm3(ct);
    double qs[3];
    if (rho0 < 1e-9) for (int a = 0; a < 3; ++a) qs[a] = c[a];
    else for (int a = 0; a < 3; ++a) qs[a] = c[a] + (ct[a] / rho0) * rs;
    double bc[3];
    barycentric(tm, prev, Hp, Fp, bc);
    double alpha = bc[0], beta = bc[1], gamma = bc[2];
    if (fabs(alpha) < 1e-6) { alpha = 1.0; beta = 0.0; gamma = 0.0; }
    double tt[3], ctt[3];
    for (int a = 0; a < 3; ++a) { tt[a] = alpha * prev[a] + beta * Hp[a] + gamma * Fp[a]; ctt[a] = tt[a] - c[a]; }
    const double rho = norm3(ctt);
    double qc[3];
    for (int a = 0; a < 3; ++a) qc[a] = qs[a] - c[a];
    const double radius = norm3(qc);
    if (rho > radius && sval < 0.0) return false;          // sign -1 (Cell.cpp:419-426)
    double q[3];
    if (rho < 1e-9) for (int a = 0; a < 3; ++a) q[a] = c[a];
    else for (int a = 0; a < 3; ++a) q[a] = c[a] + (ctt[a] / rho) * radius;
    double dv[3];
    for (int a = 0; a < 3; ++a) dv[a] = q[a] - c[a];
    for (int a = 0; a < 3; ++a) row[a] = alpha * ssw * dv[a];
    rb = ssw * ((dot3(q, dv) - beta * dot3(Hp, dv)) - gamma * dot3(Fp, dv));
    return true;
}

// Sphere rows of one chunk, summed in order from zero: 6 entries of the symmetric A^T A
// (00 01 02 11 12 22) and 3 of A^T b.
__device__ void chunk_sums(const OursParams& P, const OursCell& S, const int* fan, int nfan, const double* prev,
                           const uint32_t* sph, unsigned int lo, unsigned int hi, double ssw, double acc[9]) {
    for (int q = 0; q < 9; ++q) acc[q] = 0.0;
    for (unsigned int s = lo; s < hi; ++s) {
        double row[3], rb;
        if (!sphere_row(P, S, fan, nfan, prev, sph[s], ssw, row, rb)) continue;
        acc[0] += row[0] * row[0]; acc[1] += row[0] * row[1]; acc[2] += row[0] * row[2];
        acc[3] += row[1] * row[1]; acc[4] += row[1] * row[2]; acc[5] += row[2] * row[2];
        acc[6] += row[0] * rb; acc[7] += row[1] * rb; acc[8] += row[2] * rb;
    }
}

// The local fan of a cell: (vertex, Hermite point on edge e, face point d) for each face d
// with a point and each of its four edges with a Hermite point, in face then edge order.
__device__ int cell_fan(const OursCell& S, int fan[24]) {
    int nfan = 0;
    for (int d = 0; d < 6; ++d) {
        if (!(S.fmask & (1 << d))) continue;
        for (int u = 0; u < 4; ++u) {
            const int e = edge_of_corners(kFaceCorners[d][u], kFaceCorners[d][(u + 1) & 3]);
            if (e >= 0 && (S.hmask & (1 << e))) fan[nfan++] = e | (d << 4);
        }
    }
    return nfan;
}

// The Hermite rows dc_weight * n_e in edge order and the Hermite centroid.
__device__ void hermite_rows(const OursParams& P, const OursCell& S, double H0[9], double cen[3]) {
    for (int q = 0; q < 9; ++q) H0[q] = 0.0;
    cen[0] = cen[1] = cen[2] = 0.0;
    int m = 0;
    for (int e = 0; e < 12; ++e) {
        if (!(S.hmask & (1 << e))) continue;
        double sn[3];
        for (int d = 0; d < 3; ++d) sn[d] = P.dc_weight * S.hn[e][d];
        const double b = dot3(sn, S.hp[e]);
        H0[0] += sn[0] * sn[0]; H0[1] += sn[0] * sn[1]; H0[2] += sn[0] * sn[2];
        H0[3] += sn[1] * sn[1]; H0[4] += sn[1] * sn[2]; H0[5] += sn[2] * sn[2];
        H0[6] += sn[0] * b; H0[7] += sn[1] * b; H0[8] += sn[2] * b;
        for (int d = 0; d < 3; ++d) cen[d] += S.hp[e][d];
        ++m;
    }
    for (int d = 0; d < 3; ++d) cen[d] /= double(m);
}

// solve_quadratic_system (Cell.cpp:324-361) with the proximal rows sqrt(mu) * I added.
__device__ void inner_solve(const OursParams& P, const double Acc[9], const double* prev, const double cen[3],
                            double smu, double x[3]) {
    double A[3][3] = {{Acc[0], Acc[1], Acc[2]}, {Acc[1], Acc[3], Acc[4]}, {Acc[2], Acc[4], Acc[5]}};
    double b[3] = {Acc[6], Acc[7], Acc[8]};
    for (int a = 0; a < 3; ++a) { A[a][a] += smu * smu; b[a] += smu * (smu * prev[a]); }
    double E[3][3], U[3][3];
    for (int a = 0; a < 3; ++a) for (int c = 0; c < 3; ++c) E[a][c] = A[a][c];
    f64::jacobi3(E, U);
    double rhs[3];
    for (int a = 0; a < 3; ++a) rhs[a] = b[a] - (A[a][0] * cen[0] + A[a][1] * cen[1] + A[a][2] * cen[2]);
    x[0] = cen[0]; x[1] = cen[1]; x[2] = cen[2];
    for (int q = 0; q < 3; ++q) {
        const double sv = fabs(E[q][q]);
        if (sv > P.thr) {
            const double coef = (U[0][q] * rhs[0] + U[1][q] * rhs[1] + U[2][q] * rhs[2]) / sv;
            for (int a = 0; a < 3; ++a) x[a] += U[a][q] * coef;
        }
    }
}

// The inner loop of one cell (contouring.cpp:1288-1309): refine_vertex_from_face_intersections
// (vertex_refinement.cpp:201-280) + Cell::minimize_qef (Cell.cpp:364-473) until the vertex
// moves less than 1e-6. The sphere rows are summed in 32 chunks of consecutive spheres, each
// from zero, added in chunk order: the same sums whether a thread or a warp computes them.
__global__ void __launch_bounds__(128) k_ours_inner(OursParams P) {
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < P.nv; r += (long long)gridDim.x * blockDim.x) {
        OursCell& S = P.cells[r];
        const unsigned int nsph = P.cell_count[r];
        if (!S.fmask || !nsph || !S.hmask || nsph >= kWarpCellSpheres) continue;
        int fan[24];
        const int nfan = cell_fan(S, fan);
        if (!nfan) continue;
        const uint32_t* sph = P.cell_spheres + P.cell_start[r];
        double H0[9], cen[3];
        hermite_rows(P, S, H0, cen);
        const double ssw = sqrt(P.sphere_weight), smu = sqrt(P.mu);
        const unsigned int cs = (nsph + 31) / 32;
        double v[3] = {S.v[0], S.v[1], S.v[2]};
        for (int it = 0; it < P.inner_iters; ++it) {
            const double prev[3] = {v[0], v[1], v[2]};
            double Acc[9];
            for (int q = 0; q < 9; ++q) Acc[q] = H0[q];
            for (unsigned int l = 0; l < 32; ++l) {
                const unsigned int lo = l * cs, hi = min(nsph, lo + cs);
                if (lo >= hi) break;
                double part[9];
                chunk_sums(P, S, fan, nfan, prev, sph, lo, hi, ssw, part);
                for (int q = 0; q < 9; ++q) Acc[q] += part[q];
            }
            inner_solve(P, Acc, prev, cen, smu, v);
            double dm[3] = {v[0] - prev[0], v[1] - prev[1], v[2] - prev[2]};
            if (norm3(dm) < 1e-6) break;
        }
        for (int a = 0; a < 3; ++a) S.v[a] = v[a];
    }
}

// The same inner loop for the cells with many spheres, a warp per cell.
__global__ void __launch_bounds__(128) k_ours_inner_warp(OursParams P) {
    const int lane = threadIdx.x & 31;
    const unsigned int nheavy = *P.heavy_count;
    for (long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nheavy;
         w += ((long long)gridDim.x * blockDim.x) >> 5) {
        const long long r = P.heavy[w];
        OursCell& S = P.cells[r];
        const unsigned int nsph = P.cell_count[r];
        if (!S.fmask || !S.hmask) continue;                  // warp-uniform
        int fan[24];
        const int nfan = cell_fan(S, fan);
        if (!nfan) continue;
        const uint32_t* sph = P.cell_spheres + P.cell_start[r];
        double H0[9], cen[3];
        hermite_rows(P, S, H0, cen);
        const double ssw = sqrt(P.sphere_weight), smu = sqrt(P.mu);
        const unsigned int cs = (nsph + 31) / 32;
        const unsigned int lo = min(nsph, lane * cs), hi = min(nsph, lo + cs);
        double v[3] = {S.v[0], S.v[1], S.v[2]};
        for (int it = 0; it < P.inner_iters; ++it) {
            const double prev[3] = {v[0], v[1], v[2]};
            double part[9];
            chunk_sums(P, S, fan, nfan, prev, sph, lo, hi, ssw, part);
            double Acc[9];
            for (int q = 0; q < 9; ++q) Acc[q] = H0[q];
            const int nchunks = (int)((nsph + cs - 1) / cs);      // warp-uniform
            for (int l = 0; l < nchunks; ++l)
                for (int q = 0; q < 9; ++q) Acc[q] += __shfl_sync(0xffffffffu, part[q], l);
            inner_solve(P, Acc, prev, cen, smu, v);
            double dm[3] = {v[0] - prev[0], v[1] - prev[1], v[2] - prev[2]};
            if (norm3(dm) < 1e-6) break;
        }
        if (lane == 0) for (int a = 0; a < 3; ++a) S.v[a] = v[a];
    }
}

__global__ void k_ours_mesh(OursParams P) {
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < P.nv; r += (long long)gridDim.x * blockDim.x)
        for (int d = 0; d < 3; ++d) P.Vm[3 * r + d] = P.cells[r].v[d];
}

// The output: vertices as float; quads wound by the edge's gradient (contouring.cpp:624-641),
// or their triangles oriented like the quad (triangulate_v1 + orient_triangles_for_quad,
// contouring.cpp:40-113).
__global__ void __launch_bounds__(128) k_ours_output(OursParams P, int triangles) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < P.nv; r += stride)
        for (int d = 0; d < 3; ++d) P.out_V[3 * r + d] = (float)P.Vm[3 * r + d];
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < P.nq; q += stride) {
        const int4 f = wound_quad(P, q);
        if (!triangles) { P.out_faces[q] = f; continue; }
        int t0[3], t1[3];
        quad_triangles(P, f, t0, t1);
        int* out = reinterpret_cast<int*>(P.out_faces) + 6 * q;
        out[0] = t0[0]; out[1] = t0[1]; out[2] = t0[2];
        out[3] = t1[0]; out[4] = t1[1]; out[5] = t1[2];
    }
}

// ---- host --------------------------------------------------------------------------------

namespace {
inline unsigned grid_for(long long n, int threads, int num_sms) {
    long long b = (n + threads - 1) / threads;
    const long long cap = (long long)num_sms * 32;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (unsigned)b;
}
inline size_t al(size_t x) { return (x + 255) & ~size_t(255); }
}  // namespace

size_t ours_workspace_bytes(long long nv, long long nq, long long npts, size_t* sort_bytes) {
    const long long nt = 2 * nq;
    // radix sorts: triangle codes (32-bit keys) and point keys (64-bit keys), 32-bit values
    *sort_bytes = std::max(radix_sort_temp_bytes(std::max(1LL, nt), 4, true),
                          radix_sort_temp_bytes(std::max(1LL, npts), 8, true));
    size_t b = 0;
    b += al(sizeof(OursCell) * nv) + al(sizeof(double) * 3 * nv);            // cells, Vm
    b += al(sizeof(int4) * nq) + al(sizeof(double) * 3 * nq);               // quads, gsum
    b += 3 * al(sizeof(uint32_t) * npts) + al(sizeof(int) * npts);           // sel, band/rest, sel_cell
    b += al(sizeof(unsigned long long) * npts) * 2 + al(sizeof(uint32_t) * npts);  // fill keys/values
    b += 3 * al(sizeof(unsigned int) * (nv + 1)) + al(sizeof(uint32_t) * npts);    // count/start/fill, spheres
    b += al(sizeof(uint32_t) * (nv + 1));                                    // cells with many spheres
    b += al(sizeof(uint32_t) * npts);                                        // selected points, sorted
    b += al(sizeof(int) * npts);                                             // last closest triangle per point
    b += al(sizeof(unsigned long long) * nt) + al(sizeof(int2) * nt) + al(sizeof(int) * 2 * nt);
    b += 4 * al(sizeof(uint32_t) * nt);                                      // triangle codes / indices
    b += 2 * al(sizeof(float4) * 2 * nt) + al(sizeof(unsigned int) * nt) + al(sizeof(double) * 9 * nt);
    b += al(sizeof(uint32_t) * (scan_partials_len(nv + 1) + 1)) + al(64);    // scan partials, counters
    b += al(*sort_bytes);
    return b + 4096;
}

cudaError_t ours_run(OursRun& R, cudaStream_t s) {
    OursParams& P = R.P;
    const long long nv = P.nv, nq = P.nq, nt = 2 * nq, npts = (long long)P.g.nx * P.g.ny * P.g.nz;
    char* base = reinterpret_cast<char*>(R.workspace);
    size_t at = 0;
    auto take = [&](size_t bytes) { void* p = base + at; at += al(bytes); return p; };
    P.cells = (OursCell*)take(sizeof(OursCell) * nv);
    P.Vm = (double*)take(sizeof(double) * 3 * nv);
    P.quads = (int4*)take(sizeof(int4) * nq);
    P.gsum = (double*)take(sizeof(double) * 3 * nq);
    uint32_t* sel = (uint32_t*)take(sizeof(uint32_t) * npts);
    uint32_t* band = (uint32_t*)take(sizeof(uint32_t) * npts);
    uint32_t* rest = (uint32_t*)take(sizeof(uint32_t) * npts);
    P.sel_cell = (int*)take(sizeof(int) * npts);
    unsigned long long* fk = (unsigned long long*)take(sizeof(unsigned long long) * npts);
    unsigned long long* fk2 = (unsigned long long*)take(sizeof(unsigned long long) * npts);
    uint32_t* fv2 = (uint32_t*)take(sizeof(uint32_t) * npts);
    P.cell_count = (unsigned int*)take(sizeof(unsigned int) * (nv + 1));
    P.cell_start = (unsigned int*)take(sizeof(unsigned int) * (nv + 1));
    P.cell_fill = (unsigned int*)take(sizeof(unsigned int) * (nv + 1));
    P.cell_spheres = (uint32_t*)take(sizeof(uint32_t) * npts);
    P.heavy = (uint32_t*)take(sizeof(uint32_t) * (nv + 1));
    P.mkeys_sorted = (unsigned long long*)take(sizeof(unsigned long long) * nt);
    P.tcode = (uint32_t*)take(sizeof(uint32_t) * nt);
    P.tidx = (uint32_t*)take(sizeof(uint32_t) * nt);
    P.tcode_sorted = (uint32_t*)take(sizeof(uint32_t) * nt);
    P.tidx_sorted = (uint32_t*)take(sizeof(uint32_t) * nt);
    P.child = (int2*)take(sizeof(int2) * nt);
    P.parent = (int*)take(sizeof(int) * 2 * nt);
    P.bmin = (float4*)take(sizeof(float4) * 2 * nt);
    P.bmax = (float4*)take(sizeof(float4) * 2 * nt);
    P.flags = (unsigned int*)take(sizeof(unsigned int) * nt);
    P.tri9 = (double*)take(sizeof(double) * 9 * nt);
    uint32_t* partials = (uint32_t*)take(sizeof(uint32_t) * (scan_partials_len(nv + 1) + 1));
    unsigned int* counters = (unsigned int*)take(64);
    void* sort_temp = take(R.sort_bytes);
    uint32_t* sel_sorted = (uint32_t*)take(sizeof(uint32_t) * npts);
    P.prev_tri = (int*)take(sizeof(int) * npts);
    P.heavy_count = counters + 8;
    P.sel = sel_sorted;
    P.nt = nt;
    const int sms = R.num_sms;
    cudaError_t e;
#define OURS_TRY(x) do { e = (x); if (e != cudaSuccess) return e; } while (0)
    OURS_TRY(cudaMemsetAsync(counters, 0, 64, s));
    OURS_TRY(cudaMemsetAsync(P.prev_tri, 0xff, sizeof(int) * npts, s));
    k_ours_init<<<grid_for(nv, 128, sms), 128, 0, s>>>(P);
    k_ours_quads<<<grid_for(nq, 128, sms), 128, 0, s>>>(P);
    k_ours_select<<<grid_for(npts, 256, sms), 256, 0, s>>>(P, npts, band, rest, counters);
    OURS_TRY(cudaGetLastError());
    unsigned int hc[2] = {0, 0};
    OURS_TRY(cudaMemcpyAsync(hc, counters, sizeof(hc), cudaMemcpyDeviceToHost, s));
    OURS_TRY(cudaStreamSynchronize(s));
    const long long nband = hc[0], nrest = hc[1];
    const long long bounded = std::min<long long>(R.batch_size, npts);
    const long long nfill = nband < bounded ? std::min(bounded - nband, nrest) : 0;
    P.nsel = nband + nfill;
    // the near-surface points never change: Morton-ordered once (a warp's queries then cover
    // a compact block of the grid); a random fill is ordered again every outer iteration
    if (nband > 0) {
        k_ours_point_keys<<<grid_for(nband, 256, sms), 256, 0, s>>>(P, band, nband, fk);
        OURS_TRY(radix_sort_pairs(sort_temp, R.sort_bytes, fk, fk2, band, sel_sorted, nband, 0, 63, s));
    }
    for (int it = 0; it < R.outer_iters; ++it) {
        if (nq > 0) {
            k_ours_tris<<<grid_for(nq, 128, sms), 128, 0, s>>>(P);
            OURS_TRY(radix_sort_pairs(sort_temp, R.sort_bytes, P.tcode, P.tcode_sorted, P.tidx, P.tidx_sorted, nt, 0, 30, s));
            k_bvh_keys<<<grid_for(nt, 256, sms), 256, 0, s>>>(P);
            OURS_TRY(cudaMemsetAsync(P.flags, 0, sizeof(unsigned int) * nt, s));
            if (nt > 1) k_bvh_tree<<<grid_for(nt - 1, 128, sms), 128, 0, s>>>(P);
            else OURS_TRY(cudaMemsetAsync(P.parent, 0xff, sizeof(int) * 2, s));
            k_bvh_boxes<<<grid_for(nt, 128, sms), 128, 0, s>>>(P);
            if (nfill > 0) {
                k_ours_fill_keys<<<grid_for(nrest, 256, sms), 256, 0, s>>>(rest, nrest, R.seed, it, fk);
                OURS_TRY(radix_sort_pairs(sort_temp, R.sort_bytes, fk, fk2, rest, fv2, nrest, 0, 64, s));
                k_ours_point_keys<<<grid_for(nfill, 256, sms), 256, 0, s>>>(P, fv2, nfill, fk);
                OURS_TRY(radix_sort_pairs(sort_temp, R.sort_bytes, fk, fk2, fv2, sel_sorted + nband, nfill, 0, 63, s));
            }
            OURS_TRY(cudaMemsetAsync(P.cell_count, 0, sizeof(unsigned int) * (nv + 1), s));
            OURS_TRY(cudaMemsetAsync(P.cell_fill, 0, sizeof(unsigned int) * (nv + 1), s));
            OURS_TRY(cudaMemsetAsync(P.heavy_count, 0, sizeof(unsigned int), s));
            k_ours_query<<<grid_for(P.nsel, 128, sms), 128, 0, s>>>(P);
            OURS_TRY(launch_scan(P.cell_count, nv, partials, P.cell_start,
                                 reinterpret_cast<unsigned long long*>(counters + 4), s));
            k_ours_scatter<<<grid_for(P.nsel, 128, sms), 128, 0, s>>>(P);
            k_ours_sort<<<grid_for(nv, 128, sms), 128, 0, s>>>(P);
        } else {
            OURS_TRY(cudaMemsetAsync(P.cell_count, 0, sizeof(unsigned int) * (nv + 1), s));
            OURS_TRY(cudaMemsetAsync(P.heavy_count, 0, sizeof(unsigned int), s));
        }
        k_ours_faces<<<grid_for(nv, 128, sms), 128, 0, s>>>(P);
        if (R.hermite_update && it > 0) k_ours_hermite<<<grid_for(12 * nv, 128, sms), 128, 0, s>>>(P);
        k_ours_inner<<<grid_for(nv, 128, sms), 128, 0, s>>>(P);
        k_ours_inner_warp<<<grid_for(32 * nv, 128, sms), 128, 0, s>>>(P);
        k_ours_mesh<<<grid_for(nv, 128, sms), 128, 0, s>>>(P);
        OURS_TRY(cudaGetLastError());
    }
    if (R.outer_iters == 0) k_ours_mesh<<<grid_for(nv, 128, sms), 128, 0, s>>>(P);
    k_ours_output<<<grid_for(std::max(nv, nq), 128, sms), 128, 0, s>>>(P, R.triangles);
    OURS_TRY(cudaGetLastError());
#undef OURS_TRY
    return cudaSuccess;
}

}  // namespace dcb
