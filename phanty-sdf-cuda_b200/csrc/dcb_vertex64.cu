// dcb_vertex64.cu — FP64 vertices for cells the FP32 path does not trust, and FP64
// re-decision of uncertain face orientations. Compiled with --fmad=false: every double
// operation is rounded as written, like the reference's x86-64 CPU build, so a cell on this
// path reproduces the CPU backend's double arithmetic (Cell.cpp:57-361,
// hermite_update.cpp:171-438, contouring.cpp:141-207, 624-641).
//
// Per cell: the Hermite samples (with the three neighbours' own samples of an averaged edge),
// then A^T A, A^T b and the centroid summed in edge order (the CPU's std::map order), the
// Jacobi eigen-decomposition and the truncated pseudo-inverse; a lane per (cell, crossing
// edge) and a lane per solve when cells are few, a thread per cell when many.
#include "dcb_f64.cuh"

namespace dcb {

namespace f64 {

__device__ __forceinline__ double shfl_d(double v, int src) { return __shfl_sync(0xffffffffu, v, src); }

// One cell's rows summed in edge order (the CPU's std::map order), then the solve.
__device__ void solve_rows(const double (*rows)[8], uint32_t mask, double thr, double out[3]) {
    double ATA[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, ATb[3] = {0, 0, 0}, c[3] = {0, 0, 0};
    int m = 0;
    for (int e = 0; e < 12; ++e) {
        if (!(mask & (1u << e))) continue;
        const double* R = rows[e];
        const double pe[3] = {R[0], R[1], R[2]}, ne[3] = {R[3], R[4], R[5]};
        const double bb = R[6];
        for (int r = 0; r < 3; ++r) {
            for (int s = 0; s < 3; ++s) ATA[r][s] += ne[r] * ne[s];
            ATb[r] += ne[r] * bb;
        }
        for (int d = 0; d < 3; ++d) c[d] += pe[d];
        ++m;
    }
    solve_about_centroid(ATA, ATb, c, m, thr, out);
}

// ---- adjoint of the vertex map -----------------------------------------------------------
//
// v(cell) = c + M r with c the mean Hermite point, A = sum n n^T, r = sum n n^T (p - c) and
// M = sum over retained eigenpairs (lambda > thr) of u u^T / lambda. For a gradient g of the
// loss at v, with the rank held fixed (topology fixed), the implicit derivative of the
// truncated pseudo-inverse gives
//   r_bar = M g,   c_bar = g - A r_bar,
//   A_bar = -sym((M g)(M r)^T)
//           + sum_{q retained, p truncated} [(g.u_p)(u_q.r) + (g.u_q)(u_p.r)] sym(u_p u_q^T)
//             / ((lambda_q - lambda_p) lambda_q)
// (the retained-retained pairs combine into the -M dA M term, smooth even for equal
// eigenvalues; a retained-truncated pair has the gap lambda_q - lambda_p > 0). Then per
// Hermite sample (p_e, n_e): n_bar = 2 A_bar n + (n.(p-c)) r_bar + (r_bar.n)(p-c),
// p_bar = (r_bar.n) n + c_bar/m, back through the normalisations, the 4-cell average, the
// trilinear gradients and t = fa/(fa - fb + 1e-16) to the grid values of the 4x4x4 stencil.

// A cell's own sample on local edge e, with what its backward needs.
struct Sample {
    double t, p[3], g[3], gn, n[3];
};

__device__ bool sample_fwd(const Cell64& C, int e, Sample& S) {
    const int a = edge_a(e), b = edge_b(e);
    const double fa = C.cs[a], fb = C.cs[b];
    if (fa * fb > 0.0) return false;
    S.t = (fa - 0.0) / (fa - fb + 1e-16);
    for (int d = 0; d < 3; ++d) S.p[d] = (1.0 - S.t) * C.cp[a][d] + S.t * C.cp[b][d];
    tri_grad(C, S.p, S.g);
    S.gn = sqrt(sq3(S.g));
    for (int d = 0; d < 3; ++d) S.n[d] = S.g[d];
    if (S.gn > 0.0) normalize3(S.n);
    return true;
}

// Backward of the trilinear gradient (Cell.cpp:80-155): gbar -> corner values Sbar, point pbar.
__device__ void tri_grad_bwd(const Cell64& C, const double p[3], const double gb[3], double Sb[8], double pb[3]) {
    const double S000 = C.cs[0], S100 = C.cs[1], S110 = C.cs[2], S010 = C.cs[3];
    const double S001 = C.cs[4], S101 = C.cs[5], S111 = C.cs[6], S011 = C.cs[7];
    const double x0 = C.cp[0][0], x1 = C.cp[1][0];
    const double y0 = C.cp[0][1], y1 = C.cp[3][1];
    const double z0 = C.cp[0][2], z1 = C.cp[4][2];
    const double dx = x1 - x0, dy = y1 - y0, dz = z1 - z0;
    const double eps = 1e-12;
    double u = 0.5, v = 0.5, w = 0.5;
    bool fu = false, fv = false, fw = false;           // inside [0,1]: the point moves it
    if (fabs(dx) > eps) { u = (p[0] - x0) / dx; fu = u >= 0.0 && u <= 1.0; }
    if (fabs(dy) > eps) { v = (p[1] - y0) / dy; fv = v >= 0.0 && v <= 1.0; }
    if (fabs(dz) > eps) { w = (p[2] - z0) / dz; fw = w >= 0.0 && w <= 1.0; }
    u = fmax(0.0, fmin(1.0, u)); v = fmax(0.0, fmin(1.0, v)); w = fmax(0.0, fmin(1.0, w));
    const double omu = 1.0 - u, omv = 1.0 - v, omw = 1.0 - w;
    const double ax = fabs(dx) > eps ? gb[0] / dx : 0.0;   // d(loss)/d(df_du)
    const double ay = fabs(dy) > eps ? gb[1] / dy : 0.0;
    const double az = fabs(dz) > eps ? gb[2] / dz : 0.0;
    // corners
    Sb[1] += ax * omv * omw; Sb[0] -= ax * omv * omw; Sb[2] += ax * v * omw; Sb[3] -= ax * v * omw;
    Sb[5] += ax * omv * w;   Sb[4] -= ax * omv * w;   Sb[6] += ax * v * w;   Sb[7] -= ax * v * w;
    Sb[3] += ay * omu * omw; Sb[0] -= ay * omu * omw; Sb[2] += ay * u * omw; Sb[1] -= ay * u * omw;
    Sb[7] += ay * omu * w;   Sb[4] -= ay * omu * w;   Sb[6] += ay * u * w;   Sb[5] -= ay * u * w;
    Sb[4] += az * omu * omv; Sb[0] -= az * omu * omv; Sb[5] += az * u * omv; Sb[1] -= az * u * omv;
    Sb[7] += az * omu * v;   Sb[3] -= az * omu * v;   Sb[6] += az * u * v;   Sb[2] -= az * u * v;
    // parametric coordinates
    const double dux = -(S100 - S000) * omw + (S110 - S010) * omw - (S101 - S001) * w + (S111 - S011) * w;   // d df_du / dv
    const double dwx = -(S100 - S000) * omv - (S110 - S010) * v + (S101 - S001) * omv + (S111 - S011) * v;  // d df_du / dw
    const double duy = -(S010 - S000) * omw + (S110 - S100) * omw - (S011 - S001) * w + (S111 - S101) * w;   // d df_dv / du
    const double dwy = -(S010 - S000) * omu - (S110 - S100) * u + (S011 - S001) * omu + (S111 - S101) * u;  // d df_dv / dw
    const double duz = -(S001 - S000) * omv + (S101 - S100) * omv - (S011 - S010) * v + (S111 - S110) * v;   // d df_dw / du
    const double dvz = -(S001 - S000) * omu - (S101 - S100) * u + (S011 - S010) * omu + (S111 - S110) * u;  // d df_dw / dv
    const double ub = ay * duy + az * duz, vb = ax * dux + az * dvz, wb = ax * dwx + ay * dwy;
    if (fu) pb[0] += ub / dx;
    if (fv) pb[1] += vb / dy;
    if (fw) pb[2] += wb / dz;
}

// Backward of one sample of cell (ci,cj,ck) on local edge e: nbar at its normalised normal,
// pbar at its point; the grid values' adjoints are added into dgrid.
__device__ void sample_bwd(const GridDesc& g, const Cell64& C, int ci, int cj, int ck, int e, const Sample& S,
                           const double nb[3], const double pbar[3], float* dgrid) {
    double gb[3];
    if (S.gn > 0.0) {
        const double nn = S.n[0] * nb[0] + S.n[1] * nb[1] + S.n[2] * nb[2];
        for (int d = 0; d < 3; ++d) gb[d] = (nb[d] - S.n[d] * nn) / S.gn;
    } else {
        for (int d = 0; d < 3; ++d) gb[d] = nb[d];
    }
    double Sb[8] = {0, 0, 0, 0, 0, 0, 0, 0}, pb[3] = {pbar[0], pbar[1], pbar[2]};
    tri_grad_bwd(C, S.p, gb, Sb, pb);
    const int a = edge_a(e), b = edge_b(e);
    double tb = 0.0;
    for (int d = 0; d < 3; ++d) tb += pb[d] * (C.cp[b][d] - C.cp[a][d]);
    const double fa = C.cs[a], fb = C.cs[b];
    if (fa != 0.0 || fb != 0.0) {          // both zero: t = 0 jumps under any change, no derivative
        const double D = fa - fb + 1e-16;
        Sb[a] += tb * (-fb + 1e-16) / (D * D);
        Sb[b] += tb * fa / (D * D);
    }
#pragma unroll
    for (int q = 0; q < 8; ++q)
        if (Sb[q] != 0.0) atomicAdd(dgrid + pidx(g, ci + corner_dx(q), cj + corner_dy(q), ck + corner_dz(q)), (float)Sb[q]);
}

// The QEF part of the adjoint: from the sums A, A^T b, the centroid c and the vertex gradient
// vb, the gradients of A (symmetric, Ab), of r = A^T b - A c (rb) and of c (cb).
__device__ void qef_adjoint(const double A[3][3], const double ATb[3], const double c[3], double thr,
                            const double vb[3], double Ab[3][3], double rb[3], double cb[3]) {
    double E[3][3], U[3][3];
    for (int r = 0; r < 3; ++r) for (int s2 = 0; s2 < 3; ++s2) E[r][s2] = A[r][s2];
    jacobi3(E, U);
    double lam[3];                          // |eigenvalue| for the retained, signed for the rest
    bool keep[3];
    for (int q = 0; q < 3; ++q) { keep[q] = fabs(E[q][q]) > thr; lam[q] = keep[q] ? fabs(E[q][q]) : E[q][q]; }
    double r[3];
    for (int d = 0; d < 3; ++d) r[d] = ATb[d] - (A[d][0] * c[0] + A[d][1] * c[1] + A[d][2] * c[2]);
    // M g, M r, projections on the eigenvectors
    double ug[3], ur[3], Mg[3] = {0, 0, 0}, Mr[3] = {0, 0, 0};
    for (int q = 0; q < 3; ++q) {
        ug[q] = U[0][q] * vb[0] + U[1][q] * vb[1] + U[2][q] * vb[2];
        ur[q] = U[0][q] * r[0] + U[1][q] * r[1] + U[2][q] * r[2];
        if (!keep[q]) continue;
        for (int d = 0; d < 3; ++d) { Mg[d] += U[d][q] * ug[q] / lam[q]; Mr[d] += U[d][q] * ur[q] / lam[q]; }
    }
    for (int x = 0; x < 3; ++x)
        for (int y = 0; y < 3; ++y) Ab[x][y] = -0.5 * (Mg[x] * Mr[y] + Mr[x] * Mg[y]);
    for (int q = 0; q < 3; ++q) {
        if (!keep[q]) continue;
        for (int pp = 0; pp < 3; ++pp) {
            if (keep[pp]) continue;
            const double wpq = 1.0 / ((lam[q] - lam[pp]) * lam[q]);
            const double coef = wpq * (ug[pp] * ur[q] + ug[q] * ur[pp]);
            for (int x = 0; x < 3; ++x)
                for (int y = 0; y < 3; ++y) Ab[x][y] += 0.5 * coef * (U[x][pp] * U[y][q] + U[x][q] * U[y][pp]);
        }
    }
    for (int d = 0; d < 3; ++d) rb[d] = Mg[d];
    for (int d = 0; d < 3; ++d) cb[d] = vb[d] - (A[d][0] * rb[0] + A[d][1] * rb[1] + A[d][2] * rb[2]);
}

}  // namespace f64

__device__ __forceinline__ void store64(const Vertex64Params& P, uint32_t r, unsigned int t, const double x[3]) {
    if (P.Vf) {
        P.Vf[3 * (size_t)r + 0] = (float)x[0];
        P.Vf[3 * (size_t)r + 1] = (float)x[1];
        P.Vf[3 * (size_t)r + 2] = (float)x[2];
        if (P.vclass) P.vclass[r] = kVcFp64;
    }
    if (P.V64) {
        P.V64[3 * (size_t)t + 0] = x[0];
        P.V64[3 * (size_t)t + 1] = x[1];
        P.V64[3 * (size_t)t + 2] = x[2];
    }
}

// Listed cells' FP64 vertices: Vf[rank] (float) and/or V64[t] (double). The launch holds as
// many warps as fit on the GPU at once. With up to kGroupMax cells per warp, the warp's lanes
// take its cells' crossing edges, one (cell, edge) each: the Hermite sample with its averaged
// normal and the normalised row, into shared memory; then a lane per cell sums the rows in
// edge order and solves. With more cells, a thread takes a whole cell. Both give the bits
// of the CPU's double arithmetic.
constexpr int kGroupMax = 8;
constexpr int kV64Threads = 128;

__global__ void __launch_bounds__(kV64Threads)
k_vertex_fp64(Vertex64Params P) {
    __shared__ double s_rows[kV64Threads / 32][kGroupMax][12][8];
    __shared__ uint32_t s_mask[kV64Threads / 32][kGroupMax];
    __shared__ uint8_t s_pair[kV64Threads / 32][kGroupMax * 12];
    const unsigned int n = min(*P.count, P.cap);
    const unsigned int warps = (gridDim.x * blockDim.x) >> 5;
    const unsigned int G = (n + warps - 1) / warps;
    if (G <= (unsigned)kGroupMax) {
        const int lane = threadIdx.x & 31, wb = threadIdx.x >> 5;
        const unsigned int t0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * G;
        if (t0 >= n) return;                                  // warp-uniform
        const unsigned int cnt = min(G, n - t0);
        // lane q < cnt: crossing edges of cell q (Cell.cpp:185: no sample when fa * fb > 0)
        uint32_t emask = 0;
        if ((unsigned)lane < cnt) {
            const uint32_t r = P.cells[t0 + lane];
            int i, j, k;
            unpack_cell(P.list[r], i, j, k);
            const GridDesc g = P.B.slots[slot_of_rank(P.B, r)].g;
            double cs[8];
#pragma unroll
            for (int c = 0; c < 8; ++c)
                cs[c] = (double)__ldg(g.v + pidx(g, i + corner_dx(c), j + corner_dy(c), k + corner_dz(c)));
#pragma unroll
            for (int e = 0; e < 12; ++e)
                if (!(cs[edge_a(e)] * cs[edge_b(e)] > 0.0)) emask |= 1u << e;
            s_mask[wb][lane] = emask;
        }
        unsigned int off = __popc(emask);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int v = __shfl_up_sync(0xffffffffu, off, o);
            if (lane >= o) off += v;
        }
        const unsigned int total = __shfl_sync(0xffffffffu, off, 31);
        off -= __popc(emask);
        for (uint32_t m = emask; m; m &= m - 1) s_pair[wb][off++] = (uint8_t)((lane << 4) | (__ffs(m) - 1));
        __syncwarp();
        for (unsigned int pr = lane; pr < total; pr += 32) {
            const int q = s_pair[wb][pr] >> 4, e = s_pair[wb][pr] & 15;
            const uint32_t r = P.cells[t0 + q];
            int i, j, k;
            unpack_cell(P.list[r], i, j, k);
            const GridDesc g = P.B.slots[slot_of_rank(P.B, r)].g;
            f64::Cell64 C;
            f64::load_cell(g, i, j, k, C);
            double p[3], nn[3];
            f64::edge_sample(g, C, i, j, k, e, p, nn);
            // Cell::update row (Cell.cpp:298-311): normalise, b = n.p
            if (sqrt(f64::sq3(nn)) > 0.0) f64::normalize3(nn);
            double* R = s_rows[wb][q][e];
            R[0] = p[0]; R[1] = p[1]; R[2] = p[2];
            R[3] = nn[0]; R[4] = nn[1]; R[5] = nn[2];
            R[6] = nn[0] * p[0] + nn[1] * p[1] + nn[2] * p[2];
        }
        __syncwarp();
        if ((unsigned)lane < cnt) {
            double x[3];
            f64::solve_rows(s_rows[wb][lane], s_mask[wb][lane], P.thr, x);
            store64(P, P.cells[t0 + lane], t0 + lane, x);
        }
        return;
    }
    for (unsigned int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const uint32_t r = P.cells[t];
        int i, j, k;
        unpack_cell(P.list[r], i, j, k);
        const GridDesc g = P.B.slots[slot_of_rank(P.B, r)].g;
        double x[3];
        f64::cell_vertex_thread(g, i, j, k, P.thr, x);
        store64(P, r, t, x);
    }
}

cudaError_t launch_vertex_fp64(const Vertex64Params& P, long long max_items, int num_sms, cudaStream_t s) {
    if (max_items <= 0) return cudaSuccess;
    static int resident = 0;                           // blocks of k_vertex_fp64 per SM at once
    if (resident == 0) {
        int b = 0;
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_vertex_fp64, kV64Threads, 0);
        if (e != cudaSuccess) return e;
        resident = b > 0 ? b : 1;
    }
    long long blocks = (max_items + kV64Threads - 1) / kV64Threads;
    const long long cap = (long long)num_sms * resident;
    if (blocks > cap) blocks = cap;
    k_vertex_fp64<<<(unsigned)blocks, kV64Threads, 0, s>>>(P);
    return cudaGetLastError();
}

// Thread per uncertain face: orientation exactly as extract_mesh_from_cells decides it
// (contouring.cpp:624-641) from the FP64 vertices of its four cells and FP64 gradients.
// Uncertain faces were staged in canonical order c0, c1, c2, c3.
__global__ void __launch_bounds__(128)
k_winding_fp64(Winding64Params P) {
    const unsigned int n = min(*P.count, P.cap);
    for (unsigned int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const uint4 it = P.items[t];
        const int axis = (int)(it.y & 3u);
        const GridDesc g = P.B.slots[it.y >> 2].g;
        int i, j, k;
        unpack_cell(((uint64_t)it.w << 32) | it.z, i, j, k);
        const int4 q4 = P.quads[it.x];
        const int rr[4] = {q4.x, q4.y, q4.z, q4.w};
        double pv[4][3];
        bool ok = true;
        for (int q = 0; q < 4; ++q) {
            const int idx = P.v64_index[rr[q]];
            if (idx < 0) { ok = false; break; }
            for (int d = 0; d < 3; ++d) pv[q][d] = P.V64[3 * (size_t)idx + d];
        }
        if (!ok) { set_error(P.err, kErrInternal); continue; }
        double g0[3], g1[3];
        f64::grid_gradient(g, i, j, k, g0);
        f64::grid_gradient(g, i + (axis == 0), j + (axis == 1), k + (axis == 2), g1);
        const double gn[3] = {g0[0] + g1[0], g0[1] + g1[1], g0[2] + g1[2]};
        const double ba[3] = {pv[1][0] - pv[0][0], pv[1][1] - pv[0][1], pv[1][2] - pv[0][2]};
        const double da[3] = {pv[3][0] - pv[0][0], pv[3][1] - pv[0][1], pv[3][2] - pv[0][2]};
        double qn[3] = {ba[1] * da[2] - ba[2] * da[1], ba[2] * da[0] - ba[0] * da[2], ba[0] * da[1] - ba[1] * da[0]};
        if (f64::sq3(qn) < 1e-24) {
            const double ca[3] = {pv[2][0] - pv[0][0], pv[2][1] - pv[0][1], pv[2][2] - pv[0][2]};
            qn[0] = ca[1] * da[2] - ca[2] * da[1];
            qn[1] = ca[2] * da[0] - ca[0] * da[2];
            qn[2] = ca[0] * da[1] - ca[1] * da[0];
        }
        bool swap = false;
        if (f64::sq3(gn) > 0 && f64::sq3(qn) > 0) {
            if (qn[0] * gn[0] + qn[1] * gn[1] + qn[2] * gn[2] < 0.0) swap = true;
        }
        if (swap) P.quads[it.x] = make_int4(q4.x, q4.w, q4.z, q4.y);
    }
}

cudaError_t launch_winding_fp64(const Winding64Params& P, long long max_items, int num_sms, cudaStream_t s) {
    if (max_items <= 0) return cudaSuccess;
    long long blocks = (max_items + 127) / 128;
    const long long cap = (long long)num_sms * 8;
    if (blocks > cap) blocks = cap;
    k_winding_fp64<<<(unsigned)blocks, 128, 0, s>>>(P);
    return cudaGetLastError();
}

// Thread per listed quad: the triangle orientations of triangulate_v1 /
// orient_triangles_for_quad (contouring.cpp:40-113) from the FP64 vertices.
__global__ void __launch_bounds__(128)
k_tri_fp64(Tri64Params P) {
    const unsigned int n = min(*P.count, P.cap);
    for (unsigned int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const uint32_t f = P.items[t];
        const int4 q4 = P.quads[f];
        const int rr[4] = {q4.x, q4.y, q4.z, q4.w};
        double pv[4][3];
        bool ok = true;
        for (int q = 0; q < 4; ++q) {
            const int idx = P.v64_index[rr[q]];
            if (idx < 0) { ok = false; break; }
            for (int d = 0; d < 3; ++d) pv[q][d] = P.V64[3 * (size_t)idx + d];
        }
        if (!ok) { set_error(P.err, kErrInternal); continue; }
        const double ba[3] = {pv[1][0] - pv[0][0], pv[1][1] - pv[0][1], pv[1][2] - pv[0][2]};
        const double ca[3] = {pv[2][0] - pv[0][0], pv[2][1] - pv[0][1], pv[2][2] - pv[0][2]};
        const double da[3] = {pv[3][0] - pv[0][0], pv[3][1] - pv[0][1], pv[3][2] - pv[0][2]};
        double qn[3] = {ba[1] * da[2] - ba[2] * da[1], ba[2] * da[0] - ba[0] * da[2], ba[0] * da[1] - ba[1] * da[0]};
        if (f64::sq3(qn) < 1e-24) {
            qn[0] = ca[1] * da[2] - ca[2] * da[1];
            qn[1] = ca[2] * da[0] - ca[0] * da[2];
            qn[2] = ca[0] * da[1] - ca[1] * da[0];
        }
        bool flip0 = false, flip1 = false;
        if (!(f64::sq3(qn) < 1e-24)) {
            const double t0[3] = {ba[1] * ca[2] - ba[2] * ca[1], ba[2] * ca[0] - ba[0] * ca[2], ba[0] * ca[1] - ba[1] * ca[0]};
            const double t1[3] = {ca[1] * da[2] - ca[2] * da[1], ca[2] * da[0] - ca[0] * da[2], ca[0] * da[1] - ca[1] * da[0]};
            flip0 = t0[0] * qn[0] + t0[1] * qn[1] + t0[2] * qn[2] < 0.0;
            flip1 = t1[0] * qn[0] + t1[1] * qn[1] + t1[2] * qn[2] < 0.0;
        }
        int* o = P.tris + 6 * (size_t)f;
        o[0] = rr[0]; o[1] = flip0 ? rr[2] : rr[1]; o[2] = flip0 ? rr[1] : rr[2];
        o[3] = rr[0]; o[4] = flip1 ? rr[3] : rr[2]; o[5] = flip1 ? rr[2] : rr[3];
    }
}

// The adjoint runs in three passes. A grid edge with a crossing is shared by up to four active
// cells, each of which has a row (its Hermite sample as Cell::update uses it) for it; the first
// active cell around the edge (in the averaging's cell order, or the cell itself for an edge
// that is not averaged) owns the edge and handles all its rows, so every sample is computed
// once per pass.
//   k_adjoint_owners thread per (cell, local edge): rows without a crossing cleared, owners listed
//   k_adjoint_rows   four lanes per owner, one per cell of the edge: the edge's samples, the
//                    average, and each cell's row (normal a, point b)
//   k_adjoint_cells  thread per cell: the sums in edge order, the solve's adjoint, and per row
//                    the gradients of its normal and point (written over the row)
//   k_adjoint_push   four lanes per owner: back through the normalisations and the average to
//                    the samples, and from them to the grid values
namespace {

__device__ __forceinline__ bool cell_active_bit(const AdjointParams& P, int i, int j, int k) {
    const uint32_t w = __ldg(P.bits + ((long long)j + (long long)P.g.cy * k) * P.g.W + (i >> 5));
    return (w >> (i & 31)) & 1u;
}

// The cells of edge e of cell (i,j,k) that have a row for it: n = 1 (the cell itself) for an
// edge that is not averaged, else the four cells in averaging order with their activity. Returns
// false when another cell owns the edge.
struct EdgeGroup {
    int n;
    bool avg;
    int cc[4][3];
    int ex[4];
    bool act[4];
};

__device__ bool edge_group(const AdjointParams& P, int i, int j, int k, int e, EdgeGroup& G) {
    const bool inside = f64::edge_cells(P.g, i, j, k, e, G.cc, G.ex);
    if (!inside) {
        G.n = 1; G.avg = false;
        G.cc[0][0] = i; G.cc[0][1] = j; G.cc[0][2] = k; G.ex[0] = e; G.act[0] = true;
        return true;
    }
    G.n = 4;
    int first = -1;
    bool all = true;
    for (int q = 0; q < 4; ++q) {
        const bool own = G.cc[q][0] == i && G.cc[q][1] == j && G.cc[q][2] == k;
        G.act[q] = own || cell_active_bit(P, G.cc[q][0], G.cc[q][1], G.cc[q][2]);
        if (own) G.ex[q] = e;
        if (G.act[q] && first < 0) first = q;
        all = all && G.act[q];
    }
    G.avg = all;                 // all four active: each has a sample on the shared edge
    return G.cc[first][0] == i && G.cc[first][1] == j && G.cc[first][2] == k;
}

__device__ __forceinline__ long long row_index(const AdjointParams& P, const int c[3], int ex) {
    return 12LL * cell_rank(P.bits, P.super, P.g, c[0], c[1], c[2]) + ex;
}

}  // namespace

// Rows without a crossing are cleared; rows that own their edge are listed.
__global__ void __launch_bounds__(128)
k_adjoint_owners(AdjointParams P) {
    const long long nrow = 12 * P.nactive;
    const int lane = threadIdx.x & 31;
    const long long stride = (long long)gridDim.x * blockDim.x;
    // warp-uniform loop: one atomic per warp appends the warp's owners
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < nrow; base += stride) {
        const long long t = base + lane;
        bool own = false;
        if (t < nrow) {
            const long long r = t / 12;
            const int e = (int)(t - 12 * r);
            int i, j, k;
            unpack_cell(P.list[r], i, j, k);
            const int a = edge_a(e), b = edge_b(e);
            const float fa = __ldg(P.g.v + pidx(P.g, i + corner_dx(a), j + corner_dy(a), k + corner_dz(a)));
            const float fb = __ldg(P.g.v + pidx(P.g, i + corner_dx(b), j + corner_dy(b), k + corner_dz(b)));
            if ((double)fa * (double)fb > 0.0) {
                P.rows[t].flags = 0;
            } else {
                EdgeGroup G;
                own = edge_group(P, i, j, k, e, G);
            }
        }
        const uint32_t m = __ballot_sync(0xffffffffu, own);
        if (m == 0) continue;
        unsigned int first = 0;
        if (lane == __ffs(m) - 1) first = atomicAdd(P.owner_count, (unsigned int)__popc(m));
        first = __shfl_sync(0xffffffffu, first, __ffs(m) - 1);
        if (own) P.owners[first + __popc(m & ((1u << lane) - 1u))] = (uint32_t)t;
    }
}

// A quad of lanes per listed edge, lane q for cell q of the edge's group. Loops are warp-uniform
// (the quad shuffles need every lane).
struct QuadSlot {
    EdgeGroup G;
    bool valid, mine;
    f64::Sample S;
};

__device__ void quad_load(const AdjointParams& P, long long o, long long count, int q, QuadSlot& Q) {
    Q.valid = o < count;
    Q.mine = false;
    Q.S.t = Q.S.gn = 0.0;
    for (int d = 0; d < 3; ++d) Q.S.p[d] = Q.S.g[d] = Q.S.n[d] = 0.0;
    if (!Q.valid) return;
    const long long t = P.owners[o];
    const long long r = t / 12;
    const int e = (int)(t - 12 * r);
    int i, j, k;
    unpack_cell(P.list[r], i, j, k);
    edge_group(P, i, j, k, e, Q.G);
    Q.mine = q < Q.G.n && Q.G.act[q];
    if (!Q.mine) return;
    f64::Cell64 X;
    f64::load_cell(P.g, Q.G.cc[q][0], Q.G.cc[q][1], Q.G.cc[q][2], X);
    f64::sample_fwd(X, Q.G.ex[q], Q.S);
}

// The normalised sum of the quad's non-zero sample normals, summed in cell order
// (hermite_update.cpp:334-438); acc before normalisation in accum.
__device__ void quad_average(const f64::Sample& S, int lane, double out[3], double accum[3]) {
    double acc[3] = {0.0, 0.0, 0.0};
    for (int u = 0; u < 4; ++u) {
        double nu[3];
        for (int d = 0; d < 3; ++d) nu[d] = f64::shfl_d(S.n[d], (lane & ~3) | u);
        if (sqrt(f64::sq3(nu)) > 0) { acc[0] += nu[0]; acc[1] += nu[1]; acc[2] += nu[2]; }
    }
    for (int d = 0; d < 3; ++d) { accum[d] = acc[d]; out[d] = acc[d]; }
    f64::normalize3(out);
}

__global__ void __launch_bounds__(128)
k_adjoint_rows(AdjointParams P) {
    const long long count = *P.owner_count;
    const int lane = threadIdx.x & 31, q = lane & 3;
    const long long stride = (long long)gridDim.x * blockDim.x / 4;
    for (long long base = ((long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) / 4; base < count; base += stride) {
        QuadSlot Q;
        quad_load(P, base + (lane >> 2), count, q, Q);
        double avgn[3], acc[3];
        quad_average(Q.S, lane, avgn, acc);
        if (!Q.mine) continue;
        double n[3];
        for (int d = 0; d < 3; ++d) n[d] = Q.G.avg ? avgn[d] : Q.S.n[d];
        if (sqrt(f64::sq3(n)) > 0.0) f64::normalize3(n);      // Cell::update (Cell.cpp:298-311)
        AdjointRow& R = P.rows[row_index(P, Q.G.cc[q], Q.G.ex[q])];
        for (int d = 0; d < 3; ++d) { R.a[d] = n[d]; R.b[d] = Q.S.p[d]; }
        R.flags = 1;
    }
}

__global__ void __launch_bounds__(128)
k_adjoint_cells(AdjointParams P) {
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < P.nactive;
         r += (long long)gridDim.x * blockDim.x) {
        AdjointRow* rows = P.rows + 12 * r;
        const double vb[3] = {P.dV[3 * r], P.dV[3 * r + 1], P.dV[3 * r + 2]};
        if (vb[0] == 0.0 && vb[1] == 0.0 && vb[2] == 0.0) {
            for (int e = 0; e < 12; ++e) rows[e].flags = 0;
            continue;
        }
        double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, ATb[3] = {0, 0, 0}, c[3] = {0, 0, 0};
        int m = 0;
        for (int e = 0; e < 12; ++e) {                   // edge order = the CPU's std::map order
            const AdjointRow& R = rows[e];
            if (!R.flags) continue;
            const double bb = R.a[0] * R.b[0] + R.a[1] * R.b[1] + R.a[2] * R.b[2];
            for (int x = 0; x < 3; ++x) {
                for (int y = 0; y < 3; ++y) A[x][y] += R.a[x] * R.a[y];
                ATb[x] += R.a[x] * bb;
            }
            for (int d = 0; d < 3; ++d) c[d] += R.b[d];
            ++m;
        }
        if (m == 0) continue;
        for (int d = 0; d < 3; ++d) c[d] /= double(m);
        double Ab[3][3], rb[3], cb[3];
        f64::qef_adjoint(A, ATb, c, P.thr, vb, Ab, rb, cb);
        for (int e = 0; e < 12; ++e) {
            AdjointRow& R = rows[e];
            if (!R.flags) continue;
            const double n[3] = {R.a[0], R.a[1], R.a[2]};
            double pc[3];
            for (int d = 0; d < 3; ++d) pc[d] = R.b[d] - c[d];
            const double npc = n[0] * pc[0] + n[1] * pc[1] + n[2] * pc[2];
            const double rn = rb[0] * n[0] + rb[1] * n[1] + rb[2] * n[2];
            for (int d = 0; d < 3; ++d) {
                R.a[d] = 2.0 * (Ab[d][0] * n[0] + Ab[d][1] * n[1] + Ab[d][2] * n[2]) + npc * rb[d] + rn * pc[d];
                R.b[d] = rn * n[d] + cb[d] / double(m);
            }
            R.flags = 2;
        }
    }
}

__global__ void __launch_bounds__(128)
k_adjoint_push(AdjointParams P) {
    const long long count = *P.owner_count;
    const int lane = threadIdx.x & 31, q = lane & 3;
    const long long stride = (long long)gridDim.x * blockDim.x / 4;
    for (long long base = ((long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) / 4; base < count; base += stride) {
        QuadSlot Q;
        quad_load(P, base + (lane >> 2), count, q, Q);
        double avgn[3], acc[3];
        quad_average(Q.S, lane, avgn, acc);
        const bool avg = Q.valid && Q.G.avg;
        // this lane's row gradients, back through Cell::update's normalisation
        double nbar[3] = {0.0, 0.0, 0.0}, pb[3] = {0.0, 0.0, 0.0};
        if (Q.mine) {
            const AdjointRow& R = P.rows[row_index(P, Q.G.cc[q], Q.G.ex[q])];
            if (R.flags == 2) {
                double npre[3];
                for (int d = 0; d < 3; ++d) { npre[d] = avg ? avgn[d] : Q.S.n[d]; pb[d] = R.b[d]; }
                const double npn = sqrt(f64::sq3(npre));
                if (npn > 0.0) {
                    const double n[3] = {npre[0] / npn, npre[1] / npn, npre[2] / npn};
                    const double tt = n[0] * R.a[0] + n[1] * R.a[1] + n[2] * R.a[2];
                    for (int d = 0; d < 3; ++d) nbar[d] = (R.a[d] - n[d] * tt) / npn;
                } else {
                    for (int d = 0; d < 3; ++d) nbar[d] = R.a[d];
                }
            }
        }
        // averaged edge: n_pre = normalize(acc) is shared, so its gradient is the quad's sum
        double sum[3] = {0.0, 0.0, 0.0};
        for (int u = 0; u < 4; ++u)
            for (int d = 0; d < 3; ++d) sum[d] += f64::shfl_d(nbar[d], (lane & ~3) | u);
        if (!Q.mine) continue;
        if (avg) {
            const double accn = sqrt(f64::sq3(acc));
            const bool used = sqrt(f64::sq3(Q.S.n)) > 0;
            double ab[3] = {0.0, 0.0, 0.0};
            if (accn > 0.0 && used) {
                const double tt = avgn[0] * sum[0] + avgn[1] * sum[1] + avgn[2] * sum[2];
                for (int d = 0; d < 3; ++d) ab[d] = (sum[d] - avgn[d] * tt) / accn;
            }
            for (int d = 0; d < 3; ++d) nbar[d] = ab[d];
        }
        const bool any = nbar[0] != 0.0 || nbar[1] != 0.0 || nbar[2] != 0.0 || pb[0] != 0.0 || pb[1] != 0.0 ||
                         pb[2] != 0.0;
        if (!any) continue;
        f64::Cell64 X;
        f64::load_cell(P.g, Q.G.cc[q][0], Q.G.cc[q][1], Q.G.cc[q][2], X);
        f64::sample_bwd(P.g, X, Q.G.cc[q][0], Q.G.cc[q][1], Q.G.cc[q][2], Q.G.ex[q], Q.S, nbar, pb, P.dgrid);
    }
}

cudaError_t launch_vertex_adjoint(const AdjointParams& P, int num_sms, cudaStream_t s) {
    if (P.nactive <= 0) return cudaSuccess;
    const long long cap = (long long)num_sms * 32;
    const long long rb = std::min(cap, (12 * P.nactive + 127) / 128);
    const long long cb = std::min(cap, (P.nactive + 127) / 128);
    cudaError_t err = cudaMemsetAsync(P.owner_count, 0, sizeof(unsigned int), s);
    if (err != cudaSuccess) return err;
    // owners <= rows with a crossing; a quad of lanes each
    const long long qb = std::min(cap, (4 * 12 * P.nactive / 3 + 127) / 128 + 1);
    k_adjoint_owners<<<(unsigned)rb, 128, 0, s>>>(P);
    k_adjoint_rows<<<(unsigned)qb, 128, 0, s>>>(P);
    k_adjoint_cells<<<(unsigned)cb, 128, 0, s>>>(P);
    k_adjoint_push<<<(unsigned)qb, 128, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_tri_fp64(const Tri64Params& P, long long max_items, int num_sms, cudaStream_t s) {
    if (max_items <= 0) return cudaSuccess;
    long long blocks = (max_items + 127) / 128;
    const long long cap = (long long)num_sms * 8;
    if (blocks > cap) blocks = cap;
    k_tri_fp64<<<(unsigned)blocks, 128, 0, s>>>(P);
    return cudaGetLastError();
}

}  // namespace dcb
