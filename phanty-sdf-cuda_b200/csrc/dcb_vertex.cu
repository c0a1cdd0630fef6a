// dcb_vertex.cu — Hermite estimate, 4-cell normal averaging and QEF solve in FP32, plus
// the face mask of each cell's three min-corner edges.
//
// Semantics follow the reference CPU backend:
//   Hermite samples   Cell::fill_hermite_data (src/cpp/Cell.cpp:162-212): every edge with
//                     fa*fb <= 0, t = fa/(fa - fb + 1e-16), normal = normalised trilinear
//                     gradient of the cell at the sample (Cell.cpp:80-155)
//   averaging         average_hermite_normals / process_edge (src/cpp/hermite_update.cpp:
//                     171-438): a grid edge with an endpoint strictly inside the grid whose
//                     four cells are all active gets n = normalize(sum of the four cells' own
//                     non-zero normals), summed owner, -dir1, -dir2, diagonal; the owner is the
//                     cell at the edge's minimum endpoint
//   QEF               Cell::update / solve_quadratic_system (Cell.cpp:284-361): A^T A, A^T b,
//                     pinv truncating singular values <= svd_threshold, about the centroid
//   faces             extract_mesh_from_cells (src/cpp/contouring.cpp:607-729): a face per
//                     edge with s0*s1 < 0; cell (i,j,k) owns its three min-corner edges.
// The reference GPU kernel clamps vertices, skips the averaging and uses another lerp
// epsilon (src/cuda/dc_cuda.cu:283-423); none of that is reproduced.
//
// Work split:
//   k_edge_normals   one thread per active cell, for each of its min-corner edges (the
//                    edges it owns): the averaged normal, computed once per grid edge. On an
//                    edge every trilinear gradient reduces to the edge difference plus two
//                    bilinear differences, so the four cells' gradients need 10 grid values.
//   k_cell_qef       one thread per active cell: Hermite positions in cell-local units, the
//                    owners' averaged normals (or the own normal off the averaging set), the
//                    centred normal equations with Kahan sums, and the solve when the
//                    spectrum is provably rank 1 (power iteration + trace test); every other
//                    cell is appended to a compact list.
//   k_cell_jacobi    the listed cells: cyclic Jacobi in FP32.
// FP32 is not trusted when an eigenvalue sits within a relative band of the threshold,
// when the retained condition exceeds the limit, or when a normal's direction is decided
// by cancellation (gradient tiny against its terms, or four normals nearly cancelling);
// such cells go to the FP64 path (dcb_vertex64.cu), which repeats the CPU arithmetic.
#include "dcb_kernels.cuh"

namespace dcb {

// A gradient below 1e-2 of the bound on its terms (squared: 1e-4) has a direction that
// FP32 rounding can move by ~1e-5; such cells are re-solved in FP64.
constexpr float kNormalCond2 = 1e-4f;

__device__ __forceinline__ float ldv(const GridDesc& g, int i, int j, int k) {
    return __ldg(g.v + pidx(g, i, j, k));
}
__device__ __forceinline__ float width_axis(const GridDesc& g, int axis, int idx) {
    if (axis == 0) return pos_axis(g.ox, g.vx, idx + 1) - pos_axis(g.ox, g.vx, idx);
    if (axis == 1) return pos_axis(g.oy, g.vy, idx + 1) - pos_axis(g.oy, g.vy, idx);
    return pos_axis(g.oz, g.vz, idx + 1) - pos_axis(g.oz, g.vz, idx);
}
__device__ __forceinline__ float3 normalized(float3 a) {
    const float s = a.x * a.x + a.y * a.y + a.z * a.z;
    if (s > 0.f) {
        const float r = rsqrtf(s);
        return make_float3(a.x * r, a.y * r, a.z * r);
    }
    return a;
}
// t = fa / (fa - fb + 1e-16) (Cell.cpp:49-52); the epsilon only matters for tiny |fa - fb|.
__device__ __forceinline__ float lerp_t(float fa, float fb) {
    const float d = fa - fb;
    if (fabsf(d) < 1e-6f) return (float)((double)fa / ((double)fa - (double)fb + 1e-16));
    return fa / d;
}
__device__ __forceinline__ bool active_at(const GridDesc& g, int i, int j, int k) {
    bool neg = false, pos = false;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const float v = ldv(g, i + corner_dx(c), j + corner_dy(c), k + corner_dz(c));
        neg |= v < 0.f;
        pos |= v > 0.f;
    }
    return neg && pos;
}
__device__ __forceinline__ int3 add3(int3 a, int axis, int d) {
    if (axis == 0) a.x += d; else if (axis == 1) a.y += d; else a.z += d;
    return a;
}
__device__ __forceinline__ int comp(int3 a, int axis) { return axis == 0 ? a.x : (axis == 1 ? a.y : a.z); }
__device__ __forceinline__ float ldp(const GridDesc& g, int3 p) { return ldv(g, p.x, p.y, p.z); }

// ---- k_edge_normals ---------------------------------------------------------------------

__global__ void __launch_bounds__(128)
k_edge_normals(EdgeParams P) {
    const GridDesc& g = P.g;
    const long long cxcy = (long long)g.cx * g.cy;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < P.nactive;
         r += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        unpack_cell(P.list[r], i, j, k);
        const int3 P0 = make_int3(i, j, k);
        const float s0 = ldv(g, i, j, k);
        const bool in0 = i > 0 && i < g.nx - 1 && j > 0 && j < g.ny - 1 && k > 0 && k < g.nz - 1;
        uint8_t flags = 0, fm = 0;
        for (int a = 0; a < 3; ++a) {
            const int3 P1 = add3(P0, a, 1);
            const float s1 = ldp(g, P1);
            // faces owned by this cell (contouring.cpp:609-729 loop ranges)
            if (strict_change(s0, s1)) {
                const bool ok = (a == 0) ? (j >= 1 && k >= 1) : (a == 1) ? (i >= 1 && k >= 1) : (i >= 1 && j >= 1);
                if (ok) {
                    fm |= (uint8_t)(1 << a);
                    atomicAdd(&P.col_count[a * cxcy + (long long)i * g.cy + j], 1u);
                }
            }
            if (!hermite_crossing(s0, s1)) continue;
            const bool in1 = P1.x > 0 && P1.x < g.nx - 1 && P1.y > 0 && P1.y < g.ny - 1 && P1.z > 0 && P1.z < g.nz - 1;
            if (!(in0 || in1)) continue;
            const int d1 = a == 0 ? 1 : 0;
            const int d2 = a == 2 ? 1 : 2;
            if (!strict_change(s0, s1)) {
                // zero endpoint: the four cells are not automatically active
                bool all = true;
                for (int q = 0; q < 4 && all; ++q) {
                    int3 c = P0;
                    if (q & 1) c = add3(c, d1, -1);
                    if (q & 2) c = add3(c, d2, -1);
                    all = active_at(g, c.x, c.y, c.z);
                }
                if (!all) continue;
            }
            // Along-edge sample of each cell in its own EDGE_PAIRS orientation: X edges start
            // at local x=1 when local y=1, Y edges at local y=1 when local x=0, Z edges at z=0.
            const float t_lo = lerp_t(s0, s1), t_hi = lerp_t(s1, s0);
            const float ga = (s1 - s0) / width_axis(g, a, comp(P0, a));
            const float ba = fabsf(ga);
            // perpendicular differences at both edge ends: forward (m=0) and backward (m=1)
            const float a0p = ldp(g, add3(P0, d1, 1)) - s0, a0m = s0 - ldp(g, add3(P0, d1, -1));
            const float a1p = ldp(g, add3(P1, d1, 1)) - s1, a1m = s1 - ldp(g, add3(P1, d1, -1));
            const float b0p = ldp(g, add3(P0, d2, 1)) - s0, b0m = s0 - ldp(g, add3(P0, d2, -1));
            const float b1p = ldp(g, add3(P1, d2, 1)) - s1, b1m = s1 - ldp(g, add3(P1, d2, -1));
            const float rw1p = 1.f / width_axis(g, d1, comp(P0, d1)), rw1m = 1.f / width_axis(g, d1, comp(P0, d1) - 1);
            const float rw2p = 1.f / width_axis(g, d2, comp(P0, d2)), rw2m = 1.f / width_axis(g, d2, comp(P0, d2) - 1);
            float3 acc = make_float3(0.f, 0.f, 0.f);
            bool ill = false;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int m1 = q & 1, m2 = q >> 1;
                const bool start_high = (a == 0) ? (m1 == 1) : (a == 1) ? (m1 == 0) : false;
                const float u = start_high ? 1.f - t_hi : t_lo;
                const float e1lo = m1 ? a0m : a0p, e1hi = m1 ? a1m : a1p;
                const float e2lo = m2 ? b0m : b0p, e2hi = m2 ? b1m : b1p;
                const float rw1 = m1 ? rw1m : rw1p, rw2 = m2 ? rw2m : rw2p;
                const float g1 = ((1.f - u) * e1lo + u * e1hi) * rw1;
                const float g2 = ((1.f - u) * e2lo + u * e2hi) * rw2;
                const float bb1 = ((1.f - u) * fabsf(e1lo) + u * fabsf(e1hi)) * rw1;
                const float bb2 = ((1.f - u) * fabsf(e2lo) + u * fabsf(e2hi)) * rw2;
                float3 gv;
                if (a == 0) gv = make_float3(ga, g1, g2);
                else if (a == 1) gv = make_float3(g1, ga, g2);
                else gv = make_float3(g1, g2, ga);
                const float gn2 = gv.x * gv.x + gv.y * gv.y + gv.z * gv.z;
                if (gn2 <= kNormalCond2 * (ba * ba + bb1 * bb1 + bb2 * bb2)) ill = true;
                const float3 n = normalized(gv);
                if (gn2 > 0.f) { acc.x += n.x; acc.y += n.y; acc.z += n.z; }
            }
            if (acc.x * acc.x + acc.y * acc.y + acc.z * acc.z < 1e-4f) ill = true;
            const float3 n = normalized(acc);
            P.en[3 * r + a] = make_float4(n.x, n.y, n.z, 0.f);
            flags |= (uint8_t)(1 << a);
            if (ill) flags |= (uint8_t)(8 << a);
        }
        P.eflags[r] = flags;
        P.fmask[r] = fm;
    }
}

cudaError_t launch_edge_normals(const EdgeParams& P, int num_sms, cudaStream_t s) {
    if (P.nactive <= 0) return cudaSuccess;
    long long blocks = (P.nactive + 127) / 128;
    const long long cap = (long long)num_sms * 32;
    if (blocks > cap) blocks = cap;
    k_edge_normals<<<(unsigned)blocks, 128, 0, s>>>(P);
    return cudaGetLastError();
}

// ---- k_cell_qef -------------------------------------------------------------------------

__device__ __forceinline__ void kahan_add(float& s, float& c, float x) {
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

__device__ __forceinline__ bool bit_active(const uint32_t* __restrict__ bits, const GridDesc& g, int i, int j, int k) {
    if (i >= g.cx || j >= g.cy || k >= g.cz) return false;
    const int64_t row = (int64_t)j + (int64_t)g.cy * k;
    return (__ldg(bits + row * g.W + (i >> 5)) >> (i & 31)) & 1u;
}

// Full trilinear gradient of cell (i,j,k) at local (u,v,w) (Cell.cpp:80-155), world units,
// with the same cancellation test as the edge kernel. Only used off the averaging set.
__device__ float3 own_gradient(const GridDesc& g, const float c[8], float u, float v, float w,
                               float rdx, float rdy, float rdz, bool& ill) {
    const float S000 = c[0], S100 = c[1], S110 = c[2], S010 = c[3];
    const float S001 = c[4], S101 = c[5], S111 = c[6], S011 = c[7];
    const float omu = 1.f - u, omv = 1.f - v, omw = 1.f - w;
    const float ax0 = S100 - S000, ax1 = S110 - S010, ax2 = S101 - S001, ax3 = S111 - S011;
    const float ay0 = S010 - S000, ay1 = S110 - S100, ay2 = S011 - S001, ay3 = S111 - S101;
    const float az0 = S001 - S000, az1 = S101 - S100, az2 = S011 - S010, az3 = S111 - S110;
    const float wu0 = omv * omw, wu1 = v * omw, wu2 = omv * w, wu3 = v * w;
    const float wv0 = omu * omw, wv1 = u * omw, wv2 = omu * w, wv3 = u * w;
    const float ww0 = omu * omv, ww1 = u * omv, ww2 = omu * v, ww3 = u * v;
    const float3 gr = make_float3((ax0 * wu0 + ax1 * wu1 + ax2 * wu2 + ax3 * wu3) * rdx,
                                  (ay0 * wv0 + ay1 * wv1 + ay2 * wv2 + ay3 * wv3) * rdy,
                                  (az0 * ww0 + az1 * ww1 + az2 * ww2 + az3 * ww3) * rdz);
    const float bu = (fabsf(ax0) * wu0 + fabsf(ax1) * wu1 + fabsf(ax2) * wu2 + fabsf(ax3) * wu3) * rdx;
    const float bv = (fabsf(ay0) * wv0 + fabsf(ay1) * wv1 + fabsf(ay2) * wv2 + fabsf(ay3) * wv3) * rdy;
    const float bw = (fabsf(az0) * ww0 + fabsf(az1) * ww1 + fabsf(az2) * ww2 + fabsf(az3) * ww3) * rdz;
    if (gr.x * gr.x + gr.y * gr.y + gr.z * gr.z <= kNormalCond2 * (bu * bu + bv * bv + bw * bw)) ill = true;
    return gr;
}

// Local -> world and store (double for the final combination: one float rounding).
__device__ __forceinline__ void store_vertex(const QefParams& P, long long r, int i, int j, int k,
                                             float cu, float cv, float cw, float wx, float wy, float wz) {
    const GridDesc& g = P.g;
    const float wx1 = width_axis(g, 0, i), wy1 = width_axis(g, 1, j), wz1 = width_axis(g, 2, k);
    const double fy = (double)wy1 / (double)wx1, fz = (double)wz1 / (double)wx1;
    const double Lx = (double)cu + (double)wx, Ly = (double)cv + (double)wy / fy, Lz = (double)cw + (double)wz / fz;
    P.V[3 * r + 0] = (float)((double)pos_axis(g.ox, g.vx, i) + (double)wx1 * Lx);
    P.V[3 * r + 1] = (float)((double)pos_axis(g.oy, g.vy, j) + (double)wy1 * Ly);
    P.V[3 * r + 2] = (float)((double)pos_axis(g.oz, g.vz, k) + (double)wz1 * Lz);
}

__global__ void __launch_bounds__(128)
k_cell_qef(QefParams P) {
    const GridDesc& g = P.g;
    __shared__ unsigned int s_hist[2];
    __shared__ float s_c[8][128];    // per-thread corner values (dynamically indexed below)
    __shared__ float s_tt[12][128];  // per-thread lerp parameters
    const int tid = threadIdx.x;
    if (tid < 2) s_hist[tid] = 0;
    __syncthreads();
    for (long long r = (long long)blockIdx.x * blockDim.x + tid; r < P.nactive;
         r += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        unpack_cell(P.list[r], i, j, k);
        float c[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            c[q] = ldv(g, i + corner_dx(q), j + corner_dy(q), k + corner_dz(q));
            s_c[q][tid] = c[q];
        }

        // Pass 1: crossing edges, their t, centroid in local units.
        uint32_t hmask = 0;
        float cu = 0.f, cv = 0.f, cw = 0.f;
        int m = 0;
#pragma unroll
        for (int e = 0; e < 12; ++e) {
            const int a = edge_a(e), b = edge_b(e);
            if (!hermite_crossing(c[a], c[b])) continue;
            const float t = lerp_t(c[a], c[b]);
            s_tt[e][tid] = t;
            hmask |= 1u << e;
            float pu = (float)corner_dx(a), pv = (float)corner_dy(a), pw = (float)corner_dz(a);
            if (corner_dx(a) != corner_dx(b)) pu = corner_dx(a) ? 1.f - t : t;
            if (corner_dy(a) != corner_dy(b)) pv = corner_dy(a) ? 1.f - t : t;
            if (corner_dz(a) != corner_dz(b)) pw = corner_dz(a) ? 1.f - t : t;
            cu += pu; cv += pv; cw += pw;
            ++m;
        }
        const float invm = 1.f / (float)m;
        cu *= invm; cv *= invm; cw *= invm;
        const float wx1 = width_axis(g, 0, i), wy1 = width_axis(g, 1, j), wz1 = width_axis(g, 2, k);
        const float fy = wy1 / wx1, fz = wz1 / wx1;
        const float rdx = 1.f / wx1, rdy = 1.f / wy1, rdz = 1.f / wz1;

        // Pass 2: normals and the centred normal equations (Kahan).
        float M00 = 0, M01 = 0, M02 = 0, M11 = 0, M12 = 0, M22 = 0, R0 = 0, R1 = 0, R2 = 0;
        float K00 = 0, K01 = 0, K02 = 0, K11 = 0, K12 = 0, K22 = 0, Q0 = 0, Q1 = 0, Q2 = 0;
        bool ill = false;
        const uint8_t myflags = P.eflags[r];
        for (int e = 0; e < 12; ++e) {
            if (!(hmask & (1u << e))) continue;
            const int a = edge_a(e), b = edge_b(e);
            const int Ax = corner_dx(a), Ay = corner_dy(a), Az = corner_dz(a);
            const int Bx = corner_dx(b), By = corner_dy(b), Bz = corner_dz(b);
            const float t = s_tt[e][tid];
            float pu = (float)Ax, pv = (float)Ay, pw = (float)Az;
            int axis;
            if (Ax != Bx) { pu = Ax ? 1.f - t : t; axis = 0; }
            else if (Ay != By) { pv = Ay ? 1.f - t : t; axis = 1; }
            else { pw = Az ? 1.f - t : t; axis = 2; }
            // owner = cell at the edge's minimum endpoint
            const int ox = min(Ax, Bx), oy = min(Ay, By), oz = min(Az, Bz);
            float3 n;
            bool have = false;
            if ((ox | oy | oz) == 0) {
                if (myflags & (1 << axis)) {
                    const float4 v = P.en[3 * r + axis];
                    n = make_float3(v.x, v.y, v.z);
                    ill |= (myflags >> (3 + axis)) & 1;
                    have = true;
                }
            } else if (bit_active(P.bits, g, i + ox, j + oy, k + oz)) {
                const uint32_t ro = (ox == 1 && oy == 0 && oz == 0)
                                        ? (uint32_t)r + 1u
                                        : cell_rank(P.bits, P.super, g, i + ox, j + oy, k + oz);
                const uint8_t fl = P.eflags[ro];
                if (fl & (1 << axis)) {
                    const float4 v = P.en[3 * (size_t)ro + axis];
                    n = make_float3(v.x, v.y, v.z);
                    ill |= (fl >> (3 + axis)) & 1;
                    have = true;
                }
            }
            if (!have) {
                float cc[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) cc[q] = s_c[q][tid];
                n = normalized(own_gradient(g, cc, pu, pv, pw, rdx, rdy, rdz, ill));
            }
            const float qx = pu - cu, qy = (pv - cv) * fy, qz = (pw - cw) * fz;
            const float nb = n.x * qx + n.y * qy + n.z * qz;
            kahan_add(M00, K00, n.x * n.x); kahan_add(M01, K01, n.x * n.y); kahan_add(M02, K02, n.x * n.z);
            kahan_add(M11, K11, n.y * n.y); kahan_add(M12, K12, n.y * n.z); kahan_add(M22, K22, n.z * n.z);
            kahan_add(R0, Q0, n.x * nb); kahan_add(R1, Q1, n.y * nb); kahan_add(R2, Q2, n.z * nb);
        }

        if (ill || P.force64) {
            // FP32 cannot be trusted: the FP64 path recomputes this cell from the grid.
            const unsigned int slot = atomicAdd(P.esc_count, 1u);
            P.esc_list[slot] = (uint32_t)r;
            store_vertex(P, r, i, j, k, cu, cv, cw, 0.f, 0.f, 0.f);
            continue;
        }
        // Rank-1 certificate: lambda1 by power iteration, lambda2 + lambda3 = trace - lambda1.
        const float tr = M00 + M11 + M22;
        float x0, x1, x2;
        if (M00 >= M11 && M00 >= M22) { x0 = M00; x1 = M01; x2 = M02; }
        else if (M11 >= M22) { x0 = M01; x1 = M11; x2 = M12; }
        else { x0 = M02; x1 = M12; x2 = M22; }
#pragma unroll
        for (int it = 0; it < 4; ++it) {
            const float y0 = M00 * x0 + M01 * x1 + M02 * x2;
            const float y1 = M01 * x0 + M11 * x1 + M12 * x2;
            const float y2 = M02 * x0 + M12 * x1 + M22 * x2;
            const float nn = rsqrtf(fmaxf(y0 * y0 + y1 * y1 + y2 * y2, 1e-30f));
            x0 = y0 * nn; x1 = y1 * nn; x2 = y2 * nn;
        }
        const float lam1 = x0 * (M00 * x0 + M01 * x1 + M02 * x2) + x1 * (M01 * x0 + M11 * x1 + M12 * x2) +
                           x2 * (M02 * x0 + M12 * x1 + M22 * x2);
        const float rest = tr - lam1;
        const float thr = P.thr;
        // certified rank 1 with lambda2/lambda1 < 0.01: four power steps converge to ~1e-8
        if (lam1 > thr * (1.f + P.band) && rest < thr * (1.f - P.band) && rest < 0.01f * lam1) {
            const float proj = (x0 * R0 + x1 * R1 + x2 * R2) / lam1;
            store_vertex(P, r, i, j, k, cu, cv, cw, x0 * proj, x1 * proj, x2 * proj);
            atomicAdd(&s_hist[0], 1u);
        } else {
            const unsigned int slot = atomicAdd(P.hard_count, 1u);
            P.hard_list[slot] = (uint32_t)r;
            P.hard_data[3 * (size_t)slot + 0] = make_float4(M00, M01, M02, M11);
            P.hard_data[3 * (size_t)slot + 1] = make_float4(M12, M22, R0, R1);
            P.hard_data[3 * (size_t)slot + 2] = make_float4(R2, cu, cv, cw);
            atomicAdd(&s_hist[1], 1u);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_hist[0]) atomicAdd(P.rank_hist + 1, (unsigned long long)s_hist[0]);
    }
}

cudaError_t launch_cell_qef(const QefParams& P, int num_sms, cudaStream_t s) {
    if (P.nactive <= 0) return cudaSuccess;
    long long blocks = (P.nactive + 127) / 128;
    const long long cap = (long long)num_sms * 32;
    if (blocks > cap) blocks = cap;
    k_cell_qef<<<(unsigned)blocks, 128, 0, s>>>(P);
    return cudaGetLastError();
}

// ---- k_cell_jacobi ----------------------------------------------------------------------

// Cyclic Jacobi eigen-decomposition of a symmetric 3x3 (Golub & Van Loan 8.5) in FP32.
__device__ __forceinline__ void jacobi3f(float a[3][3], float V[3][3]) {
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) V[r][c] = (r == c) ? 1.f : 0.f;
    for (int sweep = 0; sweep < 8; ++sweep) {
        const float off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        const float diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (off <= 1e-14f * diag || off == 0.f) break;
        for (int pq = 0; pq < 3; ++pq) {
            const int p = pq == 2 ? 1 : 0;
            const int q = pq == 0 ? 1 : 2;
            const float apq = a[p][q];
            if (apq == 0.f) continue;
            const float theta = (a[q][q] - a[p][p]) / (2.f * apq);
            const float t = (theta >= 0.f ? 1.f : -1.f) / (fabsf(theta) + sqrtf(theta * theta + 1.f));
            const float c = rsqrtf(t * t + 1.f), s = t * c;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const float arp = a[r][p], arq = a[r][q];
                a[r][p] = c * arp - s * arq;
                a[r][q] = s * arp + c * arq;
            }
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const float apr = a[p][r], aqr = a[q][r];
                a[p][r] = c * apr - s * aqr;
                a[q][r] = s * apr + c * aqr;
            }
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const float vrp = V[r][p], vrq = V[r][q];
                V[r][p] = c * vrp - s * vrq;
                V[r][q] = s * vrp + c * vrq;
            }
        }
    }
}

__global__ void __launch_bounds__(128)
k_cell_jacobi(QefParams P) {
    __shared__ unsigned int s_hist[4];
    if (threadIdx.x < 4) s_hist[threadIdx.x] = 0;
    __syncthreads();
    const unsigned int n = *P.hard_count;
    for (unsigned int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const uint32_t r = P.hard_list[t];
        const float4 d0 = P.hard_data[3 * (size_t)t], d1 = P.hard_data[3 * (size_t)t + 1], d2 = P.hard_data[3 * (size_t)t + 2];
        int i, j, k;
        unpack_cell(P.list[r], i, j, k);
        float A[3][3] = {{d0.x, d0.y, d0.z}, {d0.y, d0.w, d1.x}, {d0.z, d1.x, d1.y}};
        const float R0 = d1.z, R1 = d1.w, R2 = d2.x;
        float EV[3][3];
        jacobi3f(A, EV);
        const float lam[3] = {fabsf(A[0][0]), fabsf(A[1][1]), fabsf(A[2][2])};
        int rank = 0;
        bool near = false;
        float lmax = 0.f, lmin_ret = 3.4e38f, wx = 0.f, wy = 0.f, wz = 0.f;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            lmax = fmaxf(lmax, lam[q]);
            near |= fabsf(lam[q] - P.thr) <= P.band * P.thr;
            if (lam[q] > P.thr) {
                ++rank;
                lmin_ret = fminf(lmin_ret, lam[q]);
                const float proj = (EV[0][q] * R0 + EV[1][q] * R1 + EV[2][q] * R2) / lam[q];
                wx += EV[0][q] * proj; wy += EV[1][q] * proj; wz += EV[2][q] * proj;
            }
        }
        const bool ill_cond = rank >= 1 && lmax > P.cond_max * lmin_ret;
        atomicAdd(&s_hist[rank], 1u);
        if (near || ill_cond) {
            const unsigned int slot = atomicAdd(P.esc_count, 1u);
            P.esc_list[slot] = r;
        }
        store_vertex(P, r, i, j, k, d2.y, d2.z, d2.w, wx, wy, wz);
    }
    __syncthreads();
    if (threadIdx.x < 4 && s_hist[threadIdx.x]) atomicAdd(P.rank_hist + threadIdx.x, (unsigned long long)s_hist[threadIdx.x]);
}

cudaError_t launch_cell_jacobi(const QefParams& P, long long max_items, int num_sms, cudaStream_t s) {
    if (max_items <= 0) return cudaSuccess;
    long long blocks = (max_items + 127) / 128;
    const long long cap = (long long)num_sms * 16;
    if (blocks > cap) blocks = cap;
    k_cell_jacobi<<<(unsigned)blocks, 128, 0, s>>>(P);
    return cudaGetLastError();
}

}  // namespace dcb
