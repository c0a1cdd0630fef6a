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
//   k_cell_qef       one thread per active cell. Each lane walks only its own crossing
//                    edges. On an edge every trilinear gradient reduces to the edge difference
//                    plus two bilinear differences, so the four cells' normals of an averaged
//                    edge need 10 grid values; every cell sharing the edge recomputes the same
//                    average (no storage, no neighbour lookups). Hermite positions are kept in
//                    cell-local units, the centred normal equations are summed with Kahan
//                    compensation, and the cell is solved at once when its spectrum is
//                    provably rank 1 (power iteration + trace test); every other cell is
//                    appended to a compact list. The kernel also emits the face mask of the
//                    cell's three min-corner edges and the per-column face counts.
//   k_cell_jacobi    the listed cells: cyclic Jacobi in FP32.
// FP32 is not trusted when an eigenvalue sits within a relative band of the threshold,
// when the retained condition exceeds the limit, or when a normal's direction is decided
// by cancellation (gradient tiny against its terms, or four normals nearly cancelling);
// such cells go to the FP64 path (dcb_vertex64.cu), which repeats the CPU arithmetic.
#include "dcb_qef.cuh"

namespace dcb {

// Hermite normal of one crossing edge: the 4-cell average when the edge is in the averaging
// set, else the cell's own trilinear normal at its sample. The average is a function of
// the edge alone, so every cell sharing the edge computes the same value.
// lo: global low endpoint; o1/o2: offset (0/1) of the low endpoint from the cell along d1/d2.
__device__ float3 edge_normal(const GridDesc& g, int3 lo, int axis, int o1, int o2, float s_lo, float s_hi,
                              float t_lo, float pu, float pv, float pw, const float cc[8],
                              const Widths& W, bool& ill) {
    const int3 hi = add3(lo, axis, 1);
    const bool in0 = lo.x > 0 && lo.x < g.nx - 1 && lo.y > 0 && lo.y < g.ny - 1 && lo.z > 0 && lo.z < g.nz - 1;
    const bool in1 = hi.x > 0 && hi.x < g.nx - 1 && hi.y > 0 && hi.y < g.ny - 1 && hi.z > 0 && hi.z < g.nz - 1;
    const int d1 = axis == 0 ? 1 : 0;
    const int d2 = axis == 2 ? 1 : 2;
    bool avg = in0 || in1;
    if (avg && !strict_change(s_lo, s_hi)) {
        // zero endpoint: the four cells are not automatically active
        for (int q = 0; q < 4 && avg; ++q) {
            int3 c = lo;
            if (q & 1) c = add3(c, d1, -1);
            if (q & 2) c = add3(c, d2, -1);
            avg = active_at(g, c.x, c.y, c.z);
        }
    }
    if (!avg) return normalized(own_gradient(cc, pu, pv, pw, W.r[0][1], W.r[1][1], W.r[2][1], ill));
    // Along-edge sample of each cell in its own EDGE_PAIRS orientation: X edges start at
    // local x=1 when local y=1, Y edges at local y=1 when local x=0, Z edges at z=0. A cell
    // starting at the high end samples at 1 - t_hi, which equals t_lo unless |s_lo - s_hi| is
    // tiny (both t are then formed in double, exactly as the CPU forms them).
    const float u_hi = fabsf(s_lo - s_hi) < 1e-6f ? 1.f - lerp_t(s_hi, s_lo) : t_lo;
    const int64_t st1 = d1 == 0 ? 1 : (int64_t)g.nx;
    const int64_t st2 = d2 == 1 ? (int64_t)g.nx : (int64_t)g.nx * g.ny;
    const float* plo = g.v + pidx(g, lo.x, lo.y, lo.z);
    const float* phi = g.v + pidx(g, hi.x, hi.y, hi.z);
    const float ga = (s_hi - s_lo) * (axis == 0 ? W.r[0][1] : (axis == 1 ? W.r[1][1] : W.r[2][1]));
    // perpendicular differences at both edge ends: forward (m=0) and backward (m=1)
    const float a0p = __ldg(plo + st1) - s_lo, a0m = s_lo - __ldg(plo - st1);
    const float a1p = __ldg(phi + st1) - s_hi, a1m = s_hi - __ldg(phi - st1);
    const float b0p = __ldg(plo + st2) - s_lo, b0m = s_lo - __ldg(plo - st2);
    const float b1p = __ldg(phi + st2) - s_hi, b1m = s_hi - __ldg(phi - st2);
    // widths of the cells on either side of the edge: the cell index along d is
    // (cell coordinate + o) for m = 0 and one less for m = 1
    // (d1 is y for X edges, else x; d2 is y for Z edges, else z)
    const float rw1p = d1 == 0 ? (o1 ? W.r[0][2] : W.r[0][1]) : (o1 ? W.r[1][2] : W.r[1][1]);
    const float rw1m = d1 == 0 ? (o1 ? W.r[0][1] : W.r[0][0]) : (o1 ? W.r[1][1] : W.r[1][0]);
    const float rw2p = d2 == 1 ? (o2 ? W.r[1][2] : W.r[1][1]) : (o2 ? W.r[2][2] : W.r[2][1]);
    const float rw2m = d2 == 1 ? (o2 ? W.r[1][1] : W.r[1][0]) : (o2 ? W.r[2][1] : W.r[2][0]);
    // one cancellation bound per edge (>= each cell's own bound)
    const float m1v = fmaxf(fmaxf(fabsf(a0p), fabsf(a1p)) * rw1p, fmaxf(fabsf(a0m), fabsf(a1m)) * rw1m);
    const float m2v = fmaxf(fmaxf(fabsf(b0p), fabsf(b1p)) * rw2p, fmaxf(fabsf(b0m), fabsf(b1m)) * rw2m);
    const float bound2 = kNormalCond2 * (ga * ga + m1v * m1v + m2v * m2v);
    // the four gradients (along the edge, along d1, along d2) summed in the edge's own frame,
    // then placed on x, y, z
    float sa = 0.f, s1 = 0.f, s2 = 0.f;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int m1 = q & 1, m2 = q >> 1;
        const bool start_high = (axis == 0) ? (m1 == 1) : (axis == 1) ? (m1 == 0) : false;
        const float u = start_high ? u_hi : t_lo;
        const float e1lo = m1 ? a0m : a0p, e1hi = m1 ? a1m : a1p;
        const float e2lo = m2 ? b0m : b0p, e2hi = m2 ? b1m : b1p;
        const float g1 = (e1lo + u * (e1hi - e1lo)) * (m1 ? rw1m : rw1p);
        const float g2 = (e2lo + u * (e2hi - e2lo)) * (m2 ? rw2m : rw2p);
        const float gn2 = ga * ga + g1 * g1 + g2 * g2;
        if (gn2 <= bound2) ill = true;
        if (gn2 > 0.f) {
            const float rn = rsqrtf(gn2);
            sa += ga * rn; s1 += g1 * rn; s2 += g2 * rn;
        }
    }
    float3 acc;
    if (axis == 0) acc = make_float3(sa, s1, s2);
    else if (axis == 1) acc = make_float3(s1, sa, s2);
    else acc = make_float3(s1, s2, sa);
    if (acc.x * acc.x + acc.y * acc.y + acc.z * acc.z < 1e-4f) ill = true;
    return normalized(acc);
}

// ---- cell-width tables ------------------------------------------------------------------

// Block row b fills grid b's tables: the width of cell c along an axis is the difference of
// the float positions of its two planes (grid.ox + i * grid.vx rounded in float, as the CPU
// backend forms positions, dc_backend.cpp:63-65), its reciprocal 1 / width.
__global__ void __launch_bounds__(256) k_width_tables(const BatchTable B, float* __restrict__ wt) {
    const GridSlot& S = B.n == 1 ? B.s0 : B.slots[blockIdx.y];
    const GridDesc& g = S.g;
    const int nx = g.cx + 2, ny = g.cy + 2, nz = g.cz + 2;
    const int total = nx + ny + nz;
    float* const t = wt + S.wt_off;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        float o, vv;
        int c;
        if (e < nx)           { o = g.ox; vv = g.vx; c = e - 1; }
        else if (e < nx + ny) { o = g.oy; vv = g.vy; c = e - nx - 1; }
        else                  { o = g.oz; vv = g.vz; c = e - nx - ny - 1; }
        const float w = pos_axis(o, vv, c + 1) - pos_axis(o, vv, c);
        t[e] = w;
        t[total + e] = 1.f / w;
    }
}

cudaError_t launch_width_tables(const BatchTable& B, float* wt, cudaStream_t s) {
    if (B.n <= 0) return cudaSuccess;
    k_width_tables<<<dim3(4, (unsigned)B.n), 256, 0, s>>>(B, wt);
    return cudaGetLastError();
}

// ---- k_cell_qef -------------------------------------------------------------------------

// MINB: resident blocks per SM the register allocation must allow (the register cap); the
// autotuner picks 4, 5 or 6 per handle.
template <bool ONE, int MINB>
__global__ void __launch_bounds__(128, MINB)
k_cell_qef(const __grid_constant__ QefParams P) {
    __shared__ unsigned int s_hist;
    __shared__ float s_c[8][128];    // per-thread corner values (dynamically indexed)
    __shared__ float s_t[12][128];   // per-thread lerp parameter of each crossing edge
    const int tid = threadIdx.x;
    if (tid == 0) s_hist = 0;
    __syncthreads();
    // a captured graph whose live count exceeds the capacity it was built for does nothing
    // (the host reports the overflow after the replay)
    const long long nact = P.live ? ((long long)*P.live > P.nactive ? 0 : (long long)*P.live) : P.nactive;
    // the list entry of the next grid-stride step is loaded one step ahead
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long first = (long long)blockIdx.x * blockDim.x + tid;
    uint64_t pk_next = first < nact ? P.list[first] : 0;
    for (long long r = first; r < nact; r += stride) {
        const uint64_t pk = pk_next;
        if (r + stride < nact) pk_next = P.list[r + stride];
        const GridSlot& S = slot_ref<ONE>(P.B, ONE ? 0 : slot_of_rank(P.B, (unsigned long long)r));
        const GridDesc& g = S.g;
        const long long cxcy = (long long)g.cx * g.cy;
        uint32_t* const col_count = P.col_count + S.col_off;
        int i, j, k;
        unpack_cell(pk, i, j, k);
        float c[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            c[q] = ldv(g, i + corner_dx(q), j + corner_dy(q), k + corner_dz(q));
            s_c[q][tid] = c[q];
        }
        // Faces owned by this cell: its min-corner X, Y, Z edges (contouring.cpp:609-729).
        uint8_t fm = 0;
        if (j >= 1 && k >= 1 && strict_change(c[0], c[1])) {
            fm |= 1; atomicAdd(&col_count[0 * cxcy + (long long)i * g.cy + j], 1u);
        }
        if (i >= 1 && k >= 1 && strict_change(c[0], c[3])) {
            fm |= 2; atomicAdd(&col_count[1 * cxcy + (long long)i * g.cy + j], 1u);
        }
        if (i >= 1 && j >= 1 && strict_change(c[0], c[4])) {
            fm |= 4; atomicAdd(&col_count[2 * cxcy + (long long)i * g.cy + j], 1u);
        }
        // an infinite value where the reference's face lookup interpolates from: it exits
        // (contouring.cpp:560-594); the host reports DCB_ERR_INVALID_ARGUMENT
        if (((fm & 1) && isinf(c[1])) || ((fm & 6) && isinf(c[0]))) set_error(P.err, kErrNonFinite);
        P.fmask[r] = fm;

        // Pass 1: crossing edges and the centroid in local units.
        uint32_t hmask = 0;
        float cu = 0.f, cv = 0.f, cw = 0.f;
#pragma unroll
        for (int e = 0; e < 12; ++e) {
            const int a = edge_a(e), b = edge_b(e);
            if (!hermite_crossing(c[a], c[b])) continue;
            hmask |= 1u << e;
            const float t = lerp_t(c[a], c[b]);
            s_t[e][tid] = t;
            float pu = (float)corner_dx(a), pv = (float)corner_dy(a), pw = (float)corner_dz(a);
            if (corner_dx(a) != corner_dx(b)) pu = corner_dx(a) ? 1.f - t : t;
            if (corner_dy(a) != corner_dy(b)) pv = corner_dy(a) ? 1.f - t : t;
            if (corner_dz(a) != corner_dz(b)) pw = corner_dz(a) ? 1.f - t : t;
            cu += pu; cv += pv; cw += pw;
        }
        const float invm = 1.f / (float)__popc(hmask);
        cu *= invm; cv *= invm; cw *= invm;
        // this cell's and its two neighbours' widths along each axis, from the tables
        Widths W;
        {
            const float* const t = P.wt + S.wt_off;
            const int nx = g.cx + 2, ny = g.cy + 2, nz = g.cz + 2, tot = nx + ny + nz;
            const int e0[3] = {i, nx + j, nx + ny + k};   // entry of cell index - 1
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    W.w[a][q] = __ldg(t + e0[a] + q);
                    W.r[a][q] = __ldg(t + tot + e0[a] + q);
                }
        }
        const float fy = W.w[1][1] * W.r[0][1], fz = W.w[2][1] * W.r[0][1];

        // Pass 2: each lane walks its own crossing edges (warp iterations = max count).
        float M00 = 0, M01 = 0, M02 = 0, M11 = 0, M12 = 0, M22 = 0, R0 = 0, R1 = 0, R2 = 0;
        float K00 = 0, K01 = 0, K02 = 0, K11 = 0, K12 = 0, K22 = 0, Q0 = 0, Q1 = 0, Q2 = 0;
        bool ill = false;
        uint32_t rem = hmask;
        while (rem) {
            const int e = __ffs(rem) - 1;
            rem &= rem - 1;
            const uint32_t geo = c_edge_geo[e];
            const int axis = geo & 3;
            const int lox = (geo >> 2) & 1, loy = (geo >> 3) & 1, loz = (geo >> 4) & 1;
            const bool own_low = (geo >> 5) & 1;
            const float s_lo = s_c[(geo >> 6) & 7][tid], s_hi = s_c[(geo >> 9) & 7][tid];
            // this cell's own sample (pass 1): t in its own orientation
            const float t = s_t[e][tid];
            const float along = own_low ? t : 1.f - t;
            const float t_lo = own_low ? t : lerp_t(s_lo, s_hi);
            const float pu = axis == 0 ? along : (float)lox;
            const float pv = axis == 1 ? along : (float)loy;
            const float pw = axis == 2 ? along : (float)loz;
            const int o1 = axis == 0 ? loy : lox, o2 = axis == 2 ? loy : loz;
            const float3 n = edge_normal(g, make_int3(i + lox, j + loy, k + loz), axis, o1, o2, s_lo, s_hi, t_lo,
                                         pu, pv, pw, c, W, ill);
            const float qx = pu - cu, qy = (pv - cv) * fy, qz = (pw - cw) * fz;
            const float nb = n.x * qx + n.y * qy + n.z * qz;
            kahan_add(M00, K00, n.x * n.x); kahan_add(M01, K01, n.x * n.y); kahan_add(M02, K02, n.x * n.z);
            kahan_add(M11, K11, n.y * n.y); kahan_add(M12, K12, n.y * n.z); kahan_add(M22, K22, n.z * n.z);
            kahan_add(R0, Q0, n.x * nb); kahan_add(R1, Q1, n.y * nb); kahan_add(R2, Q2, n.z * nb);
        }

        // A NaN or infinite value in the normal equations, or anywhere in the grid (the CPU
        // backend's trilinear normals then see it through zero-weighted corners, Cell.cpp:80-155,
        // and its SVD factors carry it into the vertex, Cell.cpp:324-361): only the FP64 path
        // repeats that arithmetic, so such cells go there.
        if (!isfinite(M00 + M01 + M02 + M11 + M12 + M22 + R0 + R1 + R2 + cu + cv + cw) || (P.nonfinite && *P.nonfinite))
            ill = true;
        if (ill || P.force64) {
            // FP32 cannot be trusted: the FP64 path recomputes this cell from the grid.
            const unsigned int slot = atomicAdd(P.esc_count, 1u);
            P.esc_list[slot] = (uint32_t)r;
            store_vertex(P.V, g, r, i, j, k, cu, cv, cw);
            continue;
        }
        float ox, oy, oz;
        if (qef_rank1(M00, M01, M02, M11, M12, M22, R0, R1, R2, P.thr, P.band, ox, oy, oz)) {
            store_vertex(P.V, g, r, i, j, k, cu + ox, cv + oy / fy, cw + oz / fz);
            P.vclass[r] = kVcRank1;
            atomicAdd(&s_hist, 1u);
        } else {
            const unsigned int slot = atomicAdd(P.hard_count, 1u);
            P.hard_list[slot] = (uint32_t)r;
            P.hard_data[3 * (size_t)slot + 0] = make_float4(M00, M01, M02, M11);
            P.hard_data[3 * (size_t)slot + 1] = make_float4(M12, M22, R0, R1);
            P.hard_data[3 * (size_t)slot + 2] = make_float4(R2, cu, cv, cw);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_hist) atomicAdd(P.rank_hist + 1, (unsigned long long)s_hist);
}

template <bool ONE>
void launch_cell_qef_t(const QefParams& P, unsigned blocks, int minb, cudaStream_t s) {
    if (minb <= 4)      k_cell_qef<ONE, 4><<<blocks, 128, 0, s>>>(P);
    else if (minb == 5) k_cell_qef<ONE, 5><<<blocks, 128, 0, s>>>(P);
    else                k_cell_qef<ONE, 6><<<blocks, 128, 0, s>>>(P);
}

cudaError_t launch_cell_qef(const QefParams& P, int num_sms, cudaStream_t s, int minb, int blocks_per_sm) {
    if (P.nactive <= 0) return cudaSuccess;
    long long blocks = (P.nactive + 127) / 128;
    const long long cap = (long long)num_sms * blocks_per_sm;
    if (blocks > cap) blocks = cap;
    if (P.B.n == 1) launch_cell_qef_t<true>(P, (unsigned)blocks, minb, s);
    else            launch_cell_qef_t<false>(P, (unsigned)blocks, minb, s);
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
#pragma unroll
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
        const GridDesc g = P.B.slots[slot_of_rank(P.B, r)].g;
        const float wx1 = width_axis(g, 0, i), wy1 = width_axis(g, 1, j), wz1 = width_axis(g, 2, k);
        store_vertex(P.V, g, r, i, j, k, d2.y + wx, d2.z + wy * (wx1 / wy1), d2.w + wz * (wx1 / wz1));
        P.vclass[r] = kVcJacobi;
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
