// dcb_qef.cuh — device helpers of the FP32 vertex kernels (k_cell_qef and k_cell_jacobi of
// dcb_vertex.cu): Hermite interpolation and
// trilinear normals (src/cpp/Cell.cpp:49-155), cell widths as the reference forms positions
// (src/cpp/dc_backend.cpp:63-65), compensated sums and the rank-1 certified QEF solve.
#pragma once
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
    return __fdividef(fa, d);   // |t| <= 1 here: the 2-ulp quotient is far inside the FP32 budget
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

__device__ __forceinline__ void kahan_add(float& s, float& c, float x) {
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

// Full trilinear gradient of a cell at local (u,v,w) (Cell.cpp:80-155) in world units, with
// a cancellation test. Only used for edges outside the averaging set.
static __device__ float3 own_gradient(const float c[8], float u, float v, float w,
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

// Edge geometry of a cell, packed: bits 0-1 axis, 2-4 low-endpoint offset (x,y,z),
// 5 the cell's EDGE_PAIRS orientation starts at the low endpoint, 6-8 low corner index,
// 9-11 high corner index.
__host__ __device__ constexpr uint32_t edge_geo(int e) {
    return (uint32_t)(corner_dx(edge_a(e)) != corner_dx(edge_b(e)) ? 0 : (corner_dy(edge_a(e)) != corner_dy(edge_b(e)) ? 1 : 2)) |
           ((uint32_t)corner_dx((corner_dx(edge_a(e)) + corner_dy(edge_a(e)) + corner_dz(edge_a(e)) <=
                                 corner_dx(edge_b(e)) + corner_dy(edge_b(e)) + corner_dz(edge_b(e))) ? edge_a(e) : edge_b(e)) << 2) |
           ((uint32_t)corner_dy((corner_dx(edge_a(e)) + corner_dy(edge_a(e)) + corner_dz(edge_a(e)) <=
                                 corner_dx(edge_b(e)) + corner_dy(edge_b(e)) + corner_dz(edge_b(e))) ? edge_a(e) : edge_b(e)) << 3) |
           ((uint32_t)corner_dz((corner_dx(edge_a(e)) + corner_dy(edge_a(e)) + corner_dz(edge_a(e)) <=
                                 corner_dx(edge_b(e)) + corner_dy(edge_b(e)) + corner_dz(edge_b(e))) ? edge_a(e) : edge_b(e)) << 4) |
           ((uint32_t)((corner_dx(edge_a(e)) + corner_dy(edge_a(e)) + corner_dz(edge_a(e)) <=
                        corner_dx(edge_b(e)) + corner_dy(edge_b(e)) + corner_dz(edge_b(e))) ? 1 : 0) << 5) |
           ((uint32_t)((corner_dx(edge_a(e)) + corner_dy(edge_a(e)) + corner_dz(edge_a(e)) <=
                        corner_dx(edge_b(e)) + corner_dy(edge_b(e)) + corner_dz(edge_b(e))) ? edge_a(e) : edge_b(e)) << 6) |
           ((uint32_t)((corner_dx(edge_a(e)) + corner_dy(edge_a(e)) + corner_dz(edge_a(e)) <=
                        corner_dx(edge_b(e)) + corner_dy(edge_b(e)) + corner_dz(edge_b(e))) ? edge_b(e) : edge_a(e)) << 9);
}
static __constant__ uint32_t c_edge_geo[12] = {edge_geo(0), edge_geo(1), edge_geo(2), edge_geo(3), edge_geo(4), edge_geo(5),
                                        edge_geo(6), edge_geo(7), edge_geo(8), edge_geo(9), edge_geo(10), edge_geo(11)};

// Widths (and reciprocals) of the cells i-1, i, i+1 along each axis, exact float
// differences of the float grid positions (the CPU forms positions the same way), read from
// the per-grid tables of k_width_tables.
struct Widths {
    float w[3][3];   // [axis][offset+1]
    float r[3][3];
};

// Local -> world: one double combination per axis, one float rounding.
__device__ __forceinline__ void store_vertex(float* __restrict__ V, const GridDesc& g, long long r, int i, int j, int k,
                                             float Lx, float Ly, float Lz) {
    const float wx1 = width_axis(g, 0, i), wy1 = width_axis(g, 1, j), wz1 = width_axis(g, 2, k);
    V[3 * r + 0] = (float)((double)pos_axis(g.ox, g.vx, i) + (double)wx1 * (double)Lx);
    V[3 * r + 1] = (float)((double)pos_axis(g.oy, g.vy, j) + (double)wy1 * (double)Ly);
    V[3 * r + 2] = (float)((double)pos_axis(g.oz, g.vz, k) + (double)wz1 * (double)Lz);
}


// Rank-1 certificate of the centred normal equations M (A^T A, 6 entries) with right-hand side
// R (A^T b - A^T A c): lambda1 by four power steps from M's largest diagonal column, and
// lambda2 + lambda3 = trace - lambda1. When lambda1 clears the truncation threshold by the
// band, the rest stays below it by the band and below 1% of lambda1, the truncated
// pseudo-inverse keeps only lambda1's eigenvector x and the offset is x * (x.R) / lambda1
// (Cell.cpp:324-361 with one singular value above the threshold). Returns false when the
// spectrum is not certified.
__device__ __forceinline__ bool qef_rank1(float M00, float M01, float M02, float M11, float M12, float M22,
                                          float R0, float R1, float R2, float thr, float band,
                                          float& ox, float& oy, float& oz) {
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
    // certified rank 1 with lambda2/lambda1 < 0.01: four power steps converge to ~1e-8
    if (lam1 > thr * (1.f + band) && rest < thr * (1.f - band) && rest < 0.01f * lam1) {
        const float proj = (x0 * R0 + x1 * R1 + x2 * R2) / lam1;
        ox = x0 * proj; oy = x1 * proj; oz = x2 * proj;
        return true;
    }
    return false;
}

}  // namespace dcb
