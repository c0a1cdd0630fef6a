// dcb_mesh_sdf.cu — triangle mesh -> dense signed distance grid.
//
// Semantics: compute_mesh_sdf_device_cuda without voxelisation
// (src/cuda/mesh_to_sdf_cuda.cu:740-1009, branch :862-951):
//   bins         g = max(1, n/8) per axis, bin size (n*v)/g, every triangle listed in each bin
//                its bounding box grown by 2*max(v) overlaps (:99-190)
//   active bins  some bin of the 3x3x3 block around it is non-empty (:192-224)
//   band         per grid point: closest point over the triangles of its bin, then of the 26
//                neighbours (z, y, x order), ties within 1e-5 relative sum area- (or, at a
//                vertex, angle-) weighted normals; sign from the summed normal; |d| beyond 2.5
//                bins -> far (:226-360)
//   sign fill    far points reached from the border or from a positive point through far
//                points are +10, the other far points -10 (:362-428)
//   relaxation   4 Jacobi passes of |v| <- min(|v|, |neighbour| + h) beyond 1.5 h (:430-456)
// Determinism (the reference fills bins with atomics and floods with racing in-place
// passes): bins list their triangles in ascending index, and the flood runs to its fixpoint.
// The file is compiled with --fmad=false: every float expression is rounded as written, like
// the CPU restatement it is checked against.
//
// B200 layout of the work:
//   k_tri_prep      triangle records (bounding sphere, vertices, unit normal, doubled area)
//                   + per-bin counts (atomics)
//   k_tri_bins      scatter into bins (atomics), then k_bin_order ranks each bin's entries
//                   by triangle index (CTA per bin, shared-memory tiles), so the order is the
//                   ascending one whatever the atomics did
//   k_bin_active    active flags + a compact list of the active bins; k_axis_starts the
//                   first grid point of every bin per axis; k_fill_far sets every value far
//   k_band          persistent CTAs take active bins from a work counter; the 27-bin
//                   visiting sequence is the same for every point of a bin, so its triangle
//                   records stream through shared memory once per 8 cubes of 4x4x4 points
//                   (a cube per warp, 2 points per thread). A triangle whose bounding sphere
//                   provably lies beyond a point's running minimum plus the tie tolerance is
//                   skipped — the reference loop would ignore it at that point of the
//                   sequence, so skipping it changes no bit. The test runs first for a whole
//                   warp (lane l takes the l-th of 32 triangles against the warp's point box
//                   and largest reach), then per point, then with the triangle's plane,
//                   before the exact distance.
//   k_sdf_masks     far / positive bit words (ballots over x rows)
//   k_flood         exterior flood on bit words: 4x16x16-word tiles iterate to local
//                   convergence in shared memory; the host repeats until nothing changes
//   k_sdf_finish    far -> +-10; then 4 relaxation passes (k_relax)
#include <algorithm>
#include <cfloat>
#include "dcb_kernels.cuh"

namespace dcb {

namespace {

constexpr float kFar = FLT_MAX;

// Triangle record, 5 x 16 bytes.
struct Tri {
    float4 s;   // bounding sphere: centroid xyz, radius grown by a rounding allowance
    float4 a;   // v0.xyz, doubled area (0: skipped, as the reference skips area <= 1e-12)
    float4 b;   // v1.xyz
    float4 c;   // v2.xyz
    float4 n;   // unit normal xyz
};
constexpr int kTriF4 = 5;
static_assert(sizeof(Tri) == kTriF4 * sizeof(float4), "record = kTriF4 float4s");

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sub(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 scl(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

__device__ __forceinline__ int bin_coord(float x, float o, float bd, int g) {
    return max(0, min(g - 1, (int)floorf((x - o) / bd)));
}

// Closest point on triangle abc to p and its squared distance (Ericson, Real-Time Collision
// Detection 5.1.5; the case analysis of mesh_to_sdf_cuda.cu:40-97).
__device__ float point_triangle(float3 p, float3 a, float3 b, float3 c, float3& out) {
    const float3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) { out = a; return dot(ap, ap); }
    const float3 bp = sub(p, b);
    const float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) { out = b; return dot(bp, bp); }
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        const float v = d1 / (d1 - d3);
        out = add(a, scl(v, ab));
        const float3 e = sub(p, out);
        return dot(e, e);
    }
    const float3 cp = sub(p, c);
    const float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) { out = c; return dot(cp, cp); }
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        const float w = d2 / (d2 - d6);
        out = add(a, scl(w, ac));
        const float3 e = sub(p, out);
        return dot(e, e);
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        out = add(b, scl(w, sub(c, b)));
        const float3 e = sub(p, out);
        return dot(e, e);
    }
    const float denom = 1.0f / (va + vb + vc);
    const float v = vb * denom, w = vc * denom;
    out = add(add(a, scl(v, ab)), scl(w, ac));
    const float3 e = sub(p, out);
    return dot(e, e);
}

__device__ __forceinline__ float angle_at(float3 e1, float3 e2, float fallback) {
    const float l1 = sqrtf(dot(e1, e1)), l2 = sqrtf(dot(e2, e2));
    if (l1 > 1e-6f && l2 > 1e-6f) {
        const float c = fmaxf(-1.0f, fminf(1.0f, dot(e1, e2) / (l1 * l2)));
        return (float)acos((double)c);
    }
    return fallback;
}

__device__ __forceinline__ void tri_bin_range(const SdfParams& P, float3 a, float3 b, float3 c, int* r) {
    const float mnx = fminf(a.x, fminf(b.x, c.x)) - P.margin;
    const float mny = fminf(a.y, fminf(b.y, c.y)) - P.margin;
    const float mnz = fminf(a.z, fminf(b.z, c.z)) - P.margin;
    const float mxx = fmaxf(a.x, fmaxf(b.x, c.x)) + P.margin;
    const float mxy = fmaxf(a.y, fmaxf(b.y, c.y)) + P.margin;
    const float mxz = fmaxf(a.z, fmaxf(b.z, c.z)) + P.margin;
    r[0] = bin_coord(mnx, P.ox, P.bdx, P.gx); r[1] = bin_coord(mxx, P.ox, P.bdx, P.gx);
    r[2] = bin_coord(mny, P.oy, P.bdy, P.gy); r[3] = bin_coord(mxy, P.oy, P.bdy, P.gy);
    r[4] = bin_coord(mnz, P.oz, P.bdz, P.gz); r[5] = bin_coord(mxz, P.oz, P.bdz, P.gz);
}

__device__ __forceinline__ bool load_tri(const SdfParams& P, long long f, float3& a, float3& b, float3& c) {
    const int i0 = P.faces[3 * f], i1 = P.faces[3 * f + 1], i2 = P.faces[3 * f + 2];
    if (i0 < 0 || i1 < 0 || i2 < 0 || i0 >= P.nv || i1 >= P.nv || i2 >= P.nv) {
        set_error(P.err, kErrInvalid);
        return false;
    }
    a = f3(P.verts[3 * (size_t)i0], P.verts[3 * (size_t)i0 + 1], P.verts[3 * (size_t)i0 + 2]);
    b = f3(P.verts[3 * (size_t)i1], P.verts[3 * (size_t)i1 + 1], P.verts[3 * (size_t)i1 + 2]);
    c = f3(P.verts[3 * (size_t)i2], P.verts[3 * (size_t)i2 + 1], P.verts[3 * (size_t)i2 + 2]);
    return true;
}

__global__ void __launch_bounds__(256) k_tri_prep(SdfParams P) {
    for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < P.nf; f += (long long)gridDim.x * blockDim.x) {
        float3 a, b, c;
        if (!load_tri(P, f, a, b, c)) continue;
        float3 n = cross(sub(b, a), sub(c, a));
        const float a2 = sqrtf(dot(n, n));
        const bool ok = a2 > 1e-12f;
        if (ok) n = f3(n.x / a2, n.y / a2, n.z / a2);
        // Bounding sphere about the centroid; the radius is grown by 1e-5 of the coordinate
        // magnitudes so that it bounds the float closest points as well.
        const float3 cc = f3((a.x + b.x + c.x) / 3.f, (a.y + b.y + c.y) / 3.f, (a.z + b.z + c.z) / 3.f);
        const float3 da = sub(a, cc), db = sub(b, cc), dcv = sub(c, cc);
        const float R = sqrtf(fmaxf(dot(da, da), fmaxf(dot(db, db), dot(dcv, dcv))));
        const float mag = fmaxf(fmaxf(fabsf(cc.x), fabsf(cc.y)), fabsf(cc.z)) + R;
        Tri* t = reinterpret_cast<Tri*>(P.tris) + f;
        t->s = make_float4(cc.x, cc.y, cc.z, R * 1.0001f + 1e-5f * mag);
        t->a = make_float4(a.x, a.y, a.z, ok ? a2 : 0.f);
        t->b = make_float4(b.x, b.y, b.z, 0.f);
        t->c = make_float4(c.x, c.y, c.z, 0.f);
        t->n = make_float4(n.x, n.y, n.z, 0.f);
        int r[6];
        tri_bin_range(P, a, b, c, r);
        for (int bz = r[4]; bz <= r[5]; ++bz)
            for (int by = r[2]; by <= r[3]; ++by)
                for (int bx = r[0]; bx <= r[1]; ++bx)
                    atomicAdd(&P.bin_count[bx + (long long)P.gx * (by + (long long)P.gy * bz)], 1u);
    }
}

__global__ void __launch_bounds__(256) k_tri_bins(SdfParams P) {
    for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < P.nf; f += (long long)gridDim.x * blockDim.x) {
        float3 a, b, c;
        if (!load_tri(P, f, a, b, c)) continue;
        int r[6];
        tri_bin_range(P, a, b, c, r);
        for (int bz = r[4]; bz <= r[5]; ++bz)
            for (int by = r[2]; by <= r[3]; ++by)
                for (int bx = r[0]; bx <= r[1]; ++bx) {
                    const long long bin = bx + (long long)P.gx * (by + (long long)P.gy * bz);
                    const uint32_t slot = P.bin_start[bin] + atomicAdd(&P.bin_fill[bin], 1u);
                    P.bin_scratch[slot] = (uint32_t)f;
                }
    }
}

// CTA per bin: entry e goes to position (number of entries with a smaller triangle index);
// triangle indices are unique within a bin.
constexpr int kOrderThreads = 128;
constexpr int kOrderTile = 1024;
__global__ void __launch_bounds__(kOrderThreads) k_bin_order(SdfParams P) {
    __shared__ uint32_t s_key[kOrderTile];
    for (long long bin = blockIdx.x; bin < P.nbins; bin += gridDim.x) {
        const uint32_t start = P.bin_start[bin], n = P.bin_count[bin];
        if (n == 0) continue;
        const uint32_t* in = P.bin_scratch + start;
        for (uint32_t i0 = 0; i0 < n; i0 += kOrderThreads * 8) {
            uint32_t key[8], rank[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const uint32_t i = i0 + threadIdx.x + q * kOrderThreads;
                key[q] = i < n ? in[i] : 0xffffffffu;
                rank[q] = 0;
            }
            for (uint32_t j0 = 0; j0 < n; j0 += kOrderTile) {
                const uint32_t m = min((uint32_t)kOrderTile, n - j0);
                __syncthreads();
                for (uint32_t j = threadIdx.x; j < m; j += kOrderThreads) s_key[j] = in[j0 + j];
                __syncthreads();
                for (uint32_t j = 0; j < m; ++j) {
                    const uint32_t kj = s_key[j];
#pragma unroll
                    for (int q = 0; q < 8; ++q) rank[q] += kj < key[q] ? 1u : 0u;
                }
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const uint32_t i = i0 + threadIdx.x + q * kOrderThreads;
                if (i < n) P.bin_tris[start + rank[q]] = key[q];
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) k_bin_active(SdfParams P) {
    for (long long bin = (long long)blockIdx.x * blockDim.x + threadIdx.x; bin < P.nbins; bin += (long long)gridDim.x * blockDim.x) {
        const int bx = (int)(bin % P.gx), by = (int)((bin / P.gx) % P.gy), bz = (int)(bin / ((long long)P.gx * P.gy));
        uint8_t act = 0;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int x = bx + dx, y = by + dy, z = bz + dz;
                    if (x < 0 || x >= P.gx || y < 0 || y >= P.gy || z < 0 || z >= P.gz) continue;
                    if (P.bin_count[x + (long long)P.gx * (y + (long long)P.gy * z)]) act = 1;
                }
        P.bin_active[bin] = act;
        if (act) P.active_list[atomicAdd(P.active_count, 1u)] = (uint32_t)bin;   // order is irrelevant
    }
}

// First grid point along an axis whose bin coordinate is >= b (bins are monotone in the point
// index); searched around the nominal b*n/g.
__device__ int first_point_of_bin(int b, int n, int g, float o, float v, float bd) {
    if (b <= 0) return 0;
    if (b >= g) return n;
    int x = max(0, (int)(((long long)b * n) / g) - 3);
    while (x < n && bin_coord(o + (float)x * v, o, bd, g) < b) ++x;
    return x;
}

// axis_start = [x: gx+1][y: gy+1][z: gz+1] first points of the bins along each axis.
__global__ void k_axis_starts(SdfParams P) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t <= P.gx) P.axis_start[t] = first_point_of_bin(t, P.nx, P.gx, P.ox, P.vx, P.bdx);
    else if (t <= P.gx + 1 + P.gy) P.axis_start[t] = first_point_of_bin(t - (P.gx + 1), P.ny, P.gy, P.oy, P.vy, P.bdy);
    else if (t <= P.gx + P.gy + P.gz + 2) P.axis_start[t] = first_point_of_bin(t - (P.gx + P.gy + 2), P.nz, P.gz, P.oz, P.vz, P.bdz);
}

// Every value starts far; the band kernel overwrites the points of the active bins. (Scalar
// stores: the caller's array need not be 16-byte aligned.)
__global__ void __launch_bounds__(256) k_fill_far(SdfParams P) {
    const long long n = (long long)P.nx * P.ny * P.nz;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        P.out[q] = kFar;
}

constexpr int kBandThreads = 256;
constexpr int kBandChunk = 256;   // triangle records staged per pass (20 KB)
constexpr int kBandPts = 2;       // grid points per thread (a 4x4x4 cube per warp)

// Running closest-triangle state of one grid point.
struct BandPoint {
    float3 p;
    float best, reach;            // reach: beyond it a triangle cannot reach the tie window
    float3 bp, bn;
};

__device__ __forceinline__ float reach_of(float best, float pm) {
    if (best == kFar) return kFar;
    return sqrtf(best + 1e-5f * (best + 1e-8f)) * 1.00001f + 1e-5f * pm;
}

// One triangle against one point, exactly as evaluate_sdf_grid_kernel's loop body, after two
// lower bounds of the distance: the bounding sphere, then the plane distance h and the
// lateral distance beyond the sphere (d^2 >= h^2 + (l - R)^2). A triangle beyond the point's
// reach has a float distance above best + tolerance, so the reference loop ignores it too.
// The record is read from shared memory by the caller (s_rec = the record's 5 float4s).
__device__ __forceinline__ void visit(BandPoint& q, float pm, const float4 (&s_rec)[kTriF4], float veps) {
    const float4 ts = s_rec[0];
    if (q.best != kFar) {
        const float dx = q.p.x - ts.x, dy = q.p.y - ts.y, dz = q.p.z - ts.z;
        const float d2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
        const float lim = q.reach + ts.w;
        if (d2 > __fmul_rn(__fmul_rn(lim, lim), 1.00002f)) return;
        const float4 tn = s_rec[4];
        const float reach2 = __fmul_rn(__fmul_rn(q.reach, q.reach), 1.00002f);
        const float allow = 2e-5f * (pm + fabsf(ts.x) + fabsf(ts.y) + fabsf(ts.z) + ts.w);
        const float h = __fmaf_rn(dx, tn.x, __fmaf_rn(dy, tn.y, __fmul_rn(dz, tn.z)));
        const float hh = fmaxf(0.f, fabsf(h) - allow);
        const float lat = sqrtf(fmaxf(0.f, d2 - h * h));
        const float ll = fmaxf(0.f, lat - ts.w - allow);
        if (__fmaf_rn(hh, hh, __fmul_rn(ll, ll)) > reach2) return;
    }
    const float4 ta = s_rec[1];
    if (!(ta.w > 0.f)) return;                          // area <= 1e-12: skipped
    const float4 tb = s_rec[2], tc = s_rec[3];
    const float3 v0 = f3(ta.x, ta.y, ta.z), v1 = f3(tb.x, tb.y, tb.z), v2 = f3(tc.x, tc.y, tc.z);
    float3 cp;
    const float d = point_triangle(q.p, v0, v1, v2, cp);
    const float tol = 1e-5f * (q.best + 1e-8f);
    const bool replace = d < q.best - tol;
    if (!replace && !(fabsf(d - q.best) <= tol)) return;   // ignored: its weight is never used
    // weight: the doubled area, or the angle at a vertex the closest point sits on
    float w = ta.w;
    const float3 c0v = sub(cp, v0), c1v = sub(cp, v1), c2v = sub(cp, v2);
    if (dot(c0v, c0v) < veps) w = angle_at(sub(v1, v0), sub(v2, v0), w);
    else if (dot(c1v, c1v) < veps) w = angle_at(sub(v0, v1), sub(v2, v1), w);
    else if (dot(c2v, c2v) < veps) w = angle_at(sub(v0, v2), sub(v1, v2), w);
    const float4 tn = s_rec[4];
    if (replace) {
        q.best = d;
        q.bp = cp;
        q.bn = f3(w * tn.x, w * tn.y, w * tn.z);
        q.reach = reach_of(d, pm);
    } else {
        q.bn = f3(q.bn.x + w * tn.x, q.bn.y + w * tn.y, q.bn.z + w * tn.z);
    }
}

__global__ void __launch_bounds__(kBandThreads, 2) k_band(SdfParams P) {
    __shared__ float4 s_tri[kBandChunk][kTriF4];
    __shared__ int s_seq_bin[27];
    __shared__ uint32_t s_seq_start[28];
    __shared__ uint32_t s_next;
    const uint32_t nact = *P.active_count;
    const int lane = threadIdx.x & 31;
    for (;;) {
        // next active bin from the shared work counter (bins differ a lot in cost)
        __syncthreads();
        if (threadIdx.x == 0) s_next = atomicAdd(P.work_next, 1u);
        __syncthreads();
        const uint32_t ai = s_next;
        if (ai >= nact) break;
        const long long bin = P.active_list[ai];
        const int bx = (int)(bin % P.gx), by = (int)((bin / P.gx) % P.gy), bz = (int)(bin / ((long long)P.gx * P.gy));
        const int* ys_ = P.axis_start + P.gx + 1;
        const int* zs_ = ys_ + P.gy + 1;
        const int x0 = P.axis_start[bx], x1 = P.axis_start[bx + 1];
        const int y0 = ys_[by], y1 = ys_[by + 1];
        const int z0 = zs_[bz], z1 = zs_[bz + 1];
        const int sx = x1 - x0, sy = y1 - y0, sz = z1 - z0;
        if (sx <= 0 || sy <= 0 || sz <= 0) continue;
        // points go to warps in 4x4x4 cubes (lane: 4x4x2, the second point 2 planes up), so
        // that a warp's point box, used to cull triangles, stays small
        const int cx4 = (sx + 3) / 4, cy4 = (sy + 3) / 4, cz4 = (sz + 3) / 4;
        const int ncubes = cx4 * cy4 * cz4;
        // visiting sequence: centre bin, then the shell of radius 1 in z, y, x order; lane t of
        // warp 0 takes the t-th of the 27 slots, a warp scan gives the starts
        __syncthreads();
        if (threadIdx.x < 32) {
            const int t = threadIdx.x;
            int nb = -1;
            if (t == 0) {
                nb = (int)bin;
            } else if (t < 27) {
                const int r = t <= 13 ? t - 1 : t;          // shell slots skip the centre (13)
                const int xx = bx + r % 3 - 1, yy = by + (r / 3) % 3 - 1, zz = bz + r / 9 - 1;
                if (xx >= 0 && xx < P.gx && yy >= 0 && yy < P.gy && zz >= 0 && zz < P.gz)
                    nb = (int)(xx + (long long)P.gx * (yy + (long long)P.gy * zz));
            }
            const uint32_t c = nb >= 0 ? P.bin_count[nb] : 0u;
            uint32_t incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
                if (t >= o) incl += v;
            }
            if (t < 27) { s_seq_bin[t] = nb; s_seq_start[t] = incl - c; }
            if (t == 26) s_seq_start[27] = incl;
        }
        __syncthreads();
        const uint32_t L = s_seq_start[27];
        const float veps = 1e-6f * P.min_box * P.min_box;
        for (int cube0 = 0; cube0 < ncubes; cube0 += kBandThreads / 32) {
            BandPoint q[kBandPts];
            float pm[kBandPts];
            bool mine[kBandPts];
            int pidx[kBandPts][3];
            const int cube = cube0 + (threadIdx.x >> 5);
            const int ccx = cube % cx4, ccy = (cube / cx4) % cy4, ccz = cube / (cx4 * cy4);
#pragma unroll
            for (int u = 0; u < kBandPts; ++u) {
                const int lx = 4 * ccx + (lane & 3), ly = 4 * ccy + ((lane >> 2) & 3), lz = 4 * ccz + (lane >> 4) + 2 * u;
                mine[u] = cube < ncubes && lx < sx && ly < sy && lz < sz;
                const int ix = x0 + (mine[u] ? lx : 0), iy = y0 + (mine[u] ? ly : 0), iz = z0 + (mine[u] ? lz : 0);
                pidx[u][0] = ix; pidx[u][1] = iy; pidx[u][2] = iz;
                q[u].p = f3(P.ox + (float)ix * P.vx, P.oy + (float)iy * P.vy, P.oz + (float)iz * P.vz);
                pm[u] = fmaxf(fabsf(q[u].p.x), fmaxf(fabsf(q[u].p.y), fabsf(q[u].p.z)));
                q[u].best = kFar;
                q[u].reach = kFar;
                q[u].bp = f3(0.f, 0.f, 0.f);
                q[u].bn = f3(0.f, 1.f, 0.f);
            }
            // box of this warp's points (lanes without a point add nothing)
            float3 wlo = f3(kFar, kFar, kFar), whi = f3(-kFar, -kFar, -kFar);
#pragma unroll
            for (int u = 0; u < kBandPts; ++u) {
                if (!mine[u]) continue;
                wlo = f3(fminf(wlo.x, q[u].p.x), fminf(wlo.y, q[u].p.y), fminf(wlo.z, q[u].p.z));
                whi = f3(fmaxf(whi.x, q[u].p.x), fmaxf(whi.y, q[u].p.y), fmaxf(whi.z, q[u].p.z));
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                wlo.x = fminf(wlo.x, __shfl_xor_sync(0xffffffffu, wlo.x, o));
                wlo.y = fminf(wlo.y, __shfl_xor_sync(0xffffffffu, wlo.y, o));
                wlo.z = fminf(wlo.z, __shfl_xor_sync(0xffffffffu, wlo.z, o));
                whi.x = fmaxf(whi.x, __shfl_xor_sync(0xffffffffu, whi.x, o));
                whi.y = fmaxf(whi.y, __shfl_xor_sync(0xffffffffu, whi.y, o));
                whi.z = fmaxf(whi.z, __shfl_xor_sync(0xffffffffu, whi.z, o));
            }
            for (uint32_t c0 = 0; c0 < L; c0 += kBandChunk) {
                const uint32_t m = min((uint32_t)kBandChunk, L - c0);
                __syncthreads();
                for (uint32_t ent = threadIdx.x; ent < m; ent += kBandThreads) {
                    const uint32_t sq = c0 + ent;
                    int b = 0;                                   // last slot with start <= sq
#pragma unroll
                    for (int step = 16; step > 0; step >>= 1)
                        if (b + step < 27 && s_seq_start[b + step] <= sq) b += step;
                    const uint32_t f = P.bin_tris[P.bin_start[s_seq_bin[b]] + (sq - s_seq_start[b])];
                    const float4* rec = reinterpret_cast<const float4*>(P.tris) + kTriF4 * (size_t)f;
                    float4 r[kTriF4];
#pragma unroll
                    for (int part = 0; part < kTriF4; ++part) r[part] = rec[part];
#pragma unroll
                    for (int part = 0; part < kTriF4; ++part) s_tri[ent][part] = r[part];
                }
                __syncthreads();
                // Warp culling: lane l tests entry base+l against the box of the warp's points
                // and the warp's largest reach; only entries that pass are visited by every
                // lane (each of which still applies its own exact-preserving tests).
                for (uint32_t base = 0; base < m; base += 32) {
                    float wr = 0.f;
#pragma unroll
                    for (int u = 0; u < kBandPts; ++u)
                        if (mine[u]) wr = fmaxf(wr, q[u].reach);
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) wr = fmaxf(wr, __shfl_xor_sync(0xffffffffu, wr, o));
                    const uint32_t e = base + lane;
                    bool cand = false;
                    if (e < m && s_tri[e][1].w > 0.f) {
                        cand = true;
                        if (wr != kFar) {
                            const float4 ts = s_tri[e][0];
                            const float ex = fmaxf(fmaxf(wlo.x - ts.x, ts.x - whi.x), 0.f);
                            const float ey = fmaxf(fmaxf(wlo.y - ts.y, ts.y - whi.y), 0.f);
                            const float ez = fmaxf(fmaxf(wlo.z - ts.z, ts.z - whi.z), 0.f);
                            const float dd = __fmaf_rn(ex, ex, __fmaf_rn(ey, ey, __fmul_rn(ez, ez)));
                            const float lim = wr + ts.w;
                            cand = !(dd > __fmul_rn(__fmul_rn(lim, lim), 1.00002f));
                        }
                    }
                    uint32_t live = __ballot_sync(0xffffffffu, cand);
                    while (live) {
                        const int b = __ffs(live) - 1;
                        live &= live - 1;
#pragma unroll
                        for (int u = 0; u < kBandPts; ++u)
                            if (mine[u]) visit(q[u], pm[u], s_tri[base + b], veps);
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kBandPts; ++u) {
                if (!mine[u]) continue;
                float val = kFar;
                if (q[u].best != kFar) {
                    float dist = sqrtf(q[u].best);
                    float3 bn = q[u].bn;
                    const float nl = sqrtf(dot(bn, bn));
                    if (nl > 1e-12f) bn = f3(bn.x / nl, bn.y / nl, bn.z / nl);
                    if (dot(sub(q[u].p, q[u].bp), bn) < 0.0f) dist = -dist;
                    if (!(dist > 2.5f * P.min_box || dist < -2.5f * P.min_box)) val = dist;
                }
                P.out[pidx[u][0] + (long long)P.nx * (pidx[u][1] + (long long)P.ny * pidx[u][2])] = val;
            }
        }
    }
}

// Far / positive bit words, warp per 32-word stretch of one x row.
__global__ void __launch_bounds__(256) k_sdf_masks(SdfParams P) {
    const int lane = threadIdx.x & 31;
    const long long rows = (long long)P.ny * P.nz;
    const long long per_row = (P.W + 31) / 32;
    const long long groups = rows * per_row;
    for (long long gq = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; gq < groups;
         gq += ((long long)gridDim.x * blockDim.x) >> 5) {
        const long long row = gq / per_row;
        const int w0 = (int)(gq % per_row) * 32;
        const int j = (int)(row % P.ny), k = (int)(row / P.ny);
        const bool border_row = j == 0 || j == P.ny - 1 || k == 0 || k == P.nz - 1;
        const float* src = P.out + row * P.nx;
        uint32_t my_far = 0, my_ext = 0;
        for (int q = 0; q < 32 && w0 + q < P.W; ++q) {
            const int x = 32 * (w0 + q) + lane;
            const float v = x < P.nx ? src[x] : 0.f;
            const bool far = x < P.nx && v == kFar;
            const bool pos = x < P.nx && v != kFar && v > 0.0f;
            const bool border = x < P.nx && (border_row || x == 0 || x == P.nx - 1);
            const uint32_t bf = __ballot_sync(0xffffffffu, far);
            const uint32_t be = __ballot_sync(0xffffffffu, pos || (far && border));
            if (lane == q) { my_far = bf; my_ext = be; }
        }
        if (w0 + lane < P.W) {
            P.far[row * P.W + w0 + lane] = my_far;
            P.ext[row * P.W + w0 + lane] = my_ext;
        }
    }
}

// Exterior flood on bit words. Tile = kFX words x kFY rows x kFZ planes; the neighbouring
// tiles' words are read once per launch as fixed sources; the tile iterates to its local
// fixpoint. ext <- ext | (far & (ext shifted by one point along x, y or z)). Bits only ever
// get set, so reading a word another thread is updating in the same sweep is harmless.
constexpr int kFX = 4, kFY = 16, kFZ = 16;
constexpr int kFloodThreads = 256;
constexpr int kFloodLocalCap = 4 * (32 * kFX + kFY + kFZ);   // local sweeps before yielding
__global__ void __launch_bounds__(kFloodThreads) k_flood(SdfParams P, int* changed) {
    __shared__ uint32_t s_ext[kFZ + 2][kFY + 2][kFX + 2];
    __shared__ uint32_t s_far[kFZ][kFY][kFX];
    __shared__ int s_any, s_tile_changed;
    const long long tx = (P.W + kFX - 1) / kFX, ty = (P.ny + kFY - 1) / kFY, tz = (P.nz + kFZ - 1) / kFZ;
    for (long long tile = blockIdx.x; tile < tx * ty * tz; tile += gridDim.x) {
        const int wx0 = (int)(tile % tx) * kFX, y0 = (int)((tile / tx) % ty) * kFY, z0 = (int)(tile / (tx * ty)) * kFZ;
        __syncthreads();
        if (threadIdx.x == 0) { s_any = 0; s_tile_changed = 0; }
        __syncthreads();
        for (int e = threadIdx.x; e < (kFZ + 2) * (kFY + 2) * (kFX + 2); e += kFloodThreads) {
            const int lx = e % (kFX + 2), ly = (e / (kFX + 2)) % (kFY + 2), lz = e / ((kFX + 2) * (kFY + 2));
            const int w = wx0 + lx - 1, y = y0 + ly - 1, z = z0 + lz - 1;
            uint32_t v = 0;
            if (w >= 0 && w < P.W && y >= 0 && y < P.ny && z >= 0 && z < P.nz) v = P.ext[((long long)z * P.ny + y) * P.W + w];
            s_ext[lz][ly][lx] = v;
            if (lx >= 1 && lx <= kFX && ly >= 1 && ly <= kFY && lz >= 1 && lz <= kFZ) {
                const uint32_t f = (w < P.W && y < P.ny && z < P.nz) ? P.far[((long long)z * P.ny + y) * P.W + w] : 0u;
                s_far[lz - 1][ly - 1][lx - 1] = f;
                if (f & ~v) s_any = 1;   // unreached far points here
            }
        }
        __syncthreads();
        if (!s_any) continue;
        for (int it = 0; it < kFloodLocalCap; ++it) {
            int mine = 0;
            for (int e = threadIdx.x; e < kFZ * kFY * kFX; e += kFloodThreads) {
                const int lx = e % kFX + 1, ly = (e / kFX) % kFY + 1, lz = e / (kFX * kFY) + 1;
                const uint32_t cur = s_ext[lz][ly][lx];
                const uint32_t far = s_far[lz - 1][ly - 1][lx - 1];
                const uint32_t nb = (cur << 1) | (cur >> 1) | (s_ext[lz][ly][lx - 1] >> 31) | (s_ext[lz][ly][lx + 1] << 31) |
                                    s_ext[lz][ly - 1][lx] | s_ext[lz][ly + 1][lx] | s_ext[lz - 1][ly][lx] | s_ext[lz + 1][ly][lx];
                const uint32_t nxt = cur | (far & nb);
                if (nxt != cur) { s_ext[lz][ly][lx] = nxt; mine = 1; }
            }
            const int any = __syncthreads_or(mine);
            if (!any) break;
            if (threadIdx.x == 0) s_tile_changed = 1;
        }
        __syncthreads();
        if (s_tile_changed) {
            for (int e = threadIdx.x; e < kFZ * kFY * kFX; e += kFloodThreads) {
                const int lx = e % kFX, ly = (e / kFX) % kFY, lz = e / (kFX * kFY);
                const int w = wx0 + lx, y = y0 + ly, z = z0 + lz;
                if (w < P.W && y < P.ny && z < P.nz) P.ext[((long long)z * P.ny + y) * P.W + w] = s_ext[lz + 1][ly + 1][lx + 1];
            }
            if (threadIdx.x == 0) atomicExch(changed, 1);
        }
    }
}

// Far points -> +10 (exterior) or -10; block per x row.
__global__ void __launch_bounds__(256) k_sdf_finish(SdfParams P, unsigned long long* filled) {
    const long long rows = (long long)P.ny * P.nz;
    unsigned long long cnt = 0;
    for (long long row = blockIdx.x; row < rows; row += gridDim.x) {
        float* r = P.out + row * P.nx;
        const uint32_t* e = P.ext + row * P.W;
        for (int x = threadIdx.x; x < P.nx; x += blockDim.x) {
            if (r[x] != kFar) continue;
            const bool ex = (e[x >> 5] >> (x & 31)) & 1u;
            r[x] = ex ? 10.0f : -10.0f;
            cnt += ex ? 1 : 0;
        }
    }
    if (cnt) atomicAdd(filled, cnt);
}

// One Jacobi pass of the relaxation (eikonal_relaxation_kernel); block per x row.
__global__ void __launch_bounds__(256) k_relax(SdfParams P, const float* __restrict__ in, float* __restrict__ out) {
    const long long rows = (long long)P.ny * P.nz;
    const long long plane = (long long)P.nx * P.ny;
    const float keep = fminf(P.vx, fminf(P.vy, P.vz)) * 1.5f;
    for (long long row = blockIdx.x; row < rows; row += gridDim.x) {
        const int iy = (int)(row % P.ny), iz = (int)(row / P.ny);
        const long long base = row * P.nx;
        for (int ix = threadIdx.x; ix < P.nx; ix += blockDim.x) {
            const long long q = base + ix;
            const float val = in[q];
            if (fabsf(val) <= keep) { out[q] = val; continue; }
            float a = fabsf(val);
            const float s = val < 0.0f ? -1.0f : 1.0f;
            if (ix > 0) a = fminf(a, fabsf(in[q - 1]) + P.vx);
            if (ix < P.nx - 1) a = fminf(a, fabsf(in[q + 1]) + P.vx);
            if (iy > 0) a = fminf(a, fabsf(in[q - P.nx]) + P.vy);
            if (iy < P.ny - 1) a = fminf(a, fabsf(in[q + P.nx]) + P.vy);
            if (iz > 0) a = fminf(a, fabsf(in[q - plane]) + P.vz);
            if (iz < P.nz - 1) a = fminf(a, fabsf(in[q + plane]) + P.vz);
            out[q] = s * a;
        }
    }
}

// ---- voxelize-first (compute_mesh_sdf_device_cuda with voxelize_first, :764-832) -------------

// A thread per triangle: every voxel corner of the triangle's voxel box whose squared distance
// to the triangle is within (0.866 * largest voxel side)^2 joins the shell (:458-501).
__global__ void __launch_bounds__(256) k_vox_raster(SdfParams P) {
    const int vr = P.vres;
    const float mvd = fmaxf(P.vox_vx, fmaxf(P.vox_vy, P.vox_vz)) * 0.8660254f;
    const float lim = mvd * mvd;
    for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < P.nf; f += (long long)gridDim.x * blockDim.x) {
        float3 a, b, c;
        if (!load_tri(P, f, a, b, c)) continue;
        const float mnx = fminf(a.x, fminf(b.x, c.x)), mny = fminf(a.y, fminf(b.y, c.y)), mnz = fminf(a.z, fminf(b.z, c.z));
        const float mxx = fmaxf(a.x, fmaxf(b.x, c.x)), mxy = fmaxf(a.y, fmaxf(b.y, c.y)), mxz = fmaxf(a.z, fmaxf(b.z, c.z));
        const int bx0 = bin_coord(mnx, P.ox, P.vox_vx, vr), bx1 = bin_coord(mxx, P.ox, P.vox_vx, vr);
        const int by0 = bin_coord(mny, P.oy, P.vox_vy, vr), by1 = bin_coord(mxy, P.oy, P.vox_vy, vr);
        const int bz0 = bin_coord(mnz, P.oz, P.vox_vz, vr), bz1 = bin_coord(mxz, P.oz, P.vox_vz, vr);
        for (int bz = bz0; bz <= bz1; ++bz)
            for (int by = by0; by <= by1; ++by)
                for (int bx = bx0; bx <= bx1; ++bx) {
                    const float3 q = f3(P.ox + (float)bx * P.vox_vx, P.oy + (float)by * P.vox_vy, P.oz + (float)bz * P.vox_vz);
                    float3 closest;
                    if (point_triangle(q, a, b, c, closest) <= lim)
                        atomicOr(P.vshell + ((long long)bz * vr + by) * P.Wv + (bx >> 5), 1u << (bx & 31));
                }
    }
}

// The shell dilated by one voxel (27-neighbourhood, :503-526), then the flood's inputs: the
// voxels outside the dilated shell pass the exterior flood, and those of them on the border
// seed it (init_voxel_exterior_kernel, :561-575). A thread per 32-voxel word.
__global__ void __launch_bounds__(256) k_vox_dilate(SdfParams P) {
    const int vr = P.vres;
    const long long words = (long long)vr * vr * P.Wv;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < words;
         idx += (long long)gridDim.x * blockDim.x) {
        const int w = (int)(idx % P.Wv);
        const long long row = idx / P.Wv;
        const int y = (int)(row % vr), z = (int)(row / vr);
        uint32_t dil = 0;
        for (int zz = max(0, z - 1); zz <= min(vr - 1, z + 1); ++zz)
            for (int yy = max(0, y - 1); yy <= min(vr - 1, y + 1); ++yy) {
                const uint32_t* src = P.vshell + ((long long)zz * vr + yy) * P.Wv;
                const uint32_t cur = src[w];
                const uint32_t prev = w > 0 ? src[w - 1] : 0u, next = w + 1 < P.Wv ? src[w + 1] : 0u;
                dil |= cur | (cur << 1) | (cur >> 1) | (prev >> 31) | (next << 31);
            }
        const int valid_bits = min(32, vr - 32 * w);
        const uint32_t valid = valid_bits >= 32 ? 0xffffffffu : ((1u << valid_bits) - 1u);
        const uint32_t pass = ~dil & valid;
        uint32_t border;
        if (y == 0 || y == vr - 1 || z == 0 || z == vr - 1) {
            border = valid;
        } else {
            border = 0;
            if (w == 0) border |= 1u;
            if ((vr - 1) >> 5 == w) border |= 1u << ((vr - 1) & 31);
        }
        P.vfar[idx] = pass;
        P.vext[idx] = pass & border;
    }
}

// Far grid points -> -10 inside the solid voxels (not exterior), +10 elsewhere
// (apply_solid_voxel_sign_mask_kernel, :660-690); block per x row.
__global__ void __launch_bounds__(256) k_vox_sign(SdfParams P, unsigned long long* filled) {
    const long long rows = (long long)P.ny * P.nz;
    const int vr = P.vres;
    unsigned long long cnt = 0;
    for (long long row = blockIdx.x; row < rows; row += gridDim.x) {
        const int iy = (int)(row % P.ny), iz = (int)(row / P.ny);
        float* r = P.out + row * P.nx;
        const float py = P.oy + (float)iy * P.vy, pz = P.oz + (float)iz * P.vz;
        const int vby = bin_coord(py, P.oy, P.vox_vy, vr), vbz = bin_coord(pz, P.oz, P.vox_vz, vr);
        const uint32_t* e = P.vext + ((long long)vbz * vr + vby) * P.Wv;
        for (int ix = threadIdx.x; ix < P.nx; ix += blockDim.x) {
            if (r[ix] != kFar) continue;
            const int vbx = bin_coord(P.ox + (float)ix * P.vx, P.ox, P.vox_vx, vr);
            const bool exterior = (e[vbx >> 5] >> (vbx & 31)) & 1u;
            r[ix] = exterior ? 10.0f : -10.0f;
            cnt += exterior ? 1 : 0;
        }
    }
    if (cnt) atomicAdd(filled, cnt);
}

unsigned grid_for(long long items, int per_block, int num_sms, int per_sm) {
    long long b = (items + per_block - 1) / per_block;
    const long long cap = (long long)num_sms * per_sm;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (unsigned)b;
}

}  // namespace

size_t sdf_tri_record_bytes() { return sizeof(Tri); }

void sdf_bin_geometry(SdfParams& P) {
    P.gx = std::max(1, P.nx / 8);
    P.gy = std::max(1, P.ny / 8);
    P.gz = std::max(1, P.nz / 8);
    P.bdx = ((float)P.nx * P.vx) / (float)P.gx;
    P.bdy = ((float)P.ny * P.vy) / (float)P.gy;
    P.bdz = ((float)P.nz * P.vz) / (float)P.gz;
    P.margin = 2.0f * std::max(P.vx, std::max(P.vy, P.vz));
    P.min_box = std::min(P.bdx, std::min(P.bdy, P.bdz));
    P.nbins = (long long)P.gx * P.gy * P.gz;
    P.W = (P.nx + 31) / 32;
}

cudaError_t launch_sdf_prep(const SdfParams& P, int num_sms, cudaStream_t s) {
    if (P.nf <= 0) return cudaSuccess;
    k_tri_prep<<<grid_for(P.nf, 256, num_sms, 16), 256, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_sdf_bins(const SdfParams& P, int num_sms, cudaStream_t s) {
    const int na = P.gx + P.gy + P.gz + 3;
    k_axis_starts<<<(na + 127) / 128, 128, 0, s>>>(P);
    k_fill_far<<<grid_for((long long)P.nx * P.ny * P.nz, 256, num_sms, 16), 256, 0, s>>>(P);
    if (P.nf > 0) k_tri_bins<<<grid_for(P.nf, 256, num_sms, 16), 256, 0, s>>>(P);
    k_bin_order<<<grid_for(P.nbins, 1, num_sms, 64), kOrderThreads, 0, s>>>(P);
    k_bin_active<<<grid_for(P.nbins, 256, num_sms, 16), 256, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_sdf_band(const SdfParams& P, int num_sms, cudaStream_t s) {
    k_band<<<grid_for(P.nbins, 1, num_sms, 2), kBandThreads, 0, s>>>(P);   // persistent: 2 CTAs per SM
    return cudaGetLastError();
}

cudaError_t launch_sdf_masks(const SdfParams& P, int num_sms, cudaStream_t s) {
    const long long groups = (long long)P.ny * P.nz * ((P.W + 31) / 32);
    k_sdf_masks<<<grid_for(groups * 32, 256, num_sms, 16), 256, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_sdf_flood(const SdfParams& P, int* changed, int num_sms, cudaStream_t s) {
    const long long tiles = ((P.W + kFX - 1) / kFX) * (long long)((P.ny + kFY - 1) / kFY) * ((P.nz + kFZ - 1) / kFZ);
    k_flood<<<grid_for(tiles, 1, num_sms, 8), kFloodThreads, 0, s>>>(P, changed);
    return cudaGetLastError();
}

cudaError_t launch_sdf_finish(const SdfParams& P, unsigned long long* filled, float* tmp, int num_sms, cudaStream_t s) {
    const long long rows = (long long)P.ny * P.nz;
    const unsigned g = grid_for(rows, 1, num_sms, 32);
    k_sdf_finish<<<g, 256, 0, s>>>(P, filled);
    for (int it = 0; it < 4; ++it) {
        if (it % 2 == 0) k_relax<<<g, 256, 0, s>>>(P, P.out, tmp);
        else             k_relax<<<g, 256, 0, s>>>(P, tmp, P.out);
    }
    return cudaGetLastError();
}

cudaError_t launch_vox_raster(const SdfParams& P, int num_sms, cudaStream_t s) {
    if (P.nf <= 0) return cudaSuccess;
    k_vox_raster<<<grid_for(P.nf, 256, num_sms, 16), 256, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_vox_dilate(const SdfParams& P, int num_sms, cudaStream_t s) {
    k_vox_dilate<<<grid_for((long long)P.vres * P.vres * P.Wv, 256, num_sms, 16), 256, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_vox_flood(const SdfParams& P, int* changed, int num_sms, cudaStream_t s) {
    SdfParams V = P;
    V.W = P.Wv;
    V.nx = P.vres; V.ny = P.vres; V.nz = P.vres;
    V.far = P.vfar;
    V.ext = P.vext;
    return launch_sdf_flood(V, changed, num_sms, s);
}

cudaError_t launch_vox_sign(const SdfParams& P, unsigned long long* filled, int num_sms, cudaStream_t s) {
    const long long rows = (long long)P.ny * P.nz;
    k_vox_sign<<<grid_for(rows, 1, num_sms, 8), 256, 0, s>>>(P, filled);
    return cudaGetLastError();
}

}  // namespace dcb
