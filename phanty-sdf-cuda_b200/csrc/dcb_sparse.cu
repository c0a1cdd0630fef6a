// dcb_sparse.cu — the reference's sparse (brick) dual contouring and its multi-vertex variant
// (CudaSparseDualContouringBackend / CudaSparseMvdcDualContouringBackend,
// src/cuda/dc_cuda_sparse.cu:271-1415). Compiled with --fmad=false: every float operation is
// rounded as written, so the results are the reference's arithmetic without contraction.
//
// Semantics (reference line numbers in dc_cuda_sparse.cu):
//   bricks    brick_size^3 cells; active iff its points [b*s, b*s + s] (clipped) hold a value
//             < 0 and a value > 0 (:271-308)
//   cells     a cell of an active brick is active iff it has corners of both strict signs
//             or a corner with |v| <= 0.45*vx (:321-377); vertices in ascending linear order
//   samples   crossing edges (fa*fb <= 0 in float) and thin edges (same sign, both within
//             0.45*vx of zero, end gradients with dot < -0.3: two samples) (:310-319, :676-752)
//   vertices  one QEF per cell; the multi-vertex variant splits the samples in two when the
//             most opposed normal pair has dot < -0.3 and both halves hold two samples
//             (:445-620, :753-826); max-pivot Jacobi (15 rotations), pinv above 0.01,
//             centroid fallback, clamp into the cell (:181-269, :380-443)
//   faces     each active cell's min-corner X, Y, Z edges with a strict crossing or a thin
//             edge whose four cells have vertices; a thin edge adds the reversed quad; winding
//             by the sum of the end gradients (:829-1102); order: active cell, then X, Y, Z.
//
// B200 layout: the grid is read once by a warp-ballot pass into neg / pos / near-zero bit
// words per point row; bricks and cells are decided on those bits; the active cells get the
// dense path's bitmap layout, so its scan and rank expansion give the ascending active list
// and O(1) cell -> vertex lookups (no cell-sized index map as in the reference).
#include "dcb_kernels.cuh"

namespace dcb {

namespace {

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 mul3(float s, float3 b) { return f3(s * b.x, s * b.y, s * b.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ bool finite3(float3 v) {
    return !(isnan(v.x) || isnan(v.y) || isnan(v.z) || isinf(v.x) || isinf(v.y) || isinf(v.z));
}
// bits [lo, hi) of a word, 0 <= lo <= hi <= 32
__device__ __forceinline__ uint32_t range_bits(int lo, int hi) {
    const uint32_t h = hi >= 32 ? 0xffffffffu : ((1u << hi) - 1u);
    return h & ~((1u << lo) - 1u);
}

__device__ __forceinline__ float sval(const GridDesc& g, int i, int j, int k) { return __ldg(g.v + pidx(g, i, j, k)); }

// Central differences with clamped neighbours (:155-179).
__device__ float3 sgrad(const GridDesc& g, int i, int j, int k) {
    const int im = i > 0 ? i - 1 : 0, ip = i < g.nx - 1 ? i + 1 : g.nx - 1;
    const int jm = j > 0 ? j - 1 : 0, jp = j < g.ny - 1 ? j + 1 : g.ny - 1;
    const int km = k > 0 ? k - 1 : 0, kp = k < g.nz - 1 ? k + 1 : g.nz - 1;
    float3 o = f3(0.f, 0.f, 0.f);
    const float dx = (float)(ip - im) * g.vx, dy = (float)(jp - jm) * g.vy, dz = (float)(kp - km) * g.vz;
    if (dx > 1e-12f) o.x = (sval(g, ip, j, k) - sval(g, im, j, k)) / dx;
    if (dy > 1e-12f) o.y = (sval(g, i, jp, k) - sval(g, i, jm, k)) / dy;
    if (dz > 1e-12f) o.z = (sval(g, i, j, kp) - sval(g, i, j, km)) / dz;
    return o;
}

// Thin edge between grid points a and b (:310-319).
__device__ bool thin_edge(const SparseParams& P, float fa, float fb, int ai, int aj, int ak, int bi, int bj, int bk) {
    if (fa * fb <= 0.0f) return false;
    if (fabsf(fa) > P.close || fabsf(fb) > P.close) return false;
    return dot3(sgrad(P.g, ai, aj, ak), sgrad(P.g, bi, bj, bk)) < -0.3f;
}

// Trilinear gradient of the cell at p (:91-153).
__device__ float3 tri_gradient(const float s[8], float3 c0, float x1, float y1, float z1, float3 p) {
    const float dx = x1 - c0.x, dy = y1 - c0.y, dz = z1 - c0.z;
    float u = 0.5f, v = 0.5f, w = 0.5f;
    if (fabsf(dx) > 1e-12f) u = (p.x - c0.x) / dx;
    if (fabsf(dy) > 1e-12f) v = (p.y - c0.y) / dy;
    if (fabsf(dz) > 1e-12f) w = (p.z - c0.z) / dz;
    u = fmaxf(0.0f, fminf(1.0f, u));
    v = fmaxf(0.0f, fminf(1.0f, v));
    w = fmaxf(0.0f, fminf(1.0f, w));
    const float omu = 1.0f - u, omv = 1.0f - v, omw = 1.0f - w;
    const float S000 = s[0], S100 = s[1], S110 = s[2], S010 = s[3];
    const float S001 = s[4], S101 = s[5], S111 = s[6], S011 = s[7];
    const float du = (S100 - S000) * omv * omw + (S110 - S010) * v * omw + (S101 - S001) * omv * w + (S111 - S011) * v * w;
    const float dv = (S010 - S000) * omu * omw + (S110 - S100) * u * omw + (S011 - S001) * omu * w + (S111 - S101) * u * w;
    const float dw = (S001 - S000) * omu * omv + (S101 - S100) * u * omv + (S011 - S010) * omu * v + (S111 - S110) * u * v;
    float3 gr = f3(0.f, 0.f, 0.f);
    if (fabsf(dx) > 1e-12f) gr.x = du / dx;
    if (fabsf(dy) > 1e-12f) gr.y = dv / dy;
    if (fabsf(dz) > 1e-12f) gr.z = dw / dz;
    return gr;
}

// Max-pivot Jacobi with at most 15 rotations and the pinv of the diagonal above 0.01
// (:181-269): y = V S^+ V^T d. Row-major A and V.
__device__ void pivot_jacobi_solve(float A[9], const float d[3], float y[3], bool& singular) {
    float V[9] = {1.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f};
#pragma unroll 1
    for (int it = 0; it < 15; ++it) {
        int p = 0, q = 1;
        float mv = fabsf(A[1]);
        if (fabsf(A[2]) > mv) { p = 0; q = 2; mv = fabsf(A[2]); }
        if (fabsf(A[5]) > mv) { p = 1; q = 2; mv = fabsf(A[5]); }
        if (mv < 1e-7f) break;
        const int o = 3 - p - q;                  // the third index
        const float ap = A[p * 3 + p], aq = A[q * 3 + q], apq = A[p * 3 + q];
        const float phi = 0.5f * (aq - ap) / apq;
        float t = 1.0f / (fabsf(phi) + sqrtf(phi * phi + 1.0f));
        if (phi < 0.0f) t = -t;
        const float c = 1.0f / sqrtf(t * t + 1.0f), s = t * c;
        const float aop = A[o * 3 + p], aoq = A[o * 3 + q];
        A[o * 3 + p] = A[p * 3 + o] = c * aop - s * aoq;
        A[o * 3 + q] = A[q * 3 + o] = s * aop + c * aoq;
        A[p * 3 + p] = ap - t * apq;
        A[q * 3 + q] = aq + t * apq;
        A[p * 3 + q] = A[q * 3 + p] = 0.0f;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const float vip = V[i * 3 + p], viq = V[i * 3 + q];
            V[i * 3 + p] = c * vip - s * viq;
            V[i * 3 + q] = s * vip + c * viq;
        }
    }
    const float S[3] = {A[0], A[4], A[8]};
    float Si[3];
    int ok = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        Si[i] = 0.0f;
        if (S[i] > 0.01f) { Si[i] = 1.0f / S[i]; ++ok; }
    }
    singular = ok == 0;
    float t0 = V[0] * d[0] + V[3] * d[1] + V[6] * d[2];
    float t1 = V[1] * d[0] + V[4] * d[1] + V[7] * d[2];
    float t2 = V[2] * d[0] + V[5] * d[1] + V[8] * d[2];
    t0 *= Si[0]; t1 *= Si[1]; t2 *= Si[2];
    y[0] = V[0] * t0 + V[1] * t1 + V[2] * t2;
    y[1] = V[3] * t0 + V[4] * t1 + V[5] * t2;
    y[2] = V[6] * t0 + V[7] * t1 + V[8] * t2;
}

// The vertex of the samples selected by `sel` (bit q = sample q), in sample order (:380-443).
__device__ float3 cluster_vertex(const float3* pts, const float3* nrm, int m, uint32_t sel, float3 cmin, float3 cmax,
                                 float3 half, unsigned int* cnt) {
    const int k = __popc(sel & ((1u << m) - 1u));
    if (k == 0) return add3(cmin, half);
    float3 c = f3(0.f, 0.f, 0.f);
    for (int q = 0; q < m; ++q) if (sel >> q & 1u) c = add3(c, pts[q]);
    c = mul3(1.0f / (float)k, c);
    float B[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, d[3] = {0.f, 0.f, 0.f};
    for (int q = 0; q < m; ++q) {
        if (!(sel >> q & 1u)) continue;
        const float3 n = nrm[q];
        const float dv = dot3(n, sub3(pts[q], c));
        B[0] += n.x * n.x; B[1] += n.x * n.y; B[2] += n.x * n.z;
        B[3] += n.y * n.x; B[4] += n.y * n.y; B[5] += n.y * n.z;
        B[6] += n.z * n.x; B[7] += n.z * n.y; B[8] += n.z * n.z;
        d[0] += n.x * dv; d[1] += n.y * dv; d[2] += n.z * dv;
    }
    float y[3];
    bool singular;
    pivot_jacobi_solve(B, d, y, singular);
    float3 v = add3(c, f3(y[0], y[1], y[2]));
    if (singular || !finite3(v)) { atomicAdd(cnt + kScFallback, 1u); v = c; }
    if (!finite3(v)) { atomicAdd(cnt + kScInvalid, 1u); v = add3(cmin, half); }
    if (v.x < cmin.x || v.x > cmax.x || v.y < cmin.y || v.y > cmax.y || v.z < cmin.z || v.z > cmax.z) {
        atomicAdd(cnt + kScClamp, 1u);
        v.x = fmaxf(cmin.x, fminf(cmax.x, v.x));
        v.y = fmaxf(cmin.y, fminf(cmax.y, v.y));
        v.z = fmaxf(cmin.z, fminf(cmax.z, v.z));
    }
    return v;
}

__device__ __forceinline__ float3 unit_or(float3 a, float3 fb) {
    const float l = sqrtf(dot3(a, a));
    return l > 1e-6f ? mul3(1.0f / l, a) : fb;
}

// Active-cell bit of cell (i,j,k) and its rank.
__device__ __forceinline__ bool cell_active(const SparseParams& P, int i, int j, int k) {
    const uint32_t w = __ldg(P.bits + ((int64_t)j + (int64_t)P.g.cy * k) * P.g.W + (i >> 5));
    return (w >> (i & 31)) & 1u;
}

// Vertex of face cell (i,j,k) for the gradient sum gn, or -1 (:829-851).
__device__ int face_vertex(const SparseParams& P, int i, int j, int k, float3 gn) {
    if (!cell_active(P, i, j, k)) return -1;
    const uint32_t r = cell_rank(P.bits, P.super, P.g, i, j, k);
    if (!P.mvdc) return (int)r;
    const int st = (int)__ldg(P.vstart + r);
    if (__ldg(P.vcount + r) == 1u) return st;
    const float3 n0 = f3(__ldg(P.N + 3 * (size_t)st), __ldg(P.N + 3 * (size_t)st + 1), __ldg(P.N + 3 * (size_t)st + 2));
    const float3 n1 = f3(__ldg(P.N + 3 * (size_t)st + 3), __ldg(P.N + 3 * (size_t)st + 4), __ldg(P.N + 3 * (size_t)st + 5));
    const float d0 = dot3(gn, n0), d1 = dot3(gn, n1);
    const int best = d0 >= d1 ? st : st + 1;
    return fmaxf(d0, d1) < -0.5f ? -1 : best;
}

}  // namespace

// ---- marking ----------------------------------------------------------------------------

// Negative / positive / near-zero bit words of every point row (32 points a word), a warp
// per 32 consecutive words of a row. VEC4 (rows 16-byte aligned, nx % 4 == 0): lane l loads
// points 4l..4l+3 of each 128-point chunk as one float4, builds the three nibbles and an
// 8-lane shuffle-OR forms each word; otherwise one coalesced scalar load and three ballots
// per word.
template <bool VEC4>
__global__ void __launch_bounds__(256) k_sparse_points(const __grid_constant__ SparseParams P) {
    const GridDesc& g = P.g;
    const int lane = threadIdx.x & 31;
    const int cpr = (P.Wp + 31) / 32;
    const long long nchunks = (long long)g.ny * g.nz * cpr;
    for (long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < nchunks;
         c += ((long long)gridDim.x * blockDim.x) >> 5) {
        const long long row = c / cpr;
        const int w0 = (int)(c - row * cpr) * 32;
        const float* src = g.v + row * g.nx;
        uint32_t mn = 0, mp = 0, mc = 0;
        if (VEC4) {
            float4 v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int x = w0 * 32 + 128 * q + 4 * lane;
                v[q] = x < g.nx ? __ldg(reinterpret_cast<const float4*>(src + x)) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const bool in = w0 * 32 + 128 * q + 4 * lane < g.nx;
                const float e[4] = {v[q].x, v[q].y, v[q].z, v[q].w};
                uint32_t n = 0, p = 0, z = 0;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    n |= (e[u] < 0.f ? 1u : 0u) << u;
                    p |= (e[u] > 0.f ? 1u : 0u) << u;
                    z |= (fabsf(e[u]) <= P.close ? 1u : 0u) << u;
                }
                if (!in) n = p = z = 0;
                const int sh = 4 * (lane & 7);
                n <<= sh; p <<= sh; z <<= sh;
#pragma unroll
                for (int o = 1; o < 8; o <<= 1) {
                    n |= __shfl_xor_sync(0xffffffffu, n, o);
                    p |= __shfl_xor_sync(0xffffffffu, p, o);
                    z |= __shfl_xor_sync(0xffffffffu, z, o);
                }
                // word 4q + (l >> 3) is complete in lanes 8*(l >> 3)..; lane L keeps word L
                const int src_lane = 8 * (lane & 3);
                const uint32_t tn = __shfl_sync(0xffffffffu, n, src_lane);
                const uint32_t tp = __shfl_sync(0xffffffffu, p, src_lane);
                const uint32_t tz = __shfl_sync(0xffffffffu, z, src_lane);
                if ((lane >> 2) == q) { mn = tn; mp = tp; mc = tz; }
            }
        } else {
#pragma unroll 8
            for (int u = 0; u < 32; ++u) {
                const int x = (w0 + u) * 32 + lane;
                const bool in = x < g.nx;
                const float v = in ? __ldg(src + x) : 0.f;
                const uint32_t bn = __ballot_sync(0xffffffffu, in && v < 0.f);
                const uint32_t bp = __ballot_sync(0xffffffffu, in && v > 0.f);
                const uint32_t bc = __ballot_sync(0xffffffffu, in && fabsf(v) <= P.close);
                if (lane == u) { mn = bn; mp = bp; mc = bc; }
            }
        }
        if (w0 + lane < P.Wp) {
            const long long o = row * P.Wp + w0 + lane;
            P.pn[o] = mn; P.pp[o] = mp; P.pc[o] = mc;
        }
    }
}

// Brick flags from the point words (:271-308): a block per row of bricks (by, bz). Its threads
// OR the point words of the brick row's (s+1)^2 point rows, word by word (coalesced), into
// shared memory; then a thread per brick tests its x-range of points in those words.
constexpr int kBrickThreads = 128;
constexpr int kMaxPointWords = 2048;           // nx <= 65536

__global__ void __launch_bounds__(kBrickThreads) k_sparse_bricks(const __grid_constant__ SparseParams P) {
    const GridDesc& g = P.g;
    __shared__ uint32_t s_n[kMaxPointWords], s_p[kMaxPointWords];
    __shared__ unsigned int s_active;
    if (threadIdx.x == 0) s_active = 0;
    const long long nrow = (long long)P.nby * P.nbz;
    for (long long br = blockIdx.x; br < nrow; br += gridDim.x) {
        const int by = (int)(br % P.nby), bz = (int)(br / P.nby);
        const int j0 = by * P.bs, k0 = bz * P.bs;
        const int j1 = min(j0 + P.bs + 1, g.ny), k1 = min(k0 + P.bs + 1, g.nz);
        __syncthreads();
        for (int w = threadIdx.x; w < P.Wp; w += blockDim.x) {
            uint32_t n = 0, p = 0;
            for (int k = k0; k < k1; ++k)
                for (int j = j0; j < j1; ++j) {
                    const long long o = ((long long)j + (long long)g.ny * k) * P.Wp + w;
                    n |= __ldg(P.pn + o);
                    p |= __ldg(P.pp + o);
                }
            s_n[w] = n;
            s_p[w] = p;
        }
        __syncthreads();
        for (int bx = threadIdx.x; bx < P.nbx; bx += blockDim.x) {
            const int i0 = bx * P.bs, i1 = min(i0 + P.bs + 1, g.nx);
            bool neg = false, pos = false;
            for (int w = i0 >> 5; w <= (i1 - 1) >> 5; ++w) {
                const uint32_t m = range_bits(max(i0 - 32 * w, 0), min(i1 - 32 * w, 32));
                neg |= (s_n[w] & m) != 0u;
                pos |= (s_p[w] & m) != 0u;
            }
            const bool act = neg && pos;
            P.brick[bx + (long long)P.nbx * br] = act ? 1 : 0;
            if (act) atomicAdd(&s_active, 1u);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_active) atomicAdd(P.counters + kScActiveBricks, (unsigned long long)s_active);
}

// Active-cell words (:321-377) in the dense path's layout: a warp per (cell row, 32 words),
// lane w builds cell word w from the point words of the four point rows around it.
__global__ void __launch_bounds__(256) k_sparse_cells(const __grid_constant__ SparseParams P) {
    const GridDesc& g = P.g;
    const int lane = threadIdx.x & 31;
    const long long nseg = (long long)g.cy * g.cz * P.nxt;
    for (long long sg = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; sg < nseg;
         sg += ((long long)gridDim.x * blockDim.x) >> 5) {
        const long long row = sg / P.nxt;
        const int xt = (int)(sg - row * P.nxt);
        const int j = (int)(row % g.cy), k = (int)(row / g.cy);
        const int w = xt * 32 + lane;
        uint32_t act = 0;
        if (w < g.W && 32 * w < g.cx) {
            const long long r00 = ((long long)j + (long long)g.ny * k) * P.Wp;
            const long long r10 = r00 + P.Wp, r01 = r00 + (long long)g.ny * P.Wp, r11 = r01 + P.Wp;
            const bool nxw = w + 1 < P.Wp;
            uint32_t m[3];
            const uint32_t* src[3] = {P.pn, P.pp, P.pc};
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const uint32_t* a = src[q];
                const uint32_t lo = __ldg(a + r00 + w) | __ldg(a + r10 + w) | __ldg(a + r01 + w) | __ldg(a + r11 + w);
                const uint32_t hi = nxw ? (__ldg(a + r00 + w + 1) | __ldg(a + r10 + w + 1) | __ldg(a + r01 + w + 1) |
                                           __ldg(a + r11 + w + 1)) : 0u;
                m[q] = lo | (lo >> 1) | (hi << 31);
            }
            act = (m[0] & m[1]) | m[2];
            const int c0 = 32 * w, c1 = min(32 * w + 32, g.cx);
            act &= range_bits(0, c1 - c0);
            const int by = j / P.bs, bz = k / P.bs;
            uint32_t bm = 0;
            for (int bx = c0 / P.bs; bx * P.bs < c1; ++bx)
                if (__ldg(P.brick + bx + (long long)P.nbx * (by + (long long)P.nby * bz)))
                    bm |= range_bits(max(bx * P.bs, c0) - c0, min(bx * P.bs + P.bs, c1) - c0);
            act &= bm;
        }
        if (w < g.W) P.bits[row * g.W + w] = act;
        uint32_t cnt = __popc(act);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        if (lane == 0) P.seg_count[row * P.nxt + xt] = cnt;
    }
}

// ---- vertices -----------------------------------------------------------------------------

// A thread per active cell: its Hermite samples, the vertex count and the vertices (:445-826).
// The single-vertex variant writes V[rank] directly; the multi-vertex one writes both slots of
// the cell into Vtmp / Ntmp and its count, placed after the scan by k_sparse_place.
__global__ void __launch_bounds__(128) k_sparse_vertices(const __grid_constant__ SparseParams P) {
    __shared__ unsigned int s_cnt[kScCount];
    if (threadIdx.x < kScCount) s_cnt[threadIdx.x] = 0;
    __syncthreads();
    const GridDesc& g = P.g;
    const float3 half = mul3(0.5f, f3(g.vx, g.vy, g.vz));
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < P.nactive;
         r += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        unpack_cell(P.list[r], i, j, k);
        float s[8];
        float3 cp0, cp6;
        float cx1, cy1, cz1;
#pragma unroll
        for (int c = 0; c < 8; ++c) s[c] = sval(g, i + corner_dx(c), j + corner_dy(c), k + corner_dz(c));
        cp0 = f3(g.ox + (float)i * g.vx, g.oy + (float)j * g.vy, g.oz + (float)k * g.vz);
        cx1 = g.ox + (float)(i + 1) * g.vx;
        cy1 = g.oy + (float)(j + 1) * g.vy;
        cz1 = g.oz + (float)(k + 1) * g.vz;
        cp6 = f3(cx1, cy1, cz1);
        float3 pts[12], nrm[12];
        int m = 0;
        for (int e = 0; e < 12; ++e) {
            const int a = edge_a(e), b = edge_b(e);
            const float fa = s[a], fb = s[b];
            const int ai = i + corner_dx(a), aj = j + corner_dy(a), ak = k + corner_dz(a);
            const int bi = i + corner_dx(b), bj = j + corner_dy(b), bk = k + corner_dz(b);
            const bool crossing = fa * fb <= 0.0f;
            const bool thin = !crossing && thin_edge(P, fa, fb, ai, aj, ak, bi, bj, bk);
            if (!crossing && !thin) continue;
            float t = crossing ? fa / (fa - fb + 1e-12f) : fabsf(fa) / (fabsf(fa) + fabsf(fb) + 1e-12f);
            t = fmaxf(0.0f, fminf(1.0f, t));
            const float3 pa = f3(corner_dx(a) ? cx1 : cp0.x, corner_dy(a) ? cy1 : cp0.y, corner_dz(a) ? cz1 : cp0.z);
            const float3 pb = f3(corner_dx(b) ? cx1 : cp0.x, corner_dy(b) ? cy1 : cp0.y, corner_dz(b) ? cz1 : cp0.z);
            const float3 p = add3(mul3(1.0f - t, pa), mul3(t, pb));
            if (thin) {
                float3 ga = sgrad(g, ai, aj, ak), gb = sgrad(g, bi, bj, bk);
                const float la = sqrtf(dot3(ga, ga)), lb = sqrtf(dot3(gb, gb));
                if (la > 1e-6f) ga = mul3(1.0f / la, ga);
                if (lb > 1e-6f) gb = mul3(1.0f / lb, gb);
                if (m < 11) {
                    pts[m] = p; nrm[m] = ga; ++m;
                    pts[m] = p; nrm[m] = gb; ++m;
                }
            } else {
                float3 n;
                if (P.normal_mode == 1) {
                    const float3 ga = sgrad(g, ai, aj, ak), gb = sgrad(g, bi, bj, bk);
                    n = add3(mul3(1.0f - t, ga), mul3(t, gb));
                } else {
                    n = tri_gradient(s, cp0, cx1, cy1, cz1, p);
                }
                const float ln = sqrtf(dot3(n, n));
                if (ln > 1e-6f) n = mul3(1.0f / ln, n);
                if (m < 12) { pts[m] = p; nrm[m] = n; ++m; }
            }
        }
        // the most opposed normal pair (first minimum in (i, j > i) order)
        int A = -1, B = -1;
        float mind = 1.0f;
        if (P.mvdc) {
            for (int q = 0; q < m; ++q)
                for (int u = q + 1; u < m; ++u) {
                    const float dt = dot3(nrm[q], nrm[u]);
                    if (dt < mind) { mind = dt; A = q; B = u; }
                }
        }
        uint32_t selA = 0;
        int count = 1;
        if (P.mvdc && m >= 2 && A >= 0 && mind < -0.3f) {
            const float3 nA = nrm[A], nB = nrm[B];
            for (int q = 0; q < m; ++q) if (dot3(nrm[q], nA) >= dot3(nrm[q], nB)) selA |= 1u << q;
            const int ca = __popc(selA);
            if (ca < 2 || m - ca < 2) atomicAdd(&s_cnt[kScSplitReject], 1u);
            else count = 2;
        }
        const uint32_t all = (1u << m) - 1u;
        if (count == 1) {
            const float3 v = cluster_vertex(pts, nrm, m, all, cp0, cp6, half, s_cnt);
            if (!P.mvdc) {
                P.V[3 * r] = v.x; P.V[3 * r + 1] = v.y; P.V[3 * r + 2] = v.z;
            } else {
                float3 avg = f3(0.f, 0.f, 0.f);
                for (int q = 0; q < m; ++q) avg = add3(avg, nrm[q]);
                const float3 n0 = unit_or(avg, f3(0.f, 1.f, 0.f));
                float* vt = P.vtmp + 6 * r;
                float* nt = P.ntmp + 6 * r;
                vt[0] = v.x; vt[1] = v.y; vt[2] = v.z;
                nt[0] = n0.x; nt[1] = n0.y; nt[2] = n0.z;
                P.vcount[r] = 1u;
                atomicAdd(&s_cnt[kScOne], 1u);
            }
        } else {
            const float3 nA = nrm[A], nB = nrm[B];
            const float3 v0 = cluster_vertex(pts, nrm, m, selA, cp0, cp6, half, s_cnt);
            const float3 v1 = cluster_vertex(pts, nrm, m, all & ~selA, cp0, cp6, half, s_cnt);
            float3 a0 = f3(0.f, 0.f, 0.f), a1 = f3(0.f, 0.f, 0.f);
            for (int q = 0; q < m; ++q) {
                if (selA >> q & 1u) a0 = add3(a0, nrm[q]);
                else a1 = add3(a1, nrm[q]);
            }
            const float3 n0 = unit_or(a0, nA), n1 = unit_or(a1, nB);
            float* vt = P.vtmp + 6 * r;
            float* nt = P.ntmp + 6 * r;
            vt[0] = v0.x; vt[1] = v0.y; vt[2] = v0.z; vt[3] = v1.x; vt[4] = v1.y; vt[5] = v1.z;
            nt[0] = n0.x; nt[1] = n0.y; nt[2] = n0.z; nt[3] = n1.x; nt[4] = n1.y; nt[5] = n1.z;
            P.vcount[r] = 2u;
            atomicAdd(&s_cnt[kScAmbiguous], 1u);
            atomicAdd(&s_cnt[kScMulti], 1u);
            atomicAdd(&s_cnt[kScTwo], 1u);
        }
    }
    __syncthreads();
    if (threadIdx.x < kScCount && s_cnt[threadIdx.x])
        atomicAdd(P.counters + threadIdx.x, (unsigned long long)s_cnt[threadIdx.x]);
}

// Multi-vertex variant: each cell's vertices (and normals, and the cell of each vertex) at
// their scanned positions.
__global__ void __launch_bounds__(256) k_sparse_place(const __grid_constant__ SparseParams P) {
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < P.nactive;
         r += (long long)gridDim.x * blockDim.x) {
        const uint32_t st = P.vstart[r], c = P.vcount[r];
        const uint64_t cell = P.list[r];
        for (uint32_t q = 0; q < c; ++q) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                P.V[3 * (size_t)(st + q) + d] = P.vtmp[6 * r + 3 * q + d];
                P.N[3 * (size_t)(st + q) + d] = P.ntmp[6 * r + 3 * q + d];
            }
            P.vcell[st + q] = cell;
        }
    }
}

// ---- faces ----------------------------------------------------------------------------------

// A thread per active cell: its faces in the reference's order (:853-1102) into the cell's six
// staging slots (three axes, a thin edge's reversed quad beside its own) and their count;
// k_sparse_compact moves them to their scanned positions. A cell without faces adds nothing
// to the skipped-face counter (the reference's emit pass returns for it, :954).
__global__ void __launch_bounds__(128) k_sparse_faces(const __grid_constant__ SparseParams P) {
    __shared__ unsigned int s_skipped;
    if (threadIdx.x == 0) s_skipped = 0;
    __syncthreads();
    const GridDesc& g = P.g;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < P.nactive;
         r += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        unpack_cell(P.list[r], i, j, k);
        uint32_t count = 0, skipped = 0;
        int4* const out = P.stage + 6 * r;
        const float s0 = sval(g, i, j, k);
        float3 g0 = f3(0.f, 0.f, 0.f);
        bool have_g0 = false;
#pragma unroll 1
        for (int axis = 0; axis < 3; ++axis) {
            if (axis == 0 && !(j >= 1 && k >= 1)) continue;
            if (axis == 1 && !(i >= 1 && k >= 1 && j < g.ny - 1)) continue;
            if (axis == 2 && !(i >= 1 && j >= 1 && k < g.nz - 1)) continue;
            const int i1 = i + (axis == 0), j1 = j + (axis == 1), k1 = k + (axis == 2);
            const float s1 = sval(g, i1, j1, k1);
            const bool crossing = s0 * s1 < 0.0f;
            bool thin = false;
            if (!crossing && !(s0 * s1 <= 0.0f) && !(fabsf(s0) > P.close || fabsf(s1) > P.close)) {
                if (!have_g0) { g0 = sgrad(g, i, j, k); have_g0 = true; }
                thin = dot3(g0, sgrad(g, i1, j1, k1)) < -0.3f;
            }
            if (!crossing && !thin) continue;
            if (!have_g0) { g0 = sgrad(g, i, j, k); have_g0 = true; }
            const float3 gn = add3(g0, sgrad(g, i1, j1, k1));
            int v0, v1, v2, v3;
            if (axis == 0) {
                v0 = face_vertex(P, i, j - 1, k - 1, gn); v1 = face_vertex(P, i, j, k - 1, gn);
                v2 = face_vertex(P, i, j, k, gn); v3 = face_vertex(P, i, j - 1, k, gn);
            } else if (axis == 1) {
                v0 = face_vertex(P, i - 1, j, k - 1, gn); v1 = face_vertex(P, i, j, k - 1, gn);
                v2 = face_vertex(P, i, j, k, gn); v3 = face_vertex(P, i - 1, j, k, gn);
            } else {
                v0 = face_vertex(P, i - 1, j - 1, k, gn); v1 = face_vertex(P, i, j - 1, k, gn);
                v2 = face_vertex(P, i, j, k, gn); v3 = face_vertex(P, i - 1, j, k, gn);
            }
            if (v0 < 0 || v1 < 0 || v2 < 0 || v3 < 0) {
                if (P.mvdc) ++skipped;
                continue;
            }
            auto vtx = [&](int v) {
                return f3(__ldg(P.V + 3 * (size_t)v), __ldg(P.V + 3 * (size_t)v + 1), __ldg(P.V + 3 * (size_t)v + 2));
            };
            const float3 pa = vtx(v0), pb = vtx(v1), pc = vtx(v2), pd = vtx(v3);
            float3 qn = cross3(sub3(pb, pa), sub3(pd, pa));
            if (dot3(qn, qn) < 1e-12f) qn = cross3(sub3(pc, pa), sub3(pd, pa));
            if (dot3(gn, gn) > 0.0f && dot3(qn, qn) > 0.0f && dot3(qn, gn) < 0.0f) { const int t = v1; v1 = v3; v3 = t; }
            out[count++] = make_int4(v0, v1, v2, v3);
            if (thin) out[count++] = make_int4(v0, v3, v2, v1);
        }
        P.fcount[r] = count;
        if (count && skipped) atomicAdd(&s_skipped, skipped);
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_skipped) atomicAdd(P.counters + kScSkipped, (unsigned long long)s_skipped);
}

// Each cell's staged faces to their scanned positions.
__global__ void __launch_bounds__(256) k_sparse_compact(const __grid_constant__ SparseParams P) {
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < P.nactive;
         r += (long long)gridDim.x * blockDim.x) {
        const uint32_t c = P.fcount[r], st = P.fstart[r];
        for (uint32_t q = 0; q < c; ++q) P.faces[st + q] = P.stage[6 * r + q];
    }
}

// ---- launchers --------------------------------------------------------------------------------

namespace {
unsigned blocks_for(long long items, int threads, int num_sms, int per_sm) {
    long long b = (items + threads - 1) / threads;
    const long long cap = (long long)num_sms * per_sm;
    if (b > cap) b = cap;
    return (unsigned)(b < 1 ? 1 : b);
}
}  // namespace

cudaError_t launch_sparse_mark(const SparseParams& P, int num_sms, cudaStream_t s) {
    const long long chunks = (long long)P.g.ny * P.g.nz * ((P.Wp + 31) / 32);
    const bool vec4 = P.g.nx % 4 == 0 && (reinterpret_cast<uintptr_t>(P.g.v) % 16) == 0;
    if (vec4) k_sparse_points<true><<<blocks_for(chunks * 32, 256, num_sms, 16), 256, 0, s>>>(P);
    else      k_sparse_points<false><<<blocks_for(chunks * 32, 256, num_sms, 16), 256, 0, s>>>(P);
    const long long nrow = (long long)P.nby * P.nbz;
    k_sparse_bricks<<<(unsigned)std::min<long long>(nrow, (long long)num_sms * 16), kBrickThreads, 0, s>>>(P);
    const long long nseg = (long long)P.g.cy * P.g.cz * P.nxt;
    k_sparse_cells<<<blocks_for(nseg * 32, 256, num_sms, 16), 256, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_sparse_vertices(const SparseParams& P, int num_sms, cudaStream_t s) {
    if (P.nactive <= 0) return cudaSuccess;
    k_sparse_vertices<<<blocks_for(P.nactive, 128, num_sms, 16), 128, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_sparse_place(const SparseParams& P, int num_sms, cudaStream_t s) {
    if (P.nactive <= 0) return cudaSuccess;
    k_sparse_place<<<blocks_for(P.nactive, 256, num_sms, 8), 256, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_sparse_faces(const SparseParams& P, int num_sms, cudaStream_t s) {
    if (P.nactive <= 0) return cudaSuccess;
    k_sparse_faces<<<blocks_for(P.nactive, 128, num_sms, 16), 128, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_sparse_compact(const SparseParams& P, int num_sms, cudaStream_t s) {
    if (P.nactive <= 0) return cudaSuccess;
    k_sparse_compact<<<blocks_for(P.nactive, 256, num_sms, 8), 256, 0, s>>>(P);
    return cudaGetLastError();
}

}  // namespace dcb
