// dcb_faces.cu — quad emission in the CPU backend's order and winding.
//
// The reference CPU loops (src/cpp/contouring.cpp:607-729) emit all X-edge quads, then Y,
// then Z; within an axis the loops run i outermost and k innermost, and a quad is emitted
// for every edge with s0*s1 < 0 whose four cells have vertices. Winding: swap c1 and c3
// when (pb-pa)x(pd-pa) [fallback (pc-pa)x(pd-pa) if its squared norm < 1e-24] points
// against gradientAt(p0) + gradientAt(p1) (contouring.cpp:624-641).
// The reference GPU kernels emit in edge-major order instead (src/cuda/dc_cuda.cu:425-605).
//
// Order without a global sort: each face belongs to a "column" (axis, i, j) and the CPU
// order is (axis, i, j, k). The vertex kernel counts faces per column (atomics); an
// exclusive scan of the counts gives each column's start; the scatter places faces into
// their column in arbitrary order; the ordering pass ranks each face by k inside its
// column. Columns hold a handful of faces on real surfaces.
// Winding is decided in FP32 with error margins; faces inside the margin are staged in
// canonical order and re-decided from FP64 vertices (k_winding_fp64, dcb_vertex64.cu).
#include "dcb_kernels.cuh"

namespace dcb {

// ---- exclusive scan of uint32 counts (three passes, 2048 items per block) --------------

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_warp, uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    uint32_t base = 0;
    total = 0;
#pragma unroll
    for (int q = 0; q < kScanThreads / 32; ++q) {
        const uint32_t s = s_warp[q];
        if (q < warp) base += s;
        total += s;
    }
    __syncthreads();
    return base + incl - v;
}

__global__ void __launch_bounds__(kScanThreads)
k_scan_partials(const uint32_t* __restrict__ in, long long n, uint32_t* partials) {
    __shared__ uint32_t s_warp[kScanThreads / 32];
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    uint32_t s = 0;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) s += (base + q < n) ? in[base + q] : 0u;
    uint32_t total;
    block_excl_scan(s, s_warp, total);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads)
k_scan_single(uint32_t* partials, long long nb, unsigned long long* grand_total) {
    __shared__ uint32_t s_warp[kScanThreads / 32];
    uint32_t carry = 0;
    for (long long c0 = 0; c0 < nb; c0 += kScanThreads) {
        const long long idx = c0 + threadIdx.x;
        const uint32_t v = idx < nb ? partials[idx] : 0u;
        uint32_t total;
        const uint32_t ex = block_excl_scan(v, s_warp, total);
        if (idx < nb) partials[idx] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) *grand_total = carry;
}

__global__ void __launch_bounds__(kScanThreads)
k_scan_apply(const uint32_t* __restrict__ in, long long n, const uint32_t* __restrict__ partials,
             uint32_t* __restrict__ out) {
    __shared__ uint32_t s_warp[kScanThreads / 32];
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) { v[q] = (base + q < n) ? in[base + q] : 0u; s += v[q]; }
    uint32_t total;
    uint32_t run = block_excl_scan(s, s_warp, total) + partials[blockIdx.x];
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        if (base + q < n) out[base + q] = run;
        run += v[q];
    }
}

cudaError_t launch_scan(const uint32_t* in, long long n, uint32_t* partials, uint32_t* out,
                        unsigned long long* grand_total, cudaStream_t s) {
    const long long nb = (n + kScanTile - 1) / kScanTile;
    if (nb <= 0) return cudaSuccess;
    k_scan_partials<<<(unsigned)nb, kScanThreads, 0, s>>>(in, n, partials);
    k_scan_single<<<1, kScanThreads, 0, s>>>(partials, nb, grand_total);
    k_scan_apply<<<(unsigned)nb, kScanThreads, 0, s>>>(in, n, partials, out);
    return cudaGetLastError();
}

long long scan_partials_len(long long n) { return (n + kScanTile - 1) / kScanTile; }

// ---- face scatter ----------------------------------------------------------------------

constexpr int kFaceThreads = 128;


// gradientAt (contouring.cpp:141-207) in FP32 (orientation tests only: a 2-ulp quotient is
// far inside the uncertainty margin, and uncertain faces are re-decided in FP64).
__device__ __forceinline__ float3 grid_gradient32(const GridDesc& g, int i, int j, int k) {
    const int im = max(i - 1, 0), ip = min(i + 1, g.nx - 1);
    const int jm = max(j - 1, 0), jp = min(j + 1, g.ny - 1);
    const int km = max(k - 1, 0), kp = min(k + 1, g.nz - 1);
    float3 o = make_float3(0.f, 0.f, 0.f);
    const float dx = pos_axis(g.ox, g.vx, ip) - pos_axis(g.ox, g.vx, im);
    if (fabsf(dx) > 1e-12f) o.x = __fdividef(__ldg(g.v + pidx(g, ip, j, k)) - __ldg(g.v + pidx(g, im, j, k)), dx);
    const float dy = pos_axis(g.oy, g.vy, jp) - pos_axis(g.oy, g.vy, jm);
    if (fabsf(dy) > 1e-12f) o.y = __fdividef(__ldg(g.v + pidx(g, i, jp, k)) - __ldg(g.v + pidx(g, i, jm, k)), dy);
    const float dz = pos_axis(g.oz, g.vz, kp) - pos_axis(g.oz, g.vz, km);
    if (fabsf(dz) > 1e-12f) o.z = __fdividef(__ldg(g.v + pidx(g, i, j, kp)) - __ldg(g.v + pidx(g, i, j, km)), dz);
    const float n2 = o.x * o.x + o.y * o.y + o.z * o.z;
    if (n2 > 0.f) { const float r = rsqrtf(n2); o.x *= r; o.y *= r; o.z *= r; }
    return o;
}

__device__ __forceinline__ float3 ldv(const float* V, uint32_t r) {
    return make_float3(__ldg(V + 3 * (size_t)r), __ldg(V + 3 * (size_t)r + 1), __ldg(V + 3 * (size_t)r + 2));
}
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Bound on each stored vertex's deviation from the CPU's double vertex: its solve class (in
// cell widths) plus one ulp of the stored float coordinates; the largest of the four.
__device__ __forceinline__ float quad_vertex_bound(const uint8_t* __restrict__ vclass, uint32_t r0, uint32_t r1,
                                                  uint32_t r2, uint32_t r3, float3 pa, float3 pb, float3 pc,
                                                  float3 pd, float hmax) {
    const uint8_t cls[4] = {vclass[r0], vclass[r1], vclass[r2], vclass[r3]};
    const float3 pv[4] = {pa, pb, pc, pd};
    float dv = 0.f;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float ce = cls[q] == kVcRank1 ? 2e-6f : (cls[q] == kVcJacobi ? 1e-4f : 0.f);
        const float mag = fmaxf(fabsf(pv[q].x), fmaxf(fabsf(pv[q].y), fabsf(pv[q].z)));
        dv = fmaxf(dv, ce * hmax + mag * 1.2e-7f);
    }
    return dv;
}

// Ask for the FP64 vertex of cell rank r once (v64_index: -1 none, -2 being claimed).
__device__ __forceinline__ void request_fp64_vertex(int* v64_index, uint32_t* v64_cells, unsigned int* v64_count,
                                                    unsigned long long v64_cap, int* err, uint32_t r) {
    if (atomicCAS(&v64_index[r], -1, -2) == -1) {
        const unsigned int v = atomicAdd(v64_count, 1u);
        if (v < v64_cap) {
            v64_cells[v] = r;
            v64_index[r] = (int)v;
        } else {
            set_error(err, kErrOverflow);
        }
    }
}

// One face of cell (i,j,k) (rank r) along `axis`: its four cells' ranks, the FP32 winding test
// with its error bound, the staging slot in its column, and for an uncertain face the FP64
// work items.
template <bool ONE>
__device__ __forceinline__ void emit_face(const FaceParams& P, int gi, int i, int j, int k, uint32_t r, int axis,
                                          float3 g0, uint32_t r_k1, uint32_t r_j1, uint32_t r_jk) {
    const GridSlot& S = slot_ref<ONE>(P.B, gi);
    const GridDesc& g = S.g;
    const long long cxcy = (long long)g.cx * g.cy;
    uint32_t r0, r1, r3;
    if (axis == 0) { r0 = r_jk; r1 = r_k1; r3 = r_j1; }                // (i,j-1,k-1) (i,j,k-1) (i,j-1,k)
    else if (axis == 1) { r0 = r_k1 - 1u; r1 = r_k1; r3 = r - 1u; }    // (i-1,j,k-1) (i,j,k-1) (i-1,j,k)
    else { r0 = r_j1 - 1u; r1 = r_j1; r3 = r - 1u; }                   // (i-1,j-1,k) (i,j-1,k) (i-1,j,k)
    const uint32_t r2 = r;
    // the staging slot first: it depends on the column alone, so its atomic round trip overlaps
    // the gradient and vertex loads below (col_fill starts at each column's first slot)
    const long long col = S.col_off + axis * cxcy + (long long)i * g.cy + j;
    const uint32_t slot = atomicAdd(&P.col_fill[col], 1u);
    const float3 g1 = grid_gradient32(g, i + (axis == 0), j + (axis == 1), k + (axis == 2));
    const float3 gn = make_float3(g0.x + g1.x, g0.y + g1.y, g0.z + g1.z);
    const float3 pa = ldv(P.V, r0), pb = ldv(P.V, r1), pc = ldv(P.V, r2), pd = ldv(P.V, r3);
    const float dv = quad_vertex_bound(P.vclass, r0, r1, r2, r3, pa, pb, pc, pd, S.hmax);
    const float3 ba = sub3(pb, pa), da = sub3(pd, pa), ca = sub3(pc, pa);
    float3 qn = cross3(ba, da);
    float qn2 = dot3(qn, qn);
    // |qn| error bound of the FP32 cross product from the vertex bounds
    const float lb = sqrtf(dot3(ba, ba)), ld = sqrtf(dot3(da, da)), lc = sqrtf(dot3(ca, ca));
    float dq = 2.f * dv * (lb + ld + 2.f * dv);
    // The reference switches to the other diagonal below |qn|^2 = 1e-24 (absolute):
    // decide in FP64 whenever the bound straddles that switch.
    const float qnl0 = sqrtf(qn2);
    const bool near_fallback = (qnl0 - dq) < 1e-12f && (qnl0 + dq) >= 1e-12f;
    if (qn2 < 1e-24f) { qn = cross3(ca, da); qn2 = dot3(qn, qn); dq = 2.f * dv * (lc + ld + 2.f * dv); }
    const float gn2 = dot3(gn, gn);
    const float d = dot3(qn, gn);
    const float qnl = sqrtf(qn2), gnl = sqrtf(gn2);
    // gradient sum: FP32 quotients and normalisation, ~1e-6 relative
    const bool uncertain = near_fallback || gn2 < 1e-4f ||
                           fabsf(d) <= 4.f * dq * gnl + 1e-5f * qnl * gnl;
    bool swap = !uncertain && gn2 > 0.f && qn2 > 0.f && d < 0.f;
    P.stage_quad[slot] = swap ? make_int4((int)r0, (int)r3, (int)r2, (int)r1)
                              : make_int4((int)r0, (int)r1, (int)r2, (int)r3);
    P.stage_key[slot] = make_uint2((uint32_t)k, (uint32_t)col);
    if (uncertain) {
        const unsigned int w = atomicAdd(P.wind_count, 1u);
        if (w < P.wind_cap) {
            const uint64_t pk = pack_cell(i, j, k);
            P.wind_items[w] = make_uint4(slot, (uint32_t)axis | ((uint32_t)gi << 2), (uint32_t)pk, (uint32_t)(pk >> 32));
        } else {
            set_error(P.err, kErrOverflow);
        }
        // request the FP64 vertex of each of the four cells once
        const uint32_t rq[4] = {r0, r1, r2, r3};
#pragma unroll
        for (int q = 0; q < 4; ++q)
            request_fp64_vertex(P.v64_index, P.v64_cells, P.v64_count, P.v64_cap, P.err, rq[q]);
    }
}

// A warp takes 32 consecutive active cells. Each lane reads its cell's face mask (the cell's
// min-corner edges with a strict sign change, contouring.cpp:609-729) and, when it owns a
// face, the cell's gradient and the ranks of the face neighbours; then the warp's faces
// (about one per cell) are dealt out a lane each, the owner's data passed by shuffle, so
// the per-face work runs with the lanes full.
template <bool ONE>
__global__ void __launch_bounds__(kFaceThreads)
k_face_scatter(const __grid_constant__ FaceParams P) {
    __shared__ uint8_t s_item[kFaceThreads / 32][96];
    const int lane = threadIdx.x & 31, wb = threadIdx.x >> 5;
    const long long stride = (long long)gridDim.x * blockDim.x;
    // a captured graph whose live count exceeds the capacity it was built for does nothing
    // (the host reports the overflow after the replay)
    const long long nact = P.live ? ((long long)*P.live > P.nactive ? 0 : (long long)*P.live) : P.nactive;
    // the face mask and list entry of the next grid-stride step are loaded one step ahead
    long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x - lane);
    uint32_t fm_next = 0;
    uint64_t pk_next = 0;
    if (base + lane < nact) { fm_next = P.fmask[base + lane]; pk_next = P.list[base + lane]; }
    for (; base < nact; base += stride) {                                 // warp-uniform
        const long long rr = base + lane;
        const uint32_t fm = fm_next;
        const uint64_t pk = pk_next;
        fm_next = 0;
        if (rr + stride < nact) { fm_next = P.fmask[rr + stride]; pk_next = P.list[rr + stride]; }
        int gi = 0, i = 0, j = 0, k = 0;
        float3 g0 = make_float3(0.f, 0.f, 0.f);
        uint32_t r_k1 = 0xffffffffu, r_j1 = 0xffffffffu, r_jk = 0xffffffffu;
        if (fm) {
            gi = ONE ? 0 : slot_of_rank(P.B, (unsigned long long)rr);
            const GridSlot& S = slot_ref<ONE>(P.B, gi);
            const uint32_t* const bits = P.bits + S.bits_off;
            const uint32_t* const super = P.super + S.super_off;
            unpack_cell(pk, i, j, k);
            g0 = grid_gradient32(S.g, i, j, k);
            // All four cells of a face are active, so a cell's x-1 neighbour in a face is the
            // previous active cell in linear order (rank - 1).
            if (fm & 3) r_k1 = cell_rank(bits, super, S.g, i, j, k - 1);
            if (fm & 5) r_j1 = cell_rank(bits, super, S.g, i, j - 1, k);
            if (fm & 1) r_jk = cell_rank(bits, super, S.g, i, j - 1, k - 1);
        }
        const uint32_t cnt = __popc(fm);
        uint32_t off = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, off, o);
            if (lane >= o) off += v;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, off, 31);
        off -= cnt;
        for (uint32_t m = fm; m; m &= m - 1) s_item[wb][off++] = (uint8_t)((lane << 2) | (__ffs(m) - 1));
        __syncwarp();
        for (uint32_t t0 = 0; t0 < total; t0 += 32) {                     // warp-uniform
            const uint32_t t = t0 + lane;
            const uint32_t it = t < total ? s_item[wb][t] : 0u;
            const int src = (int)(it >> 2), axis = (int)(it & 3);
            const int fi = __shfl_sync(0xffffffffu, i, src), fj = __shfl_sync(0xffffffffu, j, src);
            const int fk = __shfl_sync(0xffffffffu, k, src), fg = __shfl_sync(0xffffffffu, gi, src);
            const float3 f0 = make_float3(__shfl_sync(0xffffffffu, g0.x, src), __shfl_sync(0xffffffffu, g0.y, src),
                                          __shfl_sync(0xffffffffu, g0.z, src));
            const uint32_t fk1 = __shfl_sync(0xffffffffu, r_k1, src), fj1 = __shfl_sync(0xffffffffu, r_j1, src);
            const uint32_t fjk = __shfl_sync(0xffffffffu, r_jk, src);
            if (t < total)
                emit_face<ONE>(P, fg, fi, fj, fk, (uint32_t)(base + src), axis, f0, fk1, fj1, fjk);
        }
        __syncwarp();
    }
}

cudaError_t launch_face_scatter(const FaceParams& P, int num_sms, cudaStream_t s, int blocks_per_sm) {
    if (P.nactive <= 0) return cudaSuccess;
    long long blocks = (P.nactive + kFaceThreads - 1) / kFaceThreads;
    const long long cap = (long long)num_sms * blocks_per_sm;
    if (blocks > cap) blocks = cap;
    if (P.B.n == 1) k_face_scatter<true><<<(unsigned)blocks, kFaceThreads, 0, s>>>(P);
    else            k_face_scatter<false><<<(unsigned)blocks, kFaceThreads, 0, s>>>(P);
    return cudaGetLastError();
}

// ---- in-column ordering ----------------------------------------------------------------

__global__ void __launch_bounds__(256)
k_face_order(const int4* __restrict__ stage_quad, const uint2* __restrict__ stage_key,
             const uint32_t* __restrict__ col_start, const uint32_t* __restrict__ col_count,
             const unsigned long long* __restrict__ nfaces, int4* __restrict__ faces) {
    const long long nf = (long long)*nfaces;
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < nf;
         s += (long long)gridDim.x * blockDim.x) {
        const uint2 key = stage_key[s];
        const uint32_t start = col_start[key.y];
        const uint32_t cnt = col_count[key.y];
        uint32_t rank = 0;
        for (uint32_t q = 0; q < cnt; ++q) rank += (stage_key[start + q].x < key.x) ? 1u : 0u;
        faces[start + rank] = stage_quad[s];
    }
}

cudaError_t launch_face_order(const int4* stage_quad, const uint2* stage_key, const uint32_t* col_start,
                              const uint32_t* col_count, const unsigned long long* nfaces, int4* faces,
                              long long max_faces, int num_sms, cudaStream_t s) {
    if (max_faces <= 0) return cudaSuccess;
    long long blocks = (max_faces + 255) / 256;
    const long long cap = (long long)num_sms * 16;
    if (blocks > cap) blocks = cap;
    k_face_order<<<(unsigned)blocks, 256, 0, s>>>(stage_quad, stage_key, col_start, col_count, nfaces, faces);
    return cudaGetLastError();
}

// ---- batch bookkeeping ------------------------------------------------------------------

// face_off[b] = col_start[col_off[b]], face_off[n] = total: the first face of every grid.
__global__ void k_face_offsets(BatchTable B, const uint32_t* __restrict__ col_start,
                               const unsigned long long* __restrict__ total, unsigned long long* face_off) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b <= B.n; b += gridDim.x * blockDim.x)
        face_off[b] = b < B.n ? (unsigned long long)col_start[B.col_off[b]] : *total;
}

cudaError_t launch_face_offsets(const BatchTable& B, const uint32_t* col_start, const unsigned long long* total,
                                unsigned long long* face_off, cudaStream_t s) {
    k_face_offsets<<<(B.n + 1 + 255) / 256, 256, 0, s>>>(B, col_start, total, face_off);
    return cudaGetLastError();
}

// Face vertex indices from batch-global ranks to ranks within the face's own grid. faces
// holds vpf ints per face; face f of the batch belongs to the grid b with
// face_off[b] * fpq <= f < face_off[b+1] * fpq (fpq = faces per quad: 1, or 2 for triangles).
__global__ void __launch_bounds__(256) k_localize_faces(const unsigned long long* __restrict__ vert_off,
                                                        const unsigned long long* __restrict__ face_off, int n,
                                                        int* faces, int vpf) {
    const int fpq = vpf == 3 ? 2 : 1;
    const unsigned long long nf = face_off[n] * fpq;
    for (unsigned long long f = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; f < nf;
         f += (unsigned long long)gridDim.x * blockDim.x) {
        const int b = slot_search(face_off, n, f / fpq);
        const int base = (int)vert_off[b];
        for (int q = 0; q < vpf; ++q) faces[f * vpf + q] -= base;
    }
}

cudaError_t launch_localize_faces(const unsigned long long* vert_off, const unsigned long long* face_off, int n,
                                  int* faces, int vpf, long long max_faces, int num_sms, cudaStream_t s) {
    if (max_faces <= 0) return cudaSuccess;
    long long blocks = (max_faces + 255) / 256;
    const long long cap = (long long)num_sms * 16;
    if (blocks > cap) blocks = cap;
    k_localize_faces<<<(unsigned)blocks, 256, 0, s>>>(vert_off, face_off, n, faces, vpf);
    return cudaGetLastError();
}

// ---- quad -> triangles -----------------------------------------------------------------
//
// triangulate_v1 (contouring.cpp:88-113): quad (a,b,c,d) -> (a,b,c), (a,c,d); each triangle
// is flipped (second and third index swapped) when its normal points against the quad
// normal (pb-pa)x(pd-pa), with the fallback (pc-pa)x(pd-pa) below a squared norm of 1e-24 and
// no orientation at all when that is below 1e-24 too (orient_triangles_for_quad,
// contouring.cpp:40-86). Decided here in FP32 with the vertex error bounds; quads whose
// decision the bounds do not settle are listed and re-decided from FP64 vertices
// (k_tri_fp64).
__global__ void __launch_bounds__(256)
k_triangulate(TriParams P) {
    const long long nq = (long long)*P.nquads;
    for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < nq;
         f += (long long)gridDim.x * blockDim.x) {
        const int4 q = P.quads[f];
        const uint32_t a = (uint32_t)q.x, b = (uint32_t)q.y, c = (uint32_t)q.z, d = (uint32_t)q.w;
        const float3 pa = ldv(P.V, a), pb = ldv(P.V, b), pc = ldv(P.V, c), pd = ldv(P.V, d);
        // the quad's grid (its first vertex's) gives the cell width of the bound
        const float hmax = P.B.n == 1 ? P.B.s0.hmax : (P.B.cell_slot ? P.B.slots[P.B.cell_slot[a]].hmax : P.hmax);
        const float dv = quad_vertex_bound(P.vclass, a, b, c, d, pa, pb, pc, pd, hmax);
        const float3 ba = sub3(pb, pa), ca = sub3(pc, pa), da = sub3(pd, pa);
        const float lb = sqrtf(dot3(ba, ba)), lc = sqrtf(dot3(ca, ca)), ld = sqrtf(dot3(da, da));
        float3 qn = cross3(ba, da);
        float dq = 2.f * dv * (lb + ld + 2.f * dv);
        float qnl = sqrtf(dot3(qn, qn));
        bool uncertain = (qnl - dq) < 1e-12f && (qnl + dq) >= 1e-12f;    // straddles the switch
        if (qnl * qnl < 1e-24f) {
            qn = cross3(ca, da);
            dq = 2.f * dv * (lc + ld + 2.f * dv);
            qnl = sqrtf(dot3(qn, qn));
            uncertain |= (qnl - dq) < 1e-12f && (qnl + dq) >= 1e-12f;   // straddles "no orientation"
        }
        const bool orient = qnl * qnl >= 1e-24f;
        const float3 t0 = cross3(ba, ca), t1 = cross3(ca, da);
        const float dt0 = 2.f * dv * (lb + lc + 2.f * dv), dt1 = 2.f * dv * (lc + ld + 2.f * dv);
        const float t0l = sqrtf(dot3(t0, t0)), t1l = sqrtf(dot3(t1, t1));
        const float d0 = dot3(t0, qn), d1 = dot3(t1, qn);
        if (orient) {
            uncertain |= fabsf(d0) <= 4.f * (dt0 * qnl + t0l * dq + dt0 * dq) + 1e-5f * t0l * qnl;
            uncertain |= fabsf(d1) <= 4.f * (dt1 * qnl + t1l * dq + dt1 * dq) + 1e-5f * t1l * qnl;
        }
        const bool flip0 = orient && d0 < 0.f, flip1 = orient && d1 < 0.f;
        int* t = P.tris + 6 * f;
        t[0] = (int)a; t[1] = flip0 ? (int)c : (int)b; t[2] = flip0 ? (int)b : (int)c;
        t[3] = (int)a; t[4] = flip1 ? (int)d : (int)c; t[5] = flip1 ? (int)c : (int)d;
        if (uncertain) {
            const unsigned int w = atomicAdd(P.item_count, 1u);
            if (w < P.item_cap) P.items[w] = (uint32_t)f;
            else set_error(P.err, kErrOverflow);
            request_fp64_vertex(P.v64_index, P.v64_cells, P.v64_count, P.v64_cap, P.err, a);
            request_fp64_vertex(P.v64_index, P.v64_cells, P.v64_count, P.v64_cap, P.err, b);
            request_fp64_vertex(P.v64_index, P.v64_cells, P.v64_count, P.v64_cap, P.err, c);
            request_fp64_vertex(P.v64_index, P.v64_cells, P.v64_count, P.v64_cap, P.err, d);
        }
    }
}

cudaError_t launch_triangulate(const TriParams& P, long long max_quads, int num_sms, cudaStream_t s) {
    if (max_quads <= 0) return cudaSuccess;
    long long blocks = (max_quads + 255) / 256;
    const long long cap = (long long)num_sms * 16;
    if (blocks > cap) blocks = cap;
    k_triangulate<<<(unsigned)blocks, 256, 0, s>>>(P);
    return cudaGetLastError();
}

}  // namespace dcb
