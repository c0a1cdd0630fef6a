// dcb_band.cu — Hermite samples, 4-cell normal averaging, FP32 QEF and face staging, a tile of
// cells at a time with the tile's stencil in shared memory, over every grid of a batch.
//
// Semantics follow the reference CPU backend:
//   Hermite samples   Cell::fill_hermite_data (src/cpp/Cell.cpp:162-212), lerp t = fa/(fa-fb
//                     +1e-16) (:49-52), normalised trilinear gradient (:80-155)
//   averaging         average_hermite_normals / process_edge (src/cpp/hermite_update.cpp:
//                     171-438): an edge with an endpoint strictly inside the grid whose four
//                     cells are active gets normalize(sum of the four cells' own normals)
//   QEF               Cell::update / solve_quadratic_system (Cell.cpp:284-361)
//   faces             extract_mesh_from_cells (src/cpp/contouring.cpp:607-729): a quad per
//                     edge with a strict sign change; cell (i,j,k) owns its min-corner edges
//
// Work split. A tile is 32 x 4 x 4 cells: one 32-cell active-bit word in each of 16 cell rows.
// A CTA takes 32 consecutive chunks of up to 32 x-adjacent tiles each; the mark kernel
// recorded which tiles of each chunk hold an active cell. For each such chunk the CTA forms the
// ranks of its rows (below), and for each of its active tiles:
//   1. stages the 35 x 7 x 7 grid points around it (every 4x4x4 stencil of its cells) in
//      shared memory, with the tile's and the surrounding rows' active words and the global
//      rank of each word's first active cell (the mark segment's first rank + popcounts of
//      the segment's earlier words, a warp scan over the chunk's words; the chunk also writes
//      the super-word ranks of its rows and, per cell, the packed active-cell list, so no
//      separate rank expansion runs);
//   2. lists, row by row with ballots, the crossing edges of the tile's active cells;
//   3. computes, a thread per listed edge, the edge's averaged normal ONCE (four trilinear
//      gradients, each an edge difference plus two bilinear differences of the staged
//      points), not once per cell that shares it;
//   4. solves, a thread per active cell, its centred FP32 normal equations (Kahan sums,
//      rank-1 certificate; other cells to the Jacobi (dcb_vertex.cu) or FP64 list), writes
//      the vertex at its rank, and stages each face it owns with the ranks of its four cells
//      and the gradient sum that decides the winding (k_face_place finishes the faces once
//      every vertex exists).
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>
#include <cooperative_groups/scan.h>
#include "dcb_qef.cuh"

namespace dcb {

namespace cg = cooperative_groups;

constexpr int kBandThreads = 128;
constexpr int kTY = kBandTileRows, kTZ = kBandTilePlanes;   // cell rows and planes per tile
constexpr int kChunkGroup = 32;                 // chunks a CTA takes at a time
constexpr int kSX = 36;                         // staged points per row: x0-1 .. x0+34
constexpr int kSY = kTY + 3, kSZ = kTZ + 3;     // rows y0-1 .. y0+5, planes z0-1 .. z0+5
constexpr int kXRows = (kTY + 1) * (kTZ + 1);   // X edges (py, pz): py in [y0, y0+4], pz in [z0, z0+4]
constexpr int kYRows = kTY * (kTZ + 1);         // Y edges: py in [y0, y0+4), pz in [z0, z0+4]
constexpr int kZRows = (kTY + 1) * kTZ;         // Z edges: py in [y0, y0+4], pz in [z0, z0+4)
constexpr int kYBase = kXRows, kZBase = kXRows + kYRows;
constexpr int kERows = kXRows + kYRows + kZRows;    // 65 edge rows
constexpr int kCRows = kTY * kTZ;                   // 16 cell rows
constexpr int kRows = kERows + kCRows;              // counted rows (edges, then cells)
constexpr int kMaxEdges = 32 * kXRows + 33 * (kYRows + kZRows);   // 2,120
// Edge records kept in shared memory per tile; a tile with more listed edges (dense sign noise,
// not surfaces) has the rest recomputed by the cells that need them, with the same function.
constexpr int kEdgeCap = 512;
constexpr int kTileCells = 32 * kTY * kTZ;

// The staged grid values of one tile, 0 outside the grid.
struct Vals {
    float v[kSZ][kSY][kSX];
};

struct BandSmem {
    Vals vb[2];                        // this tile's values and the next tile's (in flight)
    float rw[3][kSX];                  // 1 / cell width along x, y, z at index (lo - 1 + q)
    float4 e[kEdgeCap];                // per listed edge: averaged normal, flags in w
    float t[12][kBandThreads];         // per cell thread: lerp parameter of each crossing edge
    unsigned long long m[kERows];      // edge rows: crossing edges of active tile cells
    uint32_t off[kRows + 1];           // exclusive prefix of the row counts
    uint16_t list[kMaxEdges];          // edge entries: row << 6 | bit
    uint16_t cells[kTileCells];        // active tile cells: (kk * 4 + jj) << 5 | bit
    uint32_t word[kTZ + 1][kTY + 1];   // active word of cell rows (y0-1+a, z0-1+b) -> [b][a]
    uint32_t rank0[kTZ + 1][kTY + 1];  // global rank of that word's first active cell
    uint32_t cw[kTZ + 1][kTY + 1][32]; // the chunk's words of those rows, [..][x-word in chunk]
    uint32_t cr[kTZ + 1][kTY + 1][32]; // global rank of each such word's first active cell
    uint32_t gtiles[32];               // active tiles of each chunk of the group
    unsigned int chunk;
    unsigned int hist;
};

// Edge flags (w of the record).
constexpr uint32_t kEdgeOwn = 1;   // not averaged: each cell uses its own trilinear normal
constexpr uint32_t kEdgeIll = 2;   // FP32 cannot be trusted with this normal

__device__ __forceinline__ float sval(const Vals& V, int xl, int yl, int zl) {
    return V.v[zl + 1][yl + 1][xl + 1];   // local coordinates relative to (x0, y0, z0)
}

// One 4-byte asynchronous global -> shared copy (cp.async); an invalid point reads nothing
// (source size 0) and is zero-filled.
__device__ __forceinline__ void copy4_async(float* dst, const float* src, const float* any_valid, bool valid) {
    const unsigned int saddr = (unsigned int)__cvta_generic_to_shared(dst);
    const int n = valid ? 4 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(saddr), "l"(valid ? src : any_valid), "r"(n)
                 : "memory");
}
__device__ __forceinline__ void copy_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void copy_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Start the copies of tile (x0, y0, z0)'s 35 x 7 x 7 points into V: a warp per point row, lane l
// copying point x0-1+l and lanes 0-3 also x0+31+l. Completes at copy_wait_all + a barrier.
__device__ __forceinline__ void stage_tile_async(Vals& V, const GridDesc& g, int x0, int y0, int z0, int warp,
                                                 int lane) {
    for (int r = warp; r < kSY * kSZ; r += kBandThreads / 32) {
        const int yl = r % kSY - 1, zl = r / kSY - 1;
        const int y = y0 + yl, z = z0 + zl;
        const bool row_in = y >= 0 && y < g.ny && z >= 0 && z < g.nz;
        const float* row = g.v + (row_in ? ((long long)y + (long long)g.ny * z) * g.nx : 0);
        const int xa = x0 - 1 + lane;
        copy4_async(&V.v[zl + 1][yl + 1][lane], row + xa, g.v, row_in && xa >= 0 && xa < g.nx);
        if (lane < kSX - 32) {
            const int xb = x0 + 31 + lane;
            copy4_async(&V.v[zl + 1][yl + 1][32 + lane], row + xb, g.v, row_in && xb < g.nx);
        }
    }
    copy_commit();
}

// Active test of the cell whose min corner is at local (xl, yl, zl) from the staged points.
__device__ __forceinline__ bool active_local(const Vals& s, int xl, int yl, int zl) {
    bool neg = false, pos = false;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const float v = sval(s, xl + corner_dx(c), yl + corner_dy(c), zl + corner_dz(c));
        neg |= v < 0.f;
        pos |= v > 0.f;
    }
    return neg && pos;
}

// gradientAt (contouring.cpp:141-207) in FP32 at grid point (x, y, z), neighbours clamped to
// the grid, from the staged points (orientation tests only: a 2-ulp quotient is far inside the
// uncertainty margin, and uncertain faces are re-decided in FP64).
__device__ __forceinline__ float3 gradient_at(const Vals& s, const GridDesc& g, int x0, int y0, int z0,
                                              int x, int y, int z) {
    const int xm = max(x - 1, 0), xp = min(x + 1, g.nx - 1);
    const int ym = max(y - 1, 0), yp = min(y + 1, g.ny - 1);
    const int zm = max(z - 1, 0), zp = min(z + 1, g.nz - 1);
    float3 o = make_float3(0.f, 0.f, 0.f);
    const int xl = x - x0, yl = y - y0, zl = z - z0;
    const float dx = pos_axis(g.ox, g.vx, xp) - pos_axis(g.ox, g.vx, xm);
    if (fabsf(dx) > 1e-12f) o.x = __fdividef(sval(s, xp - x0, yl, zl) - sval(s, xm - x0, yl, zl), dx);
    const float dy = pos_axis(g.oy, g.vy, yp) - pos_axis(g.oy, g.vy, ym);
    if (fabsf(dy) > 1e-12f) o.y = __fdividef(sval(s, xl, yp - y0, zl) - sval(s, xl, ym - y0, zl), dy);
    const float dz = pos_axis(g.oz, g.vz, zp) - pos_axis(g.oz, g.vz, zm);
    if (fabsf(dz) > 1e-12f) o.z = __fdividef(sval(s, xl, yl, zp - z0) - sval(s, xl, yl, zm - z0), dz);
    const float n2 = o.x * o.x + o.y * o.y + o.z * o.z;
    if (n2 > 0.f) { const float r = rsqrtf(n2); o.x *= r; o.y *= r; o.z *= r; }
    return o;
}

// Edge row q (0..64) -> axis and the local (y, z) of its edges' low endpoints.
__device__ __forceinline__ void edge_row(int q, int& axis, int& yl, int& zl) {
    if (q < kYBase) { axis = 0; yl = q % (kTY + 1); zl = q / (kTY + 1); }
    else if (q < kZBase) { axis = 1; yl = (q - kYBase) % kTY; zl = (q - kYBase) / kTY; }
    else { axis = 2; yl = (q - kZBase) % (kTY + 1); zl = (q - kZBase) / (kTY + 1); }
}

// Averaged normal of the crossing edge with low endpoint at local (xl, yl, zl) along axis, or
// the kEdgeOwn flag. On an edge every trilinear gradient reduces to the edge difference plus
// two bilinear differences, so the four cells' normals need the edge's 2 x 3 x 3 points.
__device__ float4 edge_record(const BandSmem& sm, const Vals& s, const GridDesc& g, int x0, int y0, int z0, int axis,
                              int xl, int yl, int zl) {
    const int lx = x0 + xl, ly = y0 + yl, lz = z0 + zl;
    const int hx = lx + (axis == 0), hy = ly + (axis == 1), hz = lz + (axis == 2);
    const bool in0 = lx > 0 && lx < g.nx - 1 && ly > 0 && ly < g.ny - 1 && lz > 0 && lz < g.nz - 1;
    const bool in1 = hx > 0 && hx < g.nx - 1 && hy > 0 && hy < g.ny - 1 && hz > 0 && hz < g.nz - 1;
    const int d1 = axis == 0 ? 1 : 0;
    const int d2 = axis == 2 ? 1 : 2;
    // unit steps along d1 and d2 in local coordinates
    const int e1x = d1 == 0, e1y = d1 == 1;
    const int e2y = d2 == 1, e2z = d2 == 2;
    const float s_lo = sval(s, xl, yl, zl);
    const float s_hi = sval(s, xl + (axis == 0), yl + (axis == 1), zl + (axis == 2));
    bool avg = in0 || in1;
    if (avg && !strict_change(s_lo, s_hi)) {
        // zero endpoint: the four cells are not automatically active
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int m1 = q & 1, m2 = q >> 1;
            avg = avg && active_local(s, xl - m1 * e1x, yl - m1 * e1y - m2 * e2y, zl - m2 * e2z);
        }
    }
    if (!avg) return make_float4(0.f, 0.f, 0.f, __uint_as_float(kEdgeOwn));
    const float t_lo = lerp_t(s_lo, s_hi);
    const float u_hi = fabsf(s_lo - s_hi) < 1e-6f ? 1.f - lerp_t(s_hi, s_lo) : t_lo;
    const int hxl = xl + (axis == 0), hyl = yl + (axis == 1), hzl = zl + (axis == 2);
    const float ga = (s_hi - s_lo) * sm.rw[axis][(axis == 0 ? xl : axis == 1 ? yl : zl) + 1];
    // perpendicular differences at both edge ends: forward (p) and backward (m)
    const float a0p = sval(s, xl + e1x, yl + e1y, zl) - s_lo, a0m = s_lo - sval(s, xl - e1x, yl - e1y, zl);
    const float a1p = sval(s, hxl + e1x, hyl + e1y, hzl) - s_hi, a1m = s_hi - sval(s, hxl - e1x, hyl - e1y, hzl);
    const float b0p = sval(s, xl, yl + e2y, zl + e2z) - s_lo, b0m = s_lo - sval(s, xl, yl - e2y, zl - e2z);
    const float b1p = sval(s, hxl, hyl + e2y, hzl + e2z) - s_hi, b1m = s_hi - sval(s, hxl, hyl - e2y, hzl - e2z);
    // widths of the cells on either side of the edge along d1 and d2
    const int c1 = d1 == 0 ? xl : yl, c2 = d2 == 1 ? yl : zl;
    const float rw1p = sm.rw[d1][c1 + 1], rw1m = sm.rw[d1][c1];
    const float rw2p = sm.rw[d2][c2 + 1], rw2m = sm.rw[d2][c2];
    const float m1v = fmaxf(fmaxf(fabsf(a0p), fabsf(a1p)) * rw1p, fmaxf(fabsf(a0m), fabsf(a1m)) * rw1m);
    const float m2v = fmaxf(fmaxf(fabsf(b0p), fabsf(b1p)) * rw2p, fmaxf(fabsf(b0m), fabsf(b1m)) * rw2m);
    const float bound2 = kNormalCond2 * (ga * ga + m1v * m1v + m2v * m2v);
    bool ill = false;
    float3 acc = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int m1 = q & 1, m2 = q >> 1;
        const bool start_high = (axis == 0) ? (m1 == 1) : (axis == 1) ? (m1 == 0) : false;
        const float u = start_high ? u_hi : t_lo;
        const float e1lo = m1 ? a0m : a0p, e1hi = m1 ? a1m : a1p;
        const float e2lo = m2 ? b0m : b0p, e2hi = m2 ? b1m : b1p;
        const float g1 = (e1lo + u * (e1hi - e1lo)) * (m1 ? rw1m : rw1p);
        const float g2 = (e2lo + u * (e2hi - e2lo)) * (m2 ? rw2m : rw2p);
        float3 gv;
        if (axis == 0) gv = make_float3(ga, g1, g2);
        else if (axis == 1) gv = make_float3(g1, ga, g2);
        else gv = make_float3(g1, g2, ga);
        const float gn2 = gv.x * gv.x + gv.y * gv.y + gv.z * gv.z;
        if (gn2 <= bound2) ill = true;
        if (gn2 > 0.f) {
            const float rn = rsqrtf(gn2);
            acc.x += gv.x * rn; acc.y += gv.y * rn; acc.z += gv.z * rn;
        }
    }
    if (acc.x * acc.x + acc.y * acc.y + acc.z * acc.z < 1e-4f) ill = true;
    const float3 n = normalized(acc);
    return make_float4(n.x, n.y, n.z, __uint_as_float(ill ? kEdgeIll : 0u));
}

// Global rank of the active cell at bit b of the word of cell row (y0-1+a, z0-1+c).
__device__ __forceinline__ uint32_t rank_in(const BandSmem& s, int a, int c, int b) {
    return s.rank0[c][a] + __popc(s.word[c][a] & ((1u << b) - 1u));
}

// Slots for n items of each thread among the threads that arrive together: one atomic per
// such group on the shared counter.
__device__ __forceinline__ unsigned int reserve_slots(unsigned int* counter, unsigned int n) {
    cg::coalesced_group grp = cg::coalesced_threads();
    const unsigned int pre = cg::exclusive_scan(grp, n);
    const unsigned int tot = cg::reduce(grp, n, cg::plus<unsigned int>());
    unsigned int base = 0;
    if (grp.thread_rank() == 0 && tot) base = atomicAdd(counter, tot);
    return grp.shfl(base, 0) + pre;
}

// Chunks of one grid: along x (32 words of 32 cells), row blocks, plane blocks.
__host__ __device__ inline void band_chunks(const GridDesc& g, int& nxc, int& nyb, int& nzb) {
    nxc = ((g.cx + 31) / 32 + 31) / 32;
    nyb = (g.cy + kTY - 1) / kTY;
    nzb = (g.cz + kTZ - 1) / kTZ;
}

template <bool ONE>
__global__ void __launch_bounds__(kBandThreads, 4)
k_band(const __grid_constant__ BandParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BandSmem& s = *reinterpret_cast<BandSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // a captured graph whose live count exceeds the capacity it was built for does nothing
    // (the host reports the overflow after the replay)
    if (P.live && *P.live > (unsigned long long)P.nv) return;
    if (tid == 0) s.hist = 0;

    for (;;) {
        // a group of 32 consecutive chunks; the mark kernel recorded each one's active tiles
        __syncthreads();
        if (tid == 0) s.chunk = atomicAdd(P.chunk_next, (unsigned int)kChunkGroup);
        __syncthreads();
        const long long c0 = s.chunk;
        if (c0 >= P.nchunks) break;
        if (warp == 0) s.gtiles[lane] = c0 + lane < P.nchunks ? __ldg(P.tilemap + c0 + lane) : 0u;
        __syncthreads();
      for (int q = 0; q < kChunkGroup; ++q) {
        uint32_t tiles = s.gtiles[q];
        if (!tiles) continue;                               // uniform: shared memory
        const long long cg_ = c0 + q;
        // the chunk's grid (batches: the grids' chunks are concatenated)
        const int gi = ONE ? 0 : slot_search(P.B.chunk_off, P.B.n, cg_);
        const GridSlot& S = slot_ref<ONE>(P.B, gi);
        const GridDesc& g = S.g;
        const long long c = ONE ? cg_ : cg_ - P.B.chunk_off[gi];
        const uint32_t* const bits = P.bits + S.bits_off;
        const long long cxcy = (long long)g.cx * g.cy;
        const int nwx = (g.cx + 31) >> 5;                 // words holding cells, per row
        int nxc, nyb, nzb;
        band_chunks(g, nxc, nyb, nzb);
        const int xc = (int)(c % nxc);
        const int jb = (int)((c / nxc) % nyb);
        const int kb = (int)(c / ((long long)nxc * nyb));
        const int y0 = jb * kTY, z0 = kb * kTZ;
        __syncthreads();   // the previous chunk's shared data is no longer read
        if (tiles) {
            // words and first ranks of the chunk's rows and the rows below / behind them: lane =
            // word; a segment's earlier words are summed by a scan of width tw (the mark's
            // segment, 32 or 8 words, aligned with the chunk)
            const int w = xc * 32 + lane;
            const int tw = S.tw;
            constexpr int kRankRows = (kTY + 1) * (kTZ + 1);
            constexpr int kPer = (kRankRows + kBandThreads / 32 - 1) / (kBandThreads / 32);
            // every row's word and segment start first (all loads in flight), then the scans
            uint32_t wv[kPer], sv[kPer];
#pragma unroll
            for (int it = 0; it < kPer; ++it) {
                const int q = warp + it * (kBandThreads / 32);
                const int a = q % (kTY + 1), cc = q / (kTY + 1);
                const int y = y0 - 1 + a, z = z0 - 1 + cc;
                const bool row_ok = q < kRankRows && y >= 0 && y < g.cy && z >= 0 && z < g.cz;
                const long long row = (long long)y + (long long)g.cy * z;
                wv[it] = (row_ok && w < nwx) ? __ldg(bits + row * g.W + w) : 0u;
                sv[it] = (row_ok && w < nwx && (lane & (tw - 1)) == 0) ? __ldg(P.seg_start + S.seg_off + row * S.nxt + w / tw) : 0u;
            }
#pragma unroll
            for (int it = 0; it < kPer; ++it) {
                const int q = warp + it * (kBandThreads / 32);
                if (q >= kRankRows) break;                       // warp-uniform
                const int a = q % (kTY + 1), cc = q / (kTY + 1);
                const int y = y0 - 1 + a, z = z0 - 1 + cc;
                const bool row_ok = y >= 0 && y < g.cy && z >= 0 && z < g.cz;
                const long long row = (long long)y + (long long)g.cy * z;
                const uint32_t word = wv[it];
                const uint32_t cnt = __popc(word);
                uint32_t incl = cnt;
                for (int o = 1; o < tw; o <<= 1) {
                    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o, tw);
                    if ((lane & (tw - 1)) >= o) incl += t;
                }
                const uint32_t start = __shfl_sync(0xffffffffu, sv[it], lane & ~(tw - 1), 32);
                const uint32_t r0 = start + incl - cnt;
                s.cw[cc][a][lane] = word;
                s.cr[cc][a][lane] = r0;
                // the chunk's own rows: rank of the first active cell of each 8-word super word
                if (row_ok && a >= 1 && cc >= 1 && w < g.W && (w & 7) == 0) P.super[S.super_off + row * g.W8 + (w >> 3)] = r0;
            }
            __syncthreads();
        }
        // the first tile's points; each later tile's are copied while the one before it is solved
        int cur = 0;
        if (tiles) stage_tile_async(s.vb[0], g, 32 * (xc * 32 + __ffs(tiles) - 1), y0, z0, warp, lane);
        while (tiles) {
            const int tb = __ffs(tiles) - 1;
            tiles &= tiles - 1;
            const int w = xc * 32 + tb;
            const int x0 = 32 * w;
            __syncthreads();   // the previous tile's shared data is no longer read
            // 2) the reciprocal widths, the words and their first ranks; the points arrive
            if (tid < kSX) {
                const int x = x0 - 1 + tid;
                s.rw[0][tid] = 1.f / (pos_axis(g.ox, g.vx, x + 1) - pos_axis(g.ox, g.vx, x));
            } else if (tid < kSX + kSY) {
                const int q = tid - kSX, y = y0 - 1 + q;
                s.rw[1][q] = 1.f / (pos_axis(g.oy, g.vy, y + 1) - pos_axis(g.oy, g.vy, y));
            } else if (tid < kSX + kSY + kSZ) {
                const int q = tid - kSX - kSY, z = z0 - 1 + q;
                s.rw[2][q] = 1.f / (pos_axis(g.oz, g.vz, z + 1) - pos_axis(g.oz, g.vz, z));
            } else if (tid >= 64 && tid < 64 + (kTY + 1) * (kTZ + 1)) {
                const int q = tid - 64, a = q % (kTY + 1), cc = q / (kTY + 1);
                s.word[cc][a] = s.cw[cc][a][tb];
                s.rank0[cc][a] = s.cr[cc][a][tb];
            }
            copy_wait_all();
            __syncthreads();
            const Vals& V = s.vb[cur];
            if (tiles) stage_tile_async(s.vb[cur ^ 1], g, 32 * (xc * 32 + __ffs(tiles) - 1), y0, z0, warp, lane);
            cur ^= 1;
            // 3) edge rows: crossing edges (Hermite test) of the tile's active cells; then the
            //    16 cell rows' active counts
            for (int q = warp; q < kERows; q += kBandThreads / 32) {
                int axis, yl, zl;
                edge_row(q, axis, yl, zl);
                // active tile cells touching the row's edges, as bits of the edge's x
                auto act = [&](int a, int cc) -> uint32_t {   // tile cell row (y0+a, z0+cc)
                    return (a >= 0 && a < kTY && cc >= 0 && cc < kTZ) ? s.word[cc + 1][a + 1] : 0u;
                };
                unsigned long long cells;
                if (axis == 0) cells = act(yl - 1, zl - 1) | act(yl, zl - 1) | act(yl - 1, zl) | act(yl, zl);
                else {
                    const unsigned long long A = axis == 1 ? (act(yl, zl - 1) | act(yl, zl)) : (act(yl - 1, zl) | act(yl, zl));
                    cells = A | (A << 1);
                }
                const float a0 = sval(V, lane, yl, zl);
                const float a1 = sval(V, lane + (axis == 0), yl + (axis == 1), zl + (axis == 2));
                unsigned long long m = __ballot_sync(0xffffffffu, hermite_crossing(a0, a1));
                if (axis != 0) {
                    const float b0 = sval(V, 32, yl, zl);
                    const float b1 = sval(V, 32, yl + (axis == 1), zl + (axis == 2));
                    if (hermite_crossing(b0, b1)) m |= 1ull << 32;
                }
                m &= cells;
                if (lane == 0) s.m[q] = m;
            }
            __syncthreads();
            if (warp == 0) {
                // exclusive prefix over the 65 edge rows and 16 cell rows, 32 rows per step
                uint32_t carry = 0;
                for (int base = 0; base < kRows; base += 32) {
                    const int q = base + lane;
                    uint32_t n = 0;
                    if (q < kERows) n = __popcll(s.m[q]);
                    else if (q < kRows) { const int cr = q - kERows; n = __popc(s.word[(cr >> 2) + 1][(cr & 3) + 1]); }
                    uint32_t incl = n;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                        if (lane >= o) incl += t;
                    }
                    if (q < kRows) s.off[q] = carry + incl - n;
                    carry += __shfl_sync(0xffffffffu, incl, 31);
                }
                if (lane == 0) s.off[kRows] = carry;
            }
            __syncthreads();
            // lists: edges by row (bit order), then active cells
            for (int q = warp; q < kRows; q += kBandThreads / 32) {
                if (q < kERows) {
                    const unsigned long long m = s.m[q];
                    const uint32_t lo = (uint32_t)m;
                    const uint32_t base = s.off[q];
                    if ((lo >> lane) & 1u) s.list[base + __popc(lo & ((1u << lane) - 1u))] = (uint16_t)((q << 6) | lane);
                    if (lane == 0 && (m >> 32)) s.list[base + __popc(lo)] = (uint16_t)((q << 6) | 32);
                } else {
                    const int cr = q - kERows;
                    const uint32_t wd = s.word[(cr >> 2) + 1][(cr & 3) + 1];
                    if ((wd >> lane) & 1u)
                        s.cells[s.off[q] - s.off[kERows] + __popc(wd & ((1u << lane) - 1u))] = (uint16_t)((cr << 5) | lane);
                }
            }
            __syncthreads();
            // 4) edge normals, a thread per listed edge
            const int nedges = min((int)s.off[kERows], kEdgeCap);
            for (int e = tid; e < nedges; e += kBandThreads) {
                const uint32_t it = s.list[e];
                int axis, yl, zl;
                edge_row((int)(it >> 6), axis, yl, zl);
                s.e[e] = edge_record(s, V, g, x0, y0, z0, axis, (int)(it & 63), yl, zl);
            }
            __syncthreads();
            // 5) cells, a thread per active cell
            const int ncells = (int)(s.off[kRows] - s.off[kERows]);
            for (int ci = tid; ci < ncells; ci += kBandThreads) {
                const uint32_t it = s.cells[ci];
                const int b = it & 31, jj = (it >> 5) & 3, kk = it >> 7;
                const int i = x0 + b, j = y0 + jj, k = z0 + kk;
                const uint32_t r = rank_in(s, jj + 1, kk + 1, b);
                if ((long long)r >= P.nv) { set_error(P.err, kErrInternal); continue; }
                P.list[r] = pack_cell(i, j, k);
                if (!ONE && P.cell_slot) P.cell_slot[r] = (uint32_t)gi;
                float c[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) c[q] = sval(V, b + corner_dx(q), jj + corner_dy(q), kk + corner_dz(q));
                // Pass 1: crossing edges and the centroid in local units.
                uint32_t hmask = 0;
                float cu = 0.f, cv = 0.f, cw = 0.f;
#pragma unroll
                for (int e = 0; e < 12; ++e) {
                    const int a = edge_a(e), bb = edge_b(e);
                    if (!hermite_crossing(c[a], c[bb])) continue;
                    hmask |= 1u << e;
                    const float t = lerp_t(c[a], c[bb]);
                    s.t[e][tid] = t;
                    float pu = (float)corner_dx(a), pv = (float)corner_dy(a), pw = (float)corner_dz(a);
                    if (corner_dx(a) != corner_dx(bb)) pu = corner_dx(a) ? 1.f - t : t;
                    if (corner_dy(a) != corner_dy(bb)) pv = corner_dy(a) ? 1.f - t : t;
                    if (corner_dz(a) != corner_dz(bb)) pw = corner_dz(a) ? 1.f - t : t;
                    cu += pu; cv += pv; cw += pw;
                }
                const float invm = 1.f / (float)__popc(hmask);
                cu *= invm; cv *= invm; cw *= invm;
                const float rdx = s.rw[0][b + 1], rdy = s.rw[1][jj + 1], rdz = s.rw[2][kk + 1];
                const float wx1 = width_axis(g, 0, i), wy1 = width_axis(g, 1, j), wz1 = width_axis(g, 2, k);
                const float fy = wy1 * rdx, fz = wz1 * rdx;
                // Pass 2: rows of the normal equations.
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
                    const float t = s.t[e][tid];
                    const float along = own_low ? t : 1.f - t;
                    const float pu = axis == 0 ? along : (float)lox;
                    const float pv = axis == 1 ? along : (float)loy;
                    const float pw = axis == 2 ? along : (float)loz;
                    // the edge's record: its row and bit among the listed edges
                    const int yl = jj + loy, zl = kk + loz, xb = b + lox;
                    const int q = axis == 0 ? zl * (kTY + 1) + yl
                                            : (axis == 1 ? kYBase + zl * kTY + yl : kZBase + zl * (kTY + 1) + yl);
                    const unsigned long long mrow = s.m[q];
                    const int slot = (int)s.off[q] + __popcll(mrow & ((1ull << xb) - 1ull));
                    const float4 rec = slot < kEdgeCap ? s.e[slot] : edge_record(s, V, g, x0, y0, z0, axis, xb, yl, zl);
                    const uint32_t fl = __float_as_uint(rec.w);
                    float3 n;
                    if (fl & kEdgeOwn) {
                        n = normalized(own_gradient(c, pu, pv, pw, rdx, rdy, rdz, ill));
                    } else {
                        n = make_float3(rec.x, rec.y, rec.z);
                        if (fl & kEdgeIll) ill = true;
                    }
                    const float qx = pu - cu, qy = (pv - cv) * fy, qz = (pw - cw) * fz;
                    const float nb = n.x * qx + n.y * qy + n.z * qz;
                    kahan_add(M00, K00, n.x * n.x); kahan_add(M01, K01, n.x * n.y); kahan_add(M02, K02, n.x * n.z);
                    kahan_add(M11, K11, n.y * n.y); kahan_add(M12, K12, n.y * n.z); kahan_add(M22, K22, n.z * n.z);
                    kahan_add(R0, Q0, n.x * nb); kahan_add(R1, Q1, n.y * nb); kahan_add(R2, Q2, n.z * nb);
                }
                float ox, oy, oz;
                // A NaN or infinite value anywhere in the normal equations (a non-finite grid value in
                // the stencil) propagates into the CPU backend's vertex through its SVD factors
                // (Cell.cpp:324-361); only the FP64 path repeats that, so such cells go there.
                if (!isfinite(M00 + M01 + M02 + M11 + M12 + M22 + R0 + R1 + R2 + cu + cv + cw)) ill = true;
                if (ill || P.force64) {
                    // FP32 cannot be trusted: the FP64 path recomputes this cell from the grid.
                    const unsigned int slot = reserve_slots(P.esc_count, 1u);
                    P.esc_list[slot] = r;
                    store_vertex(P.V, g, r, i, j, k, cu, cv, cw);
                } else if (qef_rank1(M00, M01, M02, M11, M12, M22, R0, R1, R2, P.thr, P.band, ox, oy, oz)) {
                    store_vertex(P.V, g, r, i, j, k, cu + ox, cv + oy / fy, cw + oz / fz);
                    P.vclass[r] = kVcRank1;
                    atomicAdd(&s.hist, 1u);
                } else {
                    const unsigned int slot = reserve_slots(P.hard_count, 1u);
                    P.hard_list[slot] = r;
                    P.hard_data[3 * (size_t)slot + 0] = make_float4(M00, M01, M02, M11);
                    P.hard_data[3 * (size_t)slot + 1] = make_float4(M12, M22, R0, R1);
                    P.hard_data[3 * (size_t)slot + 2] = make_float4(R2, cu, cv, cw);
                }
                // Faces owned by this cell: its min-corner X, Y, Z edges (contouring.cpp:609-729).
                const bool fx = j >= 1 && k >= 1 && strict_change(c[0], c[1]);
                const bool fyy = i >= 1 && k >= 1 && strict_change(c[0], c[3]);
                const bool fzz = i >= 1 && j >= 1 && strict_change(c[0], c[4]);
                // the reference looks each quad's Hermite normal up in the cell at (i, j-1, k-1),
                // (i-1, j, k-1) or (i-1, j-1, k); its sample interpolates from (i+1, j, k) for an
                // X edge and from (i, j, k) for Y and Z edges: infinite there, the sample is NaN
                // and the reference exits (contouring.cpp:560-594, 607-729)
                if ((fx && isinf(c[1])) || ((fyy || fzz) && isinf(c[0]))) set_error(P.err, kErrNonFinite);
                const unsigned int nfc = (unsigned int)fx + (unsigned int)fyy + (unsigned int)fzz;
                unsigned int f = reserve_slots(P.face_count, nfc);
                if (nfc) {
                    const float3 g0 = gradient_at(V, g, x0, y0, z0, i, j, k);
#pragma unroll
                    for (int axis = 0; axis < 3; ++axis) {
                        const bool has = axis == 0 ? fx : (axis == 1 ? fyy : fzz);
                        if (!has) continue;
                        // ranks of the four cells (CPU corner order); a face's x-1 neighbour is
                        // the previous active cell in linear order
                        uint32_t r0, r1, r3;
                        if (axis == 0) { r0 = rank_in(s, jj, kk, b); r1 = rank_in(s, jj + 1, kk, b); r3 = rank_in(s, jj, kk + 1, b); }
                        else if (axis == 1) { r1 = rank_in(s, jj + 1, kk, b); r0 = r1 - 1u; r3 = r - 1u; }
                        else { r1 = rank_in(s, jj, kk + 1, b); r0 = r1 - 1u; r3 = r - 1u; }
                        const float3 g1 = gradient_at(V, g, x0, y0, z0, i + (axis == 0), j + (axis == 1), k + (axis == 2));
                        const long long col = S.col_off + axis * cxcy + (long long)i * g.cy + j;
                        atomicAdd(&P.col_count[col], 1u);
                        if (f < P.face_cap) {
                            P.face_cells[f] = make_int4((int)r0, (int)r1, (int)r, (int)r3);
                            P.face_grad[f] = make_float4(g0.x + g1.x, g0.y + g1.y, g0.z + g1.z, __uint_as_float((uint32_t)col));
                        } else {
                            set_error(P.err, kErrOverflow);
                        }
                        ++f;
                    }
                }
            }
        }
      }
    }
    __syncthreads();
    if (tid == 0 && s.hist) atomicAdd(P.rank_hist + 1, (unsigned long long)s.hist);
}

template <bool ONE>
cudaError_t launch_band_t(const BandParams& P, int num_sms, cudaStream_t s) {
    const int bytes = (int)sizeof(BandSmem);
    cudaError_t e = cudaFuncSetAttribute(k_band<ONE>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_band<ONE>, kBandThreads, bytes);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    if (P.ctas_per_sm > 0 && P.ctas_per_sm < per_sm) per_sm = P.ctas_per_sm;
    long long blocks = (long long)num_sms * per_sm;
    if (blocks > P.nchunks) blocks = P.nchunks;
    k_band<ONE><<<(unsigned)blocks, kBandThreads, bytes, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_band(const BandParams& P, int num_sms, cudaStream_t s) {
    if (P.nchunks <= 0) return cudaSuccess;
    return P.B.n == 1 ? launch_band_t<true>(P, num_sms, s) : launch_band_t<false>(P, num_sms, s);
}

int band_max_ctas_per_sm() {
    const int bytes = (int)sizeof(BandSmem);
    if (cudaFuncSetAttribute(k_band<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_band<true>, kBandThreads, bytes) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return per_sm > 0 ? per_sm : 1;
}

long long band_chunk_count(int nx, int ny, int nz) {
    GridDesc g{};
    g.cx = nx - 1; g.cy = ny - 1; g.cz = nz - 1;
    int nxc, nyb, nzb;
    band_chunks(g, nxc, nyb, nzb);
    return (long long)nxc * nyb * nzb;
}

}  // namespace dcb
