// dcb_mark.cu — markActiveCells and the order-preserving active-cell compaction.
//
// Semantics (reference CPU backend): a cell is active iff some corner < 0 and some corner
// > 0 (Cell::Cell, src/cpp/Cell.cpp:57-77); vertex index = rank of the cell among active
// cells in linear (k, j, i) order (extract_mesh_from_cells, src/cpp/contouring.cpp:513-524).
// The reference GPU path uses one thread per cell, a byte flag per cell and a Thrust
// copy_if (src/cuda/dc_cuda.cu:241-281, 701-712).
//
// k_mark_zmarch: a CTA owns a tile of R cell rows x 1024 cells along x and marches through
// a chunk of KZ cell planes. Warp w streams point row j0+w of every point plane once
// (lane l loads points x0+32q+l: coalesced 128-byte rows; the next plane prefetched into
// registers while the current one is reduced), turns it into a negative-bit word and a
// positive-bit word per 32 points (one ballot each: two compares and two votes per word,
// fewer instructions than float4 loads with a nibble shuffle, which measured 10-26% slower
// here), and the cell words of plane k are bitwise ORs of the point words of
// rows j, j+1 in planes k, k+1 and their one-bit shift along x. Each grid value crosses
// HBM once and the SM (R+1)/R times. Outputs: the active bit words and the number of
// active cells of every (plane, row, x-tile) segment, in linear order.
// A scan of the segment counts gives each segment's first rank; k_expand_ranks then writes
// the 256-cell super-word ranks and the packed active-cell list.
#include "dcb_kernels.cuh"

namespace dcb {

constexpr int kMarkWarps = 8;          // point rows per tile (R + 1 <= 8)
constexpr int kTileWords = 32;         // cell words per x-tile (1024 cells)
constexpr int kNarrowTileWords = 8;    // x-tile of grids at most 256 cells wide
// TW cell words per x-tile: TW + 1 point words, loaded as 128-point chunks.
template <int TW> struct Tile {
    static constexpr int kPtWords = TW + 1;
    static constexpr int kChunks = (kPtWords + 3) / 4;
};

template <int TW>
struct RowRegs {
    float4 v[Tile<TW>::kChunks];
};

// Load the kPtWords*32 points of one point-row segment starting at x0 into registers:
// component q of chunk c holds point x0+128c+32q+lane (0 beyond the row). Words past
// kPtWords (the last chunk's unused components) are neither loaded nor voted on: the
// conditions fold at compile time.
template <int TW>
__device__ __forceinline__ void load_row(const float* __restrict__ row, int x0, int nx, int lane, RowRegs<TW>& R) {
    constexpr int kPtWords = Tile<TW>::kPtWords;
#pragma unroll
    for (int c = 0; c < Tile<TW>::kChunks; ++c) {
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        const int x = x0 + 128 * c + lane;
        if (x < nx) v.x = __ldg(row + x);
        if (4 * c + 1 < kPtWords && x + 32 < nx) v.y = __ldg(row + x + 32);
        if (4 * c + 2 < kPtWords && x + 64 < nx) v.z = __ldg(row + x + 64);
        if (4 * c + 3 < kPtWords && x + 96 < nx) v.w = __ldg(row + x + 96);
        R.v[c] = v;
    }
}

// Negative / positive bit words of the loaded segment (word q covers points x0+32q..+31).
template <int TW>
// inf_nan: stays 0 while every value is finite; fma(q, 0, x) turns it NaN for good at an
// infinite or NaN q (one instruction a point; the intrinsic is never simplified away).
__device__ __forceinline__ void row_words(const RowRegs<TW>& R, int lane, uint32_t* nw, uint32_t* pw, float& inf_nan) {
    constexpr int kPtWords = Tile<TW>::kPtWords;
#pragma unroll
    for (int c = 0; c < Tile<TW>::kChunks; ++c) {
        const float q[4] = {R.v[c].x, R.v[c].y, R.v[c].z, R.v[c].w};
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int w = 4 * c + s;
            if (w >= kPtWords) break;
            inf_nan = __fmaf_rn(q[s], 0.f, inf_nan);
            const uint32_t n = __ballot_sync(0xffffffffu, q[s] < 0.f);
            const uint32_t p = __ballot_sync(0xffffffffu, q[s] > 0.f);
            if (lane == 0) { nw[w] = n; pw[w] = p; }
        }
    }
}

// Single-grid launches fit 64 registers without spilling: 4 resident CTAs per SM instead of 3.
template <bool ONE, int TW>
__global__ void __launch_bounds__(kMarkWarps * 32, ONE ? 4 : 3)
k_mark_zmarch(const __grid_constant__ MarkParams P) {
    constexpr int kPtWords = Tile<TW>::kPtWords;
    __shared__ uint32_t s_nw[2][kMarkWarps][kPtWords];
    __shared__ uint32_t s_pw[2][kMarkWarps][kPtWords];
    // tile -> grid of the batch -> (x-tile, row block, z-chunk), x-tile fastest
    const long long tile = blockIdx.x;
    const int mi = (ONE || P.m == 1) ? 0 : slot_search(P.tile_off, P.m, tile);
    const GridSlot& S = slot_ref<ONE>(P.B, ONE ? 0 : P.tile_slot[mi]);
    const GridDesc& g = S.g;
    const int R = S.R, KZ = S.KZ, nxt = S.nxt;
    const long long local = ONE ? tile : tile - P.tile_off[mi];
    const int xt = (int)(local % nxt);         // x-tile
    const int j0 = (int)((local / nxt) % S.nrb) * R;   // first cell row
    const int kb = (int)(local / ((long long)nxt * S.nrb)) * KZ;   // first cell plane
    uint32_t* const bits = P.bits + S.bits_off;
    uint32_t* const seg_count = P.seg_count + S.seg_off;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int rows = min(R, g.cy - j0);
    const int ke = min(g.cz, kb + KZ);
    const int x0 = xt * TW * 32;               // first point / cell of the tile
    const bool loader = warp <= rows;          // point rows j0..j0+rows
    const float* base = g.v + (int64_t)(j0 + (loader ? warp : 0)) * g.nx;
    const int64_t plane = (int64_t)g.nx * g.ny;

    RowRegs<TW> cur;
    float inf_nan = 0.f;                       // NaN once a NaN or infinite value is among this lane's points
    if (loader) {
        load_row<TW>(base + (int64_t)kb * plane, x0, g.nx, lane, cur);
        row_words<TW>(cur, lane, s_nw[kb & 1][warp], s_pw[kb & 1][warp], inf_nan);
        load_row<TW>(base + (int64_t)(kb + 1) * plane, x0, g.nx, lane, cur);
    }
    const bool word_lane = TW == 32 || lane < TW;   // lanes beyond the tile's words idle
    const int wglob = xt * TW + lane;          // this lane's cell word in the row
    const int valid = g.cx - 32 * wglob;
    const uint32_t vmask = !word_lane ? 0u : valid >= 32 ? 0xffffffffu : (valid > 0 ? ((1u << valid) - 1u) : 0u);
    const int wl = word_lane ? lane : 0;

    for (int k = kb; k < ke; ++k) {
        const int p1 = (k + 1) & 1, p0 = k & 1;
        if (loader) {
            row_words<TW>(cur, lane, s_nw[p1][warp], s_pw[p1][warp], inf_nan);
            if (k + 2 <= ke) load_row<TW>(base + (int64_t)(k + 2) * plane, x0, g.nx, lane, cur);
        }
        __syncthreads();
        if (warp < rows) {
            const int r = warp;
            const uint32_t n0 = s_nw[p0][r][wl] | s_nw[p0][r + 1][wl] | s_nw[p1][r][wl] | s_nw[p1][r + 1][wl];
            const uint32_t n1 = s_nw[p0][r][wl + 1] | s_nw[p0][r + 1][wl + 1] | s_nw[p1][r][wl + 1] | s_nw[p1][r + 1][wl + 1];
            const uint32_t q0 = s_pw[p0][r][wl] | s_pw[p0][r + 1][wl] | s_pw[p1][r][wl] | s_pw[p1][r + 1][wl];
            const uint32_t q1 = s_pw[p0][r][wl + 1] | s_pw[p0][r + 1][wl + 1] | s_pw[p1][r][wl + 1] | s_pw[p1][r + 1][wl + 1];
            const uint32_t act = (n0 | (n0 >> 1) | (n1 << 31)) & (q0 | (q0 >> 1) | (q1 << 31)) & vmask;
            const int64_t row = (int64_t)(j0 + r) + (int64_t)g.cy * k;
            if (word_lane && wglob < g.W) bits[row * g.W + wglob] = act;
            uint32_t cnt = __popc(act);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
            if (lane == 0) seg_count[row * nxt + xt] = cnt;
        }
        __syncthreads();
    }
    // the host learns that the grid holds non-finite values (their cells take the FP64 path)
    if (__syncthreads_or(isnan(inf_nan)) && threadIdx.x == 0 && P.nonfinite) atomicOr(P.nonfinite, 1);
}

// Segments with at most this many active cells are expanded by one lane.
constexpr uint32_t kLaneSegmentCells = 96;

// Warp per group of 32 consecutive (row, x-tile) segments: the non-empty ones get the global
// ranks of their super words and their part of the packed active-cell list — a lane per
// segment with few active cells, the whole warp per segment with many.
template <bool ONE>
__global__ void __launch_bounds__(256)
k_expand_ranks(const __grid_constant__ ExpandParams P) {
    const int lane = threadIdx.x & 31;
    const long long nseg = P.nseg;
    const long long ngroups = (nseg + 31) / 32;
    for (long long grp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; grp < ngroups;
         grp += ((long long)gridDim.x * blockDim.x) >> 5) {
        const long long s0 = grp * 32;
        const bool have = s0 + lane < nseg;
        const uint32_t cnt = have ? P.seg_count[s0 + lane] : 0u;
        uint32_t live = __ballot_sync(0xffffffffu, cnt != 0);
        const uint32_t my_start = (have && cnt) ? P.seg_start[s0 + lane] : 0u;
        const int my_slot = (!ONE && have && cnt) ? slot_of_segment(P.B, s0 + lane) : 0;
        // segments with few active cells: a lane each (no shuffles); the rest cooperatively
        const bool light = have && cnt != 0 && cnt <= kLaneSegmentCells;
        if (light) {
            const GridSlot& S = slot_ref<ONE>(P.B, my_slot);
            const GridDesc& g = S.g;
            const long long ls = s0 + lane - S.seg_off;
            const long long row = ls / S.nxt;
            const int wb = (int)(ls - row * S.nxt) * S.tw;
            const int nw = min(S.tw, g.W - wb);
            const int j = (int)(row % g.cy), k = (int)(row / g.cy);
            const uint4* words = reinterpret_cast<const uint4*>(P.bits + S.bits_off + row * g.W + wb);
            uint32_t rank = my_start;
            for (int q4 = 0; q4 < nw; q4 += 4) {
                const uint4 v = __ldg(words + (q4 >> 2));
                const uint32_t ws[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int w = wb + q4 + u;
                    if ((w & 7) == 0) P.super[S.super_off + row * g.W8 + (w >> 3)] = rank;
                    uint32_t m = ws[u];
                    while (m) {
                        const int bb = __ffs(m) - 1;
                        m &= m - 1;
                        if (P.list_cap <= 0 || (long long)rank < P.list_cap) {
                            P.list[rank] = pack_cell(32 * w + bb, j, k);
                            if (!ONE && P.cell_slot) P.cell_slot[rank] = (uint32_t)my_slot;
                        }
                        ++rank;
                    }
                }
            }
        }
        live &= ~__ballot_sync(0xffffffffu, light);
        while (live) {
            const int b = __ffs(live) - 1;
            live &= live - 1;
            const long long s = s0 + b;
            const uint32_t seg_first = __shfl_sync(0xffffffffu, my_start, b);
            const int sslot = __shfl_sync(0xffffffffu, my_slot, b);   // converged: before the per-lane loop
            const GridSlot& S = slot_ref<ONE>(P.B, sslot);
            const GridDesc& g = S.g;
            const long long ls = s - S.seg_off;            // segment within its grid
            const long long row = ls / S.nxt;
            const int xt = (int)(ls - row * S.nxt);
            const int w = xt * S.tw + lane;
            const bool word_lane = lane < S.tw;
            const uint32_t act = (word_lane && w < g.W) ? P.bits[S.bits_off + row * g.W + w] : 0u;
            const uint32_t c = __popc(act);
            uint32_t incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            const uint32_t first = seg_first + incl - c;
            if (word_lane && w < g.W && (w & 7) == 0) P.super[S.super_off + row * g.W8 + (w >> 3)] = first;
            const int j = (int)(row % g.cy), k = (int)(row / g.cy);
            // the segment's active cells, 32 at a time: lane l takes the (base+l)-th, found by a
            // binary search over the words' inclusive counts and a popcount select in its word
            const uint32_t n = __shfl_sync(0xffffffffu, incl, 31);
            const int w0 = xt * S.tw;
            for (uint32_t base = 0; base < n; base += 32) {
                const uint32_t idx = base + lane;
                int lo = 0;                                    // first word with incl > idx
#pragma unroll
                for (int st = 16; st >= 1; st >>= 1) {
                    const uint32_t v = __shfl_sync(0xffffffffu, incl, lo + st - 1);
                    if (v <= idx) lo += st;
                }
                const uint32_t word = __shfl_sync(0xffffffffu, act, lo);
                const uint32_t before = __shfl_sync(0xffffffffu, incl - c, lo);
                if (idx >= n) continue;
                if (P.list_cap > 0 && (long long)seg_first + idx >= P.list_cap) continue;
                const uint32_t r = idx - before;               // r-th set bit of the word
                int pos = 0;
#pragma unroll
                for (int st = 16; st >= 1; st >>= 1)
                    if ((uint32_t)__popc(word & ((1u << (pos + st)) - 1u)) <= r) pos += st;
                P.list[seg_first + idx] = pack_cell(32 * (w0 + lo) + pos, j, k);
                if (!ONE && P.cell_slot) P.cell_slot[seg_first + idx] = (uint32_t)sslot;
            }
        }
    }
}

// vert_off[b] = seg_start[seg_off[b]], vert_off[n] = total: the first vertex rank of every grid.
__global__ void k_vert_offsets(BatchTable B, const uint32_t* __restrict__ seg_start,
                               const unsigned long long* __restrict__ total, unsigned long long* vert_off) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b <= B.n; b += gridDim.x * blockDim.x)
        vert_off[b] = b < B.n ? (unsigned long long)seg_start[B.seg_off[b]] : *total;
}

cudaError_t launch_vert_offsets(const BatchTable& B, const uint32_t* seg_start, const unsigned long long* total,
                                unsigned long long* vert_off, cudaStream_t s) {
    k_vert_offsets<<<(B.n + 1 + 255) / 256, 256, 0, s>>>(B, seg_start, total, vert_off);
    return cudaGetLastError();
}

template <bool ONE>
void launch_mark_tw(const MarkParams& P, int tw, cudaStream_t s) {
    if (tw == kNarrowTileWords) k_mark_zmarch<ONE, kNarrowTileWords><<<(unsigned)P.ntiles, kMarkWarps * 32, 0, s>>>(P);
    else                        k_mark_zmarch<ONE, kTileWords><<<(unsigned)P.ntiles, kMarkWarps * 32, 0, s>>>(P);
}

cudaError_t launch_mark(const MarkParams& P, int tw, cudaStream_t s) {
    if (P.ntiles <= 0) return cudaSuccess;
    if (P.B.n == 1) launch_mark_tw<true>(P, tw, s);
    else            launch_mark_tw<false>(P, tw, s);
    return cudaGetLastError();
}

cudaError_t launch_expand(const ExpandParams& P, int num_sms, cudaStream_t s) {
    const long long nseg = P.nseg;
    long long blocks = ((nseg + 31) / 32 * 32 + 255) / 256;
    const long long cap = (long long)num_sms * 32;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    if (P.B.n == 1) k_expand_ranks<true><<<(unsigned)blocks, 256, 0, s>>>(P);
    else            k_expand_ranks<false><<<(unsigned)blocks, 256, 0, s>>>(P);
    return cudaGetLastError();
}

int mark_ctas_per_sm(bool one) {
    int n = 0;
    const cudaError_t e = one ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_mark_zmarch<true, kTileWords>, kMarkWarps * 32, 0)
                              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_mark_zmarch<false, kTileWords>, kMarkWarps * 32, 0);
    if (e != cudaSuccess) { cudaGetLastError(); return 1; }
    return n > 0 ? n : 1;
}

int mark_tile_words() { return kTileWords; }
int mark_narrow_tile_words() { return kNarrowTileWords; }
int mark_max_rows() { return kMarkWarps - 1; }

}  // namespace dcb
