// dcb_common.cuh — types and device helpers shared by the dual-contouring kernels.
//
// Layout of the engine's device data (all 256-byte aligned):
//   grid      float32, x fastest: value(i,j,k) = v[i + nx*(j + ny*k)]
//             (include/dc_backend.h:13-21, src/cpp/dc_backend.cpp:61 of the reference)
//   bits      one bit per cell, cell rows (j,k) padded to W words (W a multiple of 8):
//             bits[(j + cy*k)*W + i/32] bit (i%32) = cell (i,j,k) active
//   super     uint32 per 256-cell super word: rank of its first cell among all active
//             cells in linear (k,j,i) order; rank(cell) = super + popcounts (cell_rank)
//   list      uint64 per active cell, ascending linear order, packed i | j<<21 | k<<42
//   V         float32 x3 per active cell, index = rank (= the reference's vertex index,
//             src/cpp/contouring.cpp:513-524)
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dcb {

struct GridDesc {
    int nx, ny, nz;        // grid points per axis
    int cx, cy, cz;        // cells per axis (n - 1)
    int W;                 // bit words per cell row (multiple of 8)
    int W8;                // super words per cell row (W / 8)
    float vx, vy, vz;      // spacing
    float ox, oy, oz;      // origin
    const float* __restrict__ v;
};

// Corner order of the reference's Cell (Cell.h:9-20): 0(000) 1(100) 2(110) 3(010)
// 4(001) 5(101) 6(111) 7(011); EDGE_PAIRS (Cell.h:26-30).
__host__ __device__ constexpr int corner_dx(int c) { return (c == 1 || c == 2 || c == 5 || c == 6) ? 1 : 0; }
__host__ __device__ constexpr int corner_dy(int c) { return (c == 2 || c == 3 || c == 6 || c == 7) ? 1 : 0; }
__host__ __device__ constexpr int corner_dz(int c) { return c >= 4 ? 1 : 0; }
__host__ __device__ constexpr int edge_a(int e) {
    return e < 4 ? e : (e < 8 ? e : e - 8);
}
__host__ __device__ constexpr int edge_b(int e) {
    return e < 4 ? (e + 1) % 4 : (e < 8 ? 4 + (e - 3) % 4 : e - 4);
}

__device__ __forceinline__ int64_t pidx(const GridDesc& g, int i, int j, int k) {
    return (int64_t)i + (int64_t)g.nx * ((int64_t)j + (int64_t)g.ny * (int64_t)k);
}

// Grid positions exactly as the reference's CPU backend forms them in float:
// grid.ox + i * grid.vx (src/cpp/dc_backend.cpp:63-65), no fused multiply-add.
__device__ __forceinline__ float pos_axis(float o, float v, int i) {
    return __fadd_rn(o, __fmul_rn((float)i, v));
}

__device__ __forceinline__ uint64_t pack_cell(int i, int j, int k) {
    return (uint64_t)(uint32_t)i | ((uint64_t)(uint32_t)j << 21) | ((uint64_t)(uint32_t)k << 42);
}
__device__ __forceinline__ void unpack_cell(uint64_t p, int& i, int& j, int& k) {
    i = (int)(p & 0x1FFFFF);
    j = (int)((p >> 21) & 0x1FFFFF);
    k = (int)(p >> 42);
}

// Rank of an ACTIVE cell among all active cells in linear order.
__device__ __forceinline__ uint32_t cell_rank(const uint32_t* __restrict__ bits,
                                              const uint32_t* __restrict__ super,
                                              const GridDesc& g, int i, int j, int k) {
    const int64_t row = (int64_t)j + (int64_t)g.cy * k;
    const int s = i >> 8;
    uint32_t r = __ldg(super + row * g.W8 + s);
    const uint4* p = reinterpret_cast<const uint4*>(bits + row * g.W + 8 * s);
    const uint4 a = __ldg(p), b = __ldg(p + 1);
    const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    const int wl = (i >> 5) & 7;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        if (q < wl) r += __popc(w[q]);
    }
    uint32_t cur = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) if (q == wl) cur = w[q];
    r += __popc(cur & ((1u << (i & 31)) - 1u));
    return r;
}

// Strict sign change (s0 * s1 < 0 evaluated in double in the reference; floats of opposite
// strict sign always give a negative double product, so no underflow can occur).
__device__ __forceinline__ bool strict_change(float a, float b) {
    return (a < 0.f && b > 0.f) || (a > 0.f && b < 0.f);
}
// Hermite crossing test: the reference skips an edge when fa * fb > 0 (Cell.cpp:185).
__device__ __forceinline__ bool hermite_crossing(float a, float b) {
    return !((a > 0.f && b > 0.f) || (a < 0.f && b < 0.f));
}

// Error flags written by kernels (first error wins).
// kErrNonFinite: a quad's edge whose Hermite sample the reference CPU backend cannot find
// again (an infinite value at the end its representative cell interpolates from gives a NaN
// sample), where that backend exits (src/cpp/contouring.cpp:590-594).
enum DeviceError : int { kErrNone = 0, kErrTimeout = 1, kErrInternal = 2, kErrOverflow = 3, kErrInvalid = 4,
                         kErrNonFinite = 5 };

__device__ __forceinline__ void set_error(int* flag, int code) { atomicCAS(flag, 0, code); }

}  // namespace dcb
