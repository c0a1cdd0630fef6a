// dcb_noalloc.cu — active-cell marking and compaction without any device allocation.
//
// Some callers cannot let a library call cudaMalloc: applications that hand out all device
// memory from their own fixed budget or pool, and latency-sensitive loops in which an
// allocation's implicit device synchronisation is not acceptable. For them this file
// provides dcb_mark_active_cells_noalloc: the same mark, segment-scan and rank-expansion
// kernels as the main pipeline, with every scratch buffer carved out of one file-scope
// __device__ array of fixed size. The caller passes the grid and the output buffer.
//
// The array's name is only a host-side stand-in in host code; its device address is
// looked up with cudaGetSymbolAddress on every call, with the caller's device and context
// current, and passed to the kernels. Nothing is cached between calls, so a device reset or
// another context on the same device never sees a stale address. The very first call on a
// device may load the library's device code (lazy module loading), so make it before any
// stream capture. All calls on a device share the array and it keeps the last call's
// contents, so the counter is cleared at the start of each call and two calls whose work
// overlaps on the GPU race on it.
#include <algorithm>
#include <cmath>
#include <cstring>
#include "dcb_kernels.cuh"
#include "../../include/dcb.h"

namespace dcb {

constexpr size_t kNoAllocScratchBytes = 16u << 20;   // 16 MiB, held by every device that loads the library

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

// Device address of the scratch array in the current context. Looked up on every call: the
// lookup allocates nothing, and an address kept from an earlier call could belong to a
// context that has since been reset or to another context on the same device.
cudaError_t scratch_address(void** out) {
    *out = nullptr;
    return cudaGetSymbolAddress(out, g_noalloc_scratch);
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Packed (i | j<<21 | k<<42) -> linear index i + cx*(j + cy*k), in place.
__global__ void k_packed_to_linear(uint64_t* cells, long long n, int cx, int cy) {
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        unpack_cell(cells[r], i, j, k);
        cells[r] = (uint64_t)((int64_t)i + (int64_t)cx * ((int64_t)j + (int64_t)cy * k));
    }
}

}  // namespace
}  // namespace dcb

using namespace dcb;

extern "C" int dcb_mark_active_cells_noalloc(const dcb_grid* grid, int64_t* cells, int64_t capacity,
                                             int64_t* count, void* cuda_stream) {
    if (!grid || !grid->values || !count || capacity < 0 || (capacity > 0 && !cells)) return DCB_ERR_INVALID_ARGUMENT;
    *count = 0;
    if (grid->nx < 2 || grid->ny < 2 || grid->nz < 2) return DCB_ERR_INVALID_ARGUMENT;
    if (grid->nx > 65536 || grid->ny > (1 << 21) || grid->nz > (1 << 21)) return DCB_ERR_TOO_LARGE;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) { cudaGetLastError(); return DCB_ERR_CUDA; }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(cuda_stream);

    GridDesc g;
    g.nx = grid->nx; g.ny = grid->ny; g.nz = grid->nz;
    g.cx = g.nx - 1; g.cy = g.ny - 1; g.cz = g.nz - 1;
    g.W = ((g.cx + 31) / 32 + 7) / 8 * 8;
    g.W8 = g.W / 8;
    g.vx = grid->vx; g.vy = grid->vy; g.vz = grid->vz;
    g.ox = grid->ox; g.oy = grid->oy; g.oz = grid->oz;
    g.v = grid->values;
    const long long rows = (long long)g.cy * g.cz;
    const int tile_cells = 32 * mark_tile_words();
    const int nxt = (g.cx + tile_cells - 1) / tile_cells;
    const long long nseg = rows * nxt;

    int sms = 148;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) { cudaGetLastError(); return DCB_ERR_CUDA; }
    // The grid as a batch of one. A single grid's kernels take its slot from the launch
    // parameters (BatchTable::s0) and read no device-side table, so none is stored.
    GridSlot slot;
    slot.g = g;
    slot.bits_off = 0; slot.super_off = 0; slot.seg_off = 0; slot.col_off = 0;
    slot.nxt = nxt;
    slot.tw = mark_tile_words();
    slot.hmax = std::max(std::fabs(g.vx), std::max(std::fabs(g.vy), std::fabs(g.vz)));
    slot.R = std::min(mark_max_rows(), g.cy);
    slot.nrb = (g.cy + slot.R - 1) / slot.R;
    slot.KZ = (int)std::max(8LL, std::min(64LL, ((long long)g.cz * nxt * slot.nrb + (long long)sms * 12 - 1) / ((long long)sms * 12)));
    slot.nzc = (g.cz + slot.KZ - 1) / slot.KZ;
    const long long ntiles = (long long)nxt * slot.nrb * slot.nzc;
    if (ntiles > 0x7fffffffLL) return DCB_ERR_TOO_LARGE;

    // Scratch layout, each part 256-byte aligned: total | bits | super | seg_count |
    // seg_start | scan partials. Grids that need more than the array are rejected.
    const size_t off_total = 0;
    const size_t off_bits = align256(off_total + sizeof(unsigned long long));
    const size_t off_super = align256(off_bits + sizeof(uint32_t) * (size_t)rows * g.W);
    const size_t off_count = align256(off_super + sizeof(uint32_t) * (size_t)rows * g.W8);
    const size_t off_start = align256(off_count + sizeof(uint32_t) * (size_t)nseg);
    const size_t off_part = align256(off_start + sizeof(uint32_t) * (size_t)nseg);
    const size_t need = align256(off_part + sizeof(uint32_t) * (size_t)std::max(1LL, scan_partials_len(nseg)));
    if (need > kNoAllocScratchBytes) return DCB_ERR_TOO_LARGE;

    void* base = nullptr;
    if (scratch_address(&base) != cudaSuccess) { cudaGetLastError(); return DCB_ERR_CUDA; }
    unsigned char* sb = static_cast<unsigned char*>(base);
    unsigned long long* total = reinterpret_cast<unsigned long long*>(sb + off_total);

    // The array keeps the previous call's contents: clear the counter this call reads (the
    // bits, counts and starts are all overwritten before they are read).
    if (cudaMemsetAsync(total, 0, sizeof(unsigned long long), s) != cudaSuccess) { cudaGetLastError(); return DCB_ERR_CUDA; }

    BatchTable B;
    B.s0 = slot; B.slots = nullptr; B.n = 1; B.cell_slot = nullptr; B.seg_off = nullptr; B.col_off = nullptr; B.vert_off = nullptr;
    MarkParams mp;
    mp.B = B; mp.tile_slot = nullptr; mp.tile_off = nullptr; mp.m = 1; mp.ntiles = ntiles; mp.nonfinite = nullptr;
    mp.bits = reinterpret_cast<uint32_t*>(sb + off_bits);
    mp.seg_count = reinterpret_cast<uint32_t*>(sb + off_count);
    if (launch_mark(mp, slot.tw, s) != cudaSuccess) { cudaGetLastError(); return DCB_ERR_CUDA; }
    uint32_t* seg_start = reinterpret_cast<uint32_t*>(sb + off_start);
    if (launch_scan(mp.seg_count, nseg, reinterpret_cast<uint32_t*>(sb + off_part), seg_start, total, s) != cudaSuccess) {
        cudaGetLastError();
        return DCB_ERR_CUDA;
    }
    unsigned long long n = 0;
    if (cudaMemcpyAsync(&n, total, sizeof(n), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return DCB_ERR_CUDA;
    }
    *count = (int64_t)n;
    if ((long long)n > capacity) return DCB_ERR_TOO_LARGE;   // *count tells the size needed
    if (n == 0) return DCB_OK;

    ExpandParams xp;
    xp.B = B; xp.nseg = nseg; xp.cell_slot = nullptr; xp.bits = mp.bits; xp.seg_count = mp.seg_count; xp.seg_start = seg_start;
    xp.super = reinterpret_cast<uint32_t*>(sb + off_super);
    xp.list = reinterpret_cast<uint64_t*>(cells);
    xp.list_cap = capacity;
    if (launch_expand(xp, sms, s) != cudaSuccess) { cudaGetLastError(); return DCB_ERR_CUDA; }
    long long blocks = ((long long)n + 255) / 256;
    if (blocks > (long long)sms * 16) blocks = (long long)sms * 16;
    k_packed_to_linear<<<(unsigned)blocks, 256, 0, s>>>(xp.list, (long long)n, g.cx, g.cy);
    if (cudaGetLastError() != cudaSuccess) return DCB_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) { cudaGetLastError(); return DCB_ERR_CUDA; }
    return DCB_OK;
}
