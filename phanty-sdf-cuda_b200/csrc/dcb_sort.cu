// dcb_sort.cu — device-wide sort, scan and selection of the mesh post-pass (dcb_post.cu) and the
// vertex refinement (dcb_ours.cu): a stable LSD radix sort over 8-bit digits (keys alone or
// with 32-bit values), exclusive and inclusive sums, and flagged selection. Every primitive is a
// fixed sequence of launches with no waits between blocks: a per-tile count, a scan of the
// counts, a per-tile placement. Inputs are left unmodified; the scratch space comes from the
// caller (the *_temp_bytes functions give its size).
//
// Radix sort, one pass per digit: tile t (2048 items, one block) counts its digits into
// hist[digit * tiles + t]; an exclusive scan of hist in that digit-major order gives every
// (digit, tile) its first output position; the tile then places its items, each warp ranking
// a contiguous eighth (256 items) of them in its own digit counters: an item's position is its digit's
// base, plus that digit's items in earlier warps, plus its rank in its warp. Passes alternate
// between the output and one scratch buffer, starting so that the last pass writes the output.
#include "dcb_kernels.cuh"
#include "dcb_sort.cuh"

namespace dcb {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;      // items per tile (one block)
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kWarps = kThreads / 32;

inline size_t al(size_t x) { return (x + 255) & ~size_t(255); }
inline long long tiles_of(long long n) { return (n + kTile - 1) / kTile; }

// ---- scans over uint32 / uint64 counts ----------------------------------------------------

template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T* s_warp, T& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    T base = 0;
    total = 0;
#pragma unroll
    for (int q = 0; q < kWarps; ++q) {
        const T s = s_warp[q];
        if (q < warp) base += s;
        total += s;
    }
    __syncthreads();
    return base + incl - v;
}

// thread t of tile b sums items [b*kTile + t*kItems, +kItems): consecutive items per thread
template <typename T>
__global__ void __launch_bounds__(kThreads) k_tile_sums(const T* __restrict__ in, long long n, T* __restrict__ partials) {
    __shared__ T s_warp[kWarps];
    const long long base = (long long)blockIdx.x * kTile + (long long)threadIdx.x * kItems;
    T s = 0;
#pragma unroll
    for (int q = 0; q < kItems; ++q) s += (base + q < n) ? in[base + q] : T(0);
    T total;
    block_excl_scan<T>(s, s_warp, total);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

// exclusive scan of the tile sums in one block; *grand_total = their sum
template <typename T>
__global__ void __launch_bounds__(kThreads) k_scan_tiles(T* partials, long long nb, unsigned long long* grand_total) {
    __shared__ T s_warp[kWarps];
    T carry = 0;
    for (long long c0 = 0; c0 < nb; c0 += kThreads) {
        const long long idx = c0 + threadIdx.x;
        const T v = idx < nb ? partials[idx] : T(0);
        T total;
        const T ex = block_excl_scan<T>(v, s_warp, total);
        if (idx < nb) partials[idx] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0 && grand_total) *grand_total = (unsigned long long)carry;
}

template <typename T, bool INCLUSIVE>
__global__ void __launch_bounds__(kThreads) k_scan_out(const T* __restrict__ in, long long n, const T* __restrict__ partials,
                                                       T* __restrict__ out) {
    __shared__ T s_warp[kWarps];
    const long long base = (long long)blockIdx.x * kTile + (long long)threadIdx.x * kItems;
    T v[kItems];
    T s = 0;
#pragma unroll
    for (int q = 0; q < kItems; ++q) { v[q] = (base + q < n) ? in[base + q] : T(0); s += v[q]; }
    T total;
    T run = block_excl_scan<T>(s, s_warp, total) + partials[blockIdx.x];
#pragma unroll
    for (int q = 0; q < kItems; ++q) {
        if (INCLUSIVE) run += v[q];
        if (base + q < n) out[base + q] = run;
        if (!INCLUSIVE) run += v[q];
    }
}

template <typename T, bool INCLUSIVE>
cudaError_t scan_impl(void* temp, size_t temp_bytes, const T* in, T* out, long long n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const long long nb = tiles_of(n);
    if (temp_bytes < scan_temp_bytes(n)) return cudaErrorInvalidValue;
    T* partials = reinterpret_cast<T*>(temp);
    k_tile_sums<T><<<(unsigned)nb, kThreads, 0, s>>>(in, n, partials);
    k_scan_tiles<T><<<1, kThreads, 0, s>>>(partials, nb, nullptr);
    k_scan_out<T, INCLUSIVE><<<(unsigned)nb, kThreads, 0, s>>>(in, n, partials, out);
    return cudaGetLastError();
}

}  // namespace

size_t scan_temp_bytes(long long n) { return al(sizeof(unsigned long long) * (size_t)(tiles_of(n) + 1)); }

cudaError_t exclusive_sum(void* temp, size_t temp_bytes, const uint32_t* in, uint32_t* out, long long n, cudaStream_t s) {
    return scan_impl<uint32_t, false>(temp, temp_bytes, in, out, n, s);
}
cudaError_t exclusive_sum(void* temp, size_t temp_bytes, const unsigned long long* in, unsigned long long* out, long long n,
                          cudaStream_t s) {
    return scan_impl<unsigned long long, false>(temp, temp_bytes, in, out, n, s);
}
cudaError_t inclusive_sum(void* temp, size_t temp_bytes, const uint32_t* in, uint32_t* out, long long n, cudaStream_t s) {
    return scan_impl<uint32_t, true>(temp, temp_bytes, in, out, n, s);
}

// ---- flagged selection --------------------------------------------------------------------

namespace {

__global__ void __launch_bounds__(kThreads) k_flag_sums(const uint8_t* __restrict__ flags, long long n, uint32_t* partials) {
    __shared__ uint32_t s_warp[kWarps];
    const long long base = (long long)blockIdx.x * kTile + (long long)threadIdx.x * kItems;
    uint32_t c = 0;
#pragma unroll
    for (int q = 0; q < kItems; ++q) c += (base + q < n && flags[base + q]) ? 1u : 0u;
    uint32_t total;
    block_excl_scan<uint32_t>(c, s_warp, total);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

// the flagged items of a tile in order, from the tile's first output position; INDEX: the
// item is its own index
template <bool INDEX>
__global__ void __launch_bounds__(kThreads) k_select_out(const int4* __restrict__ in, const uint8_t* __restrict__ flags,
                                                         long long n, const uint32_t* __restrict__ partials,
                                                         int4* __restrict__ out4, int* __restrict__ outi) {
    __shared__ uint32_t s_warp[kWarps];
    const long long base = (long long)blockIdx.x * kTile + (long long)threadIdx.x * kItems;
    bool f[kItems];
    uint32_t c = 0;
#pragma unroll
    for (int q = 0; q < kItems; ++q) { f[q] = base + q < n && flags[base + q]; c += f[q] ? 1u : 0u; }
    uint32_t total;
    uint32_t pos = block_excl_scan<uint32_t>(c, s_warp, total) + partials[blockIdx.x];
#pragma unroll
    for (int q = 0; q < kItems; ++q) {
        if (!f[q]) continue;
        if (INDEX) outi[pos] = (int)(base + q);
        else       out4[pos] = in[base + q];
        ++pos;
    }
}

template <bool INDEX>
cudaError_t select_impl(void* temp, size_t temp_bytes, const int4* in, const uint8_t* flags, int4* out4, int* outi,
                        unsigned long long* count, long long n, cudaStream_t s) {
    if (n <= 0) return cudaMemsetAsync(count, 0, sizeof(unsigned long long), s);
    if (temp_bytes < select_temp_bytes(n)) return cudaErrorInvalidValue;
    const long long nb = tiles_of(n);
    uint32_t* partials = reinterpret_cast<uint32_t*>(temp);
    k_flag_sums<<<(unsigned)nb, kThreads, 0, s>>>(flags, n, partials);
    k_scan_tiles<uint32_t><<<1, kThreads, 0, s>>>(partials, nb, count);
    k_select_out<INDEX><<<(unsigned)nb, kThreads, 0, s>>>(in, flags, n, partials, out4, outi);
    return cudaGetLastError();
}

}  // namespace

size_t select_temp_bytes(long long n) { return al(sizeof(uint32_t) * (size_t)(tiles_of(n) + 1)); }

cudaError_t select_flagged(void* temp, size_t temp_bytes, const int4* in, const uint8_t* flags, int4* out,
                           unsigned long long* count, long long n, cudaStream_t s) {
    return select_impl<false>(temp, temp_bytes, in, flags, out, nullptr, count, n, s);
}
cudaError_t select_flagged_index(void* temp, size_t temp_bytes, const uint8_t* flags, int* out, unsigned long long* count,
                                 long long n, cudaStream_t s) {
    return select_impl<true>(temp, temp_bytes, nullptr, flags, nullptr, out, count, n, s);
}


// ---- LSD radix sort ---------------------------------------------------------------------

namespace {

template <typename K>
__global__ void __launch_bounds__(kThreads) k_radix_hist(const K* __restrict__ keys, long long n, int shift, uint32_t mask,
                                                         uint32_t* __restrict__ hist, long long ntiles) {
    __shared__ uint32_t s_cnt[kRadix];
    for (int d = threadIdx.x; d < kRadix; d += kThreads) s_cnt[d] = 0;
    __syncthreads();
    const long long base = (long long)blockIdx.x * kTile;
#pragma unroll
    for (int q = 0; q < kItems; ++q) {
        const long long i = base + q * kThreads + threadIdx.x;
        if (i < n) atomicAdd(&s_cnt[(uint32_t)(keys[i] >> shift) & mask], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += kThreads) hist[(long long)d * ntiles + blockIdx.x] = s_cnt[d];
}

// Warp w of the tile takes items [w*256, (w+1)*256) of it, lane l of round q the item
// w*256 + 32q + l: item order is (warp, round, lane). Each warp ranks its items in its own
// digit counters (__match_any_sync groups the lanes with the same digit; the lowest of them
// advances the counter after the others have read it), then one pass over the digits turns
// the per-warp counts into each warp's first position per digit.
template <typename K, bool PAIRS>
__global__ void __launch_bounds__(kThreads)
k_radix_scatter(const K* __restrict__ kin, const uint32_t* __restrict__ vin, K* __restrict__ kout, uint32_t* __restrict__ vout,
                long long n, int shift, uint32_t mask, const uint32_t* __restrict__ offs, long long ntiles) {
    __shared__ uint32_t s_cnt[kWarps][kRadix];     // per warp: its items of each digit, then its first position
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int x = tid; x < kWarps * kRadix; x += kThreads) s_cnt[x / kRadix][x % kRadix] = 0u;
    __syncthreads();
    const long long base = (long long)blockIdx.x * kTile + (long long)warp * (kItems * 32);
    K key[kItems];
    uint32_t val[kItems], dig[kItems], rank[kItems];
#pragma unroll
    for (int q = 0; q < kItems; ++q) {
        const long long i = base + q * 32 + lane;
        const bool have = i < n;
        key[q] = have ? kin[i] : K(0);
        if (PAIRS) val[q] = have ? vin[i] : 0u;
        const uint32_t d = have ? ((uint32_t)(key[q] >> shift) & mask) : 0xffffffffu;
        dig[q] = d;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t below = __popc(peers & ((1u << lane) - 1u));
        rank[q] = have ? s_cnt[warp][d] + below : 0u;
        __syncwarp();
        if (have && below == 0) s_cnt[warp][d] += (uint32_t)__popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // digit d: the tile's first position from the global scan, then the warps in order
    for (int d = tid; d < kRadix; d += kThreads) {
        uint32_t run = offs[(long long)d * ntiles + blockIdx.x];
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t c = s_cnt[w][d];
            s_cnt[w][d] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kItems; ++q) {
        if (dig[q] == 0xffffffffu) continue;
        const uint32_t pos = s_cnt[warp][dig[q]] + rank[q];
        kout[pos] = key[q];
        if (PAIRS) vout[pos] = val[q];
    }
}

template <typename K, bool PAIRS>
cudaError_t sort_impl(void* temp, size_t temp_bytes, const K* kin, K* kout, const uint32_t* vin, uint32_t* vout, long long n,
                      int begin_bit, int end_bit, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    if (begin_bit < 0 || end_bit > (int)(8 * sizeof(K)) || begin_bit > end_bit) return cudaErrorInvalidValue;
    if (temp_bytes < radix_sort_temp_bytes(n, (int)sizeof(K), PAIRS)) return cudaErrorInvalidValue;
    const long long ntiles = tiles_of(n), nh = (long long)kRadix * ntiles;
    char* t = reinterpret_cast<char*>(temp);
    K* kalt = reinterpret_cast<K*>(t);
    t += al(sizeof(K) * (size_t)n);
    uint32_t* valt = nullptr;
    if (PAIRS) { valt = reinterpret_cast<uint32_t*>(t); t += al(sizeof(uint32_t) * (size_t)n); }
    uint32_t* hist = reinterpret_cast<uint32_t*>(t);
    t += al(sizeof(uint32_t) * (size_t)nh);
    uint32_t* offs = reinterpret_cast<uint32_t*>(t);
    t += al(sizeof(uint32_t) * (size_t)nh);
    void* scan_temp = t;
    const int npass = (end_bit - begin_bit + kRadixBits - 1) / kRadixBits;
    if (npass == 0) {
        cudaError_t e = cudaMemcpyAsync(kout, kin, sizeof(K) * (size_t)n, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess && PAIRS) e = cudaMemcpyAsync(vout, vin, sizeof(uint32_t) * (size_t)n, cudaMemcpyDeviceToDevice, s);
        return e;
    }
    // the last pass writes the output: an odd count starts there, an even one in the scratch
    const K* sk = kin;
    const uint32_t* sv = vin;
    K* dk = (npass & 1) ? kout : kalt;
    uint32_t* dv = (npass & 1) ? vout : valt;
    for (int p = 0; p < npass; ++p) {
        const int shift = begin_bit + p * kRadixBits;
        const int nbits = end_bit - shift < kRadixBits ? end_bit - shift : kRadixBits;
        const uint32_t mask = (1u << nbits) - 1u;
        k_radix_hist<K><<<(unsigned)ntiles, kThreads, 0, s>>>(sk, n, shift, mask, hist, ntiles);
        cudaError_t e = exclusive_sum(scan_temp, scan_temp_bytes(nh), hist, offs, nh, s);
        if (e != cudaSuccess) return e;
        k_radix_scatter<K, PAIRS><<<(unsigned)ntiles, kThreads, 0, s>>>(sk, sv, dk, dv, n, shift, mask, offs, ntiles);
        sk = dk;
        sv = dv;
        dk = (dk == kout) ? kalt : kout;
        dv = (dv == vout) ? valt : vout;
    }
    return cudaGetLastError();
}

}  // namespace

size_t radix_sort_temp_bytes(long long n, int key_bytes, bool pairs) {
    if (n < 1) n = 1;
    const long long nh = (long long)kRadix * tiles_of(n);
    return al((size_t)key_bytes * (size_t)n) + (pairs ? al(sizeof(uint32_t) * (size_t)n) : 0) +
           2 * al(sizeof(uint32_t) * (size_t)nh) + scan_temp_bytes(nh);
}

cudaError_t radix_sort_pairs(void* temp, size_t temp_bytes, const unsigned long long* kin, unsigned long long* kout,
                             const uint32_t* vin, uint32_t* vout, long long n, int begin_bit, int end_bit, cudaStream_t s) {
    return sort_impl<unsigned long long, true>(temp, temp_bytes, kin, kout, vin, vout, n, begin_bit, end_bit, s);
}
cudaError_t radix_sort_pairs(void* temp, size_t temp_bytes, const uint32_t* kin, uint32_t* kout, const uint32_t* vin,
                             uint32_t* vout, long long n, int begin_bit, int end_bit, cudaStream_t s) {
    return sort_impl<uint32_t, true>(temp, temp_bytes, kin, kout, vin, vout, n, begin_bit, end_bit, s);
}
cudaError_t radix_sort_keys(void* temp, size_t temp_bytes, const unsigned long long* kin, unsigned long long* kout,
                            long long n, int begin_bit, int end_bit, cudaStream_t s) {
    return sort_impl<unsigned long long, false>(temp, temp_bytes, kin, kout, nullptr, nullptr, n, begin_bit, end_bit, s);
}
}  // namespace dcb
