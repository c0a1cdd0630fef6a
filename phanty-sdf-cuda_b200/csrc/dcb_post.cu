// dcb_post.cu — the mesh post-pass on the GPU: vertex weld, floater removal and hole closing of
// a quad mesh. The semantics are the reference's postprocess_mesh and merge_vertices_in_place
// (src/cpp/dc_backend.cpp:127-558): the same vertices, faces and order, bit for bit.
//
// Stages, on one stream, with a few host reads of counts between them (sizes of what follows):
//   weld     bounding box by ordered-integer atomics; the quantisation step in the reference's
//            float expression order (one thread); a 51-bit grid-point key per vertex (17 bits per
//            axis relative to the box's low corner: the box spans at most ~1e5 steps); a stable
//            radix sort; the first vertex of each key represents it; representatives numbered by
//            a scan in index order; faces remapped, those with < 3 distinct indices dropped with
//            the order kept (dc_backend.cpp:127-215).
//   edges    the 4 edge uses of every face keyed by (min, max) vertex and radix sorted; a run of
//            one use is a boundary edge, a run of two joins its faces in a union-find whose roots
//            are the smallest face index (dc_backend.cpp:231-310).
//   keep     the component with the most faces, the one with the smallest first face on ties
//            (the reference numbers components by their first face: dc_backend.cpp:312-361).
//   holes    boundary edges of the kept faces sorted by (from, to), so each vertex's outgoing
//            edges are in the order the reference pushes them and are taken from the back. Walks
//            (dc_backend.cpp:468-503) are sequential inside a weakly connected component of the
//            boundary graph — one thread each, start vertices in ascending order — and
//            independent across components; the loops they close are put in the reference's
//            global order by (start vertex, sequence). Filling (dc_backend.cpp:376-466): a block
//            per loop, ring by ring, the running sums in the reference's order by one thread per
//            coordinate and the rest in parallel; run once for sizes and once to write.
//   renumber vertices by first use in the face list (dc_backend.cpp:537-550): atomicMin of the
//            first position of every vertex, a scan over first uses.
//   weld     again on the result when holes are closed (dc_backend.cpp:552-554).
//
// Compiled with --fmad=false: every float expression is rounded as written, like the
// reference's x86-64 build.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include "dcb_kernels.cuh"
#include "dcb_sort.cuh"

namespace dcb {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxLoop = 4096;          // loops longer than this are not filled (dc_backend.cpp:487, 497)
constexpr int kMaxRings = 8192;         // a fill that has not converged by then is reported
constexpr int kFillThreads = 256;
constexpr int kKeyBits = 17;            // per axis in the weld key
constexpr int kRankRounds = 32;         // pointer-jumping rounds: enough for cycles of 2^31 vertices

// Device-side findings (PostRun::err): a face index out of range, a non-finite vertex, a weld
// key beyond 17 bits, a bounded loop that gave up (union retries, walk steps), a hole fill that
// had not converged after kMaxRings rings.
enum PostErr { kPostBadIndex = 1, kPostNonFinite = 2, kPostWeldSpan = 4, kPostLoopGuard = 8, kPostRingGuard = 16 };

struct PostCounters {
    unsigned int box[6];                // ordered bits: min x, y, z; max x, y, z
    int err;
    int pad;
    float inv;                          // 1 / weld step
    int pad2;
    long long qlo[3];                   // grid point of the box's low corner
    unsigned long long nvw;             // welded vertices (groups)
    unsigned long long nsel;            // selection counts (faces kept by the weld, by the component)
    unsigned long long nb;              // boundary uses
    unsigned long long ncomp;           // face components
    unsigned long long best;            // size << 32 | ~root of the largest component
    unsigned long long nbk;             // boundary edges of kept faces
    unsigned long long nstarts;         // vertices with outgoing boundary edges
    unsigned long long loops_found;
    unsigned long long nloops;          // loops of 3..4096 vertices
    unsigned long long fill_v, fill_f;
    unsigned long long nout;            // vertices after renumbering
    unsigned long long cursor;          // ring vertices reserved in the fill scratch
    unsigned long long nrings;          // ring records written
    int fill_overflow;                  // the scratch or the record list was too small
    int pad3;
};

inline unsigned grid_for(long long n, int threads, int num_sms) {
    const long long blocks = (n + threads - 1) / threads;
    return (unsigned)std::max(1LL, std::min(blocks, (long long)num_sms * 16));
}

__device__ __forceinline__ unsigned int ordered(float x) {
    const unsigned int b = __float_as_uint(x);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float unordered(unsigned int o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}

// ---- union-find with roots = smallest member; finds halve the path as they go (the
// intermediate pointer jumping of Jaiganesh & Burtscher, "A high-performance connected
// components implementation for GPUs", HPDC 2018). Parents only ever point to smaller indices.
__device__ __forceinline__ int uf_find(int* parent, int x) {
    volatile int* p = parent;
    int cur = p[x];
    if (cur != x) {
        int prev = x, next;
        while (cur > (next = p[cur])) {
            p[prev] = next;
            prev = cur;
            cur = next;
        }
    }
    return cur;
}

__device__ void uf_unite(int* parent, int a, int b, int* err) {
    int ra = a, rb = b;
    for (int guard = 0;; ++guard) {
        if (guard > (1 << 24)) { atomicOr(err, kPostLoopGuard); return; }
        ra = uf_find(parent, ra);
        rb = uf_find(parent, rb);
        if (ra == rb) return;
        if (ra < rb) { const int t = ra; ra = rb; rb = t; }
        if (atomicCAS(&parent[ra], ra, rb) == ra) return;
        // ra was linked meanwhile: both roots are found again from where they are
    }
}

__global__ void k_iota(int* a, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        a[i] = (int)i;
}

// After all unions: every parent becomes its root. The walk up only reads (a path-halving
// write here could replace a root that another thread just stored with an intermediate
// ancestor); the only writes are roots.
__global__ void k_flatten(int* parent, long long n) {
    volatile int* p = parent;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int x = (int)i, up;
        while ((up = p[x]) != x) x = up;   // indices strictly decrease towards the root
        p[i] = x;
    }
}

// ---------------------------------------------------------------- weld
__global__ void k_post_reset(PostCounters* C) {
    if (threadIdx.x == 0) {
        for (int a = 0; a < 3; ++a) { C->box[a] = 0xffffffffu; C->box[3 + a] = 0u; }
        C->nvw = 0; C->nsel = 0;
    }
}

__global__ void k_bbox(const float* __restrict__ V, long long nv, PostCounters* C) {
    unsigned int lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, hi[3] = {0u, 0u, 0u};
    bool bad = false;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv; i += (long long)gridDim.x * blockDim.x)
        for (int a = 0; a < 3; ++a) {
            const float x = V[3 * i + a];
            bad |= !isfinite(x);
            const unsigned int o = ordered(x);
            lo[a] = min(lo[a], o);
            hi[a] = max(hi[a], o);
        }
    for (int a = 0; a < 3; ++a)
        for (int d = 16; d > 0; d >>= 1) {
            lo[a] = min(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], d));
            hi[a] = max(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], d));
        }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&C->err, kPostNonFinite);
    __shared__ unsigned int s_box[6];
    if (threadIdx.x < 6) s_box[threadIdx.x] = threadIdx.x < 3 ? 0xffffffffu : 0u;
    __syncthreads();
    if ((threadIdx.x & 31) == 0)
        for (int a = 0; a < 3; ++a) { atomicMin(&s_box[a], lo[a]); atomicMax(&s_box[3 + a], hi[a]); }
    __syncthreads();
    if (threadIdx.x < 3) atomicMin(&C->box[threadIdx.x], s_box[threadIdx.x]);
    else if (threadIdx.x < 6) atomicMax(&C->box[threadIdx.x], s_box[threadIdx.x]);
}

// The weld step: eps = |box diagonal| * 1e-5 (1e-5 for a point), in the reference's order.
__global__ void k_weld_params(PostCounters* C) {
    if (threadIdx.x != 0) return;
    float lo[3], hi[3];
    for (int a = 0; a < 3; ++a) { lo[a] = unordered(C->box[a]); hi[a] = unordered(C->box[3 + a]); }
    const float ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
    const float diag = sqrtf(ex * ex + ey * ey + ez * ez);
    const float eps = diag > 0.0f ? diag * 1e-5f : 1e-5f;
    const float inv = 1.0f / eps;
    C->inv = inv;
    for (int a = 0; a < 3; ++a) C->qlo[a] = (long long)roundf(lo[a] * inv);
}

__global__ void k_weld_keys(const float* __restrict__ V, long long nv, PostCounters* C,
                            unsigned long long* key, int* idx) {
    const float inv = C->inv;
    const long long q0 = C->qlo[0], q1 = C->qlo[1], q2 = C->qlo[2];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv; i += (long long)gridDim.x * blockDim.x) {
        const long long d0 = (long long)roundf(V[3 * i] * inv) - q0;
        const long long d1 = (long long)roundf(V[3 * i + 1] * inv) - q1;
        const long long d2 = (long long)roundf(V[3 * i + 2] * inv) - q2;
        const long long lim = 1LL << kKeyBits;
        if (d0 < 0 || d0 >= lim || d1 < 0 || d1 >= lim || d2 < 0 || d2 >= lim) atomicOr(&C->err, kPostWeldSpan);
        key[i] = ((unsigned long long)(d0 & (lim - 1))) | ((unsigned long long)(d1 & (lim - 1)) << kKeyBits) |
                 ((unsigned long long)(d2 & (lim - 1)) << (2 * kKeyBits));
        idx[i] = (int)i;
    }
}

// head[p]: sorted position p starts a key; rep[i]: vertex i is the first of its key.
__global__ void k_weld_heads(const unsigned long long* __restrict__ skey, const int* __restrict__ sidx, long long n,
                             unsigned int* head, unsigned int* rep) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const unsigned int h = (p == 0 || skey[p] != skey[p - 1]) ? 1u : 0u;
        head[p] = h;
        rep[sidx[p]] = h;
    }
}

// group g (1-based inclusive scan of heads) -> new index of its representative; welded vertices.
__global__ void k_weld_groups(const int* __restrict__ sidx, const unsigned int* __restrict__ head,
                              const unsigned int* __restrict__ gid, const unsigned int* __restrict__ newid,
                              const float* __restrict__ V, long long n, unsigned int* grp, float* Vw, PostCounters* C) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        if (p == n - 1) C->nvw = gid[p];
        if (!head[p]) continue;
        const int i = sidx[p];
        const unsigned int nid = newid[i];
        grp[gid[p] - 1] = nid;
        Vw[3 * (long long)nid] = V[3 * (long long)i];
        Vw[3 * (long long)nid + 1] = V[3 * (long long)i + 1];
        Vw[3 * (long long)nid + 2] = V[3 * (long long)i + 2];
    }
}

__global__ void k_weld_remap(const int* __restrict__ sidx, const unsigned int* __restrict__ gid,
                             const unsigned int* __restrict__ grp, long long n, int* remap) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        remap[sidx[p]] = (int)grp[gid[p] - 1];
}

__global__ void k_weld_faces(const int32_t* __restrict__ F, long long nf, long long nv, const int* __restrict__ remap,
                             int4* Ft, unsigned char* keep, PostCounters* C) {
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nf; f += (long long)gridDim.x * blockDim.x) {
        int c[4];
        bool ok = true;
        for (int k = 0; k < 4; ++k) {
            const int32_t v = F[4 * f + k];
            ok = ok && v >= 0 && v < nv;
            c[k] = v;
        }
        if (!ok) { atomicOr(&C->err, kPostBadIndex); keep[f] = 0; continue; }
        int distinct = 0;
        for (int k = 0; k < 4; ++k) {
            c[k] = remap[c[k]];
            bool seen = false;
            for (int j = 0; j < k; ++j) seen = seen || c[j] == c[k];
            distinct += !seen;
        }
        Ft[f] = make_int4(c[0], c[1], c[2], c[3]);
        keep[f] = distinct >= 3 ? 1 : 0;
    }
}

// ---------------------------------------------------------------- edges and components
__device__ __forceinline__ int corner(const int4& q, int e) {
    return e == 0 ? q.x : e == 1 ? q.y : e == 2 ? q.z : q.w;
}

__global__ void k_edge_uses(const int4* __restrict__ Fw, long long nf, int b, unsigned long long* key, int* val) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 4 * nf; t += (long long)gridDim.x * blockDim.x) {
        const long long f = t >> 2;
        const int e = (int)(t & 3);
        const int4 q = Fw[f];
        const int u = corner(q, e), v = corner(q, (e + 1) & 3);
        key[t] = u == v ? ~0ull : ((unsigned long long)min(u, v) << b) | (unsigned long long)max(u, v);
        val[t] = (int)t;
    }
}

struct EdgeRunParams {
    const unsigned long long* key;
    const int* val;
    long long n;
    unsigned long long invalid;         // the sentinel within the sorted bits
    const int4* Fw;
    int close, remove;
    int* parent;
    int4* bnd;                          // (from, to, face, 0)
    PostCounters* C;
};

__device__ __forceinline__ void push_boundary(const EdgeRunParams& P, int use) {
    const int f = use >> 2, e = use & 3;
    const int4 q = P.Fw[f];
    const unsigned long long at = atomicAdd(&P.C->nb, 1ull);
    P.bnd[at] = make_int4(corner(q, e), corner(q, (e + 1) & 3), f, 0);
}

__global__ void k_edge_runs(EdgeRunParams P) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P.n; p += (long long)gridDim.x * blockDim.x) {
        const unsigned long long k = P.key[p];
        if ((k & P.invalid) == P.invalid) continue;
        if (p > 0 && P.key[p - 1] == k) continue;
        long long q = p + 1;
        while (q < P.n && P.key[q] == k) ++q;
        const long long c = q - p;
        if (c == 1) {
            push_boundary(P, P.val[p]);
        } else if (c == 2) {
            if (P.remove) uf_unite(P.parent, P.val[p] >> 2, P.val[p + 1] >> 2, &P.C->err);
        } else if (P.close && P.remove) {
            for (long long x = p; x < q; ++x) push_boundary(P, P.val[x]);
        }
    }
}

// Faces per root. Components are large: each thread counts runs of one root and adds a run
// when the root changes; the last runs are added once per distinct root in the warp.
// Before the unions: every face of a two-use edge points at the smaller face of the pair (the
// smallest such neighbour wins). Each link is an edge of the face graph and points to a smaller
// index, so this is already a valid union-find forest, and most of it is flat.
__global__ void k_first_links(EdgeRunParams P) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P.n; p += (long long)gridDim.x * blockDim.x) {
        const unsigned long long k = P.key[p];
        if ((k & P.invalid) == P.invalid || (p > 0 && P.key[p - 1] == k)) continue;
        if (p + 1 >= P.n || P.key[p + 1] != k || (p + 2 < P.n && P.key[p + 2] == k)) continue;
        const int a = P.val[p] >> 2, b = P.val[p + 1] >> 2;
        if (a != b) atomicMin(&P.parent[max(a, b)], min(a, b));
    }
}

__global__ void k_comp_size(const int* __restrict__ root, long long n, unsigned int* size) {
    int cur = -1;
    unsigned int run = 0;
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < n; f += (long long)gridDim.x * blockDim.x) {
        const int r = root[f];
        if (r != cur) {
            if (run) atomicAdd(&size[cur], run);
            cur = r;
            run = 0;
        }
        ++run;
    }
    const unsigned int peers = __match_any_sync(0xffffffffu, cur);
    const unsigned int total = __reduce_add_sync(peers, run);
    if (run && cur >= 0 && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&size[cur], total);
}

__global__ void k_comp_pick(const int* __restrict__ root, const unsigned int* __restrict__ size, long long n, PostCounters* C) {
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < n; f += (long long)gridDim.x * blockDim.x) {
        if (root[f] != f) continue;
        atomicAdd(&C->ncomp, 1ull);
        atomicMax(&C->best, ((unsigned long long)size[f] << 32) | (0xffffffffull - (unsigned long long)f));
    }
}

__global__ void k_keep_flags(const int* __restrict__ root, long long n, const PostCounters* C, unsigned char* keep) {
    const int L = (int)(0xffffffffull - (C->best & 0xffffffffull));
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < n; f += (long long)gridDim.x * blockDim.x)
        keep[f] = root[f] == L ? 1 : 0;
}

// ---------------------------------------------------------------- holes
__global__ void k_bnd_keys(const int4* __restrict__ bnd, long long nb, const int* __restrict__ root, int remove, int b,
                           unsigned long long* key, unsigned int* deg, PostCounters* C) {
    const int L = remove ? (int)(0xffffffffull - (C->best & 0xffffffffull)) : 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nb; t += (long long)gridDim.x * blockDim.x) {
        const int4 e = bnd[t];
        if (remove && root[e.z] != L) { key[t] = ~0ull; continue; }
        key[t] = ((unsigned long long)e.x << b) | (unsigned long long)e.y;
        atomicAdd(&deg[e.x], 1u);
        atomicAdd(&C->nbk, 1ull);
    }
}

__global__ void k_bnd_unite(const unsigned long long* __restrict__ key, long long n, int b, int* parent, PostCounters* C) {
    const unsigned long long m = (1ull << b) - 1;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        uf_unite(parent, (int)(key[t] >> b), (int)(key[t] & m), &C->err);
}

// ---- boundary components that are simple cycles (every vertex one edge out, one in): the
// reference's walk from the component's smallest vertex s just follows the cycle back to s, so
// the loop is the cycle from s. Each vertex's place on it comes from list ranking (pointer
// jumping on (distance, next) pairs), in parallel, instead of a sequential walk.
__global__ void k_cycle_indeg(const unsigned long long* __restrict__ key, long long n, int b,
                              const unsigned int* __restrict__ deg, const int* __restrict__ root, unsigned int* indeg,
                              unsigned int* bad) {
    const unsigned long long m = (1ull << b) - 1;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const unsigned int v = (unsigned int)(key[t] & m);
        atomicAdd(&indeg[v], 1u);
        if (!deg[v]) atomicOr(&bad[root[v]], 1u);    // a sink: the walk ends there
    }
}

// Over the vertices with outgoing edges (the sorted starts): bad[root] when one lacks exactly
// one edge in and one out (sinks were marked with the in-degrees); len[root]: vertex count.
__global__ void k_cycle_marks(const unsigned long long* __restrict__ skey, long long ns, int b,
                              const unsigned int* __restrict__ deg, const unsigned int* __restrict__ indeg,
                              const int* __restrict__ root, unsigned int* bad, unsigned int* len) {
    const unsigned long long m = (1ull << b) - 1;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < ns; p += (long long)gridDim.x * blockDim.x) {
        const unsigned int u = (unsigned int)(skey[p] & m);
        if (deg[u] != 1 || indeg[u] != 1) atomicOr(&bad[root[u]], 1u);
        atomicAdd(&len[root[u]], 1u);
    }
}

// (distance to the cycle's last vertex before s, next vertex or -1) packed as dist << 32 | next.
__global__ void k_cycle_rank_init(const unsigned long long* __restrict__ skey, long long ns, int b,
                                  const unsigned int* __restrict__ bad, const int* __restrict__ root,
                                  const int* __restrict__ succ, unsigned long long* rank) {
    const unsigned long long m = (1ull << b) - 1;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < ns; p += (long long)gridDim.x * blockDim.x) {
        const unsigned int u = (unsigned int)(skey[p] & m);
        if (bad[root[u]]) continue;
        const int nx = succ[u];
        rank[u] = nx == root[u] ? 0xffffffffull : ((1ull << 32) | (unsigned int)nx);
    }
}

// One round of pointer jumping in place; a pair is read and written as one 64-bit word, so
// (distance, next) always stays consistent. changed[r] records whether round r moved
// anything; a round after one that moved nothing returns at once.
__global__ void k_cycle_rank_jump(const unsigned long long* __restrict__ skey, long long ns, int b,
                                  const unsigned int* __restrict__ bad, const int* __restrict__ root,
                                  unsigned long long* rank, int* changed, int r) {
    if (r > 0 && !changed[r - 1]) return;
    const unsigned long long m = (1ull << b) - 1;
    volatile unsigned long long* R = rank;
    bool moved = false;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < ns; p += (long long)gridDim.x * blockDim.x) {
        const unsigned int u = (unsigned int)(skey[p] & m);
        if (bad[root[u]]) continue;
        const unsigned long long me = R[u];
        const unsigned int nx = (unsigned int)me;
        if (nx == 0xffffffffu) continue;
        const unsigned long long there = R[nx];
        R[u] = (((me >> 32) + (there >> 32)) << 32) | (there & 0xffffffffull);
        moved = true;
    }
    if (__any_sync(0xffffffffu, moved) && (threadIdx.x & 31) == 0) changed[r] = 1;
}

// The loop region of every component: base[root] = its first entry (the starts' scan).
__global__ void k_cycle_bases(const unsigned long long* __restrict__ skey, const unsigned int* __restrict__ shead,
                              const unsigned long long* __restrict__ soff, long long n, int b, unsigned long long* base) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        if (shead[p]) base[skey[p] >> b] = soff[p];
}

// Every cycle vertex writes itself into the reversed loop; s records the loop.
__global__ void k_cycle_emit(const unsigned long long* __restrict__ skey, long long ns, int b,
                             const unsigned int* __restrict__ bad, const int* __restrict__ root,
                             const unsigned int* __restrict__ len, const unsigned long long* __restrict__ rank,
                             const unsigned long long* __restrict__ base, int* lverts, unsigned char* lflag,
                             unsigned long long* lkey, int* llen, PostCounters* C) {
    const unsigned long long m = (1ull << b) - 1;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < ns; p += (long long)gridDim.x * blockDim.x) {
        const unsigned int u = (unsigned int)(skey[p] & m);
        const int s = root[u];
        if (bad[s]) continue;
        const unsigned int L = len[s];
        const bool keep = L >= 3 && L <= (unsigned int)kMaxLoop;
        const unsigned long long o = base[s];
        if (keep) lverts[o + (rank[u] >> 32)] = (int)u;
        if ((int)u == s) {
            atomicAdd(&C->loops_found, 1ull);
            if (keep) {
                lflag[o] = 1;
                lkey[o] = (unsigned long long)s << 32;
                llen[o] = (int)L;
                atomicAdd(&C->nloops, 1ull);
            }
        }
    }
}

__global__ void k_start_keys(const unsigned int* __restrict__ deg, const int* __restrict__ root, long long nv, int b,
                             unsigned long long* key, PostCounters* C) {
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < nv; u += (long long)gridDim.x * blockDim.x) {
        if (!deg[u]) continue;
        key[atomicAdd(&C->nstarts, 1ull)] = ((unsigned long long)root[u] << b) | (unsigned long long)u;
    }
}

// Per sorted start: its out-degree (for the region offsets) and whether it opens a component.
__global__ void k_start_info(const unsigned long long* __restrict__ skey, long long n, int b,
                             const unsigned int* __restrict__ deg, unsigned long long* sdeg, unsigned int* shead) {
    const unsigned long long m = (1ull << b) - 1;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        sdeg[p] = deg[skey[p] & m];
        shead[p] = (p == 0 || (skey[p] >> b) != (skey[p - 1] >> b)) ? 1u : 0u;
    }
}

struct WalkParams {
    const unsigned long long* skey;     // sorted starts: root << b | vertex
    long long nstarts;
    const unsigned int* shead;
    const unsigned long long* soff;     // exclusive scan of the starts' out-degrees
    const unsigned int* sgid;           // inclusive scan of shead
    int b;
    const unsigned long long* adj;      // sorted boundary keys: from << b | to
    const unsigned int* bot;            // first adjacency entry of every vertex
    unsigned int* top;                  // one past its last unused entry
    const int* succ;                    // the target of a vertex's only edge, else -1
    const unsigned int* cbad;           // per root: the component is not a simple cycle
    int* pos;                           // position on the current path, -1 when off it
    int* stack;                         // per component: out-degree sum + 1 entries
    int* lverts;                        // per component: out-degree sum entries
    unsigned char* lflag;               // a recorded loop starts here
    unsigned long long* lkey;           // its order: start vertex << 32 | sequence
    int* llen;
    PostCounters* C;
};

// One thread per boundary component: the reference's walks (dc_backend.cpp:468-503) over the
// component's start vertices in ascending order. Every step consumes one edge, so a walk ends
// after at most the component's edge count steps.
__global__ void k_walk(WalkParams P) {
    for (long long p0 = blockIdx.x * (long long)blockDim.x + threadIdx.x; p0 < P.nstarts;
         p0 += (long long)gridDim.x * blockDim.x) {
        if (!P.shead[p0]) continue;
        const unsigned long long m = (1ull << P.b) - 1;
        const unsigned long long root = P.skey[p0] >> P.b;
        if (!P.cbad[root]) continue;   // a simple cycle: placed by the ranking kernels
        long long p1 = p0 + 1;
        while (p1 < P.nstarts && (P.skey[p1] >> P.b) == root) ++p1;
        const unsigned long long base = P.soff[p0];
        int* stk = P.stack + base + (P.sgid[p0] - 1);
        long long w = 0;               // written loop vertices
        unsigned long long found = 0, recorded = 0;
        long long guard = 0;
        for (long long p = p0; p < p1; ++p) {
            const int s = (int)(P.skey[p] & m);
            unsigned int seq = 0;
            while (P.top[s] > P.bot[s]) {
                int len = 1;
                stk[0] = s;
                P.pos[s] = 0;
                int at = s;
                bool closed = false;
                while (P.top[at] > P.bot[at]) {
                    if (++guard > (1LL << 31)) { atomicOr(&P.C->err, kPostLoopGuard); return; }
                    const unsigned int t = --P.top[at];
                    const int only = P.succ[at];
                    const int next = only >= 0 ? only : (int)(P.adj[t] & m);
                    if (next == s) { closed = true; break; }
                    const int hit = P.pos[next];
                    if (hit >= 0) {
                        const int L = len - hit;
                        ++found;
                        if (L >= 3 && L <= kMaxLoop) {
                            const long long o = (long long)base + w;
                            for (int i = 0; i < L; ++i) P.lverts[o + i] = stk[len - 1 - i];
                            P.lflag[o] = 1;
                            P.lkey[o] = ((unsigned long long)s << 32) | seq++;
                            P.llen[o] = L;
                            w += L;
                            ++recorded;
                        }
                        for (int i = hit; i < len; ++i) P.pos[stk[i]] = -1;
                        len = hit;
                    }
                    stk[len] = next;
                    P.pos[next] = len;
                    ++len;
                    at = next;
                }
                if (closed) {
                    ++found;
                    if (len >= 3 && len <= kMaxLoop) {
                        const long long o = (long long)base + w;
                        for (int i = 0; i < len; ++i) P.lverts[o + i] = stk[len - 1 - i];
                        P.lflag[o] = 1;
                        P.lkey[o] = ((unsigned long long)s << 32) | seq++;
                        P.llen[o] = len;
                        w += len;
                        ++recorded;
                    }
                }
                for (int i = 0; i < len; ++i) P.pos[stk[i]] = -1;
            }
        }
        atomicAdd(&P.C->loops_found, found);
        atomicAdd(&P.C->nloops, recorded);
    }
}

// One past every vertex's last outgoing edge, and its successor when it has exactly one (the
// walk then needs one dependent load per step instead of two).
__global__ void k_tops(const unsigned int* __restrict__ bot, const unsigned int* __restrict__ deg,
                       const unsigned long long* __restrict__ adj, int b, long long n, unsigned int* top, int* succ) {
    const unsigned long long m = (1ull << b) - 1;
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < n; u += (long long)gridDim.x * blockDim.x) {
        top[u] = bot[u] + deg[u];
        succ[u] = deg[u] == 1 ? (int)(adj[bot[u]] & m) : -1;
    }
}

__global__ void k_gather_keys(const int* __restrict__ lpos, const unsigned long long* __restrict__ lkey, long long n,
                              unsigned long long* key) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        key[i] = lkey[lpos[i]];
}

struct FillParams {
    const int* lorder;                  // loop start positions in fill order
    long long nloops;
    const int* lverts;
    const int* llen;
    const float* Vw;                    // welded vertices (loop vertices are among them)
    long long nvw;
    unsigned long long* nvl;            // sizes pass: new vertices and faces per loop
    unsigned long long* nfl;
    const unsigned long long* vb;       // write pass: exclusive scans of the sizes
    const unsigned long long* fb;
    float* fillV;                       // new vertices (global index nvw + local)
    int4* fillF;                        // new faces
    // sizes pass: ring positions kept in a scratch area (null: not kept)
    float* scratch;                     // 3 floats per ring vertex
    unsigned long long scap;            // its capacity in vertices
    longlong2* rings;                   // per ring: (loop << 32 | ring number, scratch offset)
    unsigned long long rcap;
    float* centers;                     // per loop: the centroid of its last ring (the fan's centre)
    PostCounters* C;
};

// ((a[0] + a[1]) + a[2]) + ... in float, as a sequential loop rounds it: the additions stay in
// order, one dependent chain; the shared-memory loads of the next eight are issued before the
// eight additions of the current ones, so the chain does not wait on them (a is 16-byte aligned).
__device__ __forceinline__ float ordered_sum(const float* a, int n) {
    float c = 0.0f;
    int k = 0;
    if (n >= 16) {
        float4 u = *reinterpret_cast<const float4*>(a);
        float4 v = *reinterpret_cast<const float4*>(a + 4);
        for (k = 8; k + 8 <= n; k += 8) {
            const float4 u2 = *reinterpret_cast<const float4*>(a + k);
            const float4 v2 = *reinterpret_cast<const float4*>(a + k + 4);
            c += u.x; c += u.y; c += u.z; c += u.w;
            c += v.x; c += v.y; c += v.z; c += v.w;
            u = u2;
            v = v2;
        }
        c += u.x; c += u.y; c += u.z; c += u.w;
        c += v.x; c += v.y; c += v.z; c += v.w;
    }
    for (; k < n; ++k) c += a[k];
    return c;
}

// One loop per block: rings towards the centroid (dc_backend.cpp:376-466). Shared memory holds
// two rings (x, y, z arrays) and one scratch array of kMaxLoop floats each.
template <bool WRITE>
__global__ void __launch_bounds__(kFillThreads) k_fill(FillParams P) {
    extern __shared__ float sh[];
    float* ax = sh;                      // current ring
    float* ay = ax + kMaxLoop;
    float* az = ay + kMaxLoop;
    float* bx = az + kMaxLoop;           // next ring
    float* by = bx + kMaxLoop;
    float* bz = by + kMaxLoop;
    float* sd = bz + kMaxLoop;
    __shared__ float s_step, s_c[3], s_far;
    __shared__ unsigned long long s_base;
    __shared__ int s_fits;
    const int tid = threadIdx.x;
    for (long long li = blockIdx.x; li < P.nloops; li += gridDim.x) {
        const int at = P.lorder[li];
        const int n = P.llen[at];
        const int* idx = P.lverts + at;
        for (int k = tid; k < n; k += blockDim.x) {
            const long long v = idx[k];
            ax[k] = P.Vw[3 * v]; ay[k] = P.Vw[3 * v + 1]; az[k] = P.Vw[3 * v + 2];
        }
        __syncthreads();
        for (int k = tid; k < n; k += blockDim.x) {
            const int k1 = k + 1 == n ? 0 : k + 1;
            const float dx = ax[k1] - ax[k], dy = ay[k1] - ay[k], dz = az[k1] - az[k];
            sd[k] = sqrtf(dx * dx + dy * dy + dz * dz);
        }
        __syncthreads();
        if (tid == 0) {
            float step = ordered_sum(sd, n);
            step /= (float)n;
            if (step <= 0.0001f) step = 1.0f;
            s_step = step;
        }
        __syncthreads();
        const float step = s_step;
        const long long vbase = WRITE ? P.nvw + (long long)P.vb[li] : 0;
        const long long fbase = WRITE ? (long long)P.fb[li] : 0;
        int rings = 0;
        for (;;) {
            // centroid of the current ring: one sequential sum per coordinate, in loop order
            if (tid < 3) s_c[tid] = ordered_sum(tid == 0 ? ax : tid == 1 ? ay : az, n) / (float)n;
            if (tid == 0) s_far = 0.0f;
            __syncthreads();
            const float cx = s_c[0], cy = s_c[1], cz = s_c[2];
            if (n <= 4) break;
            float far = 0.0f;
            for (int k = tid; k < n; k += blockDim.x) {
                const float dx = cx - ax[k], dy = cy - ay[k], dz = cz - az[k];
                far = fmaxf(far, sqrtf(dx * dx + dy * dy + dz * dz));
            }
            for (int d = 16; d > 0; d >>= 1) far = fmaxf(far, __shfl_xor_sync(0xffffffffu, far, d));
            if ((tid & 31) == 0) atomicMax(reinterpret_cast<int*>(&s_far), __float_as_int(far));   // far >= 0
            __syncthreads();
            if (s_far <= 1.25f * step) break;
            if (rings >= kMaxRings) {
                if (tid == 0) atomicOr(&P.C->err, kPostRingGuard);
                break;
            }
            ++rings;
            if (!WRITE && P.scratch) {
                // room for this ring in the scratch area, and its record; bounds-checked
                if (tid == 0) {
                    const unsigned long long base = atomicAdd(&P.C->cursor, (unsigned long long)n);
                    const unsigned long long rec = atomicAdd(&P.C->nrings, 1ull);
                    s_fits = base + n <= P.scap && rec < P.rcap;
                    s_base = base;
                    if (s_fits) P.rings[rec] = make_longlong2(((long long)li << 32) | rings, (long long)base);
                    else atomicOr(&P.C->fill_overflow, 1);
                }
                __syncthreads();
            }
            for (int k = tid; k < n; k += blockDim.x) {
                const float px = ax[k], py = ay[k], pz = az[k];
                float dx = cx - px, dy = cy - py, dz = cz - pz;
                const float d = sqrtf(dx * dx + dy * dy + dz * dz);
                const float move = d > step ? step : d * 0.5f;
                if (d > 0.0001f) { dx /= d; dy /= d; dz /= d; }
                else { dx = 0.0f; dy = 0.0f; dz = 0.0f; }
                bx[k] = px + dx * move; by[k] = py + dy * move; bz[k] = pz + dz * move;
                if (!WRITE && P.scratch && s_fits) {
                    float* q = P.scratch + 3 * (s_base + k);
                    q[0] = bx[k]; q[1] = by[k]; q[2] = bz[k];
                }
                if (WRITE) {
                    const long long g = vbase - P.nvw + (long long)(rings - 1) * n + k;
                    P.fillV[3 * g] = bx[k]; P.fillV[3 * g + 1] = by[k]; P.fillV[3 * g + 2] = bz[k];
                    const int k1 = k + 1 == n ? 0 : k + 1;
                    const long long prev = rings == 1 ? -1 : vbase + (long long)(rings - 2) * n;
                    const int o0 = prev < 0 ? idx[k] : (int)(prev + k), o1 = prev < 0 ? idx[k1] : (int)(prev + k1);
                    const int i0 = (int)(vbase + (long long)(rings - 1) * n + k), i1 = (int)(vbase + (long long)(rings - 1) * n + k1);
                    P.fillF[fbase + (long long)(rings - 1) * n + k] = make_int4(o0, o1, i1, i0);
                }
            }
            __syncthreads();
            float* t;
            t = ax; ax = bx; bx = t;
            t = ay; ay = by; by = t;
            t = az; az = bz; bz = t;
        }
        // the rest: a triangle, a quad or a fan around the centroid of the last ring
        if (WRITE) {
            const long long cur = rings == 0 ? -1 : vbase + (long long)(rings - 1) * n;
            auto ring_index = [&](int k) { return cur < 0 ? idx[k] : (int)(cur + k); };
            const long long f0 = fbase + (long long)rings * n;
            if (n == 3) {
                if (tid == 0) P.fillF[f0] = make_int4(ring_index(0), ring_index(1), ring_index(2), ring_index(2));
            } else if (n == 4) {
                if (tid == 0) P.fillF[f0] = make_int4(ring_index(0), ring_index(1), ring_index(2), ring_index(3));
            } else {
                const int center = (int)(vbase + (long long)rings * n);
                if (tid == 0) {
                    const long long g = center - P.nvw;
                    P.fillV[3 * g] = s_c[0]; P.fillV[3 * g + 1] = s_c[1]; P.fillV[3 * g + 2] = s_c[2];
                }
                for (int k = tid; k < n; k += blockDim.x)
                    P.fillF[f0 + k] = make_int4(ring_index(k), ring_index(k + 1 == n ? 0 : k + 1), center, center);
            }
        } else if (tid == 0) {
            P.nvl[li] = (unsigned long long)rings * n + (n > 4 ? 1 : 0);
            P.nfl[li] = (unsigned long long)rings * n + (n > 4 ? n : 1);
            if (P.centers) { P.centers[3 * li] = s_c[0]; P.centers[3 * li + 1] = s_c[1]; P.centers[3 * li + 2] = s_c[2]; }
        }
        __syncthreads();
        ax = sh; ay = ax + kMaxLoop; az = ay + kMaxLoop; bx = az + kMaxLoop; by = bx + kMaxLoop; bz = by + kMaxLoop;
    }
}

__global__ void k_fill_totals(const unsigned long long* vb, const unsigned long long* nvl, const unsigned long long* fb,
                              const unsigned long long* nfl, long long n, PostCounters* C) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        C->fill_v = n ? vb[n - 1] + nvl[n - 1] : 0;
        C->fill_f = n ? fb[n - 1] + nfl[n - 1] : 0;
    }
}

// The kept rings moved from the scratch area to their places: ring j of loop li is vertices
// vb[li] + (j-1)*n .. + n of the fill.
__global__ void k_fill_copy(const longlong2* __restrict__ rings, long long nrings, const int* __restrict__ lorder,
                            const int* __restrict__ llen, const unsigned long long* __restrict__ vb,
                            const float* __restrict__ scratch, float* fillV) {
    for (long long r = blockIdx.x; r < nrings; r += gridDim.x) {
        const longlong2 rec = rings[r];
        const long long li = rec.x >> 32, j = rec.x & 0xffffffffLL;
        const int n = llen[lorder[li]];
        const unsigned long long dst = vb[li] + (unsigned long long)(j - 1) * n;
        for (int k = threadIdx.x; k < 3 * n; k += blockDim.x) fillV[3 * dst + k] = scratch[3 * (unsigned long long)rec.y + k];
    }
}

// The fill's faces from the sizes alone (no positions needed): ring j's quads join ring j-1
// (the loop itself for j = 1) to ring j; then the triangle, quad or fan of the last ring, whose
// fan centre comes from the sizes pass.
__global__ void k_fill_faces(FillParams P) {
    for (long long li = blockIdx.x; li < P.nloops; li += gridDim.x) {
        const int at = P.lorder[li];
        const int n = P.llen[at];
        const int* idx = P.lverts + at;
        const long long rings = (long long)((P.nvl[li] - (n > 4 ? 1 : 0)) / (unsigned long long)n);
        const long long vbase = P.nvw + (long long)P.vb[li], fbase = (long long)P.fb[li];
        for (long long t = threadIdx.x; t < rings * n; t += blockDim.x) {
            const long long j = t / n + 1;
            const int k = (int)(t - (j - 1) * n), k1 = k + 1 == n ? 0 : k + 1;
            const long long prev = j == 1 ? -1 : vbase + (j - 2) * n;
            const int o0 = prev < 0 ? idx[k] : (int)(prev + k), o1 = prev < 0 ? idx[k1] : (int)(prev + k1);
            const int i0 = (int)(vbase + (j - 1) * n + k), i1 = (int)(vbase + (j - 1) * n + k1);
            P.fillF[fbase + t] = make_int4(o0, o1, i1, i0);
        }
        const long long cur = rings == 0 ? -1 : vbase + (rings - 1) * n;
        auto ring_index = [&](int k) { return cur < 0 ? idx[k] : (int)(cur + k); };
        const long long f0 = fbase + rings * n;
        if (n == 3) {
            if (threadIdx.x == 0) P.fillF[f0] = make_int4(ring_index(0), ring_index(1), ring_index(2), ring_index(2));
        } else if (n == 4) {
            if (threadIdx.x == 0) P.fillF[f0] = make_int4(ring_index(0), ring_index(1), ring_index(2), ring_index(3));
        } else {
            const int center = (int)(vbase + rings * n);
            if (threadIdx.x == 0) {
                const long long g = center - P.nvw;
                P.fillV[3 * g] = P.centers[3 * li]; P.fillV[3 * g + 1] = P.centers[3 * li + 1];
                P.fillV[3 * g + 2] = P.centers[3 * li + 2];
            }
            for (int k = threadIdx.x; k < n; k += blockDim.x)
                P.fillF[f0 + k] = make_int4(ring_index(k), ring_index(k + 1 == n ? 0 : k + 1), center, center);
        }
    }
}

// ---------------------------------------------------------------- renumber by first use
struct FaceList {                        // kept faces, then the fill's faces
    const int4* kept;
    long long nkept;
    const int4* fill;
    __device__ __forceinline__ int at(long long p) const {
        const long long f = p >> 2;
        const int4 q = f < nkept ? kept[f] : fill[f - nkept];
        return corner(q, (int)(p & 3));
    }
};

__global__ void k_first_use(FaceList A, long long n, unsigned int* first) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        atomicMin(&first[A.at(p)], (unsigned int)p);
}

__global__ void k_first_flags(FaceList A, long long n, const unsigned int* __restrict__ first, unsigned int* flag) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        flag[p] = first[A.at(p)] == (unsigned int)p ? 1u : 0u;
}

__global__ void k_renumber(FaceList A, long long n, const unsigned int* __restrict__ first,
                           const unsigned int* __restrict__ flag, const unsigned int* __restrict__ slot,
                           const float* __restrict__ Vw, long long nvw, const float* __restrict__ fillV,
                           float* outV, int32_t* outF, PostCounters* C) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const int v = A.at(p);
        outF[p] = (int32_t)slot[first[v]];
        if (flag[p]) {
            const float* src = v < nvw ? Vw + 3 * (long long)v : fillV + 3 * ((long long)v - nvw);
            const long long o = 3 * (long long)slot[p];
            outV[o] = src[0]; outV[o + 1] = src[1]; outV[o + 2] = src[2];
        }
        if (p == n - 1) C->nout = slot[p] + flag[p];
    }
}

}  // namespace

// ---------------------------------------------------------------- host side
namespace {

cudaError_t grow(PostBuf& b, size_t bytes) {
    if (bytes <= b.bytes && b.p) return cudaSuccess;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    const size_t want = std::max<size_t>(256, (bytes + 255) & ~(size_t)255);
    cudaError_t e = dev_malloc(&b.p, want);
    if (e != cudaSuccess) { cudaGetLastError(); return e; }
    b.bytes = want;
    return cudaSuccess;
}

template <class T> T* as(PostBuf& b) { return reinterpret_cast<T*>(b.p); }

int bits_for(long long n) {   // bits to hold 0..n-1
    int b = 1;
    while (b < 31 && (1LL << b) < n) ++b;
    return b;
}

#define PP_TRY(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { R.what = #x; return e_; } } while (0)

cudaError_t read_counters(PostWork& W, PostRun& R, cudaStream_t s) {
    PP_TRY(cudaMemcpyAsync(W.hcount, W.count.p, sizeof(PostCounters), cudaMemcpyDeviceToHost, s));
    PP_TRY(cudaStreamSynchronize(s));
    return cudaSuccess;
}

const PostCounters& host_counters(const PostWork& W) { return *reinterpret_cast<const PostCounters*>(W.hcount); }

// Weld V (nv) / F (nf quads) into Vout / Fout. Returns the welded counts.
cudaError_t weld(PostWork& W, PostRun& R, const float* V, long long nv, const int32_t* F, long long nf, PostBuf& Vout,
                 PostBuf& Fout, long long& nvw, long long& nfw, int sms, cudaStream_t s) {
    PostCounters* C = as<PostCounters>(W.count);
    PP_TRY(grow(W.key, sizeof(unsigned long long) * nv));
    PP_TRY(grow(W.key2, sizeof(unsigned long long) * nv));
    PP_TRY(grow(W.val, sizeof(int) * nv));
    PP_TRY(grow(W.val2, sizeof(int) * nv));
    PP_TRY(grow(W.u0, sizeof(unsigned int) * nv));
    PP_TRY(grow(W.u1, sizeof(unsigned int) * nv));
    PP_TRY(grow(W.u2, sizeof(unsigned int) * nv));
    PP_TRY(grow(W.u3, sizeof(unsigned int) * nv));
    PP_TRY(grow(W.ft, sizeof(int4) * nf));
    PP_TRY(grow(W.flag8, nf));
    PP_TRY(grow(Vout, sizeof(float) * 3 * nv));
    PP_TRY(grow(Fout, sizeof(int4) * nf));
    size_t t0 = 0, t1 = 0, t2 = 0;
    t0 = radix_sort_temp_bytes(nv, 8, true);
    t1 = scan_temp_bytes(nv);
    t2 = select_temp_bytes(nf);
    const size_t tb = std::max(t0, std::max(t1, t2));
    PP_TRY(grow(W.scratch, tb));
    const unsigned g = grid_for(nv, kThreads, sms);
    k_post_reset<<<1, 32, 0, s>>>(C);
    k_bbox<<<g, kThreads, 0, s>>>(V, nv, C);
    k_weld_params<<<1, 32, 0, s>>>(C);
    k_weld_keys<<<g, kThreads, 0, s>>>(V, nv, C, as<unsigned long long>(W.key), as<int>(W.val));
    PP_TRY(cudaGetLastError());
    PP_TRY(radix_sort_pairs(W.scratch.p, W.scratch.bytes, as<unsigned long long>(W.key),
                            as<unsigned long long>(W.key2), as<uint32_t>(W.val), as<uint32_t>(W.val2), nv, 0, 3 * kKeyBits, s));
    k_weld_heads<<<g, kThreads, 0, s>>>(as<unsigned long long>(W.key2), as<int>(W.val2), nv, as<unsigned int>(W.u0),
                                        as<unsigned int>(W.u1));
    PP_TRY(exclusive_sum(W.scratch.p, W.scratch.bytes, as<unsigned int>(W.u1), as<unsigned int>(W.u2), nv, s));
    PP_TRY(inclusive_sum(W.scratch.p, W.scratch.bytes, as<unsigned int>(W.u0), as<unsigned int>(W.u3), nv, s));
    // u0 head, u3 group (1-based), u2 new index of representatives; u1 -> group's new index
    k_weld_groups<<<g, kThreads, 0, s>>>(as<int>(W.val2), as<unsigned int>(W.u0), as<unsigned int>(W.u3),
                                         as<unsigned int>(W.u2), V, nv, as<unsigned int>(W.u1), as<float>(Vout), C);
    k_weld_remap<<<g, kThreads, 0, s>>>(as<int>(W.val2), as<unsigned int>(W.u3), as<unsigned int>(W.u1), nv,
                                        as<int>(W.val));
    k_weld_faces<<<grid_for(nf, kThreads, sms), kThreads, 0, s>>>(F, nf, nv, as<int>(W.val), as<int4>(W.ft),
                                                                   as<unsigned char>(W.flag8), C);
    PP_TRY(cudaGetLastError());
    PP_TRY(select_flagged(W.scratch.p, W.scratch.bytes, as<int4>(W.ft), as<unsigned char>(W.flag8),
                          as<int4>(Fout), &C->nsel, (int)nf, s));
    cudaError_t e = read_counters(W, R, s);
    if (e != cudaSuccess) return e;
    nvw = (long long)host_counters(W).nvw;
    nfw = (long long)host_counters(W).nsel;
    return cudaSuccess;
}

}  // namespace

void post_release(PostWork& W) {
    PostBuf* all[] = {&W.count, &W.key, &W.key2, &W.val, &W.val2, &W.u0, &W.u1, &W.u2, &W.u3, &W.ft, &W.flag8, &W.scratch,
                      &W.Vw, &W.Fw, &W.kept, &W.parent, &W.csize, &W.bnd, &W.deg, &W.bot, &W.top, &W.pos, &W.vparent,
                      &W.skey, &W.sdeg, &W.shead, &W.soff, &W.sgid, &W.stack, &W.lverts, &W.lflag, &W.lkey, &W.llen,
                      &W.lpos, &W.lorder, &W.lkey2, &W.nvl, &W.nfl, &W.vb, &W.fb, &W.fillV, &W.fillF, &W.first,
                      &W.fflag, &W.slot, &W.V1, &W.F1, &W.outV, &W.outF, &W.succ, &W.indeg, &W.cbad, &W.clen,
                      &W.cbase, &W.crank, &W.jflags, &W.fscratch, &W.frings, &W.fcenters};
    for (PostBuf* b : all) {
        if (b->p) cudaFree(b->p);
        b->p = nullptr;
        b->bytes = 0;
    }
    if (W.hcount) cudaFreeHost(W.hcount);
    W.hcount = nullptr;
}

cudaError_t post_run(PostWork& W, PostRun& R, cudaStream_t s) {
    std::memset(R.stats, 0, sizeof(R.stats));
    R.err = 0;
    R.out_V = nullptr;
    R.out_F = nullptr;
    R.nv_out = R.nf_out = 0;
    const long long nv = R.nv, nf = R.nf;
    const int sms = R.num_sms;
    if (!W.hcount) PP_TRY(host_malloc(&W.hcount, sizeof(PostCounters)));
    PP_TRY(grow(W.count, sizeof(PostCounters)));
    PP_TRY(cudaMemsetAsync(W.count.p, 0, sizeof(PostCounters), s));
    PostCounters* C = as<PostCounters>(W.count);
    auto passthrough = [&]() {
        R.out_V = R.V;
        R.out_F = R.F;
        R.nv_out = nv;
        R.nf_out = nf;
        R.stats[kPostVertexCount] = nv;
        R.stats[kPostFaceCount] = nf;
        return cudaSuccess;
    };
    if (nv == 0 || nf == 0 || (!R.close_holes && !R.remove_floaters)) return passthrough();

    long long nvw = 0, nfw = 0;
    cudaError_t e = weld(W, R, R.V, nv, R.F, nf, W.Vw, W.Fw, nvw, nfw, sms, s);
    if (e != cudaSuccess) return e;
    R.err = host_counters(W).err;
    if (R.err) return cudaSuccess;
    R.stats[kPostWeldedVertices] = nvw;
    R.stats[kPostWeldedFaces] = nfw;
    if (nvw == 0 || nfw == 0) return passthrough();

    // edges: uses sorted by undirected key; runs -> boundary edges and face unions
    const int b = bits_for(nvw);
    const long long ne = 4 * nfw;
    const unsigned long long inval = (b >= 32) ? ~0ull : ((1ull << (2 * b)) - 1);
    PP_TRY(grow(W.key, sizeof(unsigned long long) * ne));
    PP_TRY(grow(W.key2, sizeof(unsigned long long) * ne));
    PP_TRY(grow(W.val, sizeof(int) * ne));
    PP_TRY(grow(W.val2, sizeof(int) * ne));
    PP_TRY(grow(W.bnd, sizeof(int4) * ne));
    PP_TRY(grow(W.parent, sizeof(int) * nfw));
    PP_TRY(grow(W.csize, sizeof(unsigned int) * nfw));
    PP_TRY(grow(W.kept, sizeof(int4) * nfw));
    PP_TRY(grow(W.flag8, nfw));
    {
        size_t t0 = 0, t1 = 0;
        t0 = radix_sort_temp_bytes(ne, 8, true);
        t1 = select_temp_bytes(nfw);
        PP_TRY(grow(W.scratch, std::max(t0, t1)));
    }
    const int4* Fw = as<int4>(W.Fw);
    k_edge_uses<<<grid_for(ne, kThreads, sms), kThreads, 0, s>>>(Fw, nfw, b, as<unsigned long long>(W.key), as<int>(W.val));
    PP_TRY(radix_sort_pairs(W.scratch.p, W.scratch.bytes, as<unsigned long long>(W.key),
                            as<unsigned long long>(W.key2), as<uint32_t>(W.val), as<uint32_t>(W.val2), ne, 0, 2 * b, s));
    if (R.remove_floaters) {
        k_iota<<<grid_for(nfw, kThreads, sms), kThreads, 0, s>>>(as<int>(W.parent), nfw);
        PP_TRY(cudaMemsetAsync(W.csize.p, 0, sizeof(unsigned int) * nfw, s));
    }
    EdgeRunParams ep;
    ep.key = as<unsigned long long>(W.key2); ep.val = as<int>(W.val2); ep.n = ne; ep.invalid = inval; ep.Fw = Fw;
    ep.close = R.close_holes; ep.remove = R.remove_floaters; ep.parent = as<int>(W.parent); ep.bnd = as<int4>(W.bnd);
    ep.C = C;
    if (R.remove_floaters) k_first_links<<<grid_for(ne, kThreads, sms), kThreads, 0, s>>>(ep);
    k_edge_runs<<<grid_for(ne, kThreads, sms), kThreads, 0, s>>>(ep);
    PP_TRY(cudaGetLastError());
    long long nkept = nfw;
    const int4* kept = Fw;
    if (R.remove_floaters) {
        k_flatten<<<grid_for(nfw, kThreads, sms), kThreads, 0, s>>>(as<int>(W.parent), nfw);
        k_comp_size<<<grid_for(nfw, kThreads, sms), kThreads, 0, s>>>(as<int>(W.parent), nfw, as<unsigned int>(W.csize));
        k_comp_pick<<<grid_for(nfw, kThreads, sms), kThreads, 0, s>>>(as<int>(W.parent), as<unsigned int>(W.csize), nfw, C);
        k_keep_flags<<<grid_for(nfw, kThreads, sms), kThreads, 0, s>>>(as<int>(W.parent), nfw, C, as<unsigned char>(W.flag8));
        PP_TRY(cudaGetLastError());
        PP_TRY(cudaMemsetAsync(&C->nsel, 0, sizeof(unsigned long long), s));
        PP_TRY(select_flagged(W.scratch.p, W.scratch.bytes, Fw, as<unsigned char>(W.flag8), as<int4>(W.kept), &C->nsel,
                                          (int)nfw, s));
        kept = as<int4>(W.kept);
    }
    e = read_counters(W, R, s);
    if (e != cudaSuccess) return e;
    {
        const PostCounters& h = host_counters(W);
        R.err = h.err;
        if (R.err) return cudaSuccess;
        if (R.remove_floaters) nkept = (long long)h.nsel;
        R.stats[kPostComponents] = R.remove_floaters ? (long long)h.ncomp : 0;
        R.stats[kPostKeptFaces] = nkept;
        R.stats[kPostBoundaryEdges] = (long long)h.nb;
    }
    const long long nb = (long long)host_counters(W).nb;

    // holes
    long long nloops = 0, fill_v = 0, fill_f = 0;
    if (R.close_holes && nb > 0) {
        PP_TRY(grow(W.deg, sizeof(unsigned int) * nvw));
        PP_TRY(grow(W.bot, sizeof(unsigned int) * nvw));
        PP_TRY(grow(W.top, sizeof(unsigned int) * nvw));
        PP_TRY(grow(W.pos, sizeof(int) * nvw));
        PP_TRY(grow(W.vparent, sizeof(int) * nvw));
        PP_TRY(cudaMemsetAsync(W.deg.p, 0, sizeof(unsigned int) * nvw, s));
        PP_TRY(cudaMemsetAsync(W.pos.p, 0xff, sizeof(int) * nvw, s));
        k_bnd_keys<<<grid_for(nb, kThreads, sms), kThreads, 0, s>>>(as<int4>(W.bnd), nb, as<int>(W.parent),
                                                                     R.remove_floaters, b, as<unsigned long long>(W.key),
                                                                     as<unsigned int>(W.deg), C);
        size_t t0 = 0, t1 = 0;
        t0 = radix_sort_temp_bytes(nb, 8, false);
        t1 = scan_temp_bytes(nvw);
        PP_TRY(grow(W.scratch, std::max(t0, t1)));
        PP_TRY(radix_sort_keys(W.scratch.p, W.scratch.bytes, as<unsigned long long>(W.key),
                               as<unsigned long long>(W.key2), nb, 0, 2 * b, s));
        PP_TRY(exclusive_sum(W.scratch.p, W.scratch.bytes, as<unsigned int>(W.deg), as<unsigned int>(W.bot), nvw, s));
        e = read_counters(W, R, s);
        if (e != cudaSuccess) return e;
        const long long nbk = (long long)host_counters(W).nbk;
        if (nbk > 0) {
            // top = bot + deg; weak components of the boundary graph
            k_iota<<<grid_for(nvw, kThreads, sms), kThreads, 0, s>>>(as<int>(W.vparent), nvw);
            k_bnd_unite<<<grid_for(nbk, kThreads, sms), kThreads, 0, s>>>(as<unsigned long long>(W.key2), nbk, b,
                                                                           as<int>(W.vparent), C);
            k_flatten<<<grid_for(nvw, kThreads, sms), kThreads, 0, s>>>(as<int>(W.vparent), nvw);
            PP_TRY(grow(W.skey, sizeof(unsigned long long) * nvw));
            PP_TRY(grow(W.lkey2, sizeof(unsigned long long) * std::max(nvw, nbk)));
            k_start_keys<<<grid_for(nvw, kThreads, sms), kThreads, 0, s>>>(as<unsigned int>(W.deg), as<int>(W.vparent),
                                                                            nvw, b, as<unsigned long long>(W.skey), C);
            PP_TRY(cudaGetLastError());
            e = read_counters(W, R, s);
            if (e != cudaSuccess) return e;
            const long long ns = (long long)host_counters(W).nstarts;
            {
                size_t ta = 0, tb2 = 0, tc = 0;
                ta = radix_sort_temp_bytes(ns, 8, false);
                tb2 = scan_temp_bytes(ns);
                tc = scan_temp_bytes(ns);
                PP_TRY(grow(W.scratch, std::max(ta, std::max(tb2, tc))));
            }
            PP_TRY(radix_sort_keys(W.scratch.p, W.scratch.bytes, as<unsigned long long>(W.skey),
                                   as<unsigned long long>(W.lkey2), ns, 0, 2 * b, s));
            PP_TRY(grow(W.sdeg, sizeof(unsigned long long) * ns));
            PP_TRY(grow(W.shead, sizeof(unsigned int) * ns));
            PP_TRY(grow(W.soff, sizeof(unsigned long long) * ns));
            PP_TRY(grow(W.sgid, sizeof(unsigned int) * ns));
            k_start_info<<<grid_for(ns, kThreads, sms), kThreads, 0, s>>>(as<unsigned long long>(W.lkey2), ns, b,
                                                                          as<unsigned int>(W.deg),
                                                                          as<unsigned long long>(W.sdeg),
                                                                          as<unsigned int>(W.shead));
            PP_TRY(exclusive_sum(W.scratch.p, W.scratch.bytes, as<unsigned long long>(W.sdeg),
                                 as<unsigned long long>(W.soff), ns, s));
            PP_TRY(inclusive_sum(W.scratch.p, W.scratch.bytes, as<unsigned int>(W.shead),
                                 as<unsigned int>(W.sgid), ns, s));
            PP_TRY(grow(W.succ, sizeof(int) * nvw));
            k_tops<<<grid_for(nvw, kThreads, sms), kThreads, 0, s>>>(as<unsigned int>(W.bot), as<unsigned int>(W.deg),
                                                                     as<unsigned long long>(W.key2), b, nvw,
                                                                     as<unsigned int>(W.top), as<int>(W.succ));
            // simple cycles: degrees, marks, ranks
            PP_TRY(grow(W.indeg, sizeof(unsigned int) * nvw));
            PP_TRY(grow(W.cbad, sizeof(unsigned int) * nvw));
            PP_TRY(grow(W.clen, sizeof(unsigned int) * nvw));
            PP_TRY(grow(W.cbase, sizeof(unsigned long long) * nvw));
            PP_TRY(grow(W.crank, sizeof(unsigned long long) * nvw));
            PP_TRY(grow(W.jflags, sizeof(int) * kRankRounds));
            PP_TRY(cudaMemsetAsync(W.indeg.p, 0, sizeof(unsigned int) * nvw, s));
            PP_TRY(cudaMemsetAsync(W.cbad.p, 0, sizeof(unsigned int) * nvw, s));
            PP_TRY(cudaMemsetAsync(W.clen.p, 0, sizeof(unsigned int) * nvw, s));
            PP_TRY(cudaMemsetAsync(W.jflags.p, 0, sizeof(int) * kRankRounds, s));
            const unsigned long long* starts = as<unsigned long long>(W.lkey2);
            k_cycle_indeg<<<grid_for(nbk, kThreads, sms), kThreads, 0, s>>>(as<unsigned long long>(W.key2), nbk, b,
                                                                             as<unsigned int>(W.deg), as<int>(W.vparent),
                                                                             as<unsigned int>(W.indeg), as<unsigned int>(W.cbad));
            k_cycle_marks<<<grid_for(ns, kThreads, sms), kThreads, 0, s>>>(starts, ns, b, as<unsigned int>(W.deg),
                                                                            as<unsigned int>(W.indeg), as<int>(W.vparent),
                                                                            as<unsigned int>(W.cbad), as<unsigned int>(W.clen));
            k_cycle_rank_init<<<grid_for(ns, kThreads, sms), kThreads, 0, s>>>(starts, ns, b, as<unsigned int>(W.cbad),
                                                                                as<int>(W.vparent), as<int>(W.succ),
                                                                                as<unsigned long long>(W.crank));
            for (int r = 0; r < kRankRounds; ++r)
                k_cycle_rank_jump<<<grid_for(ns, kThreads, sms), kThreads, 0, s>>>(starts, ns, b, as<unsigned int>(W.cbad),
                                                                                    as<int>(W.vparent),
                                                                                    as<unsigned long long>(W.crank),
                                                                                    as<int>(W.jflags), r);
            k_cycle_bases<<<grid_for(ns, kThreads, sms), kThreads, 0, s>>>(as<unsigned long long>(W.lkey2),
                                                                            as<unsigned int>(W.shead),
                                                                            as<unsigned long long>(W.soff), ns, b,
                                                                            as<unsigned long long>(W.cbase));
            PP_TRY(cudaGetLastError());
            PP_TRY(grow(W.stack, sizeof(int) * (nbk + ns + 1)));
            PP_TRY(grow(W.lverts, sizeof(int) * nbk));
            PP_TRY(grow(W.lflag, nbk));
            PP_TRY(grow(W.lkey, sizeof(unsigned long long) * nbk));
            PP_TRY(grow(W.llen, sizeof(int) * nbk));
            PP_TRY(cudaMemsetAsync(W.lflag.p, 0, nbk, s));
            k_cycle_emit<<<grid_for(ns, kThreads, sms), kThreads, 0, s>>>(starts, ns, b, as<unsigned int>(W.cbad),
                                                                           as<int>(W.vparent), as<unsigned int>(W.clen),
                                                                           as<unsigned long long>(W.crank),
                                                                           as<unsigned long long>(W.cbase), as<int>(W.lverts),
                                                                           as<unsigned char>(W.lflag),
                                                                           as<unsigned long long>(W.lkey), as<int>(W.llen), C);
            WalkParams wp;
            wp.skey = as<unsigned long long>(W.lkey2); wp.nstarts = ns; wp.shead = as<unsigned int>(W.shead);
            wp.soff = as<unsigned long long>(W.soff); wp.sgid = as<unsigned int>(W.sgid); wp.b = b;
            wp.adj = as<unsigned long long>(W.key2); wp.bot = as<unsigned int>(W.bot); wp.top = as<unsigned int>(W.top);
            wp.succ = as<int>(W.succ);
            wp.cbad = as<unsigned int>(W.cbad);
            wp.pos = as<int>(W.pos); wp.stack = as<int>(W.stack); wp.lverts = as<int>(W.lverts);
            wp.lflag = as<unsigned char>(W.lflag); wp.lkey = as<unsigned long long>(W.lkey); wp.llen = as<int>(W.llen);
            wp.C = C;
            k_walk<<<grid_for(ns, 64, sms), 64, 0, s>>>(wp);
            PP_TRY(cudaGetLastError());
            // the recorded loops in fill order
            PP_TRY(grow(W.lpos, sizeof(int) * nbk));
            PP_TRY(grow(W.lorder, sizeof(int) * nbk));
            {
                size_t ta = 0;
                ta = select_temp_bytes(nbk);
                PP_TRY(grow(W.scratch, ta));
            }
            PP_TRY(cudaMemsetAsync(&C->nsel, 0, sizeof(unsigned long long), s));
            PP_TRY(select_flagged_index(W.scratch.p, W.scratch.bytes, as<unsigned char>(W.lflag),
                                        as<int>(W.lpos), &C->nsel, (int)nbk, s));
            e = read_counters(W, R, s);
            if (e != cudaSuccess) return e;
            R.err = host_counters(W).err;
            if (R.err) return cudaSuccess;
            nloops = (long long)host_counters(W).nloops;
            R.stats[kPostLoopsFound] = (long long)host_counters(W).loops_found;
            R.stats[kPostLoopsFilled] = nloops;
        }
    }
    if (nloops > 0) {
        PP_TRY(grow(W.key, sizeof(unsigned long long) * nloops));
        k_gather_keys<<<grid_for(nloops, kThreads, sms), kThreads, 0, s>>>(as<int>(W.lpos), as<unsigned long long>(W.lkey),
                                                                            nloops, as<unsigned long long>(W.key));
        {
            size_t ta = 0, tb2 = 0;
            ta = radix_sort_temp_bytes(nloops, 8, true);
            tb2 = scan_temp_bytes(nloops);
            PP_TRY(grow(W.scratch, std::max(ta, tb2)));
        }
        PP_TRY(grow(W.lkey2, sizeof(unsigned long long) * nloops));
        PP_TRY(radix_sort_pairs(W.scratch.p, W.scratch.bytes, as<unsigned long long>(W.key),
                                as<unsigned long long>(W.lkey2), as<uint32_t>(W.lpos), as<uint32_t>(W.lorder), nloops, 0, 64, s));
        PP_TRY(grow(W.nvl, sizeof(unsigned long long) * nloops));
        PP_TRY(grow(W.nfl, sizeof(unsigned long long) * nloops));
        PP_TRY(grow(W.vb, sizeof(unsigned long long) * nloops));
        PP_TRY(grow(W.fb, sizeof(unsigned long long) * nloops));
        FillParams fp;
        fp.lorder = as<int>(W.lorder); fp.nloops = nloops; fp.lverts = as<int>(W.lverts); fp.llen = as<int>(W.llen);
        fp.Vw = as<float>(W.Vw); fp.nvw = nvw; fp.nvl = as<unsigned long long>(W.nvl); fp.nfl = as<unsigned long long>(W.nfl);
        fp.vb = as<unsigned long long>(W.vb); fp.fb = as<unsigned long long>(W.fb); fp.fillV = nullptr; fp.fillF = nullptr;
        fp.C = C;
        // ring positions kept by the sizes pass (the capacity grows to what the last call needed)
        PP_TRY(grow(W.fscratch, sizeof(float) * 3 * W.fill_scap));
        PP_TRY(grow(W.frings, sizeof(longlong2) * W.fill_rcap));
        PP_TRY(grow(W.fcenters, sizeof(float) * 3 * nloops));
        fp.scratch = as<float>(W.fscratch); fp.scap = W.fill_scap;
        fp.rings = as<longlong2>(W.frings); fp.rcap = W.fill_rcap;
        fp.centers = as<float>(W.fcenters);
        PP_TRY(cudaMemsetAsync(&C->cursor, 0, 2 * sizeof(unsigned long long) + 2 * sizeof(int), s));
        const size_t smem = sizeof(float) * 7 * kMaxLoop;
        PP_TRY(cudaFuncSetAttribute(k_fill<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        PP_TRY(cudaFuncSetAttribute(k_fill<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const unsigned fg = (unsigned)std::min<long long>(nloops, (long long)sms * 2);
        k_fill<false><<<fg, kFillThreads, smem, s>>>(fp);
        PP_TRY(cudaGetLastError());
        PP_TRY(exclusive_sum(W.scratch.p, W.scratch.bytes, as<unsigned long long>(W.nvl),
                             as<unsigned long long>(W.vb), nloops, s));
        PP_TRY(exclusive_sum(W.scratch.p, W.scratch.bytes, as<unsigned long long>(W.nfl),
                             as<unsigned long long>(W.fb), nloops, s));
        k_fill_totals<<<1, 32, 0, s>>>(as<unsigned long long>(W.vb), as<unsigned long long>(W.nvl),
                                       as<unsigned long long>(W.fb), as<unsigned long long>(W.nfl), nloops, C);
        e = read_counters(W, R, s);
        if (e != cudaSuccess) return e;
        R.err = host_counters(W).err;
        if (R.err) return cudaSuccess;
        fill_v = (long long)host_counters(W).fill_v;
        fill_f = (long long)host_counters(W).fill_f;
        if (nvw + fill_v >= 0x7fffffffLL || 4 * (nkept + fill_f) >= 0x7fffffffLL) {   // int item counts
            R.too_large = 1;
            return cudaSuccess;
        }
        PP_TRY(grow(W.fillV, sizeof(float) * 3 * std::max(1LL, fill_v)));
        PP_TRY(grow(W.fillF, sizeof(int4) * std::max(1LL, fill_f)));
        fp.fillV = as<float>(W.fillV);
        fp.fillF = as<int4>(W.fillF);
        const PostCounters& hc = host_counters(W);
        if (!hc.fill_overflow) {
            const long long nr = (long long)hc.nrings;
            if (nr > 0)
                k_fill_copy<<<(unsigned)std::min<long long>(nr, (long long)sms * 8), kThreads, 0, s>>>(
                    fp.rings, nr, fp.lorder, fp.llen, fp.vb, fp.scratch, fp.fillV);
            k_fill_faces<<<(unsigned)std::min<long long>(nloops, (long long)sms * 8), kThreads, 0, s>>>(fp);
        } else {
            // the kept positions did not fit: recompute the rings while writing them, and let
            // the next call keep them
            W.fill_scap = std::max<unsigned long long>(W.fill_scap, hc.cursor);
            W.fill_rcap = std::max<unsigned long long>(W.fill_rcap, hc.nrings);
            fp.scratch = nullptr;
            k_fill<true><<<fg, kFillThreads, smem, s>>>(fp);
        }
        PP_TRY(cudaGetLastError());
        R.stats[kPostFillVertices] = fill_v;
        R.stats[kPostFillFaces] = fill_f;
    }

    // renumber by first use
    const long long nall = nvw + fill_v;
    const long long nA = 4 * (nkept + fill_f);
    PP_TRY(grow(W.first, sizeof(unsigned int) * nall));
    PP_TRY(grow(W.fflag, sizeof(unsigned int) * nA));
    PP_TRY(grow(W.slot, sizeof(unsigned int) * nA));
    PostBuf& dstV = R.close_holes ? W.V1 : W.outV;
    PostBuf& dstF = R.close_holes ? W.F1 : W.outF;
    PP_TRY(grow(dstV, sizeof(float) * 3 * nall));
    PP_TRY(grow(dstF, sizeof(int32_t) * nA));
    {
        size_t ta = 0;
        ta = scan_temp_bytes(nA);
        PP_TRY(grow(W.scratch, ta));
    }
    FaceList A;
    A.kept = kept; A.nkept = nkept; A.fill = as<int4>(W.fillF);
    PP_TRY(cudaMemsetAsync(W.first.p, 0xff, sizeof(unsigned int) * nall, s));
    k_first_use<<<grid_for(nA, kThreads, sms), kThreads, 0, s>>>(A, nA, as<unsigned int>(W.first));
    k_first_flags<<<grid_for(nA, kThreads, sms), kThreads, 0, s>>>(A, nA, as<unsigned int>(W.first), as<unsigned int>(W.fflag));
    PP_TRY(exclusive_sum(W.scratch.p, W.scratch.bytes, as<unsigned int>(W.fflag), as<unsigned int>(W.slot), nA, s));
    k_renumber<<<grid_for(nA, kThreads, sms), kThreads, 0, s>>>(A, nA, as<unsigned int>(W.first), as<unsigned int>(W.fflag),
                                                                 as<unsigned int>(W.slot), as<float>(W.Vw), nvw,
                                                                 as<float>(W.fillV), as<float>(dstV), as<int32_t>(dstF), C);
    PP_TRY(cudaGetLastError());
    e = read_counters(W, R, s);
    if (e != cudaSuccess) return e;
    long long nvo = (long long)host_counters(W).nout, nfo = nA / 4;
    if (R.close_holes) {
        long long nv2 = 0, nf2 = 0;
        e = weld(W, R, as<float>(W.V1), nvo, as<int32_t>(W.F1), nfo, W.outV, W.outF, nv2, nf2, sms, s);
        if (e != cudaSuccess) return e;
        R.err = host_counters(W).err;
        if (R.err) return cudaSuccess;
        nvo = nv2;
        nfo = nf2;
    }
    R.out_V = as<float>(W.outV);
    R.out_F = as<int32_t>(W.outF);
    R.nv_out = nvo;
    R.nf_out = nfo;
    R.stats[kPostVertexCount] = nvo;
    R.stats[kPostFaceCount] = nfo;
    return cudaSuccess;
}

}  // namespace dcb
