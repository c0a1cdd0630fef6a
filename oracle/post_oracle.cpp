// post_oracle.cpp — TEST INFRASTRUCTURE ONLY: a CPU restatement of the reference's mesh
// post-pass `postprocess_mesh` (src/cpp/dc_backend.cpp:217-558) and its vertex weld
// `merge_vertices_in_place` (src/cpp/dc_backend.cpp:127-215). It is the checker of the
// engine's GPU post-pass (dcb_post.cu) and is itself pinned against the reference's own
// function compiled from its source (oracle/ref_post_harness.cpp, `make ref`) and against the
// committed fixtures tests/golden/post_*.npz. Float arithmetic is written in the reference's
// order and compiled without contraction (-ffp-contract=off), as the reference's x86-64 build
// rounds it.
//
// Quads in and out (4 indices per face; a triangle from the hole fill repeats its last index).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

namespace {

struct QuadMesh {
    std::vector<float> V;     // 3 per vertex
    std::vector<int32_t> F;   // 4 per face
    int64_t nv() const { return (int64_t)V.size() / 3; }
    int64_t nf() const { return (int64_t)F.size() / 4; }
};

// Counters reported beside the mesh (the engine's dcb_post_stats in the same order).
enum PostStat {
    kWeldedVertices, kWeldedFaces, kComponents, kKeptFaces, kBoundaryEdges, kLoopsFound, kLoopsFilled,
    kFillVertices, kFillFaces, kVertexCount, kFaceCount, kNumStats
};

// Vertex weld (dc_backend.cpp:127-215): positions quantised on a grid of diag * 1e-5 (diag of
// the bounding box; 1e-5 when the box is a point); vertices on the same grid point become the
// first of them, numbered in order of first occurrence; a face left with fewer than three
// distinct indices is dropped, the others keep their four (possibly repeated) indices.
void weld(QuadMesh& m) {
    const int64_t nv = m.nv(), nf = m.nf();
    if (nv <= 0 || nf <= 0) return;
    float lo[3] = {m.V[0], m.V[1], m.V[2]}, hi[3] = {m.V[0], m.V[1], m.V[2]};
    for (int64_t i = 0; i < nv; ++i)
        for (int a = 0; a < 3; ++a) {
            const float x = m.V[3 * i + a];
            if (x < lo[a]) lo[a] = x;
            if (x > hi[a]) hi[a] = x;
        }
    const float ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
    const float diag = std::sqrt(ex * ex + ey * ey + ez * ez);
    const float eps = diag > 0.0f ? diag * 1e-5f : 1e-5f;
    const float inv = 1.0f / eps;

    // grid point of every vertex; the first vertex on each point represents it
    std::vector<std::array<int64_t, 3>> q((size_t)nv);
    for (int64_t i = 0; i < nv; ++i)
        for (int a = 0; a < 3; ++a) q[i][a] = (int64_t)std::round(m.V[3 * i + a] * inv);
    std::vector<int32_t> order((size_t)nv);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return q[a] < q[b]; });
    std::vector<int32_t> rep((size_t)nv);
    for (int64_t p = 0; p < nv; ++p) {
        const int32_t i = order[p];
        rep[i] = (p > 0 && q[order[p - 1]] == q[i]) ? rep[order[p - 1]] : i;
    }
    std::vector<int32_t> remap((size_t)nv);
    std::vector<float> V;
    V.reserve(m.V.size());
    for (int64_t i = 0; i < nv; ++i) {
        if (rep[i] == i) {
            remap[i] = (int32_t)(V.size() / 3);
            V.insert(V.end(), &m.V[3 * i], &m.V[3 * i] + 3);
        } else {
            remap[i] = remap[rep[i]];
        }
    }
    std::vector<int32_t> F;
    F.reserve(m.F.size());
    for (int64_t f = 0; f < nf; ++f) {
        int32_t c[4];
        int distinct = 0;
        for (int k = 0; k < 4; ++k) {
            c[k] = remap[m.F[4 * f + k]];
            bool seen = false;
            for (int j = 0; j < k; ++j) seen = seen || c[j] == c[k];
            distinct += !seen;
        }
        if (distinct < 3) continue;
        F.insert(F.end(), c, c + 4);
    }
    m.V.swap(V);
    m.F.swap(F);
}

// Fills one boundary loop (dc_backend.cpp:376-466): while the loop has more than four
// vertices and its farthest vertex lies more than 1.25 mean edge lengths from the centroid, a
// new ring is placed one mean edge length (half the distance, when closer) towards the
// centroid and joined by quads; the rest is closed by one triangle (3), one quad (4) or a fan
// around the centroid (more).
void fill_loop(std::vector<float>& V, std::vector<int32_t>& out, std::vector<int32_t> ring, int64_t* st) {
    const size_t n = ring.size();
    if (n < 3) return;
    ++st[kLoopsFilled];
    const int64_t v0 = (int64_t)V.size() / 3, f0 = (int64_t)out.size() / 4;
    float step = 0.0f;
    for (size_t k = 0; k < n; ++k) {
        const float* a = &V[3 * (size_t)ring[k]];
        const float* b = &V[3 * (size_t)ring[(k + 1) % n]];
        const float dx = b[0] - a[0], dy = b[1] - a[1], dz = b[2] - a[2];
        step += std::sqrt(dx * dx + dy * dy + dz * dz);
    }
    step /= (float)n;
    if (step <= 0.0001f) step = 1.0f;
    auto centroid = [&](float c[3]) {
        c[0] = c[1] = c[2] = 0.0f;
        for (size_t k = 0; k < n; ++k)
            for (int a = 0; a < 3; ++a) c[a] += V[3 * (size_t)ring[k] + a];
        for (int a = 0; a < 3; ++a) c[a] /= (float)n;
    };
    while (n > 4) {
        float c[3];
        centroid(c);
        float far = 0.0f;
        for (size_t k = 0; k < n; ++k) {
            const float dx = c[0] - V[3 * (size_t)ring[k]], dy = c[1] - V[3 * (size_t)ring[k] + 1],
                        dz = c[2] - V[3 * (size_t)ring[k] + 2];
            const float d = std::sqrt(dx * dx + dy * dy + dz * dz);
            if (d > far) far = d;
        }
        if (far <= 1.25f * step) break;
        std::vector<int32_t> inner(n);
        for (size_t k = 0; k < n; ++k) {
            const float px = V[3 * (size_t)ring[k]], py = V[3 * (size_t)ring[k] + 1], pz = V[3 * (size_t)ring[k] + 2];
            float dx = c[0] - px, dy = c[1] - py, dz = c[2] - pz;
            const float d = std::sqrt(dx * dx + dy * dy + dz * dz);
            const float move = d > step ? step : d * 0.5f;
            if (d > 0.0001f) { dx /= d; dy /= d; dz /= d; }
            else { dx = 0.0f; dy = 0.0f; dz = 0.0f; }
            inner[k] = (int32_t)(V.size() / 3);
            V.push_back(px + dx * move);
            V.push_back(py + dy * move);
            V.push_back(pz + dz * move);
        }
        for (size_t k = 0; k < n; ++k) {
            const size_t k1 = (k + 1) % n;
            const int32_t quad[4] = {ring[k], ring[k1], inner[k1], inner[k]};
            out.insert(out.end(), quad, quad + 4);
        }
        ring.swap(inner);
    }
    if (n == 3) {
        const int32_t tri[4] = {ring[0], ring[1], ring[2], ring[2]};
        out.insert(out.end(), tri, tri + 4);
    } else if (n == 4) {
        out.insert(out.end(), ring.begin(), ring.end());
    } else {
        float c[3];
        centroid(c);
        const int32_t center = (int32_t)(V.size() / 3);
        V.insert(V.end(), c, c + 3);
        for (size_t k = 0; k < n; ++k) {
            const int32_t fan[4] = {ring[k], ring[(k + 1) % n], center, center};
            out.insert(out.end(), fan, fan + 4);
        }
    }
    st[kFillVertices] += (int64_t)V.size() / 3 - v0;
    st[kFillFaces] += (int64_t)out.size() / 4 - f0;
}

struct EdgeUse {
    int32_t lo, hi;    // undirected key
    int32_t face, slot;
};

QuadMesh postprocess(const QuadMesh& in, bool close_holes, bool remove_floaters, int64_t* st) {
    if (in.V.empty() || in.F.empty() || (!close_holes && !remove_floaters)) {
        st[kVertexCount] = in.nv();
        st[kFaceCount] = in.nf();
        return in;
    }
    QuadMesh m = in;
    weld(m);
    const int64_t nv = m.nv(), nf = m.nf();
    st[kWeldedVertices] = nv;
    st[kWeldedFaces] = nf;
    if (nv == 0 || nf == 0) {   // everything welded away: the input is returned (dc_backend.cpp:226)
        st[kVertexCount] = in.nv();
        st[kFaceCount] = in.nf();
        return in;
    }

    // Edge uses grouped by undirected edge (dc_backend.cpp:231-310). Within a group the order
    // does not reach the result: two uses make the faces neighbours, and the boundary uses of
    // a group all add the same directed edge to the same vertex's list.
    std::vector<EdgeUse> uses;
    uses.reserve((size_t)nf * 4);
    for (int64_t f = 0; f < nf; ++f)
        for (int e = 0; e < 4; ++e) {
            const int32_t u = m.F[4 * f + e], v = m.F[4 * f + (e + 1) % 4];
            if (u != v) uses.push_back({std::min(u, v), std::max(u, v), (int32_t)f, e});
        }
    std::sort(uses.begin(), uses.end(), [](const EdgeUse& a, const EdgeUse& b) {
        return a.lo != b.lo ? a.lo < b.lo : a.hi != b.hi ? a.hi < b.hi : a.face != b.face ? a.face < b.face : a.slot < b.slot;
    });
    std::vector<std::vector<int32_t>> nbr((size_t)nf);
    std::vector<std::array<int32_t, 3>> boundary;   // directed (u, v) as the face walks it, face
    auto directed = [&](const EdgeUse& x) {
        return std::array<int32_t, 3>{m.F[4 * x.face + x.slot], m.F[4 * x.face + (x.slot + 1) % 4], x.face};
    };
    for (size_t i = 0; i < uses.size();) {
        size_t j = i + 1;
        while (j < uses.size() && uses[j].lo == uses[i].lo && uses[j].hi == uses[i].hi) ++j;
        if (j - i == 1) {
            boundary.push_back(directed(uses[i]));
        } else if (j - i == 2) {
            // at most four uses per face, so the reference's cap of four neighbours never binds
            nbr[uses[i].face].push_back(uses[i + 1].face);
            nbr[uses[i + 1].face].push_back(uses[i].face);
        } else if (close_holes && remove_floaters) {
            // a non-manifold edge: every use is a boundary edge (its neighbour pairs only feed
            // the component search, which runs with remove_floaters, where they are not added)
            for (size_t x = i; x < j; ++x) boundary.push_back(directed(uses[x]));
        }
        i = j;
    }
    st[kBoundaryEdges] = (int64_t)boundary.size();

    // Face components by breadth-first search in face order; the largest (first on ties) is
    // kept (dc_backend.cpp:312-361).
    std::vector<int32_t> comp((size_t)nf, 0);
    int32_t keep = 0;
    std::vector<int32_t> out;
    out.reserve(m.F.size());
    if (remove_floaters) {
        std::fill(comp.begin(), comp.end(), -1);
        std::vector<int32_t> queue((size_t)nf);
        int32_t ncomp = 0, best = -1;
        int64_t best_size = -1;
        for (int64_t f = 0; f < nf; ++f) {
            if (comp[f] != -1) continue;
            const int32_t c = ncomp++;
            size_t head = 0, tail = 0;
            queue[tail++] = (int32_t)f;
            comp[f] = c;
            while (head < tail) {
                const int32_t g = queue[head++];
                for (int32_t h : nbr[g])
                    if (comp[h] == -1) { comp[h] = c; queue[tail++] = h; }
            }
            if ((int64_t)tail > best_size) { best_size = (int64_t)tail; best = c; }
        }
        keep = best;
        st[kComponents] = ncomp;
        for (int64_t f = 0; f < nf; ++f)
            if (comp[f] == keep) out.insert(out.end(), &m.F[4 * f], &m.F[4 * f] + 4);
    } else {
        st[kComponents] = 0;
        out = m.F;
    }
    st[kKeptFaces] = (int64_t)out.size() / 4;

    // Boundary loops (dc_backend.cpp:368-503): each vertex's outgoing boundary edges in the
    // order above; walks start at every vertex in index order and take the last edge first; a
    // walk that returns to its start, or runs into a vertex already on it, closes a loop, which
    // is filled reversed when it has 3..4096 vertices.
    if (close_holes && !boundary.empty()) {
        std::vector<std::vector<int32_t>> adj((size_t)nv);
        for (const auto& b : boundary)
            if (!remove_floaters || comp[b[2]] == keep) adj[b[0]].push_back(b[1]);
        auto take = [&](const std::vector<int32_t>& path, size_t from) {
            ++st[kLoopsFound];
            const size_t len = path.size() - from;
            if (len >= 3 && len <= 4096) fill_loop(m.V, out, std::vector<int32_t>(path.rbegin(), path.rend() - from), st);
        };
        for (int32_t start = 0; start < (int32_t)nv; ++start) {
            while (!adj[start].empty()) {
                std::vector<int32_t> path{start};
                bool closed = false;
                int32_t at = start;
                while (!adj[at].empty()) {
                    const int32_t next = adj[at].back();
                    adj[at].pop_back();
                    if (next == start) { closed = true; break; }
                    const auto hit = std::find(path.begin(), path.end(), next);
                    if (hit != path.end()) {
                        const size_t from = (size_t)(hit - path.begin());
                        take(path, from);
                        path.resize(from);
                    }
                    path.push_back(next);
                    at = next;
                }
                if (closed) take(path, 0);
            }
        }
    }

    // Vertices numbered by first use in the face list (dc_backend.cpp:537-550).
    QuadMesh r;
    std::vector<int32_t> renum(m.V.size() / 3, -1);
    r.F.reserve(out.size());
    for (int32_t v : out) {
        if (renum[v] == -1) {
            renum[v] = (int32_t)(r.V.size() / 3);
            r.V.insert(r.V.end(), &m.V[3 * (size_t)v], &m.V[3 * (size_t)v] + 3);
        }
        r.F.push_back(renum[v]);
    }
    if (close_holes) weld(r);
    st[kVertexCount] = r.nv();
    st[kFaceCount] = r.nf();
    return r;
}

struct PostResult {
    QuadMesh m;
    int64_t st[kNumStats];
};

}  // namespace

extern "C" {

void* ppo_run(const float* V, int64_t nv, const int32_t* F, int64_t nf, int close_holes, int remove_floaters) {
    if (nv < 0 || nf < 0 || (nv && !V) || (nf && !F)) return nullptr;
    for (int64_t i = 0; i < 4 * nf; ++i)
        if (F[i] < 0 || F[i] >= nv) return nullptr;
    QuadMesh in;
    in.V.assign(V, V + 3 * nv);
    in.F.assign(F, F + 4 * nf);
    PostResult* R = new PostResult();
    std::memset(R->st, 0, sizeof(R->st));
    R->m = postprocess(in, close_holes != 0, remove_floaters != 0, R->st);
    return R;
}

int64_t ppo_num_vertices(void* h) { return h ? ((PostResult*)h)->m.nv() : 0; }
int64_t ppo_num_faces(void* h) { return h ? ((PostResult*)h)->m.nf() : 0; }

void ppo_copy(void* h, float* V, int32_t* F, int64_t* stats) {
    if (!h) return;
    const PostResult* R = (const PostResult*)h;
    if (V) std::memcpy(V, R->m.V.data(), R->m.V.size() * sizeof(float));
    if (F) std::memcpy(F, R->m.F.data(), R->m.F.size() * sizeof(int32_t));
    if (stats) std::memcpy(stats, R->st, sizeof(R->st));
}

void ppo_free(void* h) { delete (PostResult*)h; }

}  // extern "C"
