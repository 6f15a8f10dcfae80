// regions.cuh -- per-item bodies of the region classification
// (gcdt_classify_regions in regions.cu).
//
// depth[t] = the fewest constraint edges a path of triangles crosses from
// the box edge to triangle t; odd depth is inside the constrained polygons
// under the even-odd rule, even depth > 0 is a hole.  (The reference returns
// the whole box triangulation and classifies nothing.)
//
// 1. Components of triangles joined across unconstrained edges, by a
//    lock-free union-find: a union hooks the larger root under the smaller
//    one with a compare-and-swap, finds halve paths.  Every parent is at most
//    its child, so each component's root is its smallest triangle id, in any
//    schedule.
// 2. Breadth-first rounds over components across constrained edges: round
//    L gives every unreached component next to a component of depth L the
//    depth L + 1 (all writers of a round store the same value).
// Every loop is bounded; a bound that runs out reports ERR_LIMIT.
#pragma once
#include <climits>
#include <cstdint>

namespace gcdt_regions {

constexpr int kUnreached = INT_MAX;
constexpr int kMaxSteps = 1 << 26;       // bound of one find / one union's retries

constexpr int ERR_NEIGHBOUR = 1;         // a neighbour id outside -1..n_tris-1
constexpr int ERR_LIMIT = 2;             // a bounded loop ran out

#ifdef __CUDA_ARCH__
// Parent links change under other threads: read them from L2, not L1.
__device__ __forceinline__ int load_link(const int* p) { return __ldcg(p); }
__device__ __forceinline__ int cas_link(int* p, int cmp, int val) { return atomicCAS(p, cmp, val); }
#else
inline int load_link(const int* p) { return *p; }
inline int cas_link(int* p, int cmp, int val) { int o = *p; if (o == cmp) *p = val; return o; }
#endif

// Root of x's tree (path halving), or -1 if the bound ran out.
__host__ __device__ __forceinline__ int uf_find(int* parent, int x) {
    for (int it = 0; it < kMaxSteps; ++it) {
        int p = load_link(parent + x);
        if (p == x) return x;
        int gp = load_link(parent + p);
        if (gp != p) parent[x] = gp;     // gp is an ancestor of x: any interleaving keeps the tree
        x = gp;
    }
    return -1;
}

__host__ __device__ __forceinline__ int uf_union(int* parent, int a, int b) {
    for (int it = 0; it < kMaxSteps; ++it) {
        int ra = uf_find(parent, a), rb = uf_find(parent, b);
        if (ra < 0 || rb < 0) return ERR_LIMIT;
        if (ra == rb) return 0;
        if (ra < rb) { int t = ra; ra = rb; rb = t; }
        if (cas_link(parent + ra, ra, rb) == ra) return 0;
        a = ra;
        b = rb;
    }
    return ERR_LIMIT;
}

__host__ __device__ __forceinline__ void body_init(int t, int* parent, int* level) {
    parent[t] = t;
    level[t] = kUnreached;
}

// Join triangle t with each neighbour of larger id across an unconstrained
// edge (so every edge is joined once); check the neighbour ids.
__host__ __device__ __forceinline__ int body_hook(const int* adj, const uint8_t* cf, int nt, int t, int* parent) {
    int err = 0;
    for (int k = 0; k < 3; k++) {
        int u = adj[3ll * t + k];
        if (u == -1) continue;
        if ((unsigned)u >= (unsigned)nt) { err |= ERR_NEIGHBOUR; continue; }
        if (u > t && !((cf[t] >> k) & 1)) err |= uf_union(parent, t, u);
    }
    return err;
}

// Root of x's tree without changing any link, or -1 if the bound ran out.
__host__ __device__ __forceinline__ int uf_root(const int* parent, int x) {
    for (int it = 0; it < kMaxSteps; ++it) {
        int p = load_link(parent + x);
        if (p == x) return x;
        x = p;
    }
    return -1;
}

// After all unions: point t straight at its root.  The find here must not
// halve paths: a halving store by another thread to parent[t] could land
// after this thread has written the root and leave parent[t] at an inner
// node.  With read-only finds, only thread t writes parent[t], and the trees
// no longer change, so every entry ends at its root.
__host__ __device__ __forceinline__ int body_compress(int t, int* parent) {
    int r = uf_root(parent, t);
    if (r < 0) return ERR_LIMIT;
    parent[t] = r;
    return 0;
}

// Triangles on the box edge seed depth 0 (they all lie in one component:
// segments join input points, which are strictly inside the box).
__host__ __device__ __forceinline__ void body_seed(const int* adj, int t, const int* parent, int* level) {
    const int* a = adj + 3ll * t;
    if (a[0] == -1 || a[1] == -1 || a[2] == -1) level[parent[t]] = 0;
}

// Round L: components at depth L reach their unreached neighbours across
// constrained edges.  Returns 1 if it set any depth.
__host__ __device__ __forceinline__ int body_expand(const int* adj, const uint8_t* cf, int nt, int t, int L,
                                                    const int* parent, int* level) {
    if (level[parent[t]] != L) return 0;
    int changed = 0;
    for (int k = 0; k < 3; k++) {
        int u = adj[3ll * t + k];
        if ((unsigned)u >= (unsigned)nt || !((cf[t] >> k) & 1)) continue;
        int r = parent[u];
        if (level[r] == kUnreached) {
            level[r] = L + 1;
            changed = 1;
        }
    }
    return changed;
}

// Depth of t's component; -1 where no path from the box edge reaches it
// (a mesh with no box edge, or not connected).
__host__ __device__ __forceinline__ void body_depth(int t, const int* parent, const int* level, int* depth) {
    int lv = level[parent[t]];
    depth[t] = lv == kUnreached ? -1 : lv;
}

}  // namespace gcdt_regions
