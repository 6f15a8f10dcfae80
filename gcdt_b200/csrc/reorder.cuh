// reorder.cuh -- per-item bodies of the reference-layout export
// (gcdt_reference_layout in reorder.cu).  Each body handles one point or
// one triangle and touches no other item's outputs, so the passes give the
// same result in any item order; the GPU runs them one item per thread, the
// host test harness runs them sequentially in several orders.
//
// Codes follow yingtix/gCDT: reorderPoint_s1 (kernel.cu:1966-1984) and
// reorderFace_s1 (kernel.cu:1886-1911), a 15-bit interleave of
// (x >> 15, y >> 15), x bits at even positions (kernel.cu:1904-1908).
#pragma once
#include <cstdint>
#include <vector_types.h>

namespace gcdt_reorder {

constexpr int kBox = (1 << 30) - 1;     // box corners (0,0),(R,0),(R,R),(0,R), rawMesh.cu:5-35
constexpr int kCodeBits = 30;           // 15 interleaved bits per axis

constexpr int ERR_VERTEX = 1;           // a triangle names a vertex outside 0..n+3
constexpr int ERR_NEIGHBOUR = 2;        // a neighbour id outside -1..n_tris-1

// Bit i of v (i < 15) moves to bit 2i; the reference's loop reads exactly
// bits 0..14 of each coordinate.
__host__ __device__ __forceinline__ unsigned spread15(unsigned v) {
    v &= 0x7fffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

__host__ __device__ __forceinline__ unsigned morton(int x, int y) {
    return spread15((unsigned)x) | (spread15((unsigned)y) << 1);
}

// Vertex i of the mesh: the caller's points, then the four box corners.
__host__ __device__ __forceinline__ int2 vertex(const int2* pts, int n, int i) {
    if (i < n) return pts[i];
    int k = i - n;
    int2 r;
    r.x = (k == 1 || k == 2) ? kBox : 0;
    r.y = k >= 2 ? kBox : 0;
    return r;
}

// Point i's code (reorderPoint_s1).
__host__ __device__ __forceinline__ void body_point_key(const int2* pts, int n, int i, unsigned* keys, int* vals) {
    int2 p = vertex(pts, n, i);
    keys[i] = morton(p.x >> 15, p.y >> 15);
    vals[i] = i;
}

// Sorted point j is vertex perm[j]; labels maps a vertex to its new number
// (reorderPoint_s2, kernel.cu:1986-1995).
__host__ __device__ __forceinline__ void body_point_scatter(const int2* pts, int n, int j, const int* perm,
                                                            int2* out, int* labels) {
    int v = perm[j];
    out[j] = vertex(pts, n, v);
    labels[v] = j;
}

// Triangle t's code: the mean of its vertices' (x >> 15, y >> 15), C integer
// division (reorderFace_s1).  Returns ERR_VERTEX (and code 0) for a vertex
// id out of range, which is then never read.
__host__ __device__ __forceinline__ int body_face_key(const int2* pts, int n, const int* tris, int t,
                                                      unsigned* keys, int* vals) {
    const int* r = tris + 3ll * t;
    int a = r[0], b = r[1], c = r[2];
    unsigned nv = (unsigned)(n + 4);
    unsigned code = 0;
    int err = 0;
    if ((unsigned)a < nv && (unsigned)b < nv && (unsigned)c < nv) {
        int2 pa = vertex(pts, n, a), pb = vertex(pts, n, b), pc = vertex(pts, n, c);
        int x = ((pa.x >> 15) + (pb.x >> 15) + (pc.x >> 15)) / 3;
        int y = ((pa.y >> 15) + (pb.y >> 15) + (pc.y >> 15)) / 3;
        code = morton(x, y);
    } else {
        err = ERR_VERTEX;
    }
    keys[t] = code;
    vals[t] = t;
    return err;
}

__host__ __device__ __forceinline__ void body_face_rank(const int* order, int j, int* newpos) {
    newpos[order[j]] = j;
}

// Output triangle j is input triangle order[j] over the new vertex numbers,
// its neighbours renumbered to their new positions (reorderFace_s2 and
// reorderPoint_s3, kernel.cu:1913-1921, 1997-2006).  adj / cf may be null.
__host__ __device__ __forceinline__ int body_face_gather(const int* tris, const int* adj, const uint8_t* cf,
                                                         int nt, int nv, int j, const int* order,
                                                         const int* labels, const int* newpos, int* tris_out,
                                                         int* adj_out, uint8_t* cf_out) {
    long long t = order[j];
    int err = 0;
    for (int k = 0; k < 3; k++) {
        int v = tris[3 * t + k];
        tris_out[3ll * j + k] = (unsigned)v < (unsigned)nv ? labels[v] : -1;
    }
    if (adj) {
        for (int k = 0; k < 3; k++) {
            int a = adj[3 * t + k];
            int m = -1;
            if ((unsigned)a < (unsigned)nt) m = newpos[a];
            else if (a != -1) err = ERR_NEIGHBOUR;
            adj_out[3ll * j + k] = m;
        }
    }
    if (cf) cf_out[j] = cf[t];
    return err;
}

}  // namespace gcdt_reorder
