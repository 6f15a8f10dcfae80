// reorder.cu -- the reference's output layout for a finished triangulation.
//
// yingtix/gCDT hands its caller the mesh in Morton order: delaunayNew
// (kernel.cu:4697-4701) first renumbers the points by the Morton code of
// (x >> 15, y >> 15) (reorderPoints, kernel.cu:1966-2068; the corners at
// n..n+3 take part) and then sorts the triangles by the Morton code of their
// centroid at the same resolution (reorderFaces, kernel.cu:1886-1964).  Both
// sorts are stable radix sorts of (code, index) pairs, so the point order is
// a pure function of the input.  gcdt_reference_layout applies the same two
// orders to a triangulation in input index order (gcdt_triangulate's output)
// and carries adjacency and constraint flags along, which the reference does
// not return.
//
// Five HBM passes and two 30-bit radix sorts; every pass is a coalesced
// stream over one array plus gathers that follow the Morton-coherent slot
// order, so the gathers mostly hit L2.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <climits>
#include <cstdint>

#include "reorder.cuh"
#include "../../include/gcdt.h"

namespace gcdt_reorder {

constexpr int kBlock = 256;

__global__ void __launch_bounds__(kBlock) k_point_keys(const int2* pts, int n, unsigned* keys, int* vals) {
    int i = blockIdx.x * kBlock + threadIdx.x;
    if (i < n + 4) body_point_key(pts, n, i, keys, vals);
}

__global__ void __launch_bounds__(kBlock) k_point_scatter(const int2* pts, int n, const int* perm,
                                                          int2* out, int* labels) {
    int j = blockIdx.x * kBlock + threadIdx.x;
    if (j < n + 4) body_point_scatter(pts, n, j, perm, out, labels);
}

__global__ void __launch_bounds__(kBlock) k_face_keys(const int2* pts, int n, const int* tris, int nt,
                                                      unsigned* keys, int* vals, int* err) {
    int t = blockIdx.x * kBlock + threadIdx.x;
    if (t >= nt) return;
    int e = body_face_key(pts, n, tris, t, keys, vals);
    if (e) atomicOr(err, e);
}

__global__ void __launch_bounds__(kBlock) k_face_rank(const int* order, int nt, int* newpos) {
    int j = blockIdx.x * kBlock + threadIdx.x;
    if (j < nt) body_face_rank(order, j, newpos);
}

__global__ void __launch_bounds__(kBlock) k_face_gather(const int* tris, const int* adj, const uint8_t* cf,
                                                        int nt, int nv, const int* order, const int* labels,
                                                        const int* newpos, int* tris_out, int* adj_out,
                                                        uint8_t* cf_out, int* err) {
    int j = blockIdx.x * kBlock + threadIdx.x;
    if (j >= nt) return;
    int e = body_face_gather(tris, adj, cf, nt, nv, j, order, labels, newpos, tris_out, adj_out, cf_out);
    if (e) atomicOr(err, e);
}

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

size_t sort_bytes(int items) {
    if (items <= 0) return 0;
    cub::DoubleBuffer<unsigned> dk(nullptr, nullptr);
    cub::DoubleBuffer<int> dv(nullptr, nullptr);
    size_t bytes = 0;
    if (cub::DeviceRadixSort::SortPairs(nullptr, bytes, dk, dv, items, 0, kCodeBits) != cudaSuccess) return 0;
    return bytes;
}

// Scratch regions, each 256-byte aligned: error word, two key buffers and
// two value buffers of max(n+4, n_tris) entries, the triangle rank array,
// then the radix sort's temporary storage.
struct Scratch {
    int* err; unsigned* k0; unsigned* k1; int* v0; int* v1; int* newpos; void* tmp; size_t tmp_bytes;
};

size_t scratch_layout(int n, int nt, char* base, Scratch* s) {
    size_t m = (size_t)((n + 4) > nt ? (n + 4) : nt);
    size_t tmp = sort_bytes(n + 4);
    size_t tf = sort_bytes(nt);
    if (tf > tmp) tmp = tf;
    size_t off = 0;
    auto take = [&](size_t bytes) { char* p = base ? base + off : nullptr; off += align256(bytes); return p; };
    char* e = take(sizeof(int));
    char* k0 = take(4 * m);
    char* k1 = take(4 * m);
    char* v0 = take(4 * m);
    char* v1 = take(4 * m);
    char* np = take(4 * (size_t)nt);
    char* tp = take(tmp);
    if (s) *s = {(int*)e, (unsigned*)k0, (unsigned*)k1, (int*)v0, (int*)v1, (int*)np, tp, tmp};
    return off;
}

bool overlaps(const void* a, size_t na, const void* b, size_t nb) {
    if (!a || !b || !na || !nb) return false;
    uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
    return x < y + nb && y < x + na;
}

}  // namespace gcdt_reorder

using namespace gcdt_reorder;

extern "C" size_t gcdt_reference_layout_scratch_bytes(int32_t n_points, int32_t n_tris) {
    if (n_points < 0 || n_tris < 0 || n_points > INT_MAX - 4 || n_tris > INT_MAX / 3) return 0;
    return scratch_layout(n_points, n_tris, nullptr, nullptr);
}

extern "C" gcdt_status gcdt_reference_layout(const int32_t* d_points, int32_t n,
                                             const int32_t* d_tris, const int32_t* d_adj,
                                             const uint8_t* d_cflags, int32_t n_tris,
                                             int32_t* d_points_out, int32_t* d_labels,
                                             int32_t* d_tris_out, int32_t* d_adj_out, uint8_t* d_cflags_out,
                                             void* d_scratch, size_t scratch_bytes, void* stream) {
    if (n < 0 || n_tris < 0 || n > INT_MAX - 4 || n_tris > INT_MAX / 3) return GCDT_BAD_INPUT;
    if ((n > 0 && !d_points) || !d_points_out || !d_labels || !d_scratch) return GCDT_BAD_INPUT;
    if (n_tris > 0 && (!d_tris || !d_tris_out)) return GCDT_BAD_INPUT;
    if ((d_adj == nullptr) != (d_adj_out == nullptr)) return GCDT_BAD_INPUT;
    if ((d_cflags == nullptr) != (d_cflags_out == nullptr)) return GCDT_BAD_INPUT;
    if (((uintptr_t)d_points & 7) || ((uintptr_t)d_points_out & 7)) return GCDT_BAD_INPUT;   // int2 rows
    if ((uintptr_t)d_scratch & 255) return GCDT_BAD_INPUT;
    size_t need = scratch_layout(n, n_tris, nullptr, nullptr);
    if (scratch_bytes < need) return GCDT_OOM;
    const size_t nv = (size_t)n + 4, t3 = 12 * (size_t)n_tris;
    const void* ins[] = {d_points, d_tris, d_adj, d_cflags, d_scratch};
    const size_t in_bytes[] = {8 * (size_t)n, t3, d_adj ? t3 : 0, d_cflags ? (size_t)n_tris : 0, scratch_bytes};
    const void* outs[] = {d_points_out, d_labels, d_tris_out, d_adj_out, d_cflags_out};
    const size_t out_bytes[] = {8 * nv, 4 * nv, t3, d_adj_out ? t3 : 0, d_cflags_out ? (size_t)n_tris : 0};
    for (int o = 0; o < 5; o++) {
        for (int i = 0; i < 5; i++)
            if (overlaps(outs[o], out_bytes[o], ins[i], in_bytes[i])) return GCDT_BAD_INPUT;
        for (int p = o + 1; p < 5; p++)
            if (overlaps(outs[o], out_bytes[o], outs[p], out_bytes[p])) return GCDT_BAD_INPUT;
    }

    cudaStream_t st = (cudaStream_t)stream;
    Scratch s;
    scratch_layout(n, n_tris, (char*)d_scratch, &s);
    const int2* pts = (const int2*)d_points;
    const int nvi = n + 4;
    cudaError_t e = cudaMemsetAsync(s.err, 0, sizeof(int), st);

    // points: code, stable sort, scatter + labels
    if (e == cudaSuccess) {
        k_point_keys<<<(nvi + kBlock - 1) / kBlock, kBlock, 0, st>>>(pts, n, s.k0, s.v0);
        e = cudaGetLastError();
    }
    cub::DoubleBuffer<unsigned> dk(s.k0, s.k1);
    cub::DoubleBuffer<int> dv(s.v0, s.v1);
    if (e == cudaSuccess) {
        size_t tb = s.tmp_bytes;
        e = cub::DeviceRadixSort::SortPairs(s.tmp, tb, dk, dv, nvi, 0, kCodeBits, st);
    }
    if (e == cudaSuccess) {
        k_point_scatter<<<(nvi + kBlock - 1) / kBlock, kBlock, 0, st>>>(pts, n, dv.Current(), (int2*)d_points_out,
                                                                        d_labels);
        e = cudaGetLastError();
    }
    // triangles: centroid code, stable sort, rank, gather
    if (e == cudaSuccess && n_tris > 0) {
        unsigned grid = (unsigned)((n_tris + kBlock - 1) / kBlock);
        k_face_keys<<<grid, kBlock, 0, st>>>(pts, n, d_tris, n_tris, s.k0, s.v0, s.err);
        e = cudaGetLastError();
        cub::DoubleBuffer<unsigned> fk(s.k0, s.k1);
        cub::DoubleBuffer<int> fv(s.v0, s.v1);
        if (e == cudaSuccess) {
            size_t tb = s.tmp_bytes;
            e = cub::DeviceRadixSort::SortPairs(s.tmp, tb, fk, fv, n_tris, 0, kCodeBits, st);
        }
        if (e == cudaSuccess && d_adj) {
            k_face_rank<<<grid, kBlock, 0, st>>>(fv.Current(), n_tris, s.newpos);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) {
            k_face_gather<<<grid, kBlock, 0, st>>>(d_tris, d_adj, d_cflags, n_tris, nvi, fv.Current(), d_labels,
                                                   s.newpos, d_tris_out, d_adj_out, d_cflags_out, s.err);
            e = cudaGetLastError();
        }
    }
    int h_err = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, s.err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return GCDT_CUDA_ERROR;
    return h_err ? GCDT_BAD_INPUT : GCDT_OK;
}
