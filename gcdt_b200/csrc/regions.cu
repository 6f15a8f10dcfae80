// regions.cu -- inside/outside classification of a constrained triangulation
// by the even-odd rule (gcdt_classify_regions).  No counterpart in the
// reference, which returns the triangulation of the whole box
// (kernel.cu:5443-5448) and leaves region selection to its caller.
//
// Passes over the triangles (bodies in regions.cuh): init, hook (union-find
// across unconstrained edges), compress, seed, one expand pass per depth
// level, depth.  Each pass reads the adjacency rows (12 B) and flags (1 B)
// of its triangles in order plus the parent / level entries of neighbours,
// which follow the mesh's slot order, coherent along the sort curve; the
// expand rounds number the greatest depth + 1 (2-3 for polygons with holes)
// and each costs one 4-byte device-to-host read of its change flag.
#include <cuda_runtime.h>
#include <climits>
#include <cstdint>

#include "regions.cuh"
#include "../../include/gcdt.h"

namespace gcdt_regions {

constexpr int kBlock = 256;

__global__ void __launch_bounds__(kBlock) k_init(int nt, int* parent, int* level) {
    int t = blockIdx.x * kBlock + threadIdx.x;
    if (t < nt) body_init(t, parent, level);
}

__global__ void __launch_bounds__(kBlock) k_hook(const int* adj, const uint8_t* cf, int nt, int* parent, int* flags) {
    int t = blockIdx.x * kBlock + threadIdx.x;
    if (t >= nt) return;
    int e = body_hook(adj, cf, nt, t, parent);
    if (e) atomicOr(flags, e);
}

__global__ void __launch_bounds__(kBlock) k_compress(int nt, int* parent, int* flags) {
    int t = blockIdx.x * kBlock + threadIdx.x;
    if (t >= nt) return;
    int e = body_compress(t, parent);
    if (e) atomicOr(flags, e);
}

__global__ void __launch_bounds__(kBlock) k_seed(const int* adj, int nt, const int* parent, int* level) {
    int t = blockIdx.x * kBlock + threadIdx.x;
    if (t < nt) body_seed(adj, t, parent, level);
}

__global__ void __launch_bounds__(kBlock) k_expand(const int* adj, const uint8_t* cf, int nt, int L,
                                                   const int* parent, int* level, int* changed) {
    int t = blockIdx.x * kBlock + threadIdx.x;
    if (t < nt && body_expand(adj, cf, nt, t, L, parent, level)) *changed = 1;
}

__global__ void __launch_bounds__(kBlock) k_depth(int nt, const int* parent, const int* level, int* depth) {
    int t = blockIdx.x * kBlock + threadIdx.x;
    if (t < nt) body_depth(t, parent, level, depth);
}

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace gcdt_regions

using namespace gcdt_regions;

// Scratch: flags (error word, then one change word per round parity), the
// parent array and the per-root level array.
extern "C" size_t gcdt_classify_regions_scratch_bytes(int32_t n_tris) {
    if (n_tris < 0 || n_tris > INT_MAX / 3) return 0;
    return 256 + 2 * align256(4 * (size_t)n_tris);
}

extern "C" gcdt_status gcdt_classify_regions(const int32_t* d_adj, const uint8_t* d_cflags, int32_t n_tris,
                                             int32_t* d_depth, int32_t* max_depth, void* d_scratch,
                                             size_t scratch_bytes, void* stream) {
    if (max_depth) *max_depth = 0;
    if (n_tris < 0 || n_tris > INT_MAX / 3) return GCDT_BAD_INPUT;
    if (n_tris == 0) return GCDT_OK;
    if (!d_adj || !d_cflags || !d_depth || !d_scratch || ((uintptr_t)d_scratch & 255)) return GCDT_BAD_INPUT;
    if (scratch_bytes < gcdt_classify_regions_scratch_bytes(n_tris)) return GCDT_OOM;
    char* base = (char*)d_scratch;
    const size_t arr = align256(4 * (size_t)n_tris);
    int* flags = (int*)base;                   // [0] errors, [1..2] change flag of even / odd rounds
    int* parent = (int*)(base + 256);
    int* level = (int*)(base + 256 + arr);
    uintptr_t d0 = (uintptr_t)d_depth, s0 = (uintptr_t)d_scratch;
    if (d0 < s0 + scratch_bytes && s0 < d0 + 4 * (size_t)n_tris) return GCDT_BAD_INPUT;

    cudaStream_t st = (cudaStream_t)stream;
    const unsigned grid = (unsigned)((n_tris + kBlock - 1) / kBlock);
    cudaError_t e = cudaMemsetAsync(flags, 0, 3 * sizeof(int), st);
    if (e == cudaSuccess) { k_init<<<grid, kBlock, 0, st>>>(n_tris, parent, level); e = cudaGetLastError(); }
    if (e == cudaSuccess) { k_hook<<<grid, kBlock, 0, st>>>(d_adj, d_cflags, n_tris, parent, flags); e = cudaGetLastError(); }
    if (e == cudaSuccess) { k_compress<<<grid, kBlock, 0, st>>>(n_tris, parent, flags); e = cudaGetLastError(); }
    if (e == cudaSuccess) { k_seed<<<grid, kBlock, 0, st>>>(d_adj, n_tris, parent, level); e = cudaGetLastError(); }
    int h[3] = {0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, flags, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return GCDT_CUDA_ERROR;
    if (h[0] & ERR_NEIGHBOUR) return GCDT_BAD_INPUT;
    if (h[0]) return GCDT_ITER_LIMIT;

    // Breadth-first rounds; the change flag of round L is cleared in round
    // L-1's stream order, so each round costs one launch and one 4-byte read.
    int L = 0;
    for (;; ++L) {
        if (L >= n_tris) return GCDT_ITER_LIMIT;     // depth never exceeds the triangle count
        int* chg = flags + 1 + (L & 1);
        int* next = flags + 1 + ((L + 1) & 1);
        e = cudaMemsetAsync(next, 0, sizeof(int), st);
        if (e == cudaSuccess) { k_expand<<<grid, kBlock, 0, st>>>(d_adj, d_cflags, n_tris, L, parent, level, chg); e = cudaGetLastError(); }
        int c = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&c, chg, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return GCDT_CUDA_ERROR;
        if (!c) break;
    }
    k_depth<<<grid, kBlock, 0, st>>>(n_tris, parent, level, d_depth);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return GCDT_CUDA_ERROR;
    if (max_depth) *max_depth = L;
    return GCDT_OK;
}
