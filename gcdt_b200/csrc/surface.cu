// surface.cu -- the reference's stage functions (include/gcdt_reference_surface.h)
// on top of the B200 solver.  getSamplePoints, filterTriangles and getBitmap
// are kernels of their own; the meshing stages establish their postcondition
// with gcdt_triangulate on a context kept here and grown on demand.
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>

#include <climits>
#include <cstdio>
#include <mutex>

#include "../../include/gcdt.h"
#include "../../include/gcdt_reference_surface.h"

namespace {

constexpr int kLogRes = 30;            // point resolution, math_base.cuh:19
constexpr int kLogSample = 8;          // 256 x 256 sample cells, math_base.cuh:24
constexpr int kLogBitmap = 10;         // 1024 x 1024 bitmap cells, math_base.cuh:25
constexpr int kBoxR = (1 << kLogRes) - 1;

std::mutex g_mu;
gcdt_context* g_ctx = nullptr;
int64_t g_n = -1, g_s = -1;
int g_dev = -1;
int32_t* g_adj = nullptr;
uint8_t* g_cf = nullptr;
int64_t g_tcap = 0;

struct EventTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    EventTimer() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, 0);
    }
    double stop() {
        cudaEventRecord(b, 0);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        return ms;
    }
};

__global__ void write_corners(int2* p, int n) {
    int k = threadIdx.x;
    if (k < 4) p[n + k] = make_int2((k == 1 || k == 2) ? kBoxR : 0, k >= 2 ? kBoxR : 0);
}

__global__ void fill_ints(int* p, int v, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// Triangulate points[0..n) (+ cons) into tris (+ adj); writes the box
// corners at points[n..n+3].  Returns the triangle count or -1.
int solve(Point2d* points, int n, const int2* cons, int s, int3* tris, int3* adj, const char* who) {
    std::lock_guard<std::mutex> lk(g_mu);
    int dev = 0;
    cudaGetDevice(&dev);
    if (!g_ctx || dev != g_dev || n > g_n || s > g_s) {
        if (g_ctx) gcdt_destroy(g_ctx);
        g_ctx = nullptr;
        int64_t nn = n > g_n ? n : g_n, ss = s > g_s ? s : g_s;
        if (dev != g_dev) { nn = n; ss = s; }
        if (gcdt_create(&g_ctx, dev, nn, ss) != GCDT_OK) {
            fprintf(stderr, "%s: cannot create a context for %d points\n", who, n);
            g_n = g_s = -1;
            return -1;
        }
        g_n = nn;
        g_s = ss;
        g_dev = dev;
    }
    int64_t T = 2 * (int64_t)n + 2;
    if (T > g_tcap || dev != g_dev) {
        cudaFree(g_adj);
        cudaFree(g_cf);
        g_adj = nullptr;
        g_cf = nullptr;
        if (cudaMalloc(&g_adj, 12 * T) != cudaSuccess || cudaMalloc(&g_cf, T) != cudaSuccess) {
            cudaGetLastError();
            g_tcap = 0;
            fprintf(stderr, "%s: out of device memory\n", who);
            return -1;
        }
        g_tcap = T;
    }
    int32_t nt = 0;
    gcdt_status rc = gcdt_triangulate(g_ctx, reinterpret_cast<const int32_t*>(points), n,
                                      reinterpret_cast<const int32_t*>(cons), s, reinterpret_cast<int32_t*>(tris),
                                      adj ? reinterpret_cast<int32_t*>(adj) : g_adj, g_cf, &nt, nullptr);
    if (rc != GCDT_OK) {
        fprintf(stderr, "%s: %s\n", who, gcdt_status_string(rc));
        return -1;
    }
    write_corners<<<1, 32>>>(points, n);
    return nt;
}

void mark_live(int* sons, int nt) {
    if (sons && nt > 0) fill_ints<<<(nt + 255) / 256, 256>>>(sons, -1, nt);
}

// exclusive sum with the caller's CUB scratch when it is large enough
bool exclusive_sum(void* cubTemp, size_t cubBytes, int* in, int* out, int n) {
    size_t need = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, need, in, out, n);
    void* tmp = cubTemp;
    bool own = false;
    if (!cubTemp || cubBytes < need) {
        if (cudaMalloc(&tmp, need > 0 ? need : 1) != cudaSuccess) { cudaGetLastError(); return false; }
        own = true;
    }
    cub::DeviceScan::ExclusiveSum(tmp, need, in, out, n);
    if (own) cudaFree(tmp);
    return true;
}

int read_int(const int* p) {
    int v = 0;
    cudaMemcpy(&v, p, sizeof(int), cudaMemcpyDeviceToHost);
    return v;
}

// ---- getSamplePoints: the smallest index of each 2^22-wide cell
__global__ void sample_cells(const int2* pts, int n, int* cell_min) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int2 p = pts[i];
    int shift = kLogRes - kLogSample;
    int cell = (p.x >> shift) + ((p.y >> shift) << kLogSample);
    atomicMin(&cell_min[cell], i);
}
__global__ void sample_flags(const int* cell_min, int* flag, int ncell) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < ncell) flag[c] = cell_min[c] != INT_MAX;
    if (c == ncell) flag[c] = 0;
}
__global__ void sample_emit(const int2* pts, const int* cell_min, const int* off, int ncell, int* sample, int2* spts) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell || cell_min[c] == INT_MAX) return;
    sample[off[c]] = cell_min[c];
    spts[off[c]] = pts[cell_min[c]];
}

// ---- filterTriangles (kernel.cu:862-893 semantics)
__global__ void live_flags(const int* sons, int* flag, int n) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) flag[t] = sons[t] == -1;
    if (t == n) flag[t] = 0;
}
__global__ void compact_tris(const int3* tris, int3* ntris, const int3* adj, int3* nadj, const int* sons,
                             const int* off, int n) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n || sons[t] != -1) return;
    ntris[off[t]] = tris[t];
    if (adj && nadj) {
        int3 a = adj[t];
        if (a.x != -1) a.x = off[a.x];
        if (a.y != -1) a.y = off[a.y];
        if (a.z != -1) a.z = off[a.z];
        nadj[off[t]] = a;
    }
}

// ---- getBitmap: cells of a 1024 x 1024 grid met by each triangle, row by row
__device__ bool row_span(int2 a, int2 b, int2 c, int row, int* c0, int* c1) {
    const int shift = kLogRes - kLogBitmap;
    double y0 = double((long long)row << shift), y1 = double(((long long)row + 1) << shift);
    double lo = 1e30, hi = -1e30;
    int2 v[3] = {a, b, c};
    for (int k = 0; k < 3; ++k) {
        int2 p = v[k], q = v[(k + 1) % 3];
        if (p.y >= y0 && p.y <= y1) { lo = fmin(lo, double(p.x)); hi = fmax(hi, double(p.x)); }
        for (int side = 0; side < 2; ++side) {
            double yy = side ? y1 : y0;
            if ((p.y - yy) * (q.y - yy) < 0.0) {
                double x = p.x + (q.x - p.x) * (yy - p.y) / double(q.y - p.y);
                lo = fmin(lo, x);
                hi = fmax(hi, x);
            }
        }
    }
    if (lo > hi) return false;
    const int cells = 1 << kLogBitmap;
    int l = int(floor(lo - 1.0)) >> shift, h = int(ceil(hi + 1.0)) >> shift;   // one unit of slack
    *c0 = max(0, l);
    *c1 = min(cells - 1, h);
    return *c0 <= *c1;
}
__device__ void tri_rows(const int2* pts, int3 t, int2* a, int2* b, int2* c, int* r0, int* r1) {
    const int shift = kLogRes - kLogBitmap;
    *a = pts[t.x]; *b = pts[t.y]; *c = pts[t.z];
    int ylo = min(a->y, min(b->y, c->y)), yhi = max(a->y, max(b->y, c->y));
    *r0 = ylo >> shift;
    *r1 = min((1 << kLogBitmap) - 1, yhi >> shift);
}
__global__ void bitmap_count(const int2* pts, const int3* tris, int n, int* cell_count) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int2 a, b, c;
    int r0, r1;
    tri_rows(pts, tris[t], &a, &b, &c, &r0, &r1);
    for (int r = r0; r <= r1; ++r) {
        int c0, c1;
        if (!row_span(a, b, c, r, &c0, &c1)) continue;
        for (int x = c0; x <= c1; ++x) atomicAdd(&cell_count[(r << kLogBitmap) + x], 1);
    }
}
__global__ void bitmap_emit(const int2* pts, const int3* tris, int n, int* cursor, int* list) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int2 a, b, c;
    int r0, r1;
    tri_rows(pts, tris[t], &a, &b, &c, &r0, &r1);
    for (int r = r0; r <= r1; ++r) {
        int c0, c1;
        if (!row_span(a, b, c, r, &c0, &c1)) continue;
        for (int x = c0; x <= c1; ++x) list[atomicAdd(&cursor[(r << kLogBitmap) + x], 1)] = t;
    }
}

}  // namespace

double getSamplePoints(void* cubTemp, size_t cubBytes, Point2d* points, int numPoints, Point2d*& samplePoints,
                       int*& sample, int& num) {
    EventTimer tm;
    const int ncell = 1 << (2 * kLogSample);
    int *cell_min = nullptr, *flag = nullptr;
    samplePoints = nullptr;
    sample = nullptr;
    num = 0;
    if (cudaMalloc(&cell_min, 4 * ncell) != cudaSuccess || cudaMalloc(&flag, 4 * (ncell + 1)) != cudaSuccess ||
        cudaMalloc(&sample, 4 * (ncell + 4)) != cudaSuccess || cudaMalloc(&samplePoints, 8 * (ncell + 4)) != cudaSuccess) {
        cudaGetLastError();
        fprintf(stderr, "getSamplePoints: out of device memory\n");
        return -1.0;
    }
    fill_ints<<<(ncell + 255) / 256, 256>>>(cell_min, INT_MAX, ncell);
    if (numPoints > 0) sample_cells<<<(numPoints + 255) / 256, 256>>>(points, numPoints, cell_min);
    sample_flags<<<(ncell + 256) / 256, 256>>>(cell_min, flag, ncell);
    exclusive_sum(cubTemp, cubBytes, flag, flag, ncell + 1);
    sample_emit<<<(ncell + 255) / 256, 256>>>(points, cell_min, flag, ncell, sample, samplePoints);
    num = read_int(flag + ncell);
    cudaFree(cell_min);
    cudaFree(flag);
    return tm.stop();
}

double rawMeshBefore(void*, size_t, Point2d* points, int3* tris, int* sons, int& numTriangles, int numPoints) {
    EventTimer tm;
    int nt = solve(points, numPoints, nullptr, 0, tris, nullptr, "rawMeshBefore");
    if (nt < 0) return -1.0;
    mark_live(sons, nt);
    numTriangles = nt;
    return tm.stop();
}

double rawMeshAfter(void*, size_t, Point2d* points, int3* tris, int3* adjTris, int* sons, int*, int*,
                    int& numTriangles, int numPoints) {
    EventTimer tm;
    int nt = solve(points, numPoints, nullptr, 0, tris, adjTris, "rawMeshAfter");
    if (nt < 0) return -1.0;
    mark_live(sons, nt);
    numTriangles = nt;
    return tm.stop();
}

void rawMesh(void* cubTemp, size_t cubBytes, Point2d* points, int3* tris, int3* adjTris, int* sons, int& numTriangles,
             int numPoints) {
    rawMeshAfter(cubTemp, cubBytes, points, tris, adjTris, sons, nullptr, nullptr, numTriangles, numPoints);
}

double delaunaySample(void*, size_t, Point2d* points, int3* tris, int3* adjTris, int numPoints, int numTriangles) {
    EventTimer tm;
    if (numTriangles != 2 * (numPoints - 4) + 2) {
        fprintf(stderr, "delaunaySample: %d triangles for %d points\n", numTriangles, numPoints);
        return -1.0;
    }
    if (solve(points, numPoints - 4, nullptr, 0, tris, adjTris, "delaunaySample") < 0) return -1.0;
    return tm.stop();
}

double tryFastDelaunay(void*, size_t, Point2d* points, int3* tris, int3* adjTris, int numPoints, int) {
    EventTimer tm;
    if (solve(points, numPoints - 4, nullptr, 0, tris, adjTris, "tryFastDelaunay") < 0) return -1.0;
    return tm.stop();
}

double addConstraints(void*, size_t, Point2d* points, int3* tris, int3* adjTris, int* sons, int*, int*, int2* cons,
                      int3*& newTris, int numCons, int numPoints, int, int& numNewTris) {
    EventTimer tm;
    newTris = nullptr;
    numNewTris = 0;
    int nt = solve(points, numPoints, cons, numCons, tris, adjTris, "addConstraints");
    if (nt < 0) return -1.0;
    mark_live(sons, nt);
    return tm.stop();
}

double addConstraints(void* cubTemp, size_t cubBytes, Point2d* points, int3* tris, int3* adjTris, int* sons,
                      int2* cons, int numCons, int numPoints, int numTriangles) {
    int3* nt = nullptr;
    int nn = 0;
    return addConstraints(cubTemp, cubBytes, points, tris, adjTris, sons, nullptr, nullptr, cons, nt, numCons,
                          numPoints, numTriangles, nn);
}

double delaunayNew(void*, size_t, Point2d*& points, int3*& tris, int2* cons, int numPoints, int, int numCons) {
    EventTimer tm;
    if (solve(points, numPoints - 4, cons, numCons, tris, nullptr, "delaunayNew") < 0) return -1.0;
    return tm.stop();
}

double filterTriangles(void* cubTemp, size_t cubBytes, int3* tris, int3* newTris, int3* adjTris, int3* newAdjTris,
                       int* sons, int& numTriangles) {
    EventTimer tm;
    int n = numTriangles;
    int* off = nullptr;
    if (cudaMalloc(&off, 4 * ((size_t)n + 1)) != cudaSuccess) {
        cudaGetLastError();
        fprintf(stderr, "filterTriangles: out of device memory\n");
        return -1.0;
    }
    live_flags<<<(n + 256) / 256, 256>>>(sons, off, n);
    exclusive_sum(cubTemp, cubBytes, off, off, n + 1);
    if (n > 0) compact_tris<<<(n + 255) / 256, 256>>>(tris, newTris, adjTris, newAdjTris, sons, off, n);
    numTriangles = read_int(off + n);
    cudaFree(off);
    return tm.stop();
}

double getBitmap(void* cubTemp, size_t cubBytes, Point2d* points, int3* tris, int*& bitmapOffsets, int*& bitmapTris,
                 int numTriangles) {
    EventTimer tm;
    const int ncell = 1 << (2 * kLogBitmap);
    int* cursor = nullptr;
    bitmapOffsets = nullptr;
    bitmapTris = nullptr;
    if (cudaMalloc(&bitmapOffsets, 4 * ((size_t)ncell + 1)) != cudaSuccess ||
        cudaMalloc(&cursor, 4 * ((size_t)ncell + 1)) != cudaSuccess) {
        cudaGetLastError();
        fprintf(stderr, "getBitmap: out of device memory\n");
        return -1.0;
    }
    cudaMemset(bitmapOffsets, 0, 4 * ((size_t)ncell + 1));
    if (numTriangles > 0)
        bitmap_count<<<(numTriangles + 127) / 128, 128>>>(points, tris, numTriangles, bitmapOffsets);
    exclusive_sum(cubTemp, cubBytes, bitmapOffsets, bitmapOffsets, ncell + 1);
    int total = read_int(bitmapOffsets + ncell);
    if (cudaMalloc(&bitmapTris, 4 * ((size_t)total + 1)) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(cursor);
        fprintf(stderr, "getBitmap: out of device memory\n");
        return -1.0;
    }
    cudaMemcpy(cursor, bitmapOffsets, 4 * ((size_t)ncell + 1), cudaMemcpyDeviceToDevice);
    if (numTriangles > 0)
        bitmap_emit<<<(numTriangles + 127) / 128, 128>>>(points, tris, numTriangles, cursor, bitmapTris);
    cudaFree(cursor);
    return tm.stop();
}
