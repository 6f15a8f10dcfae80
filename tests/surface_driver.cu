// surface_driver.cu -- replays the reference driver's stage sequence
// (yingtix/gCDT kernel.cu:5398-5443) against the same-signature functions of
// include/gcdt_reference_surface.h in libgcdt_b200.so.  Test infrastructure.
//
//   surface_driver in.bin out.bin [runs]
//
// in.bin: int32 n, int32 s, 2n int32 coordinates, 2s int32 segment ends.
// The sequence runs `runs` times (default 3) on the same input, each timed
// with one cudaEvent pair around the whole sequence; the last run also
// writes its stage outputs to out.bin as sections (int32 tag, int64 byte
// count, bytes), so the run before it gives the reported times.  Tags:
//   1 sample ids          2 sample points (+4 corners)   3 sample mesh tris
//   4 sample mesh adj     5 bitmap offsets               6 bitmap triangles
//   7 rawMeshAfter tris   8 rawMeshAfter adj             9 addConstraints tris
//  10 addConstraints adj 11 filterTriangles tris        12 filterTriangles adj
//  13 delaunayNew points 14 delaunayNew tris            15 segments after delaunayNew
//  16 tryFastDelaunay tris 17 tryFastDelaunay adj       18 rawMesh tris
//  19 float64 [sequence ms, sum of stage returns, getSamplePoints, rawMeshBefore,
//     filterTriangles, delaunaySample, getBitmap, rawMeshAfter, addConstraints,
//     filterTriangles, delaunayNew] of the run before the last
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>
#include "../include/gcdt_reference_surface.h"

// sample-local vertex ids -> global ids; the sample mesh's corners
// (numSample..numSample+3) become numPoints..numPoints+3 (the reference's
// convertSample, kernel.cu:833-860)
__global__ void to_global(int3* tris, const int* sample, int numSample, int numPoints, int nt) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    int3 v = tris[t];
    int* p = &v.x;
    for (int k = 0; k < 3; ++k) p[k] = p[k] < numSample ? sample[p[k]] : numPoints + (p[k] - numSample);
    tris[t] = v;
}

static FILE* g_out = nullptr;
static void section(int tag, const void* dptr, long long bytes, bool device = true) {
    std::vector<char> h((size_t)(bytes > 0 ? bytes : 0));
    if (bytes > 0) {
        if (device) cudaMemcpy(h.data(), dptr, (size_t)bytes, cudaMemcpyDeviceToHost);
        else memcpy(h.data(), dptr, (size_t)bytes);
    }
    fwrite(&tag, 4, 1, g_out);
    fwrite(&bytes, 8, 1, g_out);
    if (bytes > 0) fwrite(h.data(), 1, (size_t)bytes, g_out);
}

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    const int runs = argc > 3 ? atoi(argv[3]) : 3;
    FILE* f = fopen(argv[1], "rb");
    int n = 0, s = 0;
    if (!f || fread(&n, 4, 1, f) != 1 || fread(&s, 4, 1, f) != 1) return 2;
    std::vector<int2> xy(n), cons(s > 0 ? s : 1);
    if (fread(xy.data(), 8, n, f) != (size_t)n || (s > 0 && fread(cons.data(), 8, s, f) != (size_t)s)) return 2;
    fclose(f);
    size_t cubBytes = 64 << 20;
    void* cub = nullptr;
    Point2d* points0 = nullptr;
    int2* d_cons = nullptr;
    int3 *tris = nullptr, *adj = nullptr;
    int* sons = nullptr;
    const int maxT = 4 * n + 8;
    cudaMalloc(&cub, cubBytes);
    cudaMalloc(&points0, 8 * ((size_t)n + 4));
    cudaMalloc(&d_cons, 8 * (size_t)(s > 0 ? s : 1));
    cudaMalloc(&tris, 12 * (size_t)maxT);
    cudaMalloc(&adj, 12 * (size_t)maxT);
    cudaMalloc(&sons, 4 * (size_t)maxT);
    // the caller's own buffers, allocated once as the reference driver's
    // MemCache pre-pool would hand them out (no allocation inside the timing)
    int3 *trisSample = nullptr, *newTris = nullptr, *newAdj = nullptr;
    cudaMalloc(&trisSample, 12 * (size_t)maxT);
    cudaMalloc(&newTris, 12 * (size_t)maxT);
    cudaMalloc(&newAdj, 12 * (size_t)maxT);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int rc = 0;
    double times[11] = {0};
    for (int run = 0; run < runs; ++run) {
        const bool last = run == runs - 1;
        cudaMemcpy(points0, xy.data(), 8 * (size_t)n, cudaMemcpyHostToDevice);
        if (s > 0) cudaMemcpy(d_cons, cons.data(), 8 * (size_t)s, cudaMemcpyHostToDevice);
        Point2d* points = points0;
        if (last) {
            g_out = fopen(argv[2], "wb");
            if (!g_out) return 2;
        }
        double st[9] = {0};
        cudaDeviceSynchronize();
        cudaEventRecord(e0, 0);
        Point2d* sp = nullptr;
        int* sid = nullptr;
        int ns = 0, nt = 0;
        st[0] = getSamplePoints(cub, cubBytes, points, n, sp, sid, ns);
        st[1] = rawMeshBefore(cub, cubBytes, sp, tris, sons, nt, ns);
        st[2] = filterTriangles(cub, cubBytes, tris, trisSample, nullptr, nullptr, sons, nt);
        st[3] = delaunaySample(cub, cubBytes, sp, trisSample, adj, ns + 4, nt);
        if (last) {
            section(1, sid, 4LL * ns);
            section(2, sp, 8LL * (ns + 4));
            section(3, trisSample, 12LL * nt);
            section(4, adj, 12LL * nt);
        }
        int *bo = nullptr, *bt = nullptr;
        st[4] = getBitmap(cub, cubBytes, sp, trisSample, bo, bt, nt);
        if (last) {
            int total = 0;
            cudaMemcpy(&total, bo + (1 << 20), 4, cudaMemcpyDeviceToHost);
            section(5, bo, 4LL * ((1 << 20) + 1));
            section(6, bt, 4LL * total);
        }
        to_global<<<(nt + 127) / 128, 128>>>(trisSample, sid, ns, n, nt);
        cudaMemcpy(tris, trisSample, 12 * (size_t)nt, cudaMemcpyDeviceToDevice);
        st[5] = rawMeshAfter(cub, cubBytes, points, tris, adj, sons, bo, bt, nt, n);
        if (last) {
            section(7, tris, 12LL * nt);
            section(8, adj, 12LL * nt);
        }
        int3* consTris = nullptr;
        int nct = 0;
        if (s > 0) st[6] = addConstraints(cub, cubBytes, points, tris, adj, sons, bo, bt, d_cons, consTris, s, n, nt, nct);
        if (last) {
            section(9, tris, 12LL * nt);
            section(10, adj, 12LL * nt);
        }
        st[7] = filterTriangles(cub, cubBytes, tris, newTris, adj, newAdj, sons, nt);
        if (last) {
            section(11, newTris, 12LL * nt);
            section(12, newAdj, 12LL * nt);
        }
        if (nct) cudaMemcpy(newTris + nt, consTris, 12 * (size_t)nct, cudaMemcpyDeviceToDevice);
        nt += nct;
        int3* finalTris = newTris;
        st[8] = delaunayNew(cub, cubBytes, points, finalTris, s > 0 ? d_cons : nullptr, n + 4, nt, s);
        cudaEventRecord(e1, 0);
        if (cudaEventSynchronize(e1) != cudaSuccess) return 3;
        float seq_ms = 0.f;
        cudaEventElapsedTime(&seq_ms, e0, e1);
        double sum = 0;
        for (double v : st) {
            if (v < 0) rc = 4;
            sum += v;
        }
        if (!last || runs == 1) {
            const double t[11] = {seq_ms, sum, st[0], st[1], st[2], st[3], st[4], st[5], st[6], st[7], st[8]};
            for (int k = 0; k < 11; ++k) times[k] = t[k];
        }
        if (last) {
            section(13, points, 8LL * (n + 4));
            section(14, finalTris, 12LL * nt);
            section(15, d_cons, 8LL * s);
            // the other two meshing entry points, on the original points
            cudaMemcpy(points0, xy.data(), 8 * (size_t)n, cudaMemcpyHostToDevice);
            int nt2 = 2 * n + 2;
            if (tryFastDelaunay(cub, cubBytes, points0, tris, adj, n + 4, nt2) < 0) rc = 5;
            section(16, tris, 12LL * nt2);
            section(17, adj, 12LL * nt2);
            int nt3 = 0;
            rawMesh(cub, cubBytes, points0, tris, adj, sons, nt3, n);
            section(18, tris, 12LL * nt3);
            section(19, times, sizeof(times), false);
            fclose(g_out);
            printf("samples %d triangles %d sequence_ms %f stage_ms %f\n", ns, nt, times[0], times[1]);
        }
        // buffers the stages handed over (the reference leaves them to its
        // pool); the surface documents cudaFree for them
        void* handed[] = {sp, sid, bo, bt, finalTris != newTris ? finalTris : nullptr,
                          points != points0 ? points : nullptr};
        for (void* p : handed)
            if (p && cudaFree(p) != cudaSuccess) rc = 6;
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return 3;
    return rc;
}
