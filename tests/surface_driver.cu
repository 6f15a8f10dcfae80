// surface_driver.cu -- replays the reference driver's stage sequence
// (yingtix/gCDT kernel.cu:5398-5443) against the same-signature functions of
// include/gcdt_reference_surface.h in libgcdt_b200.so.  Test infrastructure.
//   surface_driver in.bin out.bin   (file formats as oracle/ref_harness.cu)
#include <cstdio>
#include <vector>
#include <cuda_runtime.h>
#include "../include/gcdt_reference_surface.h"

// sample-local vertex ids -> global ids; the sample mesh's corners
// (numSample..numSample+3) become numPoints..numPoints+3
__global__ void to_global(int3* tris, const int* sample, int numSample, int numPoints, int nt) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    int3 v = tris[t];
    int* p = &v.x;
    for (int k = 0; k < 3; ++k) p[k] = p[k] < numSample ? sample[p[k]] : numPoints + (p[k] - numSample);
    tris[t] = v;
}

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    FILE* f = fopen(argv[1], "rb");
    int n = 0, s = 0;
    if (!f || fread(&n, 4, 1, f) != 1 || fread(&s, 4, 1, f) != 1) return 2;
    std::vector<int2> xy(n), cons(s > 0 ? s : 1);
    if (fread(xy.data(), 8, n, f) != (size_t)n || (s > 0 && fread(cons.data(), 8, s, f) != (size_t)s)) return 2;
    fclose(f);
    size_t cubBytes = 64 << 20;
    void* cub = nullptr;
    Point2d* points = nullptr;
    int2* d_cons = nullptr;
    int3 *tris = nullptr, *adj = nullptr;
    int* sons = nullptr;
    const int maxT = 4 * n + 8;
    cudaMalloc(&cub, cubBytes);
    cudaMalloc(&points, 8 * (n + 4));
    cudaMalloc(&d_cons, 8 * (s > 0 ? s : 1));
    cudaMalloc(&tris, 12 * maxT);
    cudaMalloc(&adj, 12 * maxT);
    cudaMalloc(&sons, 4 * maxT);
    cudaMemcpy(points, xy.data(), 8 * n, cudaMemcpyHostToDevice);
    if (s > 0) cudaMemcpy(d_cons, cons.data(), 8 * s, cudaMemcpyHostToDevice);
    double t = 0;
    Point2d* sp = nullptr;
    int* sid = nullptr;
    int ns = 0, nt = 0;
    t += getSamplePoints(cub, cubBytes, points, n, sp, sid, ns);
    t += rawMeshBefore(cub, cubBytes, sp, tris, sons, nt, ns);
    int3* trisSample = nullptr;
    cudaMalloc(&trisSample, 12 * (nt + 8));
    t += filterTriangles(cub, cubBytes, tris, trisSample, nullptr, nullptr, sons, nt);
    t += delaunaySample(cub, cubBytes, sp, trisSample, adj, ns + 4, nt);
    int *bo = nullptr, *bt = nullptr;
    t += getBitmap(cub, cubBytes, sp, trisSample, bo, bt, nt);
    to_global<<<(nt + 127) / 128, 128>>>(trisSample, sid, ns, n, nt);
    cudaMemcpy(tris, trisSample, 12 * nt, cudaMemcpyDeviceToDevice);
    t += rawMeshAfter(cub, cubBytes, points, tris, adj, sons, bo, bt, nt, n);
    int3* consTris = nullptr;
    int nct = 0;
    if (s > 0) t += addConstraints(cub, cubBytes, points, tris, adj, sons, bo, bt, d_cons, consTris, s, n, nt, nct);
    int3 *newTris = nullptr, *newAdj = nullptr;
    cudaMalloc(&newTris, 12 * (nt + nct + 8));
    cudaMalloc(&newAdj, 12 * (nt + 8));
    t += filterTriangles(cub, cubBytes, tris, newTris, adj, newAdj, sons, nt);
    if (nct) cudaMemcpy(newTris + nt, consTris, 12 * nct, cudaMemcpyDeviceToDevice);
    nt += nct;
    t += delaunayNew(cub, cubBytes, points, newTris, s > 0 ? d_cons : nullptr, n + 4, nt, s);
    if (cudaDeviceSynchronize() != cudaSuccess) return 3;
    std::vector<int3> out(nt);
    cudaMemcpy(out.data(), newTris, 12 * nt, cudaMemcpyDeviceToHost);
    printf("samples %d triangles %d stage_ms %f\n", ns, nt, t);
    FILE* g = fopen(argv[2], "wb");
    fwrite(&nt, 4, 1, g);
    fwrite(out.data(), 12, nt, g);
    fclose(g);
    return t < 0 ? 4 : 0;
}
