// ref_harness.cu -- runs the reference's own device pipeline (yingtix/gCDT)
// on one input file.  TEST INFRASTRUCTURE ONLY (built by oracle/build_ref.sh
// together with the reference sources; never part of the product).
//
// The call sequence is the one of the reference driver, kernel.cu:5398-5443:
// getSamplePoints, rawMeshBefore, filterTriangles, delaunaySample, getBitmap,
// convertSample, rawMeshAfter, addConstraints, filterTriangles, append the
// constraint triangles, delaunayNew.  The CUB scratch size is the driver's
// (kernel.cu:5386).
//
//   gcdt_ref <in.bin> <out.bin> [repeat]
// in.bin : int32 n, int32 s, 2n int32 coordinates, 2s int32 segment ends
// out.bin: int32 ntri, 3*ntri int32 triangles (ids into the returned point
//          array), 2(n+4) int32 points in the reference's final (Morton)
//          order, float64 event ms of the last repetition, float64 the
//          reference's own summed stage times
// The reference's own progress lines ("mark ...", "sum ig: ...") go to stdout.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "utils.cuh"
#include "math_base.cuh"
#include "rawMesh.h"
#include "boostmap.h"
#include "addConstraints.h"

double delaunaySample(void* cubTemp, size_t cubBytes, Point2d* points, int3* tris, int3* adjTris,
                      int numPoints, int numTriangles);
double filterTriangles(void* cubTemp, size_t cubBytes, int3* tris, int3* newTris, int3* adjTris,
                       int3* newAdjTris, int* sons, int& numTriangles);
double delaunayNew(void* cubTemp, size_t cubBytes, Point2d*& points, int3*& tris, int2* cons,
                   int numPoints, int numTriangles, int numCons);
__global__ void convertSample(int3* tris, int* sampleId, int numSamples, int numPoints, int numT);

static bool read_all(FILE* f, void* dst, size_t bytes) { return fread(dst, 1, bytes, f) == bytes; }

int main(int argc, char** argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s in.bin out.bin [repeat]\n", argv[0]);
        return 2;
    }
    int repeat = argc > 3 ? atoi(argv[3]) : 1;
    FILE* fi = fopen(argv[1], "rb");
    if (!fi) { perror("input"); return 2; }
    int n = 0, s = 0;
    if (!read_all(fi, &n, 4) || !read_all(fi, &s, 4) || n < 1 || s < 0) { fprintf(stderr, "bad header\n"); return 2; }
    std::vector<int2> xy(n), cons(s > 0 ? s : 1);
    if (!read_all(fi, xy.data(), sizeof(int2) * n) || (s > 0 && !read_all(fi, cons.data(), sizeof(int2) * s))) {
        fprintf(stderr, "short input\n");
        return 2;
    }
    fclose(fi);

    getMemCacheRef().initAbtrtMem();
    size_t cubBytes = 983743231;
    unsigned char* cubTemp = nullptr;
    utils::malloc(cubTemp, (int)cubBytes);

    std::vector<int3> h_tris;
    std::vector<int2> h_points(n + 4);
    int ntri = 0;
    float ms = 0.f;
    double cost = 0.0;
    for (int rep = 0; rep < repeat; ++rep) {
        Point2d* points = nullptr;
        utils::malloc(points, n + 4);
        checkCudaErrors(cudaMemcpy(points, xy.data(), sizeof(int2) * n, cudaMemcpyHostToDevice));
        int2* d_cons = nullptr;
        if (s > 0) {
            utils::malloc(d_cons, s);
            checkCudaErrors(cudaMemcpy(d_cons, cons.data(), sizeof(int2) * s, cudaMemcpyHostToDevice));
        }
        const int maxTriangles = n * 4;
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        checkCudaErrors(cudaDeviceSynchronize());
        cudaEventRecord(e0, 0);
        cost = 0.0;

        Point2d* samplePoints = nullptr;
        int* sampleId = nullptr;
        int numSample = 0;
        cost += getSamplePoints(cubTemp, cubBytes, points, n, samplePoints, sampleId, numSample);
        int3 *tris = nullptr, *adjTris = nullptr;
        int* sons = nullptr;
        int numTriangles = 0;
        utils::malloc(tris, maxTriangles);
        utils::malloc(adjTris, maxTriangles);
        utils::malloc(sons, maxTriangles);
        cost += rawMeshBefore(cubTemp, cubBytes, samplePoints, tris, sons, numTriangles, numSample);
        int3* newTrisSample = nullptr;
        utils::malloc(newTrisSample, numTriangles);
        cost += filterTriangles(cubTemp, cubBytes, tris, newTrisSample, nullptr, nullptr, sons, numTriangles);
        cost += delaunaySample(cubTemp, cubBytes, samplePoints, newTrisSample, adjTris, numSample + 4, numTriangles);
        int *bitmapOffsets = nullptr, *bitmapTris = nullptr;
        cost += getBitmap(cubTemp, cubBytes, samplePoints, newTrisSample, bitmapOffsets, bitmapTris, numTriangles);
        convertSample<<<(numTriangles + 127) / 128, 128>>>(newTrisSample, sampleId, numSample, n, numTriangles);
        checkCudaErrors(cudaMemcpy(tris, newTrisSample, sizeof(int3) * numTriangles, cudaMemcpyDeviceToDevice));
        cost += rawMeshAfter(cubTemp, cubBytes, points, tris, adjTris, sons, bitmapOffsets, bitmapTris, numTriangles, n);
        int3* consTris = nullptr;
        int numConsTris = 0;
        if (s > 0)
            cost += addConstraints(cubTemp, cubBytes, points, tris, adjTris, sons, bitmapOffsets, bitmapTris, d_cons,
                                   consTris, s, n, numTriangles, numConsTris);
        int3 *newTris = nullptr, *newAdjTris = nullptr;
        utils::malloc(newTris, numTriangles);
        utils::malloc(newAdjTris, numTriangles);
        cost += filterTriangles(cubTemp, cubBytes, tris, newTris, adjTris, newAdjTris, sons, numTriangles);
        if (numConsTris != 0)
            checkCudaErrors(cudaMemcpy(newTris + numTriangles, consTris, sizeof(int3) * numConsTris, cudaMemcpyDeviceToDevice));
        numTriangles += numConsTris;
        cost += delaunayNew(cubTemp, cubBytes, points, newTris, d_cons, n + 4, numTriangles, s);

        cudaEventRecord(e1, 0);
        checkCudaErrors(cudaEventSynchronize(e1));
        cudaEventElapsedTime(&ms, e0, e1);
        printf("harness rep %d event_ms %f sum_time %f ntri %d\n", rep, ms, cost, numTriangles);
        fflush(stdout);
        ntri = numTriangles;
        h_tris.resize(ntri);
        checkCudaErrors(cudaMemcpy(h_tris.data(), newTris, sizeof(int3) * ntri, cudaMemcpyDeviceToHost));
        checkCudaErrors(cudaMemcpy(h_points.data(), points, sizeof(int2) * (n + 4), cudaMemcpyDeviceToHost));
    }

    FILE* fo = fopen(argv[2], "wb");
    if (!fo) { perror("output"); return 2; }
    fwrite(&ntri, 4, 1, fo);
    fwrite(h_tris.data(), sizeof(int3), ntri, fo);
    fwrite(h_points.data(), sizeof(int2), n + 4, fo);
    double dms = ms;
    fwrite(&dms, 8, 1, fo);
    fwrite(&cost, 8, 1, fo);
    fclose(fo);
    return 0;
}
