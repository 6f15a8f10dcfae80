/*
 * gcdt_reference_surface.h -- the reference's own entry surface, same C++
 * signatures, backed by the B200 solver.
 *
 * yingtix/gCDT declares these stage functions with MSVC forward
 * declarations (`typename Point2d; struct int3;`, include/rawMesh.h:2-3 and
 * the other headers); here the CUDA vector types are included instead.
 * Linking the reference's driver sequence (kernel.cu:5395-5448) against
 * libgcdt_b200.so yields the constrained Delaunay triangulation computed by
 * the B200 path.  Each function establishes the postcondition its stage has
 * in that sequence:
 *
 *   getSamplePoints   one point per 2^22-wide grid cell (256x256 cells over
 *                     the 2^30 box, rawMesh.cu:678-746), cells numbered
 *                     x * 256 + y and the samples in that order as in the
 *                     reference (rawMesh.cu:686); the smallest index of each
 *                     cell (the reference keeps an arbitrary one). (rawMesh.h:6)
 *   rawMeshBefore     triangulation of the samples + 4 box corners
 *                     (corners written at points[n..n+3]); every triangle
 *                     live (sons[t] = -1).                           (rawMesh.h:4)
 *   filterTriangles   compaction of the live triangles (sons == -1) with
 *                     adjacency remapped, as kernel.cu:5293-5324.     (kernel.cu:5293)
 *   delaunaySample    the Delaunay triangulation of points[0..numPoints-4)
 *                     and its adjacency.                              (kernel.cu:5038)
 *   getBitmap         CSR grid: for each cell (X, Y) of the 1024x1024 grid
 *                     over the 2^30 box (the closed square of side 2^20,
 *                     numbered X * 1024 + Y as in the reference), the
 *                     triangles whose closed area meets it, by exact
 *                     integer tests (the reference's boostmap.cu:30-145
 *                     decides the same), in increasing id.    (boostmap.h:4)
 *   rawMeshAfter,     the Delaunay triangulation of all points + corners
 *   rawMesh           with adjacency; every triangle live, so the history
 *                     arrays carry no dead entries.       (rawMesh.h:5, rawMesh.h:7)
 *   addConstraints    the constrained Delaunay triangulation written over
 *                     tris/adjTris; no separate constraint triangles
 *                     (newTris = nullptr, numNewTris = 0).      (addConstraints.h:5-6)
 *   delaunayNew       the constrained Delaunay triangulation of
 *                     points[0..numPoints-4) and cons in the reference's
 *                     returned layout (kernel.cu:4697-4701, 1886-2068):
 *                     `points` and `tris` are replaced by new buffers
 *                     holding the Morton-renumbered points (corners
 *                     included) and the triangles over those numbers sorted
 *                     by centroid code; cons is renumbered in place.  The
 *                     new buffers are cudaMalloc'ed and belong to the
 *                     caller; the replaced ones are left untouched (the
 *                     reference returns them to its own pool).   (kernel.cu:4697)
 *   tryFastDelaunay   the Delaunay triangulation, tris and adjTris in place
 *                     (the reference's host experiment writes nothing).
 *                                                                  (fastDelaunay.h:5)
 *
 * The stages reuse one another's work: a stage whose inputs (points, and
 * segments) are those of the previous solve -- compared by a
 * device-computed fingerprint -- copies that solve's result (delaunaySample
 * after rawMeshBefore, delaunayNew after addConstraints), so the reference's
 * driver sequence costs two full solves (rawMeshAfter without and
 * addConstraints with the segments) plus the sample stages.
 *
 * Pointers are device pointers; out-parameters that receive new buffers
 * (samplePoints, sample, bitmapOffsets, bitmapTris, and delaunayNew's
 * points and tris) are cudaMalloc'ed and belong to the caller (cudaFree).
 * Scratch is pooled inside the library.  Return values are CUDA-event
 * milliseconds, as in the reference, or a negative value on failure (bad
 * input or crossing constraints), with a message on stderr.  Inputs must
 * satisfy the reference's preconditions: distinct points with
 * 0 < x, y < 2^30 - 1 and non-crossing constraints.
 */
#ifndef GCDT_REFERENCE_SURFACE_H
#define GCDT_REFERENCE_SURFACE_H

#include <cstddef>
#include <vector_types.h>

typedef int2 Point2d;

double getSamplePoints(void* cubTemp, size_t cubBytes, Point2d* points, int numPoints,
                       Point2d*& samplePoints, int*& sample, int& num);
double rawMeshBefore(void* cubTempStorage, size_t cubTempStorageBytes, Point2d* points, int3* tris, int* sons,
                     int& numTriangles, int numPoints);
double rawMeshAfter(void* cubTempStorage, size_t cubTempStorageBytes, Point2d* points, int3* tris, int3* adjTris,
                    int* sons, int* bitmapOffsets, int* bitmapTriIds, int& numTriangles, int numPoints);
void rawMesh(void* cubTempStorage, size_t cubTempStorageBytes, Point2d* points, int3* tris, int3* adjTris, int* sons,
             int& numTriangles, int numPoints);
double getBitmap(void* cubTempStorage, size_t cubTempStorageBytes, Point2d* points, int3* tris, int*& bitmapOffsets,
                 int*& bitmapTris, int numTriangles);
double addConstraints(void* cubTemp, size_t cubBytes, Point2d* points, int3* tris, int3* adjTris, int* sons,
                      int* bitmapOffsets, int* bitmapTris, int2* cons, int3*& newTris, int numCons, int numPoints,
                      int numTriangles, int& numNewTris);
double addConstraints(void* cubTemp, size_t cubBytes, Point2d* points, int3* tris, int3* adjTris, int* sons,
                      int2* cons, int numCons, int numPoints, int numTriangles);
double tryFastDelaunay(void* cubTemp, size_t cubBytes, Point2d* points, int3* tris, int3* adjTris, int numPoints,
                       int numTriangles);
double delaunayNew(void* cubTemp, size_t cubBytes, Point2d*& points, int3*& tris, int2* cons, int numPoints,
                   int numTriangles, int numCons);
double delaunaySample(void* cubTemp, size_t cubBytes, Point2d* points, int3* tris, int3* adjTris, int numPoints,
                      int numTriangles);
double filterTriangles(void* cubTemp, size_t cubBytes, int3* tris, int3* newTris, int3* adjTris, int3* newAdjTris,
                       int* sons, int& numTriangles);

#endif /* GCDT_REFERENCE_SURFACE_H */
