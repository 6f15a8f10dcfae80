"""Host restatements of the reference's auxiliary stage functions, the
checkers of the same-signature surface (include/gcdt_reference_surface.h).

TEST INFRASTRUCTURE ONLY: numpy, int64 exact arithmetic.

  sample_points   getSamplePoints, rawMesh.cu:678-746 (samplePoints_s1 puts
                  point i in cell x * 256 + y of the 2^22-wide grid; the
                  cells' points come out in cell order).  The reference keeps
                  whichever point of a cell wrote last; the surface keeps the
                  smallest index, one of the reference's possible results.
  bitmap          getBitmap, boostmap.cu:30-181: for every cell (X, Y) of the
                  1024 x 1024 grid -- the closed square [X a, X a + a - 1] x
                  [Y a, Y a + a - 1], a = 2^20, number X * 1024 + Y -- the
                  triangles meeting it, found as the reference finds them: a
                  cell corner inside the triangle (closed), a triangle edge
                  meeting the square (bounding boxes overlap and the edge's
                  line separates or touches the two corners chosen by its
                  slope), or a vertex in the square.  Listed in increasing
                  triangle id (the reference's order within a cell depends on
                  atomics).
  filter          filterTriangles, kernel.cu:862-893, 5293-5324.
"""
import numpy as np

LOG_RES, LOG_SAMPLE, LOG_BITMAP = 30, 8, 10


def sample_points(xy):
    """-> (sample ids (k,), sample points (k, 2)) in cell order."""
    xy = np.asarray(xy, np.int64).reshape(-1, 2)
    sh = LOG_RES - LOG_SAMPLE
    cell = (xy[:, 0] >> sh) * (1 << LOG_SAMPLE) + (xy[:, 1] >> sh)
    order = np.lexsort((np.arange(len(xy)), cell))
    first = np.ones(len(order), bool)
    first[1:] = cell[order][1:] != cell[order][:-1]
    ids = order[first]
    return ids.astype(np.int32), xy[ids].astype(np.int32)


def _orient(ax, ay, bx, by, cx, cy):
    return np.sign((ax - cx) * (by - cy) - (ay - cy) * (bx - cx))


def _edge_meets_box(ax, ay, bx, by, x0, y0, x1, y1):
    """The reference's segment test (boostmap.cu:30-39), vectorised."""
    out = ((ax < x0) & (bx < x0)) | ((ax > x1) & (bx > x1)) | ((ay < y0) & (by < y0)) | ((ay > y1) & (by > y1))
    f = ((bx >= ax) & (by >= ay)) | ((bx <= ax) & (by <= ay))
    # box corners p[0] = (x0, y0), p[1] = (x1, y0), p[2] = (x1, y1), p[3] = (x0, y1)
    px = np.where(f, x1, x0)
    py = np.where(f, y0, y0)
    qx = np.where(f, x0, x1)
    qy = np.where(f, y1, y1)
    o1 = _orient(ax, ay, bx, by, px, py)
    o2 = _orient(ax, ay, bx, by, qx, qy)
    return ~out & (o1 * o2 <= 0)


def _in_box(px, py, x0, y0, x1, y1):
    return (x0 <= px) & (px <= x1) & (y0 <= py) & (py <= y1)


def bitmap(points, tris, chunk=1 << 18):
    """-> (offsets (2^20 + 1,), triangle list) of the CSR grid."""
    P = np.asarray(points, np.int64).reshape(-1, 2)
    T = np.asarray(tris, np.int64).reshape(-1, 3)
    sh = LOG_RES - LOG_BITMAP
    side = 1 << sh
    ncell = 1 << (2 * LOG_BITMAP)
    keys = []
    for s0 in range(0, len(T), chunk):
        t = np.arange(s0, min(len(T), s0 + chunk))
        a, b, c = P[T[t, 0]], P[T[t, 1]], P[T[t, 2]]
        lo = np.minimum(np.minimum(a, b), c) >> sh
        hi = np.maximum(np.maximum(a, b), c) >> sh
        nx, ny = hi[:, 0] - lo[:, 0] + 1, hi[:, 1] - lo[:, 1] + 1
        cnt = nx * ny
        tid = np.repeat(np.arange(len(t)), cnt)
        start = np.concatenate([[0], np.cumsum(cnt)[:-1]])
        k = np.arange(cnt.sum()) - start[tid]
        X = lo[tid, 0] + k // ny[tid]
        Y = lo[tid, 1] + k % ny[tid]
        x0, y0 = X * side, Y * side
        x1, y1 = x0 + side - 1, y0 + side - 1
        A, B, C = a[tid], b[tid], c[tid]
        hit = np.zeros(len(tid), bool)
        for cx, cy in ((x0, y0), (x1, y0), (x1, y1), (x0, y1)):
            hit |= ((_orient(A[:, 0], A[:, 1], B[:, 0], B[:, 1], cx, cy) >= 0) &
                    (_orient(B[:, 0], B[:, 1], C[:, 0], C[:, 1], cx, cy) >= 0) &
                    (_orient(C[:, 0], C[:, 1], A[:, 0], A[:, 1], cx, cy) >= 0))
        for U, V in ((A, B), (B, C), (C, A)):
            hit |= _edge_meets_box(U[:, 0], U[:, 1], V[:, 0], V[:, 1], x0, y0, x1, y1)
        for U in (A, B, C):
            hit |= _in_box(U[:, 0], U[:, 1], x0, y0, x1, y1)
        cell = X * (1 << LOG_BITMAP) + Y
        keys.append((cell[hit] << 32) | t[tid[hit]])
    keys = np.sort(np.concatenate(keys)) if keys else np.zeros(0, np.int64)
    counts = np.bincount(keys >> 32, minlength=ncell)
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    return offsets, (keys & 0xffffffff).astype(np.int32)


def filter_triangles(tris, adj, sons):
    """Live triangles (sons == -1) compacted in order, neighbours renumbered."""
    tris = np.asarray(tris).reshape(-1, 3)
    live = np.asarray(sons).reshape(-1) == -1
    off = np.cumsum(live) - live
    out_t = tris[live]
    if adj is None:
        return out_t, None
    a = np.asarray(adj, np.int64).reshape(-1, 3)[live]
    return out_t, np.where(a >= 0, off[np.maximum(a, 0)], -1).astype(np.int32)
