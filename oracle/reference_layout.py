"""CPU restatement of the reference's output renumbering (numpy).

TEST INFRASTRUCTURE ONLY: the checker for gcdt_reference_layout; imported by
tests/ alone.

yingtix/gCDT's delaunayNew (kernel.cu:4697-4701) renumbers the points and
sorts the triangles before returning them:
  - reorderPoint_s1 (kernel.cu:1966-1984): code = 15-bit interleave of
    (x >> 15, y >> 15), x bits at even positions (kernel.cu:1978-1982);
  - utils::sort: stable radix sort of (code, index) pairs, so equal codes
    keep index order; reorderPoint_s2 (kernel.cu:1986-1995) gathers the
    sorted points and sets labels[old] = new;
  - reorderPoint_s3 (kernel.cu:1997-2006) renumbers the triangle vertices;
  - reorderFace_s1 (kernel.cu:1886-1911): triangle code = interleave of
    ((xa>>15)+(xb>>15)+(xc>>15))/3 and the same for y, C integer division;
    reorderFace_s2 (kernel.cu:1913-1921) gathers the triangles in that
    stable order.
The corners (0,0), (R,0), (R,R), (0,R), R = 2^30-1 (rawMesh.cu:5-35), are
vertices n..n+3 and are renumbered with the points (numPoints = n+4,
kernel.cu:5443).
"""
import numpy as np

R = (1 << 30) - 1


def interleave15(x, y):
    """Bits 0..14 of x to even, of y to odd positions (kernel.cu:1904-1908)."""
    x = np.asarray(x, np.int64)
    y = np.asarray(y, np.int64)
    c = np.zeros(x.shape, np.int64)
    for i in range(15):
        c |= ((x >> i) & 1) << (2 * i)
        c |= ((y >> i) & 1) << (2 * i + 1)
    return c


def vertices(xy):
    """The caller's points followed by the four box corners, int64."""
    xy = np.asarray(xy, np.int64).reshape(-1, 2)
    return np.concatenate([xy, np.array([[0, 0], [R, 0], [R, R], [0, R]], np.int64)])


def point_order(xy):
    """-> (perm, labels): sorted point j is vertex perm[j]; labels[v] is v's
    new number (reorderPoint_s1/_s2)."""
    v = vertices(xy)
    code = interleave15(v[:, 0] >> 15, v[:, 1] >> 15)
    perm = np.argsort(code, kind="stable")
    labels = np.empty(len(v), np.int64)
    labels[perm] = np.arange(len(v))
    return perm, labels


def face_codes(xy, tris):
    """reorderFace_s1: code of the mean of the vertices' (x >> 15, y >> 15)."""
    v = vertices(xy)
    t = np.asarray(tris, np.int64).reshape(-1, 3)
    s = (v[t] >> 15).sum(axis=1)                      # (T, 2)
    mean = np.where(s >= 0, s // 3, -((-s) // 3))     # C division truncates
    return interleave15(mean[:, 0], mean[:, 1])


def reference_layout(xy, tris, adj=None, cflags=None):
    """-> (points (n+4,2), labels (n+4,), tris (T,3), adj (T,3) or None,
    cflags (T,) or None): the mesh renumbered as the reference returns it;
    triangles with equal codes keep their input order."""
    perm, labels = point_order(xy)
    pts = vertices(xy)[perm].astype(np.int32)
    t = np.asarray(tris, np.int64).reshape(-1, 3)
    order = np.argsort(face_codes(xy, t), kind="stable")
    tris_out = labels[t[order]].astype(np.int32)
    adj_out = cf_out = None
    if adj is not None:
        a = np.asarray(adj, np.int64).reshape(-1, 3)[order]
        newpos = np.empty(len(t), np.int64)
        newpos[order] = np.arange(len(t))
        adj_out = np.where(a >= 0, newpos[np.maximum(a, 0)], -1).astype(np.int32)
    if cflags is not None:
        cf_out = np.asarray(cflags, np.uint8).reshape(-1)[order]
    return pts, labels.astype(np.int32), tris_out, adj_out, cf_out
