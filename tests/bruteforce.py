"""Independent brute-force definitions used to pin the oracle on small inputs.

Everything here is plain Python integer arithmetic, written from the
definitions rather than from the oracle's code:
  - orient / inCircle exactly as in the reference (yingtix/gCDT
    include/math_base.cuh:68-76, 267-328);
  - the symbolic tie-break (lift x^2+y^2+eps_i, eps larger for larger (x, y));
  - the global empty-circumcircle property of a (constrained) Delaunay
    triangulation, checked triangle against every vertex.
"""
R = (1 << 30) - 1


def with_corners(xy):
    pts = [(int(x), int(y)) for x, y in xy]
    return pts + [(0, 0), (R, 0), (R, R), (0, R)]


def orient(a, b, c):
    v = (a[0] - c[0]) * (b[1] - c[1]) - (a[1] - c[1]) * (b[0] - c[0])
    return (v > 0) - (v < 0)


def incircle(a, b, c, d):
    adx, ady = a[0] - d[0], a[1] - d[1]
    bdx, bdy = b[0] - d[0], b[1] - d[1]
    cdx, cdy = c[0] - d[0], c[1] - d[1]
    det = ((adx * adx + ady * ady) * (bdx * cdy - cdx * bdy)
           + (bdx * bdx + bdy * bdy) * (cdx * ady - adx * cdy)
           + (cdx * cdx + cdy * cdy) * (adx * bdy - bdx * ady))
    return (det > 0) - (det < 0)


def incircle_sos(a, b, c, d):
    s = incircle(a, b, c, d)
    if s:
        return s
    terms = [(a, orient(b, c, d)), (b, orient(c, a, d)), (c, orient(a, b, d)), (d, -orient(a, b, c))]
    for _, coef in sorted(terms, key=lambda t: t[0], reverse=True):
        if coef:
            return coef
    return 0


def _proper_cross(p, q, r, s):
    return (orient(p, q, r) * orient(p, q, s) < 0) and (orient(r, s, p) * orient(r, s, q) < 0)


def check_empty_circles(xy, tris, cons=()):
    """Return the list of (triangle index, vertex) violations of the global
    (constrained) empty-circle property.  A vertex hidden from the
    triangle's centroid by a constraint segment does not count."""
    pts = with_corners(xy)
    segs = [(pts[a], pts[b]) for a, b in cons]
    bad = []
    for k, (a, b, c) in enumerate(tris):
        A, B, C = pts[a], pts[b], pts[c]
        # centroid scaled by 3 to stay integral; scale the other points to match
        G = (A[0] + B[0] + C[0], A[1] + B[1] + C[1])
        for v, P in enumerate(pts):
            if v in (a, b, c):
                continue
            if incircle_sos(A, B, C, P) <= 0:
                continue
            if segs:
                P3 = (3 * P[0], 3 * P[1])
                hidden = any(_proper_cross(G, P3, (3 * s0[0], 3 * s0[1]), (3 * s1[0], 3 * s1[1]))
                             for s0, s1 in segs)
                if hidden:
                    continue
            bad.append((k, v))
    return bad
