// predicates.cuh -- exact orient2d / incircle for 30-bit integer points.
//
// Reference semantics (yingtix/gCDT include/math_base.cuh):
//   orient2d(a,b,c) = sign((a.x-c.x)(b.y-c.y) - (a.y-c.y)(b.x-c.x))      (68-76)
//   inCircle(a,b,c,p) = sign of | ap.x ap.y |ap|^2 ; bp.. ; cp.. |         (267-328)
//       > 0  <=>  p strictly inside the circumcircle of CCW (a,b,c).
// The reference evaluates inCircle with a vendored multi-word integer type
// (include/intX_t.cuh).  Here coordinates are < 2^30, so every difference fits
// in 31 bits, every lifted term in 61 bits and the determinant in 124 bits:
// orient2d is exact in int64 and inCircle is exact in native __int128.
//
// inCircle runs a floating-point filter first: the determinant is evaluated
// in double and accepted when its magnitude exceeds Shewchuk's static bound
// for this expression (errboundA = (10 + 96 eps) eps times the permanent,
// J. R. Shewchuk, "Adaptive Precision Floating-Point Arithmetic and Fast
// Robust Geometric Predicates", 1997).  Otherwise the exact __int128
// evaluation decides, so every returned sign equals the exact sign.
//
// incircle_sos() adds the symbolic tie-break shared with the oracle: point i
// is lifted to |p_i|^2 + eps_i with eps larger for lexicographically larger
// (x, y).  An exactly cocircular quadruple then resolves to the sign of the
// cofactor of its highest-priority point, which makes the (constrained)
// Delaunay triangulation unique.
#pragma once
#include <cstdint>

namespace gcdt {

__host__ __device__ __forceinline__ int orient2d(int2 a, int2 b, int2 c) {
    long long o1 = (long long)(a.x - c.x) * (long long)(b.y - c.y);
    long long o2 = (long long)(a.y - c.y) * (long long)(b.x - c.x);
    return (o1 > o2) - (o1 < o2);
}

__host__ __device__ __forceinline__ int incircle_exact(int2 a, int2 b, int2 c, int2 d) {
    long long adx = a.x - d.x, ady = a.y - d.y;
    long long bdx = b.x - d.x, bdy = b.y - d.y;
    long long cdx = c.x - d.x, cdy = c.y - d.y;
    long long al = adx * adx + ady * ady;
    long long bl = bdx * bdx + bdy * bdy;
    long long cl = cdx * cdx + cdy * cdy;
    long long bc = bdx * cdy - cdx * bdy;
    long long ca = cdx * ady - adx * cdy;
    long long ab = adx * bdy - bdx * ady;
    __int128 det = (__int128)al * bc + (__int128)bl * ca + (__int128)cl * ab;
    return (det > 0) - (det < 0);
}

// Filtered incircle; returns the exact sign.
__host__ __device__ __forceinline__ int incircle(int2 a, int2 b, int2 c, int2 d) {
    double adx = double(a.x - d.x), ady = double(a.y - d.y);
    double bdx = double(b.x - d.x), bdy = double(b.y - d.y);
    double cdx = double(c.x - d.x), cdy = double(c.y - d.y);
    double bdxcdy = bdx * cdy, cdxbdy = cdx * bdy;
    double cdxady = cdx * ady, adxcdy = adx * cdy;
    double adxbdy = adx * bdy, bdxady = bdx * ady;
    double alift = adx * adx + ady * ady;
    double blift = bdx * bdx + bdy * bdy;
    double clift = cdx * cdx + cdy * cdy;
    double det = alift * (bdxcdy - cdxbdy) + blift * (cdxady - adxcdy) + clift * (adxbdy - bdxady);
    double perm = (fabs(bdxcdy) + fabs(cdxbdy)) * alift + (fabs(cdxady) + fabs(adxcdy)) * blift +
                  (fabs(adxbdy) + fabs(bdxady)) * clift;
    // (10 + 96 eps) eps with eps = 2^-53
    const double errA = 1.1102230246251577e-15;
    double bound = errA * perm;
    if (det > bound) return 1;
    if (-det > bound) return -1;
    return incircle_exact(a, b, c, d);
}

__host__ __device__ __forceinline__ bool prio_gt(int2 p, int2 q) {
    return p.x > q.x || (p.x == q.x && p.y > q.y);
}

// Perturbed incircle for a CCW triangle (a,b,c); never returns 0.
__host__ __device__ __forceinline__ int incircle_sos(int2 a, int2 b, int2 c, int2 d) {
    int s = incircle(a, b, c, d);
    if (s) return s;
    int2 v[4] = {a, b, c, d};
    int coef[4];
    coef[0] = orient2d(b, c, d);
    coef[1] = orient2d(c, a, d);
    coef[2] = orient2d(a, b, d);
    coef[3] = -orient2d(a, b, c);
    unsigned used = 0;
    for (int k = 0; k < 4; ++k) {
        int best = -1;
        for (int i = 0; i < 4; ++i)
            if (!(used >> i & 1) && (best < 0 || prio_gt(v[i], v[best]))) best = i;
        used |= 1u << best;
        if (coef[best]) return coef[best];
    }
    return 0;
}

}  // namespace gcdt
