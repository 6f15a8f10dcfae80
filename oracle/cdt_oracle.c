/*
 * cdt_oracle.c -- CPU oracle for the gCDT hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path in
 * gcdt_b200/csrc; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  The product never links or calls it.
 *
 * What it restates (reference = yingtix/gCDT):
 *   - points are int2 with 30-bit resolution, R = 2^30-1   (include/math_base.cuh:19-29)
 *   - the 4 box corners (0,0),(R,0),(R,R),(0,R) stored at points[N..N+3],
 *     and the two root triangles (N,N+1,N+3),(N+1,N+2,N+3) (rawMesh.cu:5-22)
 *   - orient2d = sign((a-c) x (b-c)), exact                  (math_base.cuh:68-76)
 *   - inCircle = sign of the 3x3 lifted determinant relative to p,
 *     > 0 iff p is strictly inside the circle of CCW abc     (math_base.cuh:267-328)
 *   - triangle (x,y,z) is CCW; adj.x is the neighbour across the edge
 *     opposite x, -1 = none                                  (rawMesh.cu:16-21, 269-276)
 *   - an edge is flipped iff inCircle > 0                    (kernel.cu:2218-2219, 3679)
 *   - constraint edges are never flipped                      (kernel.cu:2203-2205, 3670)
 *
 * Algorithm (sequential, deliberately different from the GPU path):
 *   1. insert points one at a time in Morton order, locating by a visibility
 *      walk from the previous point and restoring Delaunay by Lawson flips;
 *   2. insert each constraint segment by Sloan's flip method (edges crossing
 *      the segment are flipped until the segment is an edge); a segment that
 *      passes exactly through a vertex is split there;
 *   3. run a global constrained Lawson pass until every unconstrained edge is
 *      locally Delaunay.
 *
 * Tie-break.  Cocircular quadruples make the Delaunay triangulation
 * non-unique, and the reference keeps whichever diagonal it happens to hold.
 * The oracle and the CUDA path both use the same symbolic perturbation of the
 * lifting map (simulation of simplicity, Edelsbrunner & Muecke 1990): point i
 * is lifted to x^2+y^2+eps_i, with eps_i larger for points that are larger in
 * (x, y) lexicographic order.  The perturbed constrained Delaunay
 * triangulation is unique, so on every input -- lattice included -- any
 * correct algorithm must return the same triangle set.  On inputs in general
 * position (no exactly cocircular quadruple) the perturbation never fires and
 * the result is the ordinary CDT the reference computes.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

typedef __int128 i128;

#define ORACLE_R ((int64_t)((1 << 30) - 1))

enum { OK = 0, BAD_INPUT = 1, OOM = 2, ITER_LIMIT = 3, CONSTRAINT_FAIL = 4 };

typedef struct {
    int n, nv;           /* input points, n + 4 corners */
    int64_t *px, *py;    /* coordinates, corners at n..n+3 */
    int ntri, cap;
    int32_t *tv;         /* 3 vertices per triangle, CCW */
    int32_t *tn;         /* neighbour across the edge opposite each vertex */
    uint8_t *tc;         /* bit k: edge opposite vertex k is constrained */
    int32_t *vt;         /* vertex -> one incident triangle */
    int64_t *stack; int64_t sp, scap;   /* (tri<<2|slot) work stack */
    long long flips;
} mesh_t;

/* ---------------------------------------------------------------- predicates */

int oracle_orient(int64_t ax, int64_t ay, int64_t bx, int64_t by, int64_t cx, int64_t cy)
{
    /* math_base.cuh:68-76: o1 = (a.x-c.x)(b.y-c.y), o2 = (a.y-c.y)(b.x-c.x) */
    int64_t o1 = (ax - cx) * (by - cy);
    int64_t o2 = (ay - cy) * (bx - cx);
    return (o1 > o2) - (o1 < o2);
}

int oracle_incircle(int64_t ax, int64_t ay, int64_t bx, int64_t by,
                    int64_t cx, int64_t cy, int64_t dx, int64_t dy)
{
    /* math_base.cuh:267-328, same determinant, evaluated in native 128-bit */
    int64_t adx = ax - dx, ady = ay - dy;
    int64_t bdx = bx - dx, bdy = by - dy;
    int64_t cdx = cx - dx, cdy = cy - dy;
    i128 al = (i128)(adx * adx) + (i128)(ady * ady);
    i128 bl = (i128)(bdx * bdx) + (i128)(bdy * bdy);
    i128 cl = (i128)(cdx * cdx) + (i128)(cdy * cdy);
    i128 ab = (i128)(adx * bdy - bdx * ady);
    i128 bc = (i128)(bdx * cdy - cdx * bdy);
    i128 ca = (i128)(cdx * ady - adx * cdy);
    i128 det = al * bc + bl * ca + cl * ab;
    return (det > 0) - (det < 0);
}

static inline int prio_gt(const mesh_t *m, int p, int q)
{
    return m->px[p] > m->px[q] || (m->px[p] == m->px[q] && m->py[p] > m->py[q]);
}

static inline int orient_v(const mesh_t *m, int a, int b, int c)
{
    return oracle_orient(m->px[a], m->py[a], m->px[b], m->py[b], m->px[c], m->py[c]);
}

/* Perturbed incircle: never 0 when a,b,c is a proper CCW triangle.
   With z_i = |p_i|^2 + eps_i the determinant gains
   eps_a*orient(b,c,d) + eps_b*orient(c,a,d) + eps_c*orient(a,b,d) - eps_d*orient(a,b,c);
   the sign is that of the term of the highest-priority point whose
   coefficient is non-zero. */
static int incircle_sos_v(const mesh_t *m, int a, int b, int c, int d)
{
    int s = oracle_incircle(m->px[a], m->py[a], m->px[b], m->py[b],
                            m->px[c], m->py[c], m->px[d], m->py[d]);
    if (s) return s;
    int v[4] = {a, b, c, d};
    int coef[4];
    coef[0] = orient_v(m, b, c, d);
    coef[1] = orient_v(m, c, a, d);
    coef[2] = orient_v(m, a, b, d);
    coef[3] = -orient_v(m, a, b, c);
    int used[4] = {0, 0, 0, 0};
    for (int k = 0; k < 4; ++k) {
        int best = -1;
        for (int i = 0; i < 4; ++i)
            if (!used[i] && (best < 0 || prio_gt(m, v[i], v[best]))) best = i;
        used[best] = 1;
        if (coef[best]) return coef[best];
    }
    return 0;
}

int oracle_incircle_sos(const int64_t *xy4)
{
    mesh_t m; int64_t px[4], py[4];
    for (int i = 0; i < 4; ++i) { px[i] = xy4[2 * i]; py[i] = xy4[2 * i + 1]; }
    m.px = px; m.py = py;
    return incircle_sos_v(&m, 0, 1, 2, 3);
}

/* The three predicates of n cases: quads holds 8 int32 per case (points a,
   b, c, d); out receives orient2d(a,b,c), incircle(a,b,c,d) and the
   perturbed incircle(a,b,c,d), 3 int32 per case -- the layout of the
   device's gcdt_eval_predicates. */
void oracle_predicates_batch(const int32_t *quads, int64_t n, int32_t *out)
{
    for (int64_t i = 0; i < n; ++i) {
        const int32_t *q = quads + 8 * i;
        int64_t xy4[8];
        for (int k = 0; k < 8; ++k) xy4[k] = q[k];
        out[3 * i] = oracle_orient(xy4[0], xy4[1], xy4[2], xy4[3], xy4[4], xy4[5]);
        out[3 * i + 1] = oracle_incircle(xy4[0], xy4[1], xy4[2], xy4[3], xy4[4], xy4[5], xy4[6], xy4[7]);
        out[3 * i + 2] = oracle_incircle_sos(xy4);
    }
}

/* ---------------------------------------------------------------- mesh ops */

static int push(mesh_t *m, int t, int s)
{
    if (m->sp == m->scap) {
        int64_t nc = m->scap ? m->scap * 2 : 1024;
        int64_t *ns = (int64_t *)realloc(m->stack, (size_t)nc * sizeof(int64_t));
        if (!ns) return OOM;
        m->stack = ns; m->scap = nc;
    }
    m->stack[m->sp++] = ((int64_t)t << 2) | s;
    return OK;
}

static inline int slot_of(const mesh_t *m, int t, int v)
{
    const int32_t *T = m->tv + 3 * t;
    return T[0] == v ? 0 : (T[1] == v ? 1 : 2);
}

static inline int nb_slot(const mesh_t *m, int n, int t)
{
    const int32_t *N = m->tn + 3 * n;
    return N[0] == t ? 0 : (N[1] == t ? 1 : 2);
}

static inline void set_tri(mesh_t *m, int t, int a, int b, int c, int na, int nb, int nc, int flags)
{
    int32_t *T = m->tv + 3 * t, *N = m->tn + 3 * t;
    T[0] = a; T[1] = b; T[2] = c;
    N[0] = na; N[1] = nb; N[2] = nc;
    m->tc[t] = (uint8_t)flags;
    m->vt[a] = t; m->vt[b] = t; m->vt[c] = t;
}

static inline void repoint(mesh_t *m, int nbr, int from, int to)
{
    if (nbr >= 0) m->tn[3 * nbr + nb_slot(m, nbr, from)] = to;
}

/* Flip the edge opposite slot i of t.  t=(A,B,C), n=(D,C,B) across BC.
   Afterwards t=(A,B,D) and n=(A,D,C); A sits in slot 0 of both. */
static void flip(mesh_t *m, int t, int i)
{
    int A = m->tv[3 * t + i], B = m->tv[3 * t + (i + 1) % 3], C = m->tv[3 * t + (i + 2) % 3];
    int n = m->tn[3 * t + i];
    int j = nb_slot(m, n, t);
    int D = m->tv[3 * n + j];
    int nCA = m->tn[3 * t + (i + 1) % 3], fCA = (m->tc[t] >> ((i + 1) % 3)) & 1;
    int nAB = m->tn[3 * t + (i + 2) % 3], fAB = (m->tc[t] >> ((i + 2) % 3)) & 1;
    int nBD = m->tn[3 * n + (j + 1) % 3], fBD = (m->tc[n] >> ((j + 1) % 3)) & 1;
    int nDC = m->tn[3 * n + (j + 2) % 3], fDC = (m->tc[n] >> ((j + 2) % 3)) & 1;
    set_tri(m, t, A, B, D, nBD, n, nAB, fBD | (fAB << 2));
    set_tri(m, n, A, D, C, nDC, nCA, t, fDC | (fCA << 1));
    repoint(m, nBD, n, t);
    repoint(m, nCA, t, n);
    m->flips++;
}

static int legal_edge(const mesh_t *m, int t, int i)
{
    int n = m->tn[3 * t + i];
    if (n < 0 || ((m->tc[t] >> i) & 1)) return 1;
    int j = nb_slot(m, n, t);
    int D = m->tv[3 * n + j];
    const int32_t *T = m->tv + 3 * t;
    return incircle_sos_v(m, T[0], T[1], T[2], D) <= 0;
}

/* Lawson pass over the work stack.  When `apex_mode` the stack holds edges
   opposite a freshly inserted apex (slot 0 after a flip); otherwise it holds
   arbitrary edges and the four outer edges of each flipped quad are pushed. */
static int lawson(mesh_t *m, int apex_mode)
{
    while (m->sp) {
        int64_t e = m->stack[--m->sp];
        int t = (int)(e >> 2), i = (int)(e & 3);
        if (legal_edge(m, t, i)) continue;
        int n = m->tn[3 * t + i];
        flip(m, t, i);
        int rc;
        if (apex_mode) {
            if ((rc = push(m, t, 0)) || (rc = push(m, n, 0))) return rc;
        } else {
            if ((rc = push(m, t, 0)) || (rc = push(m, t, 2)) ||
                (rc = push(m, n, 0)) || (rc = push(m, n, 1))) return rc;
        }
    }
    return OK;
}

/* Visibility walk (exact); returns the triangle whose closed interior holds
   p, and in *edge the slot of the edge p lies on (-1 if strictly inside). */
static int locate(const mesh_t *m, int p, int t, int *edge)
{
    int64_t limit = 4 * (int64_t)m->ntri + 64;
    unsigned rot = 0;
    for (int64_t it = 0; it < limit; ++it) {
        const int32_t *T = m->tv + 3 * t;
        int o[3];
        o[0] = orient_v(m, T[1], T[2], p);
        o[1] = orient_v(m, T[2], T[0], p);
        o[2] = orient_v(m, T[0], T[1], p);
        int moved = 0;
        for (int k = 0; k < 3; ++k) {
            int s = (int)((k + rot) % 3);
            if (o[s] < 0) { t = m->tn[3 * t + s]; moved = 1; break; }
        }
        rot++;
        if (t < 0) return -1;
        if (moved) continue;
        *edge = -1;
        for (int s = 0; s < 3; ++s) if (o[s] == 0) *edge = s;
        return t;
    }
    return -1;
}

static int insert_point(mesh_t *m, int p, int t, int e)
{
    int rc;
    if (e < 0) {
        int A = m->tv[3 * t], B = m->tv[3 * t + 1], C = m->tv[3 * t + 2];
        int nA = m->tn[3 * t], nB = m->tn[3 * t + 1], nC = m->tn[3 * t + 2];
        int f = m->tc[t];
        int t1 = m->ntri, t2 = m->ntri + 1;
        m->ntri += 2;
        set_tri(m, t, p, B, C, nA, t1, t2, f & 1);
        set_tri(m, t1, A, p, C, t, nB, t2, f & 2);
        set_tri(m, t2, A, B, p, t, t1, nC, f & 4);
        repoint(m, nB, t, t1);
        repoint(m, nC, t, t2);
        if ((rc = push(m, t, 0)) || (rc = push(m, t1, 1)) || (rc = push(m, t2, 2))) return rc;
    } else {
        /* p on the edge BC opposite slot e of t=(A,B,C); n=(D,C,B) */
        int A = m->tv[3 * t + e], B = m->tv[3 * t + (e + 1) % 3], C = m->tv[3 * t + (e + 2) % 3];
        int n = m->tn[3 * t + e];
        if (n < 0) return BAD_INPUT;   /* on the box: excluded by the input range */
        int j = nb_slot(m, n, t);
        int D = m->tv[3 * n + j];
        int tB = m->tn[3 * t + (e + 1) % 3], fB = (m->tc[t] >> ((e + 1) % 3)) & 1;
        int tC = m->tn[3 * t + (e + 2) % 3], fC = (m->tc[t] >> ((e + 2) % 3)) & 1;
        int nC_ = m->tn[3 * n + (j + 1) % 3], gC = (m->tc[n] >> ((j + 1) % 3)) & 1;  /* across BD */
        int nB_ = m->tn[3 * n + (j + 2) % 3], gB = (m->tc[n] >> ((j + 2) % 3)) & 1;  /* across DC */
        int fE = (m->tc[t] >> e) & 1;
        int t2 = m->ntri, n2 = m->ntri + 1;
        m->ntri += 2;
        set_tri(m, t, A, B, p, n2, t2, tC, fE | (fC << 2));
        set_tri(m, t2, A, p, C, n, tB, t, fE | (fB << 1));
        set_tri(m, n, D, C, p, t2, n2, nB_, fE | (gB << 2));
        set_tri(m, n2, D, p, B, t, nC_, n, fE | (gC << 1));
        repoint(m, tB, t, t2);
        repoint(m, nC_, n, n2);
        if ((rc = push(m, t, 2)) || (rc = push(m, t2, 1)) ||
            (rc = push(m, n, 2)) || (rc = push(m, n2, 1))) return rc;
    }
    return lawson(m, 1);
}

/* ---------------------------------------------------------------- constraints */

/* Find the triangle around `a` containing `a`-`x`-`y` as a CCW corner with x == v.  */
static int find_edge(const mesh_t *m, int a, int b, int *slot_b)
{
    int t0 = m->vt[a], t = t0;
    for (int guard = 0; guard < m->ntri + 8; ++guard) {
        int i = slot_of(m, t, a);
        int u = m->tv[3 * t + (i + 1) % 3];
        if (u == b) { *slot_b = (i + 1) % 3; return t; }
        /* rotate CW around a: neighbour across edge (a,u), opposite slot i+2 */
        t = m->tn[3 * t + (i + 2) % 3];
        if (t < 0 || t == t0) return -1;
    }
    return -1;
}

static int mark_constrained(mesh_t *m, int a, int b)
{
    int sb;
    int t = find_edge(m, a, b, &sb);
    if (t < 0) return CONSTRAINT_FAIL;
    /* edge (a,b) of t is opposite the third vertex */
    int i = slot_of(m, t, a);
    int k = 3 - i - sb;
    m->tc[t] |= (uint8_t)(1u << k);
    int n = m->tn[3 * t + k];
    if (n >= 0) m->tc[n] |= (uint8_t)(1u << nb_slot(m, n, t));
    return OK;
}

static int64_t dot_v(const mesh_t *m, int a, int b, int c)  /* (b-a).(c-a) */
{
    return (m->px[b] - m->px[a]) * (m->px[c] - m->px[a]) + (m->py[b] - m->py[a]) * (m->py[c] - m->py[a]);
}

/* Insert constraint (a,b).  Returns OK or an error code. */
static int insert_segment(mesh_t *m, int a, int b, int64_t *ebuf, int64_t ecap)
{
    int64_t iter_guard = 0;
    while (a != b) {
        if (++iter_guard > (int64_t)m->nv + 8) return ITER_LIMIT;
        /* find the wedge at a containing direction ab */
        int t0 = m->vt[a], t = t0, found = -1, via = -1;
        for (int guard = 0; guard < m->ntri + 8; ++guard) {
            int i = slot_of(m, t, a);
            int u = m->tv[3 * t + (i + 1) % 3], w = m->tv[3 * t + (i + 2) % 3];
            if (u == b || w == b) { found = -2; via = b; break; }
            int ou = orient_v(m, a, u, b), ow = orient_v(m, a, w, b);
            if (ou == 0 && dot_v(m, a, u, b) > 0) { found = -2; via = u; break; }
            if (ow == 0 && dot_v(m, a, w, b) > 0) { found = -2; via = w; break; }
            if (ou > 0 && ow < 0) { found = t; break; }
            t = m->tn[3 * t + (i + 2) % 3];
            if (t < 0 || t == t0) break;
        }
        if (found == -1) return CONSTRAINT_FAIL;
        if (found == -2) {           /* (a,via) is already an edge along ab */
            int rc = mark_constrained(m, a, via);
            if (rc) return rc;
            a = via;
            continue;
        }
        /* walk across the triangles crossed by ab, recording crossed edges */
        int64_t ne = 0;
        int i = slot_of(m, found, a);
        int u = m->tv[3 * found + (i + 1) % 3], w = m->tv[3 * found + (i + 2) % 3];
        int cur = found, cs = i;   /* crossed edge is opposite slot cs of cur */
        int stop_at = -1;
        for (int64_t steps = 0;; ++steps) {
            if (steps > (int64_t)m->ntri) return ITER_LIMIT;
            if ((m->tc[cur] >> cs) & 1) return CONSTRAINT_FAIL;  /* crosses another constraint */
            if (ne == ecap) return OOM;
            ebuf[ne++] = ((int64_t)u << 32) | (uint32_t)w;
            int n = m->tn[3 * cur + cs];
            if (n < 0) return CONSTRAINT_FAIL;
            int j = nb_slot(m, n, cur);
            int x = m->tv[3 * n + j];
            if (x == b) { stop_at = b; break; }
            int ox = orient_v(m, a, b, x);
            if (ox == 0) { stop_at = x; break; }   /* segment passes through x */
            /* n = (x, w, u) in CCW order from slot j */
            if (ox < 0) {            /* x right of ab, like u: cross edge (x,w) */
                u = x;               /* edge (x,w) is opposite u in n: slot j+2 */
                cur = n; cs = (j + 2) % 3;
            } else {                 /* x left: cross edge (u,x), opposite w: slot j+1 */
                w = x;
                cur = n; cs = (j + 1) % 3;
            }
        }
        /* Sloan: flip crossing edges until none crosses (a, stop_at) */
        int c = stop_at;
        int64_t head = 0, tail = ne, qcap = ecap;
        int64_t stall = 0;
        while (head < tail) {
            if (++stall > 64 * (int64_t)(ne + 4) * (ne + 4)) return ITER_LIMIT;
            int64_t e = ebuf[head % qcap]; head++;
            int eu = (int)(e >> 32), ew = (int)(uint32_t)e;
            int sw;
            int tt = find_edge(m, eu, ew, &sw);
            if (tt < 0) return CONSTRAINT_FAIL;
            int iu = slot_of(m, tt, eu);
            int k = 3 - iu - sw;     /* slot opposite the edge (eu,ew) */
            int X = m->tv[3 * tt + k];
            int nn = m->tn[3 * tt + k];
            int Y = m->tv[3 * nn + nb_slot(m, nn, tt)];
            int s1 = orient_v(m, X, Y, eu), s2 = orient_v(m, X, Y, ew);
            if ((s1 > 0 && s2 < 0) || (s1 < 0 && s2 > 0)) {
                flip(m, tt, k);
                int oX = orient_v(m, a, c, X), oY = orient_v(m, a, c, Y);
                if ((oX > 0 && oY < 0) || (oX < 0 && oY > 0)) {
                    if (tail - head >= qcap) return OOM;
                    ebuf[tail % qcap] = ((int64_t)X << 32) | (uint32_t)Y; tail++;
                }
            } else {
                if (tail - head >= qcap) return OOM;
                ebuf[tail % qcap] = e; tail++;
            }
        }
        int rcm = mark_constrained(m, a, c);
        if (rcm) return rcm;
        a = c;
    }
    return OK;
}

/* ---------------------------------------------------------------- driver */

static void morton_order(const mesh_t *m, int32_t *order)
{
    int n = m->n;
    uint64_t *key = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n * 2);
    int32_t *tmp = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
    uint64_t *k2 = key + n;
    for (int i = 0; i < n; ++i) {
        uint64_t x = (uint64_t)m->px[i], y = (uint64_t)m->py[i], k = 0;
        for (int bit = 29; bit >= 0; --bit)
            k = (k << 2) | (((y >> bit) & 1) << 1) | ((x >> bit) & 1);
        key[i] = k; order[i] = i;
    }
    /* LSD radix sort, 8 passes of 8 bits over the 60-bit key */
    for (int pass = 0; pass < 8; ++pass) {
        int shift = pass * 8;
        size_t cnt[257] = {0};
        for (int i = 0; i < n; ++i) cnt[((key[i] >> shift) & 255) + 1]++;
        for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
        for (int i = 0; i < n; ++i) {
            size_t pos = cnt[(key[i] >> shift) & 255]++;
            k2[pos] = key[i]; tmp[pos] = order[i];
        }
        memcpy(key, k2, sizeof(uint64_t) * (size_t)n);
        memcpy(order, tmp, sizeof(int32_t) * (size_t)n);
    }
    free(key); free(tmp);
}

static void mesh_free(mesh_t *m)
{
    free(m->px); free(m->py); free(m->tv); free(m->tn); free(m->tc); free(m->vt); free(m->stack);
}

/* Full CDT.  xy: 2n int32 (x,y); cons: 2s int32 index pairs.
   Outputs (capacity 2n+2 triangles): tris 3 per triangle (input indices,
   corners n..n+3), adj 3 per triangle, cflags 1 per triangle.
   stats (optional, 4 int64): flips, ntri, constraint-splits, 0. */
int oracle_cdt(const int32_t *xy, int n, const int32_t *cons, int s,
               int32_t *tris, int32_t *adj, uint8_t *cflags, int *ntri_out, int64_t *stats)
{
    if (n < 0 || s < 0) return BAD_INPUT;
    mesh_t m; memset(&m, 0, sizeof m);
    m.n = n; m.nv = n + 4; m.cap = 2 * n + 2;
    m.px = (int64_t *)malloc(sizeof(int64_t) * (size_t)m.nv);
    m.py = (int64_t *)malloc(sizeof(int64_t) * (size_t)m.nv);
    m.tv = (int32_t *)malloc(sizeof(int32_t) * 3 * (size_t)m.cap);
    m.tn = (int32_t *)malloc(sizeof(int32_t) * 3 * (size_t)m.cap);
    m.tc = (uint8_t *)calloc((size_t)m.cap, 1);
    m.vt = (int32_t *)malloc(sizeof(int32_t) * (size_t)m.nv);
    int32_t *order = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int rc = OK;
    if (!m.px || !m.py || !m.tv || !m.tn || !m.tc || !m.vt || !order) { rc = OOM; goto done; }
    for (int i = 0; i < n; ++i) {
        int64_t x = xy[2 * i], y = xy[2 * i + 1];
        if (x < 1 || y < 1 || x > ORACLE_R - 1 || y > ORACLE_R - 1) { rc = BAD_INPUT; goto done; }
        m.px[i] = x; m.py[i] = y;
    }
    for (int k = 0; k < s; ++k) {
        int a = cons[2 * k], b = cons[2 * k + 1];
        if (a < 0 || b < 0 || a >= n || b >= n || a == b) { rc = BAD_INPUT; goto done; }
    }
    /* corners and the two root triangles (rawMesh.cu:5-22) */
    m.px[n] = 0;        m.py[n] = 0;
    m.px[n + 1] = ORACLE_R; m.py[n + 1] = 0;
    m.px[n + 2] = ORACLE_R; m.py[n + 2] = ORACLE_R;
    m.px[n + 3] = 0;    m.py[n + 3] = ORACLE_R;
    m.ntri = 2;
    set_tri(&m, 0, n, n + 1, n + 3, 1, -1, -1, 0);
    set_tri(&m, 1, n + 1, n + 2, n + 3, -1, 0, -1, 0);

    morton_order(&m, order);
    for (int k = 1; k < n; ++k) {
        int a = order[k - 1], b = order[k];
        if (m.px[a] == m.px[b] && m.py[a] == m.py[b]) { rc = BAD_INPUT; goto done; }
    }
    int last = 0;
    for (int k = 0; k < n; ++k) {
        int p = order[k], e;
        int t = locate(&m, p, last, &e);
        if (t < 0) { rc = ITER_LIMIT; goto done; }
        if ((rc = insert_point(&m, p, t, e))) goto done;
        last = m.vt[p];
    }
    if (s > 0) {
        int64_t ecap = 4 * (int64_t)m.ntri + 64;
        int64_t *ebuf = (int64_t *)malloc(sizeof(int64_t) * (size_t)ecap);
        if (!ebuf) { rc = OOM; goto done; }
        for (int k = 0; k < s && rc == OK; ++k)
            rc = insert_segment(&m, cons[2 * k], cons[2 * k + 1], ebuf, ecap);
        free(ebuf);
        if (rc) goto done;
        for (int t = 0; t < m.ntri; ++t)
            for (int i = 0; i < 3; ++i)
                if (m.tn[3 * t + i] > t && (rc = push(&m, t, i))) goto done;
        if ((rc = lawson(&m, 0))) goto done;
    }
    *ntri_out = m.ntri;
    memcpy(tris, m.tv, sizeof(int32_t) * 3 * (size_t)m.ntri);
    memcpy(adj, m.tn, sizeof(int32_t) * 3 * (size_t)m.ntri);
    memcpy(cflags, m.tc, (size_t)m.ntri);
    if (stats) { stats[0] = m.flips; stats[1] = m.ntri; stats[2] = 0; stats[3] = 0; }
done:
    free(order);
    mesh_free(&m);
    return rc;
}

/* ---------------------------------------------------------------- validator */

static int edge_cmp(const void *x, const void *y)
{
    uint64_t a = *(const uint64_t *)x, b = *(const uint64_t *)y;
    return (a > b) - (a < b);
}

static int edge_in(const uint64_t *set, size_t n, int a, int b)
{
    uint64_t key = a < b ? ((uint64_t)a << 32) | (uint32_t)b : ((uint64_t)b << 32) | (uint32_t)a;
    return bsearch(&key, set, n, sizeof(uint64_t), edge_cmp) != NULL;
}

/* Exact validator of a CDT over points + corners.  Checks: triangle count
   2n+2, CCW orientation, adjacency symmetry, hull = the 4 box sides, every
   vertex used, every constraint present as a chain of constrained edges
   (split at collinear vertices), no other constrained edge, and every
   unconstrained interior edge locally Delaunay under the perturbed incircle.
   Because the perturbed CDT is unique, passing this check pins the triangle
   set.  Returns 0 on success, else a code with a message in msg. */
int oracle_validate(const int32_t *xy, int n, const int32_t *cons, int s,
                    const int32_t *tris, const int32_t *adj, const uint8_t *cflags, int ntri,
                    char *msg, int msglen)
{
#define FAIL(...) do { if (msg) snprintf(msg, (size_t)msglen, __VA_ARGS__); rc = 1; goto out; } while (0)
    int rc = 0;
    int nv = n + 4;
    mesh_t m; memset(&m, 0, sizeof m);
    m.n = n; m.nv = nv; m.ntri = ntri; m.cap = ntri;
    m.px = (int64_t *)malloc(sizeof(int64_t) * (size_t)nv);
    m.py = (int64_t *)malloc(sizeof(int64_t) * (size_t)nv);
    m.vt = (int32_t *)malloc(sizeof(int32_t) * (size_t)nv);
    uint64_t *cedges = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(3 * (size_t)ntri + 1));
    size_t nce = 0;
    if (!m.px || !m.py || !m.vt || !cedges) FAIL("oom");
    for (int i = 0; i < n; ++i) { m.px[i] = xy[2 * i]; m.py[i] = xy[2 * i + 1]; }
    m.px[n] = 0; m.py[n] = 0; m.px[n + 1] = ORACLE_R; m.py[n + 1] = 0;
    m.px[n + 2] = ORACLE_R; m.py[n + 2] = ORACLE_R; m.px[n + 3] = 0; m.py[n + 3] = ORACLE_R;
    m.tv = (int32_t *)tris; m.tn = (int32_t *)adj; m.tc = (uint8_t *)cflags;
    if (ntri != 2 * n + 2) FAIL("triangle count %d != 2n+2 = %d", ntri, 2 * n + 2);
    for (int v = 0; v < nv; ++v) m.vt[v] = -1;
    int hull = 0;
    for (int t = 0; t < ntri; ++t) {
        const int32_t *T = tris + 3 * t;
        for (int i = 0; i < 3; ++i) if (T[i] < 0 || T[i] >= nv) FAIL("tri %d bad vertex %d", t, T[i]);
        if (orient_v(&m, T[0], T[1], T[2]) <= 0) FAIL("tri %d not CCW", t);
        for (int i = 0; i < 3; ++i) m.vt[T[i]] = t;
        for (int i = 0; i < 3; ++i) {
            int a = T[(i + 1) % 3], b = T[(i + 2) % 3];
            int nb = adj[3 * t + i];
            if (nb < 0) {
                hull++;
                if (!(a >= n && b >= n)) FAIL("tri %d edge %d on hull but not a box side", t, i);
                if (cflags[t] >> i & 1) FAIL("hull edge flagged constrained");
                continue;
            }
            if (nb >= ntri) FAIL("tri %d bad neighbour %d", t, nb);
            const int32_t *N = tris + 3 * nb;
            int j = -1;
            for (int q = 0; q < 3; ++q) if (adj[3 * nb + q] == t) j = q;
            if (j < 0) FAIL("adjacency not symmetric at tri %d slot %d", t, i);
            if (!(N[(j + 1) % 3] == b && N[(j + 2) % 3] == a)) FAIL("neighbour %d of %d does not share edge", nb, t);
            int fa = cflags[t] >> i & 1, fb = cflags[nb] >> j & 1;
            if (fa != fb) FAIL("constraint flag asymmetric at tri %d slot %d", t, i);
            if (fa && t < nb) cedges[nce++] = a < b ? ((uint64_t)a << 32) | (uint32_t)b : ((uint64_t)b << 32) | (uint32_t)a;
            if (!fa && t < nb) {
                if (incircle_sos_v(&m, T[0], T[1], T[2], N[j]) > 0)
                    FAIL("edge (%d,%d) between tris %d,%d not locally Delaunay", a, b, t, nb);
            }
        }
    }
    if (hull != 4) FAIL("hull has %d edges, expected 4", hull);
    for (int v = 0; v < nv; ++v) if (m.vt[v] < 0) FAIL("vertex %d unused", v);
    qsort(cedges, nce, sizeof(uint64_t), edge_cmp);
    /* every constraint = chain of constrained edges through collinear vertices */
    {
        size_t ucap = nce + 16, nused = 0;
        uint64_t *used = (uint64_t *)malloc(sizeof(uint64_t) * ucap);
        if (!used) FAIL("oom");
        for (int k = 0; k < s; ++k) {
            int a = cons[2 * k], b = cons[2 * k + 1];
            int guard = 0;
            while (a != b) {
                if (++guard > nv) { free(used); FAIL("constraint %d chain too long", k); }
                /* edges at a along direction ab */
                int t0 = m.vt[a], t = t0, nxt = -1;
                for (int g2 = 0; g2 < ntri + 4; ++g2) {
                    int i = slot_of(&m, t, a);
                    int u = tris[3 * t + (i + 1) % 3];
                    if (u == b || (orient_v(&m, a, u, b) == 0 && dot_v(&m, a, u, b) > 0)) { nxt = u; break; }
                    t = adj[3 * t + (i + 2) % 3];
                    if (t < 0 || t == t0) break;
                }
                if (nxt < 0) {
                    /* star of a may be open only for corners, which are never constraint ends */
                    free(used); FAIL("constraint %d (%d,%d) missing at vertex %d", k, cons[2 * k], cons[2 * k + 1], a);
                }
                if (!edge_in(cedges, nce, a, nxt)) { free(used); FAIL("constraint %d edge (%d,%d) not flagged", k, a, nxt); }
                if (nused == ucap) {   /* overlapping constraints repeat edges */
                    uint64_t *nu = (uint64_t *)realloc(used, sizeof(uint64_t) * ucap * 2);
                    if (!nu) { free(used); FAIL("oom"); }
                    used = nu; ucap *= 2;
                }
                used[nused++] = a < nxt ? ((uint64_t)a << 32) | (uint32_t)nxt : ((uint64_t)nxt << 32) | (uint32_t)a;
                a = nxt;
            }
        }
        qsort(used, nused, sizeof(uint64_t), edge_cmp);
        size_t uq = 0;
        for (size_t i = 0; i < nused; ++i) if (i == 0 || used[i] != used[i - 1]) uq++;
        free(used);
        if (uq != nce) FAIL("%zu constrained edges flagged, %zu expected", nce, uq);
    }
out:
    free(m.px); free(m.py); free(m.vt); free(cedges);
    return rc;
#undef FAIL
}
