// mesh.cuh -- data layout and per-element bodies of every kernel of the
// CDT path.  The bodies are __host__ __device__ so that the same code is
// what the CUDA kernels (gcdt.cu, batch.cu) run, one body call per thread,
// and what the host test harness runs on the CPU.
//
// Layout in HBM (structure of arrays, one row per point or triangle):
//   P[v]      int2   point v in space-filling-curve order; corners at N..N+3
//   perm[v]   int    input index of sorted point v (corners map to N+k)
//   tri[2t]   int4   TV: (v0, v1, v2, w) -- CCW vertices; w bit k set when the
//                    edge opposite v_k is a constraint edge (k < 3), bit 3 the
//                    triangle's side of its last flip (or, after a split,
//                    whether it was the second triangle of an edge split),
//                    bits 4.. the flip sub-round of that flip (0: made by a
//                    split or a constraint flip)
//   tri[2t+1] int4   TA: (a0, a1, a2, -)  a_k = 4*n + j: neighbour n across the
//                    edge opposite v_k, which is opposite slot j in n; -1 = box;
//                    .w = the insertion round that last changed the triangle
//                    (TV and TA of a triangle share one 32-byte sector: most
//                    visits read both)
// Triangle slots never move: the two root triangles are 0 and 1, and sorted
// point q creates exactly two new slots, 2+2q and 3+2q, when it is inserted
// (1->3 split of one triangle, or 2->4 split of the two triangles sharing the
// edge q lies on).  The final mesh therefore has exactly 2N+2 triangles
// (reference count T = 2N+2 with the 4 box corners).
//
// Reference conventions kept (yingtix/gCDT): int2 points at 30-bit resolution
// (include/math_base.cuh:19-29), box corners (0,0),(R,0),(R,R),(0,R) at
// N..N+3 and root triangles (N,N+1,N+3),(N+1,N+2,N+3) (rawMesh.cu:5-22), CCW
// triangles whose adj.x is the neighbour across the edge opposite .x
// (rawMesh.cu:269-276), flips iff inCircle > 0 (kernel.cu:2218-2219) and
// constraint edges never flipped (kernel.cu:2203-2205).
#pragma once
#include <cstdint>
#include "predicates.cuh"

#if defined(__CUDACC__)
#include <cooperative_groups.h>
#endif

#define GCDT_HD __host__ __device__ __forceinline__

namespace gcdt {

constexpr int kBoxMax = (1 << 30) - 1;   // R = 2^30 - 1
constexpr int kMaxPhaseKinds = 24;

enum StatusBits : int {
    ST_OK = 0,
    ST_BAD_INPUT = 1,
    ST_OOM = 2,
    ST_ITER_LIMIT = 4,
    ST_CONSTRAINT_FAIL = 8,
    ST_INTERNAL = 16,
    ST_BARRIER = 64,     // a grid barrier wait ran out of iterations
};

// Device-resident counters.  Every list has a monotone 64-bit append
// cursor: a phase appends at [base, cursor) where base is the cursor value
// when the phase began, so no counter is ever reset between phases.
struct Counters {
    int status;                  // OR of StatusBits (host launches, final result)
    int err[2];                  // errors of the persistent phases, by phase parity
    int pad0;
    unsigned long long cur_act0; // lists built by activation
    unsigned long long cur_act;  // active point lists
    unsigned long long cur_win;  // inserted points of a round
    unsigned long long cur_q;    // flip queues
    unsigned long long cur_flip; // flips of a sub-round
    unsigned long long cur_pend; // pending segment lists
    unsigned long long cur_law;  // constrained flip pass queue
    unsigned long long cur_scr;  // constraint scratch
    unsigned int bar_count;      // grid barrier (top bit flips once per barrier)
    unsigned int pad_bar;
    long long rounds, flip_subrounds, constraint_rounds;
    long long grid_blocks;       // blocks of the persistent launch
    long long pad1[2];
    long long phase_cyc[kMaxPhaseKinds];   // SM cycles per phase kind (block 0's view)
    long long phase_cnt[kMaxPhaseKinds];
    unsigned long long handoff[24];        // driver state handed back by a single-block tail
    long long handoff_nq;
    int handoff_rc;
    int pad2;
    // Balance of the grid phases: per phase kind, the sum over its runs of
    // the longest and of the summed per-block work time (SM cycles from the
    // phase's start to the block's arrival at the barrier).  wcur_* collect
    // one run, double-buffered by phase parity.
    long long phase_wmax[kMaxPhaseKinds];
    long long phase_wsum[kMaxPhaseKinds];
    unsigned long long wcur_max[2];
    unsigned long long wcur_sum[2];
};

// The persistent kernel's phases see the launch's context with the fields
// the stage driver changes between phases copied in (phase_view in
// exec.cuh): a field the driver starts to change goes into that list.
struct Ctx {
    int n;          // input points
    int s;          // input segments
    int ntri;       // 2n + 2
    unsigned round; // insertion round / epoch stamp
    unsigned sr;    // flip sub-round stamp (monotone over the whole solve)
    int eslot;      // error word of the running phase (phase parity)
    unsigned lawson_sr;  // queue stamp of the constrained flip pass
    int list_n;     // length of the list a launch iterates over
    int carry_n;    // leading flip-queue entries carried over from the previous round

    const int2* in_xy;
    const int2* in_cons;

    unsigned long long* keys;
    unsigned long long* keys_alt;
    int* vals;
    int* vals_alt;

    int2* P;
    int* perm;
    int* rank;

    int4* tri;      // per triangle: vertices (TV) then adjacency (TA), 32 bytes

    int* loc;                 // triangle holding an uninserted point, -1 once inserted
    signed char* pedge;       // slot of the edge the point lies on, -1 inside
    int* act;                 // active point list (read)
    int* act_next;            // active point list (append)
    unsigned long long* vote; // per triangle: (round<<32) | ~hash(point)
    int2* winners;            // (q, t) inserted this round

    unsigned long long* claim;  // per triangle: (stamp<<32) | ~key
    int2* cand;                 // per queue entry: (4t+i, 4n+j) or (-1,-1)
    int* qst;                   // per triangle: queue stamp (dedup)
    int* queue;                 // flip queue (read)
    int* queue_next;            // flip queue (append)

    int4* seg;          // per segment: (a, b, stop, -)  sorted ids; a advances
    int* pend;          // pending segment list (read)
    int* pend_next;     // pending segment list (append)
    int4* pinfo;        // per pending entry: (start 4t+i, ncross, scratch base, ring size | -1)
    int* scratch;       // constraint scratch
    int scratch_cap;
    int* vt;            // vertex -> incident triangle
    int* lq;            // triangles queued for the constrained flip pass

    // append bases of the lists the current phase writes (see Counters)
    unsigned long long base_act, base_win, base_q, base_flip, base_pend, base_law, base_scr;

    unsigned char* lvl; // insertion level of each sorted point
    int level;          // level being activated / the live levels are < level
    int nlevels;
    int stride[4];      // level l holds the points i with i % stride[l] == 0 not in a lower level

    int* out_tris;
    int* out_adj;
    unsigned char* out_cflags;

    // Budgets of the bounded driver loops (0: the built-in bound): grid
    // insertion rounds per solve, flip sub-rounds per flip loop, constraint
    // rounds.  A budget that runs out ends the solve with ST_ITER_LIMIT.
    int lim_rounds;
    int lim_subrounds;
    int lim_crounds;

    // Scheduling of the whole-grid solve (set by bind_ctx, tunable per
    // context): flip sub-rounds of a round stop once the queue is at most
    // carry_q long (the rest is carried into the next round; 0: never);
    // flip queues of at most narrow_q entries and insertion tails of at most
    // narrow_act points run in one block (0: never).
    int carry_q;
    int narrow_q;
    int narrow_act;

    Counters* cnt;
};

// ---------------------------------------------------------------- helpers

GCDT_HD int enc(int t, int s) { return (t << 2) | s; }
GCDT_HD int nx3(int i) { return i == 2 ? 0 : i + 1; }
GCDT_HD int pv3(int i) { return i == 0 ? 2 : i - 1; }
GCDT_HD int comp(const int4& v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
GCDT_HD void setc(int4& v, int i, int x) {
    if (i == 0) v.x = x; else if (i == 1) v.y = x; else v.z = x;
}
GCDT_HD int slot_of(const int4& tv, int v) { return tv.x == v ? 0 : (tv.y == v ? 1 : 2); }
GCDT_HD int slot_of_or_none(const int4& tv, int v) { return tv.x == v ? 0 : (tv.y == v ? 1 : (tv.z == v ? 2 : -1)); }
// The flip sub-round kept in a vertex row's spare bits (see the layout).
GCDT_HD int flip_stamp(int w) { return (int)((unsigned)w >> 4); }

// A host test build may count triangle-record accesses by defining
// GCDT_TOUCH; the library defines nothing here.
#ifndef GCDT_TOUCH
#define GCDT_TOUCH(t)
#endif

// Vertex row (TV) and adjacency row (TA) of triangle t.
GCDT_HD int4& tri_v(const Ctx& c, int t) { GCDT_TOUCH(t); return c.tri[2 * (size_t)(unsigned)t]; }
GCDT_HD int4& tri_a(const Ctx& c, int t) { GCDT_TOUCH(t); return c.tri[2 * (size_t)(unsigned)t + 1]; }

GCDT_HD uint32_t hash32(uint32_t x) {  // bijective 32-bit mix
    x ^= x >> 16; x *= 0x7feb352dU;
    x ^= x >> 15; x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

GCDT_HD unsigned long long at_max64(unsigned long long* p, unsigned long long v) {
#if defined(__CUDA_ARCH__)
    return atomicMax(p, v);
#else
    unsigned long long o = *p; if (v > o) *p = v; return o;
#endif
}
GCDT_HD int at_add(int* p, int v) {
#if defined(__CUDA_ARCH__)
    return atomicAdd(p, v);
#else
    int o = *p; *p = o + v; return o;
#endif
}
GCDT_HD unsigned long long at_add64(unsigned long long* p, unsigned long long v) {
#if defined(__CUDA_ARCH__)
    return atomicAdd(p, v);
#else
    unsigned long long o = *p; *p = o + v; return o;
#endif
}
GCDT_HD int at_exch(int* p, int v) {
#if defined(__CUDA_ARCH__)
    return atomicExch(p, v);
#else
    int o = *p; *p = v; return o;
#endif
}
GCDT_HD int at_or(int* p, int v) {
#if defined(__CUDA_ARCH__)
    return atomicOr(p, v);
#else
    int o = *p; *p = o | v; return o;
#endif
}
// Errors go to the word of the running phase's parity: the driver reads
// that word after the phase's barrier, while the next phase writes the
// other one, so every thread sees the same error state.
GCDT_HD void fail(const Ctx& c, int bits) { at_or(&c.cnt->err[c.eslot], bits); }

// Append one element to a list with cursor *cur and phase base `base`;
// returns the element's index in the list.  On the GPU the threads of a warp
// that append together take one atomic between them.
GCDT_HD int append_slot(unsigned long long* cur, unsigned long long base) {
#if defined(__CUDA_ARCH__)
    namespace cg = cooperative_groups;
    cg::coalesced_group g = cg::coalesced_threads();
    unsigned long long b = 0;
    if (g.thread_rank() == 0) b = atomicAdd(cur, (unsigned long long)g.size());
    b = g.shfl(b, 0);
    return (int)(b - base) + (int)g.thread_rank();
#else
    unsigned long long o = *cur; *cur = o + 1; return (int)(o - base);
#endif
}

// Append `cnt` consecutive elements (0 <= cnt <= 7); returns the index of
// the first.  One atomic per warp; each thread's offset is the sum of the
// counts of the lower lanes, taken bit by bit from three ballots.
GCDT_HD int append_slots(unsigned long long* cur, unsigned long long base, int cnt) {
#if defined(__CUDA_ARCH__)
    const unsigned mask = __activemask();
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt = mask & ((1u << lane) - 1u);
    const unsigned b0 = __ballot_sync(mask, cnt & 1), b1 = __ballot_sync(mask, cnt & 2),
                   b2 = __ballot_sync(mask, cnt & 4);
    const unsigned before = __popc(b0 & lt) + 2u * __popc(b1 & lt) + 4u * __popc(b2 & lt);
    const unsigned total = __popc(b0) + 2u * __popc(b1) + 4u * __popc(b2);
    const int leader = __ffs(mask) - 1;
    unsigned long long b = 0;
    if ((int)lane == leader) b = atomicAdd(cur, (unsigned long long)total);
    b = __shfl_sync(mask, b, leader);
    return (int)(b - base) + (int)before;
#else
    unsigned long long o = *cur; *cur = o + (unsigned long long)cnt; return (int)(o - base);
#endif
}

GCDT_HD unsigned long long morton60(int2 p) {
    unsigned long long x = (unsigned)p.x, y = (unsigned)p.y;
    auto spread = [](unsigned long long v) {
        v &= 0x3fffffffULL;
        v = (v | (v << 16)) & 0x0000FFFF0000FFFFULL;
        v = (v | (v << 8)) & 0x00FF00FF00FF00FFULL;
        v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0FULL;
        v = (v | (v << 2)) & 0x3333333333333333ULL;
        v = (v | (v << 1)) & 0x5555555555555555ULL;
        return v;
    };
    return spread(x) | (spread(y) << 1);
}

// ---------------------------------------------------------------- set-up

// One thread per input point: sort key + range check.
// Four levels of the Hilbert index at a time: entry [frame][x bits << 4 |
// y bits] holds the four quadrant digits (low 8 bits) and the frame after
// them (bits 8-9).  Per level from the top bit, the quadrant of the point in
// the current sub-square gives two bits of the index; the sub-square's frame
// is the transform that maps the raw coordinates onto its canonical
// orientation: a swap of x and y (bit 0) composed with the complement of
// both (bit 1).  Both are involutions and commute, so the two bits track it.
// The index is the usual one: quadrant digit (3*rx) ^ ry, and a lower
// quadrant (ry = 0) swaps the frame, complemented first when rx = 1.
struct HilbertTable { unsigned short v[4][256]; };
__host__ __device__ constexpr HilbertTable make_hilbert_table() {
    HilbertTable T{};
    for (int frame = 0; frame < 4; ++frame)
        for (int in = 0; in < 256; ++in) {
            unsigned sw = frame & 1, cp = frame >> 1, d = 0;
            for (int l = 3; l >= 0; --l) {
                const unsigned a = ((in >> (4 + l)) & 1u) ^ cp, b = ((in >> l) & 1u) ^ cp;
                const unsigned rx = sw ? b : a, ry = sw ? a : b;
                d = (d << 2) | ((3u * rx) ^ ry);
                const unsigned lower = ry ^ 1u;
                sw ^= lower;
                cp ^= lower & rx;
            }
            T.v[frame][in] = (unsigned short)(d | ((sw | (cp << 1)) << 8));
        }
    return T;
}
#if defined(__CUDACC__)
__device__ constexpr HilbertTable kHilbertTableDev = make_hilbert_table();
#endif
constexpr HilbertTable kHilbertTable = make_hilbert_table();

// Position of p along the Hilbert curve over the 2^30 x 2^30 grid (the
// standard construction: at each level the quadrant's index, then the
// coordinates rotated into that quadrant's frame), a bijection onto
// [0, 2^60) like the Morton code, with no jumps between quadrants.  The
// coordinates are taken as 32-bit numbers: the two leading zero levels have
// digit 0 and swap the frame twice, so the index is the 30-level one.
GCDT_HD unsigned long long hilbert60(int2 p) {
    const unsigned x = (unsigned)p.x & 0x3fffffffu, y = (unsigned)p.y & 0x3fffffffu;
    unsigned frame = 0;
    unsigned long long d = 0;
#pragma unroll
    for (int k = 28; k >= 0; k -= 4) {
        const unsigned in = (((x >> k) & 15u) << 4) | ((y >> k) & 15u);
#if defined(__CUDA_ARCH__)
        const unsigned e = __ldg(&kHilbertTableDev.v[frame][in]);
#else
        const unsigned e = kHilbertTable.v[frame][in];
#endif
        d = (d << 8) | (e & 255u);
        frame = e >> 8;
    }
    return d;
}

#ifndef GCDT_SORT_CURVE
#define GCDT_SORT_CURVE 1   // 0: Morton, 1: Hilbert
#endif
// The key points are sorted by: the order of insertion levels, of the
// samples a point's activation walk starts from, and of triangle slots.
// The Hilbert order keeps consecutive points adjacent, so triangles near
// each other in the plane sit nearer each other in memory than in Morton
// order (headline solve 28.20 -> 27.88 ms, 305 -> 267 flip sub-rounds).
GCDT_HD unsigned long long sort_key60(int2 p) { return GCDT_SORT_CURVE ? hilbert60(p) : morton60(p); }

GCDT_HD void body_keys(const Ctx& c, int i) {
    int2 p = c.in_xy[i];
    if (p.x < 1 || p.y < 1 || p.x > kBoxMax - 1 || p.y > kBoxMax - 1) fail(c, ST_BAD_INPUT);
    c.keys[i] = sort_key60(p);
    c.vals[i] = i;
}

// After the sort (sorted keys/vals in keys/vals): gather points, permutation,
// inverse permutation; adjacent equal keys are duplicate points.
GCDT_HD void body_gather(const Ctx& c, int i) {
    if (i < c.n) {
        int j = c.vals[i];
        c.P[i] = c.in_xy[j];
        c.perm[i] = j;
        c.rank[j] = i;
        if (i > 0 && c.keys[i] == c.keys[i - 1]) fail(c, ST_BAD_INPUT);
    } else if (i < c.n + 4) {
        int k = i - c.n;
        int2 corner;
        corner.x = (k == 1 || k == 2) ? kBoxMax : 0;
        corner.y = (k >= 2) ? kBoxMax : 0;
        c.P[i] = corner;
        c.perm[i] = i;
    }
}

// Per-solve reset of the per-triangle state, for solves whose arrays are
// not cleared by the host (the batched path).
GCDT_HD void body_clear(const Ctx& c, int t) {
    c.vote[t] = 0;
    c.claim[t] = 0;
    c.qst[t] = 0;
}

// Root triangles (rawMesh.cu:16-21) -- one thread.
GCDT_HD void body_root(const Ctx& c, int) {
    int n = c.n;
    tri_v(c, 0) = make_int4(n, n + 1, n + 3, 0);
    tri_v(c, 1) = make_int4(n + 1, n + 2, n + 3, 0);
    tri_a(c, 0) = make_int4(enc(1, 1), -1, -1, 0);
    tri_a(c, 1) = make_int4(-1, enc(0, 0), -1, 0);
}

// Level of each sorted point: a curve-stratified sample first (every
// stride[0]-th point), then denser samples, then the rest (a biased
// randomized insertion order over the spatial sort).
GCDT_HD void body_level(const Ctx& c, int i) {
    int l = c.nlevels - 1;
    for (int k = 0; k + 1 < c.nlevels; ++k)
        if (i % c.stride[k] == 0) { l = k; break; }
    c.lvl[i] = (unsigned char)l;
}

GCDT_HD void body_seg_level0(const Ctx& c, int k) {
    int4 sg = c.seg[k];
    if (sg.z == -1) { c.lvl[sg.x] = 0; c.lvl[sg.y] = 0; }
}

GCDT_HD long long dot3(int2 a, int2 u, int2 b) {  // (u-a).(b-a)
    return (long long)(u.x - a.x) * (b.x - a.x) + (long long)(u.y - a.y) * (b.y - a.y);
}

// Straight-line walk from vertex a (t: a triangle incident to a) to the
// triangle whose closed interior holds p (p is not a vertex).  Each step
// advances along the segment a->p, so the walk ends in any triangulation,
// constrained or not; a line through a vertex restarts from that vertex.
GCDT_HD int locate_from_vertex(const Ctx& c, int a, int t, int2 p) {
    for (int restart = 0; restart < 4096; ++restart) {
        int2 pa = c.P[a];
        int t0 = t, found = -1, fslot = 0, u = -1, w = -1;
        for (int g = 0; g < 4096; ++g) {
            int4 tv = tri_v(c, t);
            int i = slot_of(tv, a), i1 = nx3(i), i2 = nx3(i1);
            u = comp(tv, i1); w = comp(tv, i2);
            int2 pu = c.P[u], pw = c.P[w];
            int ou = orient2d(pa, pu, p), ow = orient2d(pa, pw, p);
            if (ou == 0 && dot3(pa, pu, p) > 0) {
                if (dot3(pa, p, pu) > dot3(pa, p, p)) return t;   // p inside edge (a,u)
                found = -2; a = u; break;                          // continue from u
            }
            if (ow == 0 && dot3(pa, pw, p) > 0) {
                if (dot3(pa, p, pw) > dot3(pa, p, p)) return t;
                found = -2; a = w; break;
            }
            if (ou > 0 && ow < 0) {
                if (orient2d(pu, pw, p) >= 0) return t;
                found = t; fslot = i; break;
            }
            int nb = comp(tri_a(c, t), i2);
            if (nb < 0) return -1;
            t = nb >> 2;
            if (t == t0) return -1;
        }
        if (found == -2) continue;          // t contains the new a
        if (found < 0) return -1;
        int cur = found, cs = fslot;
        int next_a = -1;
        for (int steps = 0; steps < (1 << 22); ++steps) {
            int en = comp(tri_a(c, cur), cs);
            if (en < 0) return -1;
            int n = en >> 2, j = en & 3;
            int x = comp(tri_v(c, n), j);
            int2 px = c.P[x];
            // n = (x, w, u): p is inside iff it is left of (u,x) and (x,w)
            if (orient2d(c.P[u], px, p) >= 0 && orient2d(px, c.P[w], p) >= 0) return n;
            int ox = orient2d(pa, p, px);
            if (ox == 0) { next_a = x; t = n; break; }
            cur = n;
            if (ox < 0) { u = x; cs = nx3(nx3(j)); } else { w = x; cs = nx3(j); }
        }
        if (next_a < 0) return -1;
        a = next_a;
    }
    return -1;
}

// Put the points of level c.level into the active list with their
// triangle: the root triangles for level 0 (orient against the diagonal
// (R,0)-(0,R), rawMesh.cu:37-57), otherwise a straight-line walk from the
// nearer of the previous level's preceding and following points along the
// sort curve, which are already vertices.
GCDT_HD void body_activate(const Ctx& c, int i) {
    if (c.lvl[i] != c.level) return;
    int t;
    if (c.level == 0) {
        int2 rd = make_int2(kBoxMax, 0), lt = make_int2(0, kBoxMax);
        t = orient2d(rd, lt, c.P[i]) >= 0 ? 0 : 1;
    } else {
        // start from the nearer of the two previous-level samples around i
        // in curve order (both are vertices already)
        const int s = c.stride[c.level - 1];
        int sv = i - i % s;
        const int hi = sv + s;
        const int2 p = c.P[i];
        if (hi < c.n) {
            int2 a = c.P[sv], b = c.P[hi];
            long long da = (long long)(a.x - p.x) * (a.x - p.x) + (long long)(a.y - p.y) * (a.y - p.y);
            long long db = (long long)(b.x - p.x) * (b.x - p.x) + (long long)(b.y - p.y) * (b.y - p.y);
            if (db < da) sv = hi;
        }
        t = locate_from_vertex(c, sv, c.vt[sv], p);
        if (t < 0) { fail(c, ST_ITER_LIMIT); return; }
    }
    c.loc[i] = t;
    c.act_next[append_slot(&c.cnt->cur_act0, c.base_act)] = i;
}

GCDT_HD int at_min(int* p, int v) {
#if defined(__CUDA_ARCH__)
    return atomicMin(p, v);
#else
    int o = *p; if (v < o) *p = v; return o;
#endif
}

GCDT_HD void body_vt_reset(const Ctx& c, int v) { c.vt[v] = 0x7fffffff; }

// vt[v] = the smallest live triangle incident to v (deterministic, so walks
// that start from vt give the same result on every run).  Live triangles:
// the root slots 0 and 1, and the two slots of each inserted point (points
// of level < c.level); k < n + 2.
GCDT_HD void body_vt_live(const Ctx& c, int k) {
    if (k >= 2 && c.lvl[k - 2] >= c.level) return;
    int t0 = k < 2 ? k : 2 * k - 2, nt = k < 2 ? 1 : 2;
    for (int t = t0; t < t0 + nt; ++t) {
        int4 tv = tri_v(c, t);
        at_min(&c.vt[tv.x], t); at_min(&c.vt[tv.y], t); at_min(&c.vt[tv.z], t);
    }
}

// ---------------------------------------------------------------- insertion

// Visibility walk from t to the triangle whose closed interior holds p.
// Terminates in a Delaunay triangulation (acyclic in-front-of relation).
// On success *edge is the slot of the edge p lies on, or -1 (p is not a
// vertex, so it lies on at most one edge).
GCDT_HD int walk(const Ctx& c, int t, int2 p, int limit, int* edge) {
    for (int it = 0; it < limit; ++it) {
        int4 tv = tri_v(c, t);
        int2 a = c.P[tv.x], b = c.P[tv.y], cc = c.P[tv.z];
        int side = -1, zero = -1;
        int r = it % 3;
        for (int k = 0; k < 3 && side < 0; ++k) {
            int s = r + k; if (s >= 3) s -= 3;
            int o = s == 0 ? orient2d(b, cc, p) : (s == 1 ? orient2d(cc, a, p) : orient2d(a, b, p));
            if (o < 0) side = s;
            else if (o == 0) zero = s;
        }
        if (side < 0) { *edge = zero; return t; }
        int nb = comp(tri_a(c, t), side);
        if (nb < 0) return -1;
        t = nb >> 2;
    }
    return -1;
}

// Slot of the edge of t that p lies on, or -1; flags p outside t.
GCDT_HD int edge_of(const Ctx& c, int t, int2 p) {
    int4 tv = tri_v(c, t);
    int2 a = c.P[tv.x], b = c.P[tv.y], cc = c.P[tv.z];
    int o0 = orient2d(b, cc, p), o1 = orient2d(cc, a, p), o2 = orient2d(a, b, p);
    if (o0 < 0 || o1 < 0 || o2 < 0) fail(c, ST_INTERNAL);
    return o0 == 0 ? 0 : (o1 == 0 ? 1 : (o2 == 0 ? 2 : -1));
}

// Active point q (its location t = loc[q] and coordinates p loaded by the
// caller): relocate if its triangle changed in the previous round, keep it
// in the next list, and vote for the triangle(s) it will split.  Winner per
// triangle = minimum hash32(q): random insertion order per triangle,
// independent of thread scheduling.
GCDT_HD void body_reloc_vote_qt(const Ctx& c, int q, int t, int2 p) {
    if (t < 0) return;                       // inserted last round
    int e;
    if (tri_a(c, t).w == (int)c.round - 1) {
        int nt = walk(c, t, p, 256, &e);
        if (nt < 0) {
            nt = locate_from_vertex(c, tri_v(c, t).x, t, p);
            if (nt < 0) { fail(c, ST_ITER_LIMIT); return; }
            e = edge_of(c, nt, p);
        }
        t = nt;
        c.loc[q] = t;
    } else {
        e = edge_of(c, t, p);
    }
    c.act_next[append_slot(&c.cnt->cur_act, c.base_act)] = q;
    c.pedge[q] = (signed char)e;
    unsigned long long key = ((unsigned long long)c.round << 32) | (0xffffffffu - hash32((uint32_t)q));
    if (c.vote[t] < key) at_max64(&c.vote[t], key);
    if (e >= 0) {
        int n = comp(tri_a(c, t), e) >> 2;
        if (c.vote[n] < key) at_max64(&c.vote[n], key);
    }
}
GCDT_HD void body_reloc_vote(const Ctx& c, int k) {
    const int q = c.act[k], t = c.loc[q];
    if (t >= 0) body_reloc_vote_qt(c, q, t, c.P[q]);
}

// Winners split their triangle(s).  Child j of a split triangle is the
// triangle with vertex j replaced by q; it keeps the old edge j in slot j.
// Outer adjacency is written as the old neighbour and resolved in body_fix.
GCDT_HD void split_winner(const Ctx& c, int q, int t, unsigned long long key) {
    int e = c.pedge[q];
    int T1 = 2 + 2 * q, T2 = 3 + 2 * q;
    int4 tv = tri_v(c, t), ta = tri_a(c, t);
    int fl = tv.w;
    int code = e;
    if (e < 0) {
        int ch[3] = {t, T1, T2};
        for (int j = 0; j < 3; ++j) {
            int4 v = tv; setc(v, j, q); v.w = fl & (1 << j);
            int4 a;
            a.w = (int)c.round;
            for (int kk = 0; kk < 3; ++kk)
                setc(a, kk, kk == j ? comp(ta, j) : enc(ch[kk], j));
            tri_v(c, ch[j]) = v;
            tri_a(c, ch[j]) = a;
        }
        code = 7;
    } else {
        int en = comp(ta, e);
        int n = en >> 2, e2 = en & 3;
        if (c.vote[n] != key) return;
        int4 nv = tri_v(c, n), na = tri_a(c, n);
        int gl = nv.w;
        // children: A1 = child_{e+1}(t) -> t, A2 = child_{e+2}(t) -> T1,
        //           B1 = child_{e2+1}(n) -> n, B2 = child_{e2+2}(n) -> T2
        int e1 = nx3(e), e_2 = nx3(e1), f1 = nx3(e2), f2 = nx3(f1);
        int A1 = t, A2 = T1, B1 = n, B2 = T2;
        int4 v, a;
        // A1
        v = tv; setc(v, e1, q); v.w = fl & ((1 << e1) | (1 << e));
        a = make_int4(0, 0, 0, (int)c.round);
        setc(a, e1, comp(ta, e1)); setc(a, e_2, enc(A2, e1)); setc(a, e, enc(B2, e2));
        tri_v(c, A1) = v; tri_a(c, A1) = a;
        // A2
        v = tv; setc(v, e_2, q); v.w = fl & ((1 << e_2) | (1 << e));
        a = make_int4(0, 0, 0, (int)c.round);
        setc(a, e_2, comp(ta, e_2)); setc(a, e1, enc(A1, e_2)); setc(a, e, enc(B1, e2));
        tri_v(c, A2) = v; tri_a(c, A2) = a;
        // B1 (bit 3: the second triangle of an edge split)
        v = nv; setc(v, f1, q); v.w = (gl & ((1 << f1) | (1 << e2))) | 8;
        a = make_int4(0, 0, 0, (int)c.round);
        setc(a, f1, comp(na, f1)); setc(a, f2, enc(B2, f1)); setc(a, e2, enc(A2, e));
        tri_v(c, B1) = v; tri_a(c, B1) = a;
        // B2
        v = nv; setc(v, f2, q); v.w = gl & ((1 << f2) | (1 << e2));
        a = make_int4(0, 0, 0, (int)c.round);
        setc(a, f2, comp(na, f2)); setc(a, f1, enc(B1, f2)); setc(a, e2, enc(A1, e));
        tri_v(c, B2) = v; tri_a(c, B2) = a;
    }
    c.loc[q] = -1;
    c.winners[append_slot(&c.cnt->cur_win, c.base_win)] = make_int2(q * 8 + code, t);
}

GCDT_HD void body_split_qt(const Ctx& c, int q, int t) {
    unsigned long long key = ((unsigned long long)c.round << 32) | (0xffffffffu - hash32((uint32_t)q));
    if (c.vote[t] != key) return;
    split_winner(c, q, t, key);
}
GCDT_HD void body_split(const Ctx& c, int k) {
    const int q = c.act[k];
    body_split_qt(c, q, c.loc[q]);
}

// Child of triangle m (split this round) that now holds m's old edge `ms`.
// Triangle m was split this round too (its record mv is the child that kept
// the slot m): the child of m that now holds the old edge in slot ms, whose
// endpoints are the edge in slot s of triangle cv.  A child keeps the old
// edge of the vertex it replaced; m's other children are 2+2q' and 3+2q'
// for m's point q'.  A 1->3 split leaves q' in position 0 of m and edges 1,
// 2 in 2+2q', 3+2q'; an edge split leaves q' where m's one outer edge it
// keeps faces and its other outer edge in 2+2q' (first triangle) or 3+2q'
// (second triangle, bit 3 of the flags).
GCDT_HD int split_child(const int4& cv, int s, const int4& mv, int m, int ms) {
    const int u = comp(cv, nx3(s)), v = comp(cv, nx3(nx3(s)));
    const int p1 = nx3(ms), p2 = nx3(p1);
    const int w1 = comp(mv, p1), w2 = comp(mv, p2);
    const bool k1 = w1 == u || w1 == v, k2 = w2 == u || w2 == v;
    if (k1 && k2) return m;
    const int p = k1 ? p2 : p1;
    const int qm = comp(mv, p);
    return 2 + 2 * qm + (ms == nx3(p) ? ((mv.w >> 3) & 1) : 1);
}

// Flip-queue entry: triangle id << 3 | mask of the slots whose edges may
// not be locally Delaunay (the others are known to be).
GCDT_HD int qentry(int t, int mask) { return (int)(((unsigned)t << 3) | (unsigned)mask); }
GCDT_HD int qtri(int e) { return (int)((unsigned)e >> 3); }

// The children of the inserted points are distinct triangles, so the first
// flip queue of a round needs no de-duplication.

// The edge in slot s of split child ch names its old neighbour: point it at
// the neighbour's child that holds the edge when the neighbour was split in
// this round too (its adjacency row's round stamp; flips of the round come
// after this phase), else write ch into the neighbour's row.  The
// neighbour's record is the sector the second case writes anyway.
GCDT_HD void resolve_split_edge(const Ctx& c, int ch, int s) {
    int4* row = &tri_a(c, ch);
    int old = comp(*row, s);
    if (old < 0) return;
    int m = old >> 2, ms = old & 3;
    const int4 mv = tri_v(c, m), ma = tri_a(c, m);
    if (ma.w == (int)c.round) {
        ((int*)row)[s] = enc(split_child(tri_v(c, ch), s, mv, m, ms), ms);
    } else {
        ((int*)&tri_a(c, m))[ms] = enc(ch, s);
    }
}

// Resolve outer adjacency of the children of one inserted point and queue
// them for the flip phase (c.sr = first sub-round of this round).
GCDT_HD void body_fix_f(const Ctx& c, int2 w) {
    int q = w.x >> 3, t = w.y;
    int T1 = 2 + 2 * q, T2 = 3 + 2 * q;
    int code = w.x & 7;
    // Only the old edges need a test: a spoke from q to a corner of the split
    // triangle is locally Delaunay (q lies inside the old empty circumcircle,
    // so the circle through q and the spoke's far edge excludes the third
    // corner; on an edge split the spoke's quadrilateral is not even convex).
    if (code == 7) {
        resolve_split_edge(c, t, 0);
        resolve_split_edge(c, T1, 1);
        resolve_split_edge(c, T2, 2);
        int* qn = c.queue_next + append_slots(&c.cnt->cur_q, c.base_q, 3);
        qn[0] = qentry(t, 1); qn[1] = qentry(T1, 2); qn[2] = qentry(T2, 4);
    } else {
        int e = code;
        int e1 = nx3(e), e_2 = nx3(e1);
        int en = comp(tri_a(c, T1), e);     // A2 slot e = enc(B1, e2)
        int n = en >> 2, e2 = en & 3;
        int f1 = nx3(e2), f2 = nx3(f1);
        resolve_split_edge(c, t, e1);
        resolve_split_edge(c, T1, e_2);
        resolve_split_edge(c, n, f1);
        resolve_split_edge(c, T2, f2);
        // outer edge and the half of the split edge
        int* qn = c.queue_next + append_slots(&c.cnt->cur_q, c.base_q, 4);
        qn[0] = qentry(t, (1 << e1) | (1 << e)); qn[1] = qentry(T1, (1 << e_2) | (1 << e));
        qn[2] = qentry(n, (1 << f1) | (1 << e2)); qn[3] = qentry(T2, (1 << f2) | (1 << e2));
    }
}
GCDT_HD void body_fix(const Ctx& c, int k) { body_fix_f(c, c.winners[k]); }

// ---------------------------------------------------------------- flips

// Queue entry t: find the first edge of t that is not locally Delaunay
// (perturbed incircle > 0, not a constraint) and claim both triangles.
// The claim priority hash32(4t+i) is unique (hash32 is a bijection); the
// smallest wins both triangles (atomicMax of its complement), so conflicts
// resolve like a random-priority independent set, whatever the schedule.
GCDT_HD void body_flip_check(const Ctx& c, int k) {
    int qe = c.queue[k];
    int t = qtri(qe), mask = qe & 7;
    int4 tv = tri_v(c, t), ta = tri_a(c, t);
    // a carried entry (first sub-round of a round, before its flips) whose
    // triangle was split this round: the split's own queue entries test
    // every old edge of it
    if (k < c.carry_n && ta.w == (int)c.round) { c.cand[k] = make_int2(-1, -1); return; }
    // the edges to test: in the mask, with a neighbour, not constraints
    int live = mask & ~tv.w & ((ta.x >= 0) | ((ta.y >= 0) << 1) | ((ta.z >= 0) << 2));
    // issue every test's loads before the first test, so the neighbour rows
    // and the opposite points of up to three edges are in flight together
    int d0 = 0, d1 = 0, d2 = 0;
    if (live & 1) d0 = comp(tri_v(c, ta.x >> 2), ta.x & 3);
    if (live & 2) d1 = comp(tri_v(c, ta.y >> 2), ta.y & 3);
    if (live & 4) d2 = comp(tri_v(c, ta.z >> 2), ta.z & 3);
    int2 a = c.P[tv.x], b = c.P[tv.y], cc = c.P[tv.z];
    int2 p0 = c.P[d0], p1 = c.P[d1], p2 = c.P[d2];
    // first edge in slot order that is not locally Delaunay
    int i = -1;
    if ((live & 1) && incircle_sos(a, b, cc, p0) > 0) i = 0;
    else if ((live & 2) && incircle_sos(a, b, cc, p1) > 0) i = 1;
    else if ((live & 4) && incircle_sos(a, b, cc, p2) > 0) i = 2;
    if (i < 0) { c.cand[k] = make_int2(-1, -1); return; }
    int en = comp(ta, i);
    int n = en >> 2;
    int key = enc(t, i);
    unsigned long long ck = ((unsigned long long)c.sr << 32) | (0xffffffffu - hash32((uint32_t)key));
    at_max64(&c.claim[t], ck);
    at_max64(&c.claim[n], ck);
    c.cand[k] = make_int2(key, en);
}

// Two queue entries per thread (k1 < 0: only k0), each stage's loads issued
// for both entries before either is used: twice the loads in flight per
// thread for this latency-bound pass.  Same result as body_flip_check on
// each entry.
template <int W>
GCDT_HD void flip_check_multi_f(const Ctx& c, const int (&ks)[W], const int2 (&f)[W]) {
    bool on[W];
    int t[W], mask[W];
#pragma unroll
    for (int u = 0; u < W; ++u) {
        on[u] = ks[u] >= 0;
        int qe = on[u] ? f[u].x : 0;
        t[u] = qtri(qe);
        mask[u] = qe & 7;
    }
    int4 tv[W], ta[W];
#pragma unroll
    for (int u = 0; u < W; ++u) {
        tv[u] = on[u] ? tri_v(c, t[u]) : make_int4(0, 0, 0, 7);
        ta[u] = on[u] ? tri_a(c, t[u]) : make_int4(-1, -1, -1, 0);
        // a carried entry whose triangle was split this round (as above)
        if (on[u] && ks[u] < c.carry_n && ta[u].w == (int)c.round) {
            on[u] = false;
            tv[u] = make_int4(0, 0, 0, 7);
            ta[u] = make_int4(-1, -1, -1, 0);
        }
    }
    int live[W], d[W][3];
#pragma unroll
    for (int u = 0; u < W; ++u) {
        live[u] = mask[u] & ~tv[u].w & ((ta[u].x >= 0) | ((ta[u].y >= 0) << 1) | ((ta[u].z >= 0) << 2));
        d[u][0] = (live[u] & 1) ? comp(tri_v(c, ta[u].x >> 2), ta[u].x & 3) : 0;
        d[u][1] = (live[u] & 2) ? comp(tri_v(c, ta[u].y >> 2), ta[u].y & 3) : 0;
        d[u][2] = (live[u] & 4) ? comp(tri_v(c, ta[u].z >> 2), ta[u].z & 3) : 0;
    }
    int2 a[W], b[W], cc[W], p[W][3];
#pragma unroll
    for (int u = 0; u < W; ++u) {
        a[u] = c.P[tv[u].x]; b[u] = c.P[tv[u].y]; cc[u] = c.P[tv[u].z];
        p[u][0] = c.P[d[u][0]]; p[u][1] = c.P[d[u][1]]; p[u][2] = c.P[d[u][2]];
    }
#pragma unroll
    for (int u = 0; u < W; ++u) {
        if (ks[u] < 0) continue;
        if (!on[u]) { c.cand[ks[u]] = make_int2(-1, -1); continue; }   // dropped carried entry
        int i = -1;
        if ((live[u] & 1) && incircle_sos(a[u], b[u], cc[u], p[u][0]) > 0) i = 0;
        else if ((live[u] & 2) && incircle_sos(a[u], b[u], cc[u], p[u][1]) > 0) i = 1;
        else if ((live[u] & 4) && incircle_sos(a[u], b[u], cc[u], p[u][2]) > 0) i = 2;
        if (i < 0) { c.cand[ks[u]] = make_int2(-1, -1); continue; }
        int en = comp(ta[u], i);
        int n = en >> 2;
        int key = enc(t[u], i);
        unsigned long long ck = ((unsigned long long)c.sr << 32) | (0xffffffffu - hash32((uint32_t)key));
        at_max64(&c.claim[t[u]], ck);
        at_max64(&c.claim[n], ck);
        c.cand[ks[u]] = make_int2(key, en);
    }
}

// The first word item k of a flip pass loads (the check: its queue entry;
// the flip: its candidate; the fix: a flipped pair's queue entry or a
// candidate), so that a caller can issue it early.
enum FlipPass : int { FP_CHECK, FP_DO, FP_FIX };
GCDT_HD int2 flip_first(const Ctx& c, int pass, int k) {
    if (k < 0) return make_int2(-1, -1);
    if (pass == FP_CHECK) return make_int2(c.queue[k], 0);
    if (pass == FP_DO) return c.cand[k];
    // a flipped pair: both its queue entries (t's, then n's; 8-byte aligned)
    return k >= c.list_n ? c.cand[k - c.list_n] : *reinterpret_cast<const int2*>(c.queue_next + 2 * k);
}

template <int W>
GCDT_HD void flip_check_multi(const Ctx& c, const int (&ks)[W]) {
    int2 f[W];
#pragma unroll
    for (int u = 0; u < W; ++u) f[u] = flip_first(c, FP_CHECK, ks[u]);
    flip_check_multi_f<W>(c, ks, f);
}

GCDT_HD void body_flip_check_pair(const Ctx& c, int k0, int k1) {
    const int ks[2] = {k0, k1};
    flip_check_multi<2>(c, ks);
}

// Winners flip: t=(A,B,C) with A in slot i, n=(D,C,B) with D in slot j
// become t=(A,B,D), n=(A,D,C), and both go to the next queue.  Losers are
// re-queued by body_flip_fix once it is known that nobody flipped them, so
// every triangle enters the next queue at most once without any
// de-duplication.
// The flip of claimed candidate (t slot i, n slot j) given both rows, by
// value (the rows are overwritten here): writes the two new triangles and
// their flip maps.
GCDT_HD void do_flip(const Ctx& c, int t, int i, int n, int j,
                     const int4 tv, const int4 ta, const int4 nv, const int4 na) {
    int i1 = nx3(i), i2 = nx3(i1), j1 = nx3(j), j2 = nx3(j1);
    int A = comp(tv, i), B = comp(tv, i1), C = comp(tv, i2), D = comp(nv, j);
    int ft = tv.w, fn = nv.w;
    // t keeps side 0 of the flip, n side 1; both carry the sub-round
    const int stamp = (int)c.sr << 4;
    tri_v(c, t) = make_int4(A, B, D, ((fn >> j1) & 1) | (((ft >> i2) & 1) << 2) | stamp);
    tri_a(c, t) = make_int4(comp(na, j1), enc(n, 2), comp(ta, i2), (int)c.round);
    tri_v(c, n) = make_int4(A, D, C, ((fn >> j2) & 1) | (((ft >> i1) & 1) << 1) | 8 | stamp);
    tri_a(c, n) = make_int4(comp(na, j2), comp(ta, i1), enc(t, 1), (int)c.round);
}

// The edge in slot s of flipped triangle tt (vertex row tv) had the old
// neighbour `old`; mv is that neighbour's vertex row now and mp its partner
// slots (adjacency slots 1 and 2).  If that neighbour flipped in this
// sub-round too, returns the triangle and slot that now hold the edge: its
// own new triangle when both endpoints are in it, else its partner's --
// the pair (A,B,D) side 0 / (A,D,C) side 1 has the outer edges BD, AB and
// DC, CA, so the partner's slot follows from whether the edge ends at D.
// Otherwise -1 (the old neighbour keeps the edge).  The partner slots are
// the flip's new diagonal, which no fix pass writes.
GCDT_HD int moved_edge(const Ctx& c, const int4& tv, int s, int old, const int4& mv, int2 mp) {
    if (flip_stamp(mv.w) != (int)c.sr) return -1;
    const int u = comp(tv, nx3(s)), v = comp(tv, nx3(nx3(s)));
    const int su = slot_of_or_none(mv, u), sv = slot_of_or_none(mv, v);
    if (su >= 0 && sv >= 0) return enc(old >> 2, 3 - su - sv);
    if (((mv.w >> 3) & 1) == 0) {           // it became (A,B,D): the edge is DC or CA of (A,D,C)
        const int D = mv.z;
        return enc(mp.x >> 2, (u == D || v == D) ? 0 : 1);
    }
    const int D = mv.y;                      // it became (A,D,C): the edge is BD or AB of (A,B,D)
    return enc(mp.y >> 2, (u == D || v == D) ? 0 : 2);
}

// The partner slots (adjacency slots 1 and 2) of triangle m.
GCDT_HD int2 partner_slots(const Ctx& c, int m) {
    const int* a = reinterpret_cast<const int*>(&tri_a(c, m));
    return make_int2(a[1], a[2]);
}

GCDT_HD void body_flip_do(const Ctx& c, int k) {
    int2 cd = c.cand[k];
    if (cd.x < 0) return;
    int t = cd.x >> 2, i = cd.x & 3;
    int n = cd.y >> 2, j = cd.y & 3;
    unsigned long long ck = ((unsigned long long)c.sr << 32) | (0xffffffffu - hash32((uint32_t)cd.x));
    if (c.claim[t] != ck || c.claim[n] != ck) return;
    do_flip(c, t, i, n, j, tri_v(c, t), tri_a(c, t), tri_v(c, n), tri_a(c, n));
    // The new diagonal AD is locally Delaunay: queue the four outer edges.
    // Flip number f of the sub-round owns entries 2f, 2f+1 of the next
    // queue; body_flip_fix reads the pairs from there and appends the
    // re-queued losers after them.
    int* qn = c.queue_next + 2 * append_slot(&c.cnt->cur_flip, c.base_flip);
    qn[0] = qentry(t, 5);    // (A,B,D): BD and AB
    qn[1] = qentry(n, 3);    // (A,D,C): DC and CA
}

// Two candidates per thread (k1 < 0: only k0): the candidate and claim
// loads of both are in flight together; the winners (a minority) then
// flip one at a time, so only one pair of rows is live at once.
GCDT_HD void body_flip_do_pair_f(const Ctx& c, const int (&ks)[2], const int2 (&first)[2]) {
    int2 cd[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) cd[u] = ks[u] >= 0 ? first[u] : make_int2(-1, -1);
    bool win[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        unsigned long long ck = ((unsigned long long)c.sr << 32) | (0xffffffffu - hash32((uint32_t)cd[u].x));
        unsigned long long c0 = cd[u].x >= 0 ? c.claim[cd[u].x >> 2] : 0ull;
        unsigned long long c1 = cd[u].x >= 0 ? c.claim[cd[u].y >> 2] : 0ull;
        win[u] = cd[u].x >= 0 && c0 == ck && c1 == ck;
    }
    const int nw = (int)win[0] + (int)win[1];
    if (nw == 0) return;
    int f = append_slots(&c.cnt->cur_flip, c.base_flip, nw);
#pragma unroll 1
    for (int u = 0; u < 2; ++u) {
        if (!win[u]) continue;
        int t = cd[u].x >> 2, n = cd[u].y >> 2;
        do_flip(c, t, cd[u].x & 3, n, cd[u].y & 3, tri_v(c, t), tri_a(c, t), tri_v(c, n), tri_a(c, n));
        int* qn = c.queue_next + 2 * f++;
        qn[0] = qentry(t, 5);
        qn[1] = qentry(n, 3);
    }
}

GCDT_HD void body_flip_do_pair(const Ctx& c, int k0, int k1) {
    const int ks[2] = {k0, k1};
    const int2 f[2] = {flip_first(c, FP_DO, k0), flip_first(c, FP_DO, k1)};
    body_flip_do_pair_f(c, ks, f);
}

GCDT_HD void resolve_flip_edge(const Ctx& c, int tt, int s) {
    int4* row = &tri_a(c, tt);
    int old = comp(*row, s);
    if (old < 0) return;
    int m = old >> 2, ms = old & 3;
    const int e = moved_edge(c, tri_v(c, tt), s, old, tri_v(c, m), partner_slots(c, m));
    if (e >= 0) ((int*)row)[s] = e;
    else ((int*)&tri_a(c, m))[ms] = enc(tt, s);
}

// k < c.list_n: resolve the outer adjacency of flipped pair k.
// Otherwise queue entry k - c.list_n: a candidate that did not flip and
// whose triangle nobody flipped goes back to the queue, after the
// 2 * c.list_n entries of the flipped pairs.
GCDT_HD void body_flip_fix(const Ctx& c, int k) {
    if (k >= c.list_n) {
        int2 cd = c.cand[k - c.list_n];
        if (cd.x >= 0 && flip_stamp(tri_v(c, cd.x >> 2).w) != (int)c.sr)
            c.queue_next[2 * c.list_n + append_slot(&c.cnt->cur_q, c.base_q)] = c.queue[k - c.list_n];
        return;
    }
    int t = qtri(c.queue_next[2 * k]);
    int n = tri_a(c, t).y >> 2;
    resolve_flip_edge(c, t, 0);
    resolve_flip_edge(c, t, 2);
    resolve_flip_edge(c, n, 0);
    resolve_flip_edge(c, n, 1);
}

// The edge in slot s of flipped triangle tt (vertex row tv) named the old
// neighbour `old` (mv, mp: its vertex row and partner slots now): the write
// resolve_flip_edge would make.
GCDT_HD void resolve_flip_loaded(const Ctx& c, int tt, const int4& tv, int s, int old, const int4& mv, int2 mp) {
    if (old < 0) return;
    const int e = moved_edge(c, tv, s, old, mv, mp);
    if (e >= 0) ((int*)&tri_a(c, tt))[s] = e;
    else ((int*)&tri_a(c, old >> 2))[old & 3] = enc(tt, s);
}

// Two items per thread (k1 < 0: only k0), as body_flip_fix on each, with
// every stage's loads issued for both items first.
GCDT_HD void body_flip_fix_pair_f(const Ctx& c, const int (&ks)[2], const int2 (&f)[2]) {
    const int4 none = make_int4(-1, -1, -1, -1);
    int kind[2], t[2], n[2];    // kind 0: nothing, 1: flipped pair, 2: candidate of the queue
    int2 cd[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        kind[u] = ks[u] < 0 ? 0 : (ks[u] >= c.list_n ? 2 : 1);
        cd[u] = kind[u] == 2 ? f[u] : make_int2(-1, -1);
        t[u] = kind[u] == 1 ? qtri(f[u].x) : 0;
        n[u] = kind[u] == 1 ? qtri(f[u].y) : 0;
    }
    // both triangles of a flipped pair at once (the pair's two queue entries
    // name them), so their old neighbours are one load further on
    int4 tv[2], ta[2], nv[2], na[2];
    int flw[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        tv[u] = kind[u] == 1 ? tri_v(c, t[u]) : none;
        ta[u] = kind[u] == 1 ? tri_a(c, t[u]) : none;
        nv[u] = kind[u] == 1 ? tri_v(c, n[u]) : none;
        na[u] = kind[u] == 1 ? tri_a(c, n[u]) : none;
        flw[u] = (kind[u] == 2 && cd[u].x >= 0) ? tri_v(c, cd[u].x >> 2).w : 0;
    }
    // re-queue the candidates that did not flip and whose triangle nobody flipped
    int rq[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) rq[u] = (kind[u] == 2 && cd[u].x >= 0 && flip_stamp(flw[u]) != (int)c.sr) ? 1 : 0;
    if (rq[0] | rq[1]) {
        int at = 2 * c.list_n + append_slots(&c.cnt->cur_q, c.base_q, rq[0] + rq[1]);
#pragma unroll
        for (int u = 0; u < 2; ++u)
            if (rq[u]) c.queue_next[at++] = c.queue[ks[u] - c.list_n];
    }
    // flipped pairs: t's outer edges 0, 2 and n's outer edges 0, 1; each old
    // neighbour's row (one sector, which the fix writes when that neighbour
    // did not flip) tells whether it flipped and where the edge went
    int4 m0[2], m2[2];
    int2 p0[2], p2[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const bool l0 = kind[u] == 1 && ta[u].x >= 0, l2 = kind[u] == 1 && ta[u].z >= 0;
        m0[u] = l0 ? tri_v(c, ta[u].x >> 2) : none;
        p0[u] = l0 ? partner_slots(c, ta[u].x >> 2) : make_int2(-1, -1);
        m2[u] = l2 ? tri_v(c, ta[u].z >> 2) : none;
        p2[u] = l2 ? partner_slots(c, ta[u].z >> 2) : make_int2(-1, -1);
    }
    int4 g0[2], g1[2];
    int2 q0[2], q1[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const bool l0 = kind[u] == 1 && na[u].x >= 0, l1 = kind[u] == 1 && na[u].y >= 0;
        g0[u] = l0 ? tri_v(c, na[u].x >> 2) : none;
        q0[u] = l0 ? partner_slots(c, na[u].x >> 2) : make_int2(-1, -1);
        g1[u] = l1 ? tri_v(c, na[u].y >> 2) : none;
        q1[u] = l1 ? partner_slots(c, na[u].y >> 2) : make_int2(-1, -1);
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        if (kind[u] != 1) continue;
        resolve_flip_loaded(c, t[u], tv[u], 0, ta[u].x, m0[u], p0[u]);
        resolve_flip_loaded(c, t[u], tv[u], 2, ta[u].z, m2[u], p2[u]);
        resolve_flip_loaded(c, n[u], nv[u], 0, na[u].x, g0[u], q0[u]);
        resolve_flip_loaded(c, n[u], nv[u], 1, na[u].y, g1[u], q1[u]);
    }
}

GCDT_HD void body_flip_fix_pair(const Ctx& c, int k0, int k1) {
    const int ks[2] = {k0, k1};
    const int2 f[2] = {flip_first(c, FP_FIX, k0), flip_first(c, FP_FIX, k1)};
    body_flip_fix_pair_f(c, ks, f);
}

// ---------------------------------------------------------------- constraints

// Map segment endpoints to sorted ids; reject malformed segments.
GCDT_HD void body_seg_init(const Ctx& c, int k) {
    int2 ab = c.in_cons[k];
    if (ab.x < 0 || ab.y < 0 || ab.x >= c.n || ab.y >= c.n || ab.x == ab.y) {
        fail(c, ST_BAD_INPUT);
        c.seg[k] = make_int4(0, 0, 0, 0);   // .z != -1: not a valid segment
    } else {
        c.seg[k] = make_int4(c.rank[ab.x], c.rank[ab.y], -1, 0);
    }
    c.pend[k] = k;
}

GCDT_HD void mark_edge(const Ctx& c, int t, int s) {
    at_or(&tri_v(c, t).w, 1 << s);
    int en = comp(tri_a(c, t), s);
    if (en >= 0) at_or(&tri_v(c, en >> 2).w, 1 << (en & 3));
}

// Walk from the current start vertex a of a pending segment towards b.
// Existing edges along ab (through collinear vertices) are flagged and
// skipped; the first sub-segment (a, stop) that crosses triangles is
// recorded: pinfo = (4*t+i of the first crossed edge, triangles crossed).
// A crossed constraint edge means the input constraints cross.
GCDT_HD void body_cwalk(const Ctx& c, int k) {
    int sk = c.pend[k];
    int4 sg = c.seg[sk];
    int a = sg.x, b = sg.y;
    int2 pb = c.P[b];
    for (int guard = 0; guard <= c.n + 4; ++guard) {
        if (a == b) {
            c.seg[sk].x = a;
            c.pinfo[k] = make_int4(-1, 0, 0, 0);
            return;
        }
        int2 pa = c.P[a];
        int t0 = c.vt[a], t = t0;
        int found = -1, fslot = 0, via = -1, et = -1, es = 0;
        for (int g2 = 0; g2 < (1 << 16); ++g2) {
            int4 tv = tri_v(c, t);
            int i = slot_of(tv, a), i1 = nx3(i), i2 = nx3(i1);
            int u = comp(tv, i1), w = comp(tv, i2);
            if (u == b) { via = b; et = t; es = i2; break; }
            if (w == b) { via = b; et = t; es = i1; break; }
            int2 pu = c.P[u], pw = c.P[w];
            int ou = orient2d(pa, pu, pb), ow = orient2d(pa, pw, pb);
            if (ou == 0 && dot3(pa, pu, pb) > 0) { via = u; et = t; es = i2; break; }
            if (ow == 0 && dot3(pa, pw, pb) > 0) { via = w; et = t; es = i1; break; }
            if (ou > 0 && ow < 0) { found = t; fslot = i; break; }
            int nb = comp(tri_a(c, t), i2);
            if (nb < 0) break;
            t = nb >> 2;
            if (t == t0) break;
        }
        if (via >= 0) {
            mark_edge(c, et, es);
            a = via;
            continue;
        }
        if (found < 0) { fail(c, ST_CONSTRAINT_FAIL); c.pinfo[k] = make_int4(-1, 0, 0, 0); return; }
        int cur = found, cs = fslot, count = 1, stop = -1;
        for (int steps = 0; steps <= c.ntri; ++steps) {
            int4 tv = tri_v(c, cur);
            if ((tv.w >> cs) & 1) { fail(c, ST_CONSTRAINT_FAIL); c.pinfo[k] = make_int4(-1, 0, 0, 0); return; }
            int en = comp(tri_a(c, cur), cs);
            if (en < 0) { fail(c, ST_CONSTRAINT_FAIL); c.pinfo[k] = make_int4(-1, 0, 0, 0); return; }
            int n = en >> 2, j = en & 3;
            int x = comp(tri_v(c, n), j);
            count++;
            if (x == b) { stop = b; break; }
            int ox = orient2d(pa, pb, c.P[x]);
            if (ox == 0) { stop = x; break; }
            cur = n;
            cs = ox < 0 ? nx3(nx3(j)) : nx3(j);
        }
        if (stop < 0) { fail(c, ST_ITER_LIMIT); c.pinfo[k] = make_int4(-1, 0, 0, 0); return; }
        c.seg[sk] = make_int4(a, b, stop, 0);
        c.pinfo[k] = make_int4(enc(found, fslot), count, 0, -1);
        return;
    }
    fail(c, ST_ITER_LIMIT);
    c.pinfo[k] = make_int4(-1, 0, 0, 0);
}

// Record the crossed triangles of the pending sub-segment and the triangles
// around them, and claim all of them for this segment (smallest hash32 of
// the segment id wins, so chains of adjacent segments progress in parallel).
// Scratch per entry: [0,kt) crossed chain, [kt, 2kt+2) ring, [2kt+2, 3kt+2) queue.
GCDT_HD void body_cclaim(const Ctx& c, int k) {
    int4 pi = c.pinfo[k];
    if (pi.x < 0) return;
    int sk = c.pend[k];
    int4 sg = c.seg[sk];
    int kt = pi.y;
    int cap = 3 * kt + 4;
    unsigned long long b0 = at_add64(&c.cnt->cur_scr, (unsigned long long)cap) - c.base_scr;
    if (b0 + cap > (unsigned long long)c.scratch_cap) { c.pinfo[k].w = -2; return; }
    int base = (int)b0;
    int* L = c.scratch + base;
    int* R = L + kt;
    unsigned long long key = ((unsigned long long)c.sr << 32) | (0xffffffffu - hash32((uint32_t)sk));
    int2 pa = c.P[sg.x], pb = c.P[sg.y];
    int cur = pi.x >> 2, cs = pi.x & 3;
    L[0] = cur;
    for (int m = 1; m < kt; ++m) {
        int en = comp(tri_a(c, cur), cs);
        int n = en >> 2, j = en & 3;
        L[m] = n;
        if (m == kt - 1) break;
        int x = comp(tri_v(c, n), j);
        int ox = orient2d(pa, pb, c.P[x]);
        cur = n;
        cs = ox < 0 ? nx3(nx3(j)) : nx3(j);
    }
    int nr = 0;
    for (int m = 0; m < kt; ++m) {
        int4 ta = tri_a(c, L[m]);
        for (int s = 0; s < 3; ++s) {
            int en = comp(ta, s);
            if (en < 0) continue;
            int nb = en >> 2;
            if ((m > 0 && nb == L[m - 1]) || (m + 1 < kt && nb == L[m + 1])) continue;
            if (nr < kt + 2) R[nr++] = nb;
        }
    }
    for (int m = 0; m < kt; ++m) at_max64(&c.claim[L[m]], key);
    for (int r = 0; r < nr; ++r) at_max64(&c.claim[R[r]], key);
    c.pinfo[k] = make_int4(pi.x, kt, base, nr);
}

// Flip the edge opposite slot i of t and update every neighbour in place
// (the caller owns t, its partner and their neighbours).
GCDT_HD int flip_local(const Ctx& c, int t, int i) {
    int4 tv = tri_v(c, t), ta = tri_a(c, t);
    int en = comp(ta, i);
    int n = en >> 2, j = en & 3;
    int4 nv = tri_v(c, n), na = tri_a(c, n);
    int i1 = nx3(i), i2 = nx3(i1), j1 = nx3(j), j2 = nx3(j1);
    int A = comp(tv, i), B = comp(tv, i1), C = comp(tv, i2), D = comp(nv, j);
    int ft = tv.w, fn = nv.w;
    int oBD = comp(na, j1), oAB = comp(ta, i2), oDC = comp(na, j2), oCA = comp(ta, i1);
    tri_v(c, t) = make_int4(A, B, D, ((fn >> j1) & 1) | (((ft >> i2) & 1) << 2));
    tri_a(c, t) = make_int4(oBD, enc(n, 2), oAB, (int)c.round);
    tri_v(c, n) = make_int4(A, D, C, ((fn >> j2) & 1) | (((ft >> i1) & 1) << 1));
    tri_a(c, n) = make_int4(oDC, oCA, enc(t, 1), (int)c.round);
    if (oBD >= 0) ((int*)&tri_a(c, oBD >> 2))[oBD & 3] = enc(t, 0);
    if (oAB >= 0) ((int*)&tri_a(c, oAB >> 2))[oAB & 3] = enc(t, 2);
    if (oDC >= 0) ((int*)&tri_a(c, oDC >> 2))[oDC & 3] = enc(n, 0);
    if (oCA >= 0) ((int*)&tri_a(c, oCA >> 2))[oCA & 3] = enc(n, 1);
    c.vt[A] = t; c.vt[B] = t; c.vt[D] = t; c.vt[C] = n;
    return n;
}

GCDT_HD void push_lawson(const Ctx& c, int t) {
    if (at_exch(&c.qst[t], (int)c.lawson_sr) != (int)c.lawson_sr)
        c.lq[append_slot(&c.cnt->cur_law, c.base_law)] = qentry(t, 7);
}

// Owners of all their triangles recover the sub-segment (a, stop) by
// Sloan's method: flip crossing edges whose quadrilateral is strictly
// convex until none crosses.  Others retry next round.
GCDT_HD void body_cproc(const Ctx& c, int k) {
    int4 pi = c.pinfo[k];
    int sk = c.pend[k];
    if (pi.x < 0) return;                              // finished in the walk
    if (pi.w < 0) { c.pend_next[append_slot(&c.cnt->cur_pend, c.base_pend)] = sk; return; }
    int kt = pi.y;
    int* L = c.scratch + pi.z;
    int* R = L + kt;
    int* Q = R + kt + 2;
    unsigned long long key = ((unsigned long long)c.sr << 32) | (0xffffffffu - hash32((uint32_t)sk));
    bool own = true;
    for (int m = 0; m < kt && own; ++m) own = c.claim[L[m]] == key;
    for (int r = 0; r < pi.w && own; ++r) own = c.claim[R[r]] == key;
    if (!own) { c.pend_next[append_slot(&c.cnt->cur_pend, c.base_pend)] = sk; return; }
    int4 sg = c.seg[sk];
    int a = sg.x, b = sg.y, stop = sg.z;
    int2 pa = c.P[a], pb = c.P[b];
    // crossing edges between consecutive chain triangles
    int qn = 0;
    for (int m = 0; m + 1 < kt; ++m) {
        int4 ta = tri_a(c, L[m]);
        int s = (ta.x >> 2) == L[m + 1] ? 0 : ((ta.y >> 2) == L[m + 1] ? 1 : 2);
        Q[qn++] = enc(L[m], s);
    }
    int head = 0, size = qn;
    long long guard = 0, limit = 64LL * (kt + 4) * (kt + 4);
    while (size > 0) {
        if (++guard > limit) { fail(c, ST_ITER_LIMIT); return; }
        int e = Q[head]; head = head + 1 == kt ? 0 : head + 1; size--;
        int t = e >> 2, i = e & 3;
        int4 tv = tri_v(c, t);
        int en = comp(tri_a(c, t), i);
        int n = en >> 2, j = en & 3;
        int A = comp(tv, i), B = comp(tv, nx3(i)), C = comp(tv, nx3(nx3(i)));
        int D = comp(tri_v(c, n), j);
        int2 PA = c.P[A], PD = c.P[D];
        int s1 = orient2d(PA, PD, c.P[B]), s2 = orient2d(PA, PD, c.P[C]);
        int tail = head + size; if (tail >= kt) tail -= kt;
        if (!((s1 > 0 && s2 < 0) || (s1 < 0 && s2 > 0))) { Q[tail] = e; size++; continue; }
        int i1 = nx3(i), i2 = nx3(i1), j1 = nx3(j), j2 = nx3(j1);
        flip_local(c, t, i);
        for (int r = 0, pos = head; r < size; ++r, pos = pos + 1 == kt ? 0 : pos + 1) {
            int q = Q[pos];
            if (q == enc(t, i1)) Q[pos] = enc(n, 1);
            else if (q == enc(t, i2)) Q[pos] = enc(t, 2);
            else if (q == enc(n, j1)) Q[pos] = enc(t, 0);
            else if (q == enc(n, j2)) Q[pos] = enc(n, 0);
        }
        int oA = orient2d(pa, pb, PA), oD = orient2d(pa, pb, PD);
        if ((oA > 0 && oD < 0) || (oA < 0 && oD > 0)) { Q[tail] = enc(t, 1); size++; }
    }
    // flag the recovered edge (a, stop) on both sides
    for (int m = 0; m < kt; ++m) {
        int4 tv = tri_v(c, L[m]);
        bool ha = tv.x == a || tv.y == a || tv.z == a;
        bool hs = tv.x == stop || tv.y == stop || tv.z == stop;
        if (ha && hs) {
            int s3 = 3 - slot_of(tv, a) - slot_of(tv, stop);
            mark_edge(c, L[m], s3);
            break;
        }
    }
    for (int m = 0; m < kt; ++m) push_lawson(c, L[m]);
    c.seg[sk].x = stop;
    if (stop != b) c.pend_next[append_slot(&c.cnt->cur_pend, c.base_pend)] = sk;
}

// ---------------------------------------------------------------- output

GCDT_HD void body_output(const Ctx& c, int t) {
    int4 tv = tri_v(c, t), ta = tri_a(c, t);
    c.out_tris[3 * t + 0] = c.perm[tv.x];
    c.out_tris[3 * t + 1] = c.perm[tv.y];
    c.out_tris[3 * t + 2] = c.perm[tv.z];
    c.out_adj[3 * t + 0] = ta.x < 0 ? -1 : ta.x >> 2;
    c.out_adj[3 * t + 1] = ta.y < 0 ? -1 : ta.y >> 2;
    c.out_adj[3 * t + 2] = ta.z < 0 ? -1 : ta.z >> 2;
    c.out_cflags[t] = (unsigned char)(tv.w & 7);
}

}  // namespace gcdt
