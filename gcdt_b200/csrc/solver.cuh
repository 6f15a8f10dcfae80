// solver.cuh -- round structure of one CDT solve, written once against a
// launch backend (kernels.cu supplies the CUDA one).
//
// Phases (reference stage it replaces, yingtix/gCDT):
//   0  Morton keys, radix sort, gather: points in spatial order
//      (kernel.cu:1966-2019 reorderPoint, there applied before the flip stage)
//   1  insertion rounds: every uninserted point votes for its triangle, one
//      winner per triangle splits it (1->3, or 2->4 on an edge), adjacency is
//      resolved, then compacted flip sub-rounds restore the Delaunay property
//      and points of changed triangles re-locate by walking
//      (rawMesh.cu:867-908 rawMeshInsert + kernel.cu:4697-4860 delaunayNew)
//   2  constraint recovery by walk-and-flip, then constrained flips
//      (addConstraints.cu:1723-1835 + the delaunayNew flip loop with noFlips)
//   3  output in input index order with adjacency and constraint flags
#pragma once
#include "layout.cuh"
#include "mesh.cuh"

namespace gcdt {

enum Kern : int {
    K_KEYS, K_GATHER, K_ROOT, K_INITLOC, K_RELOC_VOTE, K_SPLIT, K_FIX,
    K_FLIP_CHECK, K_FLIP_DO, K_FLIP_FIX, K_OUTPUT,
    K_VT, K_SEG_INIT, K_CWALK, K_CCLAIM, K_CPROC,
    K_COUNT
};

struct SolveStats {
    long long rounds = 0;
    long long flip_subrounds = 0;
    long long flips = 0;
    long long constraint_rounds = 0;
    long long constraint_flips = 0;
    long long host_syncs = 0;
};

inline Ctx bind_ctx(char* base, const Plan& p) {
    Ctx c{};
    c.n = (int)p.n; c.s = (int)p.s; c.ntri = (int)p.ntri;
    c.keys = (unsigned long long*)(base + p.o_keys);
    c.keys_alt = (unsigned long long*)(base + p.o_keys_alt);
    c.vals = (int*)(base + p.o_vals);
    c.vals_alt = (int*)(base + p.o_vals_alt);
    c.P = (int2*)(base + p.o_P);
    c.perm = (int*)(base + p.o_perm);
    c.rank = (int*)(base + p.o_rank);
    c.TV = (int4*)(base + p.o_TV);
    c.TA = (int4*)(base + p.o_TA);
    c.loc = (int*)(base + p.o_loc);
    c.pedge = (signed char*)(base + p.o_pedge);
    c.act = (int*)(base + p.o_actA);
    c.act_next = (int*)(base + p.o_actB);
    c.vote = (unsigned long long*)(base + p.o_vote);
    c.ins = (int2*)(base + p.o_ins);
    c.modR = (int*)(base + p.o_modR);
    c.winners = (int2*)(base + p.o_win);
    c.claim = (unsigned long long*)(base + p.o_claim);
    c.cand = (int2*)(base + p.o_cand);
    c.fmap = (int4*)(base + p.o_fmap);
    c.fst = (int*)(base + p.o_fst);
    c.qst = (int*)(base + p.o_qst);
    c.queue = (int*)(base + p.o_qA);
    c.queue_next = (int*)(base + p.o_qB);
    c.flipped = (int*)(base + p.o_flipped);
    c.seg = (int4*)(base + p.o_seg);
    c.pend = (int*)(base + p.o_pendA);
    c.pend_next = (int*)(base + p.o_pendB);
    c.pinfo = (int4*)(base + p.o_pinfo);
    c.scratch = (int*)(base + p.o_scratch);
    c.scratch_cap = (int)p.scratch_cap;
    c.vt = (int*)(base + p.o_vt);
    c.cnt = (Counters*)(base + p.o_cnt);
    return c;
}

// One element of kernel `k`; the CUDA backend instantiates one kernel per id.
GCDT_HD void dispatch(int k, const Ctx& c, int i) {
    switch (k) {
    case K_KEYS: body_keys(c, i); break;
    case K_GATHER: body_gather(c, i); break;
    case K_ROOT: body_root(c, i); break;
    case K_INITLOC: body_initloc(c, i); break;
    case K_RELOC_VOTE: body_reloc_vote(c, i); break;
    case K_SPLIT: body_split(c, i); break;
    case K_FIX: body_fix(c, i); break;
    case K_FLIP_CHECK: body_flip_check(c, i); break;
    case K_FLIP_DO: body_flip_do(c, i); break;
    case K_FLIP_FIX: body_flip_fix(c, i); break;
    case K_OUTPUT: body_output(c, i); break;
    case K_VT: body_vt(c, i); break;
    case K_SEG_INIT: body_seg_init(c, i); break;
    case K_CWALK: body_cwalk(c, i); break;
    case K_CCLAIM: body_cclaim(c, i); break;
    case K_CPROC: body_cproc(c, i); break;
    default: break;
    }
}

constexpr long long kMaxSubrounds = 1 << 20;
constexpr long long kMaxRounds = 1 << 16;
constexpr unsigned kMaxConstraintRounds = 1 << 14;

// Flip sub-rounds until the queue is empty.  `qa` holds nq entries stamped
// `sr`; returns the next free stamp through `sr`.
template <class BK>
int flip_until_delaunay(BK& bk, Ctx& c, int*& qa, int*& qb, int nq, unsigned& sr, SolveStats& st) {
    Counters h;
    long long guard = 0;
    while (nq > 0) {
        if (++guard > kMaxSubrounds) return ST_ITER_LIMIT;
        c.queue = qa; c.queue_next = qb; c.sr = sr;
        bk.reset_lists();
        bk.launch(K_FLIP_CHECK, c, nq);
        bk.launch(K_FLIP_DO, c, nq);
        bk.read(&h); st.host_syncs++;
        if (h.status) return h.status;
        bk.launch(K_FLIP_FIX, c, h.n_flip);
        st.flips += h.n_flip;
        st.flip_subrounds++;
        sr++;
        nq = h.n_next;
        int* t = qa; qa = qb; qb = t;
    }
    return 0;
}

template <class BK>
int run_solve(BK& bk, Ctx c, SolveStats& st) {
    Counters h;
    const int n = c.n;
    const long long T = c.ntri;
    bk.fill(c.cnt, 0, sizeof(Counters));
    bk.fill(c.vote, 0, 8 * T);
    bk.fill(c.claim, 0, 8 * T);
    bk.fill(c.ins, 0, 8 * T);
    bk.fill(c.modR, 0xff, 4 * T);
    bk.fill(c.fst, 0xff, 4 * T);
    bk.fill(c.qst, 0, 4 * T);
    if (n > 0) {
        bk.launch(K_KEYS, c, n);
        bk.sort(c, n);
    }
    bk.launch(K_GATHER, c, n + 4);
    bk.launch(K_ROOT, c, 1);
    if (n > 0) bk.launch(K_INITLOC, c, n);
    bk.read(&h); st.host_syncs++;
    if (h.status) return h.status;

    // ---- phase 1: insertion rounds
    int* actA = c.act;
    int* actB = c.act_next;
    int* qa = c.queue;
    int* qb = c.queue_next;
    int nact = n;
    unsigned round = 0, sr = 0;
    while (nact > 0) {
        if (++round > kMaxRounds) return ST_ITER_LIMIT;
        c.round = round;
        c.act = actA; c.act_next = actB;
        bk.reset_lists();
        bk.launch(K_RELOC_VOTE, c, nact);
        bk.read(&h); st.host_syncs++;
        if (h.status) return h.status;
        nact = h.n_next;
        { int* t = actA; actA = actB; actB = t; }
        if (nact == 0) break;
        c.act = actA; c.act_next = actB;
        bk.launch(K_SPLIT, c, nact);
        bk.read(&h); st.host_syncs++;
        int nwin = h.n_win;
        sr++;
        c.sr = sr; c.queue_next = qa;
        bk.reset_lists();
        bk.launch(K_FIX, c, nwin);
        bk.read(&h); st.host_syncs++;
        if (h.status) return h.status;
        st.rounds++;
        int rc = flip_until_delaunay(bk, c, qa, qb, h.n_next, sr, st);
        if (rc) return rc;
    }

    // ---- phase 2: constraints
    if (c.s > 0) {
        bk.launch(K_VT, c, T);
        bk.launch(K_SEG_INIT, c, c.s);
        bk.read(&h); st.host_syncs++;
        if (h.status) return h.status;
        int* pa = c.pend;
        int* pb = c.pend_next;
        int npend = c.s;
        unsigned lawson_sr = sr + kMaxConstraintRounds + 2;
        c.lawson_sr = lawson_sr;
        c.lq = qa;
        unsigned cr = 0;
        while (npend > 0) {
            if (++cr > kMaxConstraintRounds) return ST_ITER_LIMIT;
            sr++;
            c.sr = sr;
            c.pend = pa; c.pend_next = pb;
            bk.reset_lists();
            bk.set_scratch_top(0);
            bk.launch(K_CWALK, c, npend);
            bk.launch(K_CCLAIM, c, npend);
            bk.launch(K_CPROC, c, npend);
            bk.read(&h); st.host_syncs++;
            if (h.status) return h.status;
            npend = h.n_next;
            int* t = pa; pa = pb; pb = t;
            st.constraint_rounds++;
        }
        sr = lawson_sr;
        int rc = flip_until_delaunay(bk, c, qa, qb, h.n_lawson, sr, st);
        if (rc) return rc;
    }
    c.sr = sr;

    // ---- phase 3: output
    bk.launch(K_OUTPUT, c, T);
    bk.read(&h); st.host_syncs++;
    return h.status;
}

}  // namespace gcdt
