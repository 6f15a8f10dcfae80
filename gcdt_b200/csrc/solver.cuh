// solver.cuh -- round structure of one CDT solve, written once against a
// launch backend (gcdt.cu supplies the CUDA one: the persistent stage
// kernel with its grid executor from exec.cuh).
//
// Phases (reference stage it replaces, yingtix/gCDT):
//   0  Hilbert keys, radix sort, gather: points in spatial order
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
#include <cstring>
#include "layout.cuh"
#include "mesh.cuh"

namespace gcdt {

enum Kern : int {
    K_KEYS, K_GATHER, K_ROOT, K_LEVEL, K_SEG_LEVEL0, K_ACTIVATE, K_VT_RESET, K_VT_LIVE,
    K_RELOC_VOTE, K_SPLIT, K_FIX,
    K_FLIP_CHECK, K_FLIP_DO, K_FLIP_FIX, K_OUTPUT,
    K_SEG_INIT, K_CWALK, K_CCLAIM, K_CPROC,
    K_NARROW_FLIPS, K_NARROW_ROUNDS,     // timing labels of the single-block tails
    K_CLEAR,
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

constexpr long long kMaxSubrounds = 1 << 20;
// A flip queue or an active list this short is finished by one block with
// block barriers instead of the whole grid with grid barriers.
constexpr long long kNarrowQueue = 1024;
constexpr long long kNarrowActive = 1024;
// On the whole grid, a round's flip sub-rounds stop (after the first) once
// the queue has at most this many entries; the rest of the queue is carried
// into the next round's first flip queue and drained before the level ends
// or the insertion tail moves to one block, so the shrinking sub-rounds of
// one round run together with the next round's large first one.  Insertion
// and location work on any triangulation; only the final mesh must be
// Delaunay.  (Measured on the 10M-point workload: 1K 33.0 ms, 64K 31.6,
// 256K 31.3, 4M 30.8, 16M 31.3; no carry 35.4.)
constexpr long long kCarryQueue = 1 << 22;
constexpr long long kMaxRounds = 1 << 16;
constexpr unsigned kMaxConstraintRounds = 1 << 14;

__host__ __device__ inline Ctx bind_ctx(char* base, const Plan& p) {
    Ctx c{};
    c.n = (int)p.n; c.s = (int)p.s; c.ntri = (int)p.ntri;
    c.keys = (unsigned long long*)(base + p.o_keys);
    c.keys_alt = (unsigned long long*)(base + p.o_keys_alt);
    c.vals = (int*)(base + p.o_vals);
    c.vals_alt = (int*)(base + p.o_vals_alt);
    c.P = (int2*)(base + p.o_P);
    c.perm = (int*)(base + p.o_perm);
    c.rank = (int*)(base + p.o_rank);
    c.tri = (int4*)(base + p.o_tri);
    c.loc = (int*)(base + p.o_loc);
    c.pedge = (signed char*)(base + p.o_pedge);
    c.act = (int*)(base + p.o_actA);
    c.act_next = (int*)(base + p.o_actB);
    c.vote = (unsigned long long*)(base + p.o_vote);
    c.winners = (int2*)(base + p.o_win);
    c.claim = (unsigned long long*)(base + p.o_claim);
    c.cand = (int2*)(base + p.o_cand);
    c.qst = (int*)(base + p.o_qst);
    c.queue = (int*)(base + p.o_qA);
    c.queue_next = (int*)(base + p.o_qB);
    c.seg = (int4*)(base + p.o_seg);
    c.pend = (int*)(base + p.o_pendA);
    c.pend_next = (int*)(base + p.o_pendB);
    c.pinfo = (int4*)(base + p.o_pinfo);
    c.scratch = (int*)(base + p.o_scratch);
    c.scratch_cap = (int)p.scratch_cap;
    c.vt = (int*)(base + p.o_vt);
    c.lvl = (unsigned char*)(base + p.o_lvl);
    c.cnt = (Counters*)(base + p.o_cnt);
    // three levels: every 512th point of the curve order plus all segment
    // endpoints, then every 8th, then the rest
    c.nlevels = 3;
    c.stride[0] = 512; c.stride[1] = 8; c.stride[2] = 1; c.stride[3] = 1;
    c.carry_q = (int)kCarryQueue;
    c.narrow_q = (int)kNarrowQueue;
    c.narrow_act = (int)kNarrowActive;
    return c;
}

// One element of kernel `k`; the CUDA backend instantiates one kernel per id.
GCDT_HD void dispatch(int k, const Ctx& c, int i) {
    switch (k) {
    case K_KEYS: body_keys(c, i); break;
    case K_GATHER: body_gather(c, i); break;
    case K_ROOT: body_root(c, i); break;
    case K_LEVEL: body_level(c, i); break;
    case K_SEG_LEVEL0: body_seg_level0(c, i); break;
    case K_ACTIVATE: body_activate(c, i); break;
    case K_VT_RESET: body_vt_reset(c, i); break;
    case K_VT_LIVE: body_vt_live(c, i); break;
    case K_RELOC_VOTE: body_reloc_vote(c, i); break;
    case K_SPLIT: body_split(c, i); break;
    case K_FIX: body_fix(c, i); break;
    case K_FLIP_CHECK: body_flip_check(c, i); break;
    case K_FLIP_DO: body_flip_do(c, i); break;
    case K_FLIP_FIX: body_flip_fix(c, i); break;
    case K_OUTPUT: body_output(c, i); break;
    case K_SEG_INIT: body_seg_init(c, i); break;
    case K_CWALK: body_cwalk(c, i); break;
    case K_CCLAIM: body_cclaim(c, i); break;
    case K_CPROC: body_cproc(c, i); break;
    case K_CLEAR: body_clear(c, i); break;
    default: break;
    }
}


// The budgets a solve runs under: the context's, where set and within the
// built-in bound (the constraint rounds' bound also spaces the queue stamps).
GCDT_HD long long budget_subrounds(const Ctx& c) {
    return c.lim_subrounds > 0 && c.lim_subrounds < kMaxSubrounds ? c.lim_subrounds : kMaxSubrounds;
}
GCDT_HD long long budget_rounds(const Ctx& c) {
    return c.lim_rounds > 0 && c.lim_rounds < kMaxRounds ? c.lim_rounds : kMaxRounds;
}
GCDT_HD unsigned budget_crounds(const Ctx& c) {
    return c.lim_crounds > 0 && (unsigned)c.lim_crounds < kMaxConstraintRounds ? (unsigned)c.lim_crounds
                                                                              : kMaxConstraintRounds;
}

// The stage driver runs the same control flow on every GPU thread of the
// persistent kernel (EX = grid executor: a phase is a grid-stride loop
// followed by a grid barrier) and on the host for the CPU emulation
// (EX = sequential executor).  Every value the driver branches on is read
// right after a barrier and cannot change before the next barrier, so all
// threads take the same branches:
//   - a list cursor is read right after the phase that appended to it, and
//     the phase after that never appends to the same cursor;
//   - errors of phase k go to err[k & 1], read after phase k's barrier
//     while phase k+1 writes err[(k+1) & 1].
//
// EX provides: phase(kernel, ctx, count), cursor(u64*) -> u64,
// word(int*) -> int, finish(...), and kCanNarrow: whether small flip queues
// and small insertion tails can be handed to one block (narrow_flips,
// narrow_rounds), which runs this same driver with block barriers.

struct Driver {
    int* actA; int* actB; int* qa; int* qb;
    long long carry;        // entries left in qa by the last round's flips
    long long drop;         // leading entries of the next flip queue that were carried
    unsigned round, sr;
    long long rounds, subrounds, crounds;
    unsigned long long e_act0, e_act, e_win, e_q, e_flip, e_pend, e_law, e_scr;
    int nphase;
    int errs;
};

// The driver state handed between the grid and a single-block tail through
// the counters' hand-off area, copied word by word through memcpy, which
// keeps the copy well defined whatever the field types.
GCDT_HD void save_driver(Counters* cnt, const Driver& D) {
    unsigned long long w[sizeof(Driver) / 8];
    memcpy(w, &D, sizeof(Driver));
    for (unsigned k = 0; k < sizeof(Driver) / 8; ++k) cnt->handoff[k] = w[k];
}
GCDT_HD void load_driver(Counters* cnt, Driver& D) {
    unsigned long long w[sizeof(Driver) / 8];
    const volatile unsigned long long* src = cnt->handoff;
    for (unsigned k = 0; k < sizeof(Driver) / 8; ++k) w[k] = src[k];
    memcpy(&D, w, sizeof(Driver));
}

template <class EX>
GCDT_HD void run_phase(EX& ex, Ctx& c, Driver& D, int k, long long count) {
    c.eslot = D.nphase & 1;
    ex.phase(k, c, count);
    D.errs |= ex.word(&c.cnt->err[c.eslot]);
    D.nphase++;
}

// Flip sub-rounds on the queue `D.qa` (nq entries, stamped D.sr) until it
// has at most `stop` entries after at least one sub-round, or -- for the
// single-block tail -- until it grows past max_nq.  The first sub-round
// always runs, so an entry is carried over at most one round.
template <class EX>
GCDT_HD int flip_loop(EX& ex, Ctx& c, Driver& D, long long& nq, long long max_nq, long long stop = 0) {
    long long guard = 0;
    const long long budget = budget_subrounds(c);
    while (nq > 0 && nq <= max_nq && (guard == 0 || nq > stop)) {
        if (++guard > budget) return ST_ITER_LIMIT;
        if (EX::kCanNarrow && nq <= c.narrow_q) {
            int rc = ex.narrow_flips(c, D, nq);
            if (rc || D.errs) return rc ? rc : D.errs;
            continue;
        }
        c.queue = D.qa; c.queue_next = D.qb; c.sr = D.sr;
        c.base_q = D.e_q;
        c.base_flip = D.e_flip;
        c.carry_n = (int)D.drop;
        D.drop = 0;
        run_phase(ex, c, D, K_FLIP_CHECK, nq);
        run_phase(ex, c, D, K_FLIP_DO, nq);
        D.e_flip = ex.cursor(&c.cnt->cur_flip);
        if (D.errs) return D.errs;
        long long nflip = (long long)(D.e_flip - c.base_flip);
        c.list_n = (int)nflip;
        // next queue: the flipped pairs' 2 * nflip entries, then the losers
        // FLIP_FIX appends through cur_q
        run_phase(ex, c, D, K_FLIP_FIX, nflip + nq);
        D.e_q = ex.cursor(&c.cnt->cur_q);
        D.subrounds++;
        D.sr++;
        nq = 2 * nflip + (long long)(D.e_q - c.base_q);
        int* t = D.qa; D.qa = D.qb; D.qb = t;
    }
    return 0;
}

template <class EX>
GCDT_HD int flip_until_delaunay(EX& ex, Ctx& c, Driver& D, long long nq) {
    return flip_loop(ex, c, D, nq, (long long)1 << 62);
}

template <class EX>
GCDT_HD int insert_rounds(EX& ex, Ctx& c, Driver& D, long long nact) {
    while (nact > 0) {
        if (EX::kCanNarrow && nact <= c.narrow_act) {
            // the single-block tail starts from a Delaunay mesh: the carried
            // flips are finished by the whole grid first
            if (D.carry > 0) {
                long long nq = D.carry;
                D.carry = 0;
                int rc = flip_until_delaunay(ex, c, D, nq);
                if (rc) return rc;
            }
            return ex.narrow_rounds(c, D, nact);
        }
        if (++D.round > budget_rounds(c)) return ST_ITER_LIMIT;
        c.round = D.round;
        c.act = D.actA; c.act_next = D.actB;
        c.base_act = D.e_act;
        run_phase(ex, c, D, K_RELOC_VOTE, nact);
        D.e_act = ex.cursor(&c.cnt->cur_act);
        if (D.errs) return D.errs;
        nact = (long long)(D.e_act - c.base_act);
        { int* t = D.actA; D.actA = D.actB; D.actB = t; }
        if (nact == 0) break;
        c.act = D.actA; c.act_next = D.actB;
        c.base_win = D.e_win;
        run_phase(ex, c, D, K_SPLIT, nact);
        D.e_win = ex.cursor(&c.cnt->cur_win);
        long long nwin = (long long)(D.e_win - c.base_win);
        D.sr++;
        // the children go into the queue after the entries carried from the
        // previous round, which sit at the front of the same buffer
        c.sr = D.sr; c.queue_next = D.qa;
        c.base_q = D.e_q - (unsigned long long)D.carry;
        run_phase(ex, c, D, K_FIX, nwin);
        D.e_q = ex.cursor(&c.cnt->cur_q);
        if (D.errs) return D.errs;
        D.rounds++;
        long long nq = (long long)(D.e_q - c.base_q);
        D.drop = D.carry;
        D.carry = 0;
        int rc = flip_loop(ex, c, D, nq, (long long)1 << 62, EX::kCanNarrow ? (long long)c.carry_q : 0);
        if (rc) return rc;
        D.carry = nq;
    }
    // end of the level: no flip is left pending
    if (D.carry > 0) {
        long long nq = D.carry;
        D.carry = 0;
        int rc = flip_until_delaunay(ex, c, D, nq);
        if (rc) return rc;
    }
    return 0;
}

// Recover every segment on the current (coarse) mesh, then restore the
// constrained Delaunay property.
template <class EX>
GCDT_HD int insert_constraints(EX& ex, Ctx& c, Driver& D) {
    c.level = 1;
    run_phase(ex, c, D, K_VT_RESET, c.n + 4);
    run_phase(ex, c, D, K_VT_LIVE, c.n + 2);
    int* pa = c.pend;
    int* pb = c.pend_next;
    long long npend = c.s;
    unsigned lawson_sr = D.sr + kMaxConstraintRounds + 2;
    c.lawson_sr = lawson_sr;
    c.lq = D.qa;
    c.base_law = D.e_law;
    unsigned cr = 0;
    const unsigned cbudget = budget_crounds(c);
    while (npend > 0) {
        if (++cr > cbudget) return ST_ITER_LIMIT;
        D.sr++;
        c.sr = D.sr;
        c.pend = pa; c.pend_next = pb;
        c.base_pend = D.e_pend;
        c.base_scr = D.e_scr;
        run_phase(ex, c, D, K_CWALK, npend);
        run_phase(ex, c, D, K_CCLAIM, npend);
        D.e_scr = ex.cursor(&c.cnt->cur_scr);
        run_phase(ex, c, D, K_CPROC, npend);
        D.e_pend = ex.cursor(&c.cnt->cur_pend);
        D.e_law = ex.cursor(&c.cnt->cur_law);
        if (D.errs) return D.errs;
        npend = (long long)(D.e_pend - c.base_pend);
        int* t = pa; pa = pb; pb = t;
        D.crounds++;
    }
    long long nlaw = (long long)(D.e_law - c.base_law);
    D.sr = lawson_sr;
    return flip_until_delaunay(ex, c, D, nlaw);
}

// Everything after the sort: the insertion levels, the constraint stage
// after level 0, and the output.  Cursors start at 0 (cleared by the host).
template <class EX>
GCDT_HD int run_stages(EX& ex, Ctx c) {
    const int n = c.n;
    Driver D;
    D.actA = c.act; D.actB = c.act_next; D.qa = c.queue; D.qb = c.queue_next;
    D.carry = 0; D.drop = 0;
    D.round = 0; D.sr = 0; D.rounds = 0; D.subrounds = 0; D.crounds = 0;
    D.e_act0 = D.e_act = D.e_win = D.e_q = D.e_flip = D.e_pend = D.e_law = D.e_scr = 0;
    D.nphase = 0; D.errs = 0;
    // set-up (keys, gather, segments) flagged bad input: stop before any phase
    if (ex.word(&c.cnt->status) | ex.word(&c.cnt->err[0]) | ex.word(&c.cnt->err[1])) {
        ex.finish(c, 0, 0, 0, 0);
        return ST_BAD_INPUT;
    }
    int rc = 0;
    for (int l = 0; l < c.nlevels && n > 0 && rc == 0; ++l) {
        c.level = l;
        if (l > 0) {
            run_phase(ex, c, D, K_VT_RESET, n + 4);
            run_phase(ex, c, D, K_VT_LIVE, n + 2);
        }
        c.act_next = D.actA;
        c.base_act = D.e_act0;
        run_phase(ex, c, D, K_ACTIVATE, n);
        D.e_act0 = ex.cursor(&c.cnt->cur_act0);
        if ((rc = D.errs)) break;
        rc = insert_rounds(ex, c, D, (long long)(D.e_act0 - c.base_act));
        if (rc == 0 && l == 0 && c.s > 0) rc = insert_constraints(ex, c, D);
    }
    if (rc == 0 && n == 0 && c.s > 0) rc = ST_BAD_INPUT;
    if (rc == 0) {
        run_phase(ex, c, D, K_OUTPUT, c.ntri);
        rc = D.errs;
    }
    ex.finish(c, D.rounds, D.subrounds, D.crounds, rc | D.errs);
    return rc;
}

// Host part: clear the per-solve arrays, key sort, gather, levels and
// segment set-up, then hand over to the stages (one persistent kernel on the
// GPU).  Everything is enqueued on the backend's stream without waiting:
// errors found by the set-up kernels make the stage kernel stop at once.
template <class BK>
void enqueue_solve(BK& bk, Ctx c) {
    const int n = c.n;
    const long long T = c.ntri;
    bk.fill(c.cnt, 0, sizeof(Counters));
    bk.fill(c.vote, 0, 8 * T);
    bk.fill(c.claim, 0, 8 * T);
    bk.fill(c.qst, 0, 4 * T);
    if (n > 0) {
        bk.launch(K_KEYS, c, n);
        bk.sort(c, n);
    }
    bk.launch(K_GATHER, c, n + 4);
    bk.launch(K_ROOT, c, 1);
    if (n > 0) bk.launch(K_LEVEL, c, n);
    if (c.s > 0) {
        bk.launch(K_SEG_INIT, c, c.s);
        bk.launch(K_SEG_LEVEL0, c, c.s);
    }
    bk.stages(c);
}

// Status bits and statistics of a finished solve from its counters.
inline int solve_result(const Counters& h, SolveStats& st) {
    st.rounds = h.rounds;
    st.flip_subrounds = h.flip_subrounds;
    st.constraint_rounds = h.constraint_rounds;
    st.flips = (long long)h.cur_flip;
    return h.status | h.err[0] | h.err[1];
}

// One solve, then one read of the counters.
template <class BK>
int run_solve(BK& bk, Ctx c, SolveStats& st) {
    enqueue_solve(bk, c);
    Counters h;
    bk.read(&h);
    st.host_syncs++;
    return solve_result(h, st);
}

}  // namespace gcdt
