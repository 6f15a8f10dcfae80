// exec.cuh -- the two executors of the stage driver on the GPU.
//
//   GridExec   every block of a cooperative persistent launch: a phase is a
//              grid-stride loop followed by a bounded grid barrier;
//   BlockExec  one block: a phase is a block-stride loop followed by
//              __syncthreads (the single-block tails of a solve, and every
//              instance of the batched path).
#pragma once
#include "solver.cuh"

namespace gcdt {

// ---------------------------------------------------------------------------
// Persistent stage kernel.  One cooperative launch runs every insertion
// round, flip sub-round and constraint round of a solve; phases are
// grid-stride loops separated by a grid barrier, so the round structure
// costs no kernel launches and no host round trips.

#ifndef GCDT_PERSIST_BLOCK
#define GCDT_PERSIST_BLOCK 512
#endif
#ifndef GCDT_PERSIST_MINB
#define GCDT_PERSIST_MINB 1
#endif
constexpr int kPersistBlock = GCDT_PERSIST_BLOCK;   // 512: one block per SM (128 registers per thread)
constexpr int kPersistMinBlocks = GCDT_PERSIST_MINB;

// The context a phase's items see: the launch's context `param` (in kernel
// parameter space) with the fields the driver changes between phases taken
// from the driver's copy `c`.  The other fields (the array pointers and
// sizes) stay reads of parameter space, so the item loops keep them in no
// register.
__device__ __forceinline__ Ctx phase_view(const Ctx& param, const Ctx& c) {
    Ctx v = param;
    v.round = c.round; v.sr = c.sr; v.eslot = c.eslot; v.lawson_sr = c.lawson_sr;
    v.list_n = c.list_n; v.carry_n = c.carry_n; v.level = c.level;
    v.act = c.act; v.act_next = c.act_next; v.queue = c.queue; v.queue_next = c.queue_next;
    v.pend = c.pend; v.pend_next = c.pend_next; v.lq = c.lq;
    v.base_act = c.base_act; v.base_win = c.base_win; v.base_q = c.base_q; v.base_flip = c.base_flip;
    v.base_pend = c.base_pend; v.base_law = c.base_law; v.base_scr = c.base_scr;
    return v;
}

struct GridExec {
    static constexpr bool kCanNarrow = true;
    Counters* cnt;
    unsigned nblocks;
    __device__ int narrow_flips(Ctx& c, Driver& D, long long& nq);
    __device__ int narrow_rounds(Ctx& c, Driver& D, long long nact);

    // Snapshot of the head of Counters (status, error words, list cursors)
    // taken by thread 0 right after each grid barrier: the driver's reads of
    // these values come from shared memory instead of every thread reading
    // the same L2 line.
    static constexpr int kSnapWords = 12;   // 96 bytes: status..cur_scr
    unsigned long long* snap;                // shared memory, kSnapWords entries
    unsigned spin_limit = 1u << 24;          // polls before a barrier wait gives up
    int* work = nullptr;                     // shared memory: the block's next item (dynamic phases)
    const Ctx* param = nullptr;              // the launch's context, in kernel parameter space
    bool prof = false;                       // record the phase profile and balance (a launch constant)

    __device__ void take_snapshot() {
        volatile unsigned long long* src = reinterpret_cast<volatile unsigned long long*>(cnt);
        for (int k = 0; k < kSnapWords; ++k) snap[k] = src[k];
    }

    // Grid barrier on one counter whose top bit flips once per barrier:
    // block 0 adds 2^31 - (blocks - 1), every other block adds 1, so the
    // count's low 31 bits are back at 0 and its top bit has flipped once
    // every block has arrived, and a block waits for the top bit to differ
    // from the value its own add saw.  One atomic per block and no reset
    // (2.9 -> 2.35 us per barrier against a counter reset by the last
    // arrival plus a generation word).  The counter starts each launch at
    // 0 (the solve clears its counters).  Every wait is bounded: after
    // spin_limit polls (2^24, about a second, in a solve) the block records
    // ST_BARRIER and stops waiting, and once that bit is set no block waits
    // or works any more, so the kernel always ends.
    __device__ void barrier() { barrier_timed(-1, 0, 0); }
    // The barrier ending a phase: with k >= 0, thread 0 first records the
    // block's work time (cycles since t0) for the phase balance.
    __device__ void barrier_timed(int k, long long t0, int slot) {
        __syncthreads();
        if (threadIdx.x == 0 && k >= 0) {
            unsigned long long w = (unsigned long long)(clock64() - t0);
            atomicMax(&cnt->wcur_max[slot], w);
            atomicAdd(&cnt->wcur_sum[slot], w);
        }
        if (threadIdx.x < 32) {
            if (threadIdx.x == 0) {
                volatile unsigned* vcount = &cnt->bar_count;
                volatile int* vst = &cnt->status;
                if (!(*vst & ST_BARRIER)) {
                    const unsigned add = blockIdx.x == 0 ? 0x80000000u - (nblocks - 1) : 1u;
                    __threadfence();
                    const unsigned old = atomicAdd(&cnt->bar_count, add);
                    // the arrival that completes the count flips the top bit itself
                    const bool last = (((old + add) ^ old) & 0x80000000u) != 0;
                    unsigned spins = 0;
                    while (!last && ((old ^ *vcount) & 0x80000000u) == 0) {
                        if (++spins > spin_limit) { atomicOr(&cnt->status, ST_BARRIER); break; }
                        if (*vst & ST_BARRIER) break;
                        __nanosleep(64);
                    }
                }
                __threadfence();
            }
            // the snapshot words read by the first lanes of warp 0 at once,
            // after lane 0 has seen the barrier open (3.20 -> 2.90 us per
            // barrier against one lane reading all of them)
            __syncwarp();
            if (threadIdx.x < kSnapWords)
                snap[threadIdx.x] = reinterpret_cast<volatile unsigned long long*>(cnt)[threadIdx.x];
        }
        __syncthreads();
    }
    __device__ void phase(int k, const Ctx& cd, long long count) {
        const Ctx c = phase_view(*param, cd);
        long long t0 = threadIdx.x == 0 ? clock64() : 0;
        // the rounds' and flip sub-rounds' phases take their items in warp
        // chunks (28.45 -> 28.03 ms on the headline solve); the others, one
        // or a few runs per solve, keep the plain grid-stride loop
        if (!(word(&cnt->status) & ST_BARRIER) && work &&
            (k == K_FLIP_CHECK || k == K_FLIP_DO || k == K_FLIP_FIX || k == K_RELOC_VOTE || k == K_SPLIT ||
             k == K_FIX)) {
            dynamic_items(k, c, count);
        } else if (!(word(&cnt->status) & ST_BARRIER)) {
            long long stride = (long long)gridDim.x * blockDim.x;
            long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
            // latency-bound passes: two items per thread and trip (i, i + stride)
            if (k == K_FLIP_CHECK) {
                for (; i < count; i += 2 * stride)
                    body_flip_check_pair(c, (int)i, i + stride < count ? (int)(i + stride) : -1);
            } else if (k == K_FLIP_DO) {
                for (; i < count; i += 2 * stride)
                    body_flip_do_pair(c, (int)i, i + stride < count ? (int)(i + stride) : -1);
            } else if (k == K_FLIP_FIX) {
                for (; i < count; i += 2 * stride)
                    body_flip_fix_pair(c, (int)i, i + stride < count ? (int)(i + stride) : -1);
            } else {
                for (; i < count; i += stride) dispatch(k, c, (int)i);
            }
        }
        const int slot = c.eslot & 1;
        const bool timer = prof && blockIdx.x == 0 && threadIdx.x == 0;
        barrier_timed(prof && k < kMaxPhaseKinds ? k : -1, t0, slot);
        if (timer && k < kMaxPhaseKinds) {   // phase time incl. the barrier, as block 0 sees it
            cnt->phase_cyc[k] += clock64() - t0;
            cnt->phase_cnt[k] += 1;
            // every block added this run's work time before it arrived; no
            // block writes this slot again before the next barrier, which
            // block 0 passes only after clearing it
            cnt->phase_wmax[k] += (long long)*(volatile unsigned long long*)&cnt->wcur_max[slot];
            cnt->phase_wsum[k] += (long long)*(volatile unsigned long long*)&cnt->wcur_sum[slot];
            cnt->wcur_max[slot] = 0;
            cnt->wcur_sum[slot] = 0;
        }
    }
    // Items of a phase in chunks of one warp's worth, chunk j of block b
    // being chunk b + j * blocks of the phase (the grid-stride interleave);
    // the block's warps take its chunks in turn from a shared-memory
    // counter, so a warp that finishes early takes more.
    __device__ int take_chunk() {
        int j = 0;
        if ((threadIdx.x & 31) == 0) j = atomicAdd(work, 1);
        return __shfl_sync(0xffffffffu, j, 0);
    }
    // The flip passes' chunk loop: each lane's two items of the next chunk
    // have their first word (queue entry or candidate) loaded while the
    // current chunk runs.
    // The flip pass two chunks ahead: chunk j+2's candidates are loaded, and
    // the claims chunk j+1's candidates name are prefetched into L2, while
    // chunk j runs.  (The same second stage in the check and the fix, an L2
    // prefetch of the rows their next chunk names, made them slower.)
    __device__ void flip_do_pipelined(const Ctx& c, long long count, int j) {
        const int lane = threadIdx.x & 31;
        auto chunk_at = [&](int jj) { return ((long long)blockIdx.x + (long long)jj * gridDim.x) * 64; };
        auto item = [&](long long b, int o) { return b + lane + o < count ? (int)(b + lane + o) : -1; };
        long long base = chunk_at(j);
        int k0 = item(base, 0), k1 = item(base, 32);
        int2 f0 = flip_first(c, FP_DO, k0), f1 = flip_first(c, FP_DO, k1);
        j = take_chunk();
        long long nb = chunk_at(j);
        int n0 = item(nb, 0), n1 = item(nb, 32);
        int2 g0 = flip_first(c, FP_DO, n0), g1 = flip_first(c, FP_DO, n1);
        while (base < count) {
            j = take_chunk();
            const long long nnb = chunk_at(j);
            const int m0 = item(nnb, 0), m1 = item(nnb, 32);
            const int2 h0 = flip_first(c, FP_DO, m0), h1 = flip_first(c, FP_DO, m1);
            if (n0 >= 0 && g0.x >= 0) prefetch_l2(&c.claim[g0.x >> 2], &c.claim[g0.y >> 2]);
            if (n1 >= 0 && g1.x >= 0) prefetch_l2(&c.claim[g1.x >> 2], &c.claim[g1.y >> 2]);
            if (k0 >= 0) {
                const int ks[2] = {k0, k1};
                const int2 f[2] = {f0, f1};
                body_flip_do_pair_f(c, ks, f);
            }
            base = nb; k0 = n0; k1 = n1; f0 = g0; f1 = g1;
            nb = nnb; n0 = m0; n1 = m1; g0 = h0; g1 = h1;
        }
    }
    __device__ static void prefetch_l2(const void* a, const void* b) {
        asm volatile("prefetch.global.L2 [%0];" :: "l"(a));
        asm volatile("prefetch.global.L2 [%0];" :: "l"(b));
    }
    template <int P>
    __device__ void pipelined(const Ctx& c, long long count, int j) {
        const int lane = threadIdx.x & 31;
        long long base = ((long long)blockIdx.x + (long long)j * gridDim.x) * 64;
        int k0 = base + lane < count ? (int)(base + lane) : -1;
        int k1 = base + lane + 32 < count ? (int)(base + lane + 32) : -1;
        int2 f0 = flip_first(c, P, k0), f1 = flip_first(c, P, k1);
        while (base < count) {
            j = take_chunk();
            const long long nb = ((long long)blockIdx.x + (long long)j * gridDim.x) * 64;
            const int n0 = nb + lane < count ? (int)(nb + lane) : -1;
            const int n1 = nb + lane + 32 < count ? (int)(nb + lane + 32) : -1;
            const int2 g0 = flip_first(c, P, n0), g1 = flip_first(c, P, n1);
            if (k0 >= 0) {
                const int ks[2] = {k0, k1};
                const int2 f[2] = {f0, f1};
                if (P == FP_CHECK) flip_check_multi_f<2>(c, ks, f);
                else if (P == FP_DO) body_flip_do_pair_f(c, ks, f);
                else body_flip_fix_pair_f(c, ks, f);
            }
            base = nb; k0 = n0; k1 = n1; f0 = g0; f1 = g1;
        }
    }
    __device__ void dynamic_items(int k, const Ctx& c, long long count) {
        if (threadIdx.x == 0) *work = 0;
        __syncthreads();
        const bool pair = k == K_FLIP_CHECK || k == K_FLIP_DO || k == K_FLIP_FIX;
        const long long chunk = pair ? 64 : 32;
        const int lane = threadIdx.x & 31;
        int j = take_chunk();
        if (pair) {
            if (k == K_FLIP_CHECK) pipelined<FP_CHECK>(c, count, j);
            else if (k == K_FLIP_DO) flip_do_pipelined(c, count, j);
            else pipelined<FP_FIX>(c, count, j);
            return;
        }
        if (k == K_RELOC_VOTE || k == K_SPLIT) {
            // two chunks ahead: the active points of chunk j+2 and the
            // locations (and, for the relocation, coordinates) of chunk j+1's
            // points are loaded while chunk j runs (each point's item is the
            // only one that writes its location)
            const bool rv = k == K_RELOC_VOTE;
            long long base = ((long long)blockIdx.x + (long long)j * gridDim.x) * chunk;
            int q = base + lane < count ? c.act[base + lane] : -1;
            int t = q >= 0 ? c.loc[q] : -1;
            int2 p = (rv && t >= 0) ? c.P[q] : make_int2(0, 0);
            j = take_chunk();
            long long nb = ((long long)blockIdx.x + (long long)j * gridDim.x) * chunk;
            int nq = nb + lane < count ? c.act[nb + lane] : -1;
            while (base < count) {
                j = take_chunk();
                const long long nnb = ((long long)blockIdx.x + (long long)j * gridDim.x) * chunk;
                const int nnq = nnb + lane < count ? c.act[nnb + lane] : -1;
                const int nt = nq >= 0 ? c.loc[nq] : -1;
                const int2 np = (rv && nq >= 0) ? c.P[nq] : make_int2(0, 0);
                if (q >= 0) {
                    if (rv) body_reloc_vote_qt(c, q, t, p);
                    else body_split_qt(c, q, t);
                }
                base = nb; q = nq; t = nt; p = np; nb = nnb; nq = nnq;
            }
            return;
        }
        if (k == K_FIX) {
            long long base = ((long long)blockIdx.x + (long long)j * gridDim.x) * chunk;
            int2 w = base + lane < count ? c.winners[base + lane] : make_int2(-1, -1);
            while (base < count) {
                j = take_chunk();
                const long long nb = ((long long)blockIdx.x + (long long)j * gridDim.x) * chunk;
                const int2 nw = nb + lane < count ? c.winners[nb + lane] : make_int2(-1, -1);
                if (w.x >= 0) body_fix_f(c, w);
                base = nb; w = nw;
            }
            return;
        }
        for (;;) {
            const long long base = ((long long)blockIdx.x + (long long)j * gridDim.x) * chunk;
            if (base >= count) break;
            const long long i0 = base + lane;
            if (i0 < count) dispatch(k, c, (int)i0);
            j = take_chunk();
        }
    }
    // Values read after a barrier come from the block's snapshot.
    __device__ unsigned long long cursor(unsigned long long* p) {
        size_t off = (size_t)((char*)p - (char*)cnt);
        if (off + 8 <= kSnapWords * 8) return *reinterpret_cast<unsigned long long*>((char*)snap + off);
        return *(volatile unsigned long long*)p;
    }
    __device__ int word(int* p) {
        size_t off = (size_t)((char*)p - (char*)cnt);
        if (off + 4 <= kSnapWords * 8) return *reinterpret_cast<int*>((char*)snap + off);
        return *(volatile int*)p;
    }
    __device__ void finish(const Ctx&, long long rounds, long long subrounds, long long crounds, int rc) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            cnt->grid_blocks = nblocks;
            cnt->rounds = rounds;
            cnt->flip_subrounds = subrounds;
            cnt->constraint_rounds = crounds;
            if (rc) atomicOr(&cnt->status, rc);
        }
    }
};

// Executor of one block: a phase is a block-stride loop and a block barrier.
// Used by block 0 for the short tails while the other blocks wait, and by
// every block of the batched kernel (kView: the items see phase_view of
// the block's context in shared memory).
template <bool kView>
struct BlockExecT {
    static constexpr bool kCanNarrow = false;
    Counters* cnt;
    const Ctx* base = nullptr;
    __device__ void phase(int k, const Ctx& cd, long long count) {
        if constexpr (kView) items(k, phase_view(*base, cd), count);
        else items(k, cd, count);
        __syncthreads();
    }
    __device__ void items(int k, const Ctx& c, long long count) {
        const long long stride = blockDim.x;
        long long i = threadIdx.x;
        // the latency-bound flip passes: two items per thread and trip, as
        // on the grid, so a queue of up to two blocks' worth is one trip
#ifndef GCDT_BLOCK_PAIRS
#define GCDT_BLOCK_PAIRS 1
#endif
        if (!GCDT_BLOCK_PAIRS) {
            for (; i < count; i += stride) dispatch(k, c, (int)i);
        } else if (k == K_FLIP_CHECK) {
            for (; i < count; i += 2 * stride)
                body_flip_check_pair(c, (int)i, i + stride < count ? (int)(i + stride) : -1);
        } else if (k == K_FLIP_DO) {
            for (; i < count; i += 2 * stride)
                body_flip_do_pair(c, (int)i, i + stride < count ? (int)(i + stride) : -1);
        } else if (k == K_FLIP_FIX) {
            for (; i < count; i += 2 * stride)
                body_flip_fix_pair(c, (int)i, i + stride < count ? (int)(i + stride) : -1);
        } else {
            for (; i < count; i += stride) dispatch(k, c, (int)i);
        }
    }
    __device__ unsigned long long cursor(unsigned long long* p) { return *(volatile unsigned long long*)p; }
    __device__ int word(int* p) { return *(volatile int*)p; }
    __device__ void finish(const Ctx&, long long rounds, long long subrounds, long long crounds, int rc) {
        if (threadIdx.x == 0) {
            cnt->rounds = rounds;
            cnt->flip_subrounds = subrounds;
            cnt->constraint_rounds = crounds;
            if (rc) atomicOr(&cnt->status, rc);
        }
    }
    __device__ int narrow_flips(Ctx&, Driver&, long long&) { return ST_INTERNAL; }
    __device__ int narrow_rounds(Ctx&, Driver&, long long) { return ST_INTERNAL; }
};
using BlockExec = BlockExecT<false>;

static_assert(sizeof(Driver) <= sizeof(((Counters*)0)->handoff), "driver state fits the hand-off area");
static_assert(sizeof(Driver) % 8 == 0, "driver state is whole 8-byte words");

__device__ inline void store_handoff(Counters* cnt, const Driver& D, long long nq, int rc) {
    save_driver(cnt, D);
    cnt->handoff_nq = nq;
    cnt->handoff_rc = rc;
}

__device__ inline int load_handoff(Counters* cnt, Driver& D, long long& nq) {
    load_driver(cnt, D);
    nq = *(volatile long long*)&cnt->handoff_nq;
    return *(volatile int*)&cnt->handoff_rc;
}

__device__ inline int GridExec::narrow_flips(Ctx& c, Driver& D, long long& nq) {
    const bool timer = prof && blockIdx.x == 0 && threadIdx.x == 0;
    long long t0 = timer ? clock64() : 0;
    if (blockIdx.x == 0) {
        BlockExec bx{cnt};
        Driver Db = D;
        Ctx cb = c;
        long long left = nq;
        int rc = flip_loop(bx, cb, Db, left, 4 * (long long)c.narrow_q);
        if (threadIdx.x == 0) store_handoff(cnt, Db, left, rc);
    }
    barrier();
    int rc = load_handoff(cnt, D, nq);
    if (timer) { cnt->phase_cyc[K_NARROW_FLIPS] += clock64() - t0; cnt->phase_cnt[K_NARROW_FLIPS] += 1; }
    return rc;
}

__device__ inline int GridExec::narrow_rounds(Ctx& c, Driver& D, long long nact) {
    const bool timer = prof && blockIdx.x == 0 && threadIdx.x == 0;
    long long t0 = timer ? clock64() : 0;
    if (blockIdx.x == 0) {
        BlockExec bx{cnt};
        Driver Db = D;
        Ctx cb = c;
        int rc = insert_rounds(bx, cb, Db, nact);
        if (threadIdx.x == 0) store_handoff(cnt, Db, 0, rc);
    }
    barrier();
    long long dummy;
    int rc = load_handoff(cnt, D, dummy);
    if (timer) { cnt->phase_cyc[K_NARROW_ROUNDS] += clock64() - t0; cnt->phase_cnt[K_NARROW_ROUNDS] += 1; }
    return rc;
}


}  // namespace gcdt
