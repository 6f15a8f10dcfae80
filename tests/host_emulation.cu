// host_emulation.cu -- test harness: the solver's kernel bodies and stage
// driver compiled for the host and run sequentially, one body call per item,
// in a chosen item order.  The GPU runs the same bodies in parallel; running
// them forward, reversed and shuffled on the host checks that a phase's
// result does not depend on the order its items run in, and the paired
// bodies (two items per call) are checked against the one-item bodies.
// Built by tests/test_host_emulation.py into tests/_bin/libhostemu.so.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>
#pragma nv_diag_suppress 20011
#pragma nv_diag_suppress 20014
// Triangle records (the 32-byte vertex + adjacency row pair, read or
// written) touched per phase kind, counted once per item (per body call:
// an item that reads a record and writes it back touches one sector), by
// the host runs of the bodies.
long long gcdt_host_touch[64];
long long gcdt_host_items[64];
// Flip-queue outcomes: entries checked, entries with a candidate edge,
// distinct candidate edges, flips.
long long g_fq[4];
int gcdt_host_phase = 63;
static int g_item_tris[64];
static int g_item_n = 0;
__host__ __device__ inline void gcdt_host_touch_one(int t) {
#ifndef __CUDA_ARCH__
    for (int k = 0; k < g_item_n; ++k)
        if (g_item_tris[k] == t) return;
    if (g_item_n < 64) g_item_tris[g_item_n++] = t;
    ++gcdt_host_touch[gcdt_host_phase];
#endif
}
inline void gcdt_host_new_item() { g_item_n = 0; }
#define GCDT_TOUCH(t) gcdt_host_touch_one(t)
#include "../gcdt_b200/csrc/solver.cuh"

using namespace gcdt;

namespace {

int g_order = 0;          // 0 forward, 1 reversed, 2 shuffled
int g_width = 1;          // items per call in the flip passes (1: one-item bodies)
bool g_check = false;     // mesh consistency after every split fix and flip fix
int g_bad = 0;
std::mt19937 g_rng(1);
int g_lim[3] = {0, 0, 0};   // loop budgets of the next solves (0: built-in bound)
int g_tune[7] = {0};         // scheduling of the next solves: levels, strides[3], carry, narrow q/act (levels 0: default)

// Every live triangle CCW, every adjacency mutual.
void check_mesh(int kind, const Ctx& c) {
    if (g_bad) return;
    for (int t = 0; t < c.ntri; ++t) {
        bool live = t < 2 || c.loc[(t - 2) / 2] == -1;
        if (!live) continue;
        int4 v = tri_v(c, t), a = tri_a(c, t);
        if (orient2d(c.P[v.x], c.P[v.y], c.P[v.z]) <= 0) { g_bad = 100 + kind; return; }
        for (int s = 0; s < 3; ++s) {
            int en = comp(a, s);
            if (en < 0) continue;
            if (comp(tri_a(c, en >> 2), en & 3) != ((t << 2) | s)) { g_bad = 200 + kind; return; }
        }
    }
}

void host_phase(int k, const Ctx& c, long long n) {
    gcdt_host_phase = k >= 0 && k < 63 ? k : 63;
    gcdt_host_items[gcdt_host_phase] += n;
    std::vector<int> idx((size_t)n);
    std::iota(idx.begin(), idx.end(), 0);
    if (g_order == 1) std::reverse(idx.begin(), idx.end());
    if (g_order == 2) std::shuffle(idx.begin(), idx.end(), g_rng);
    if (g_width > 1 && (k == K_FLIP_CHECK || k == K_FLIP_DO || k == K_FLIP_FIX)) {
        const size_t w = k == K_FLIP_CHECK ? (size_t)g_width : 2;
        for (size_t m = 0; m < idx.size(); m += w) {
            int ks[4];
            for (size_t u = 0; u < 4; ++u) ks[u] = m + u < idx.size() && u < w ? idx[m + u] : -1;
            gcdt_host_new_item();
            if (k == K_FLIP_CHECK && w == 2) body_flip_check_pair(c, ks[0], ks[1]);
            else if (k == K_FLIP_CHECK && w == 3) { const int k3[3] = {ks[0], ks[1], ks[2]}; flip_check_multi<3>(c, k3); }
            else if (k == K_FLIP_CHECK) { const int k4[4] = {ks[0], ks[1], ks[2], ks[3]}; flip_check_multi<4>(c, k4); }
            else if (k == K_FLIP_DO) body_flip_do_pair(c, ks[0], ks[1]);
            else body_flip_fix_pair(c, ks[0], ks[1]);
        }
    } else {
        for (int i : idx) {
            gcdt_host_new_item();
            dispatch(k, c, i);
        }
    }
    gcdt_host_phase = 63;
    gcdt_host_new_item();
    if (k == K_FLIP_CHECK) {
        std::vector<long long> edges;
        for (long long i = 0; i < n; ++i) {
            int2 cd = c.cand[i];
            if (cd.x < 0) continue;
            edges.push_back(cd.x < cd.y ? cd.x : cd.y);
        }
        std::sort(edges.begin(), edges.end());
        g_fq[0] += n;
        g_fq[1] += (long long)edges.size();
        g_fq[2] += (long long)(std::unique(edges.begin(), edges.end()) - edges.begin());
    }
    if (k == K_FLIP_DO) g_fq[3] += (long long)(c.cnt->cur_flip - c.base_flip);
    if (g_check && (k == K_FIX || k == K_FLIP_FIX)) check_mesh(k, c);
}

// One block's executor: no single-block hand-off.
struct HostBlock {
    static constexpr bool kCanNarrow = false;
    Counters* cnt;
    void phase(int k, const Ctx& c, long long n) { host_phase(k, c, n); }
    unsigned long long cursor(unsigned long long* p) { return *p; }
    int word(int* p) { return *p; }
    int narrow_flips(Ctx&, Driver&, long long&) { return ST_INTERNAL; }
    int narrow_rounds(Ctx&, Driver&, long long) { return ST_INTERNAL; }
    void finish(const Ctx&, long long, long long, long long, int) {}
};

// The whole grid's executor, with the single-block tails run as HostBlock.
struct HostGrid {
    static constexpr bool kCanNarrow = true;
    Counters* cnt;
    int narrow_flips(Ctx& c, Driver& D, long long& nq) {
        HostBlock bx{cnt};
        Driver Db = D;
        Ctx cb = c;
        long long left = nq;
        int rc = flip_loop(bx, cb, Db, left, 4 * (long long)c.narrow_q);
        D = Db;
        nq = left;
        return rc;
    }
    int narrow_rounds(Ctx& c, Driver& D, long long nact) {
        HostBlock bx{cnt};
        Driver Db = D;
        Ctx cb = c;
        int rc = insert_rounds(bx, cb, Db, nact);
        D = Db;
        return rc;
    }
    void phase(int k, const Ctx& c, long long n) { host_phase(k, c, n); }
    unsigned long long cursor(unsigned long long* p) { return *p; }
    int word(int* p) { return *p; }
    void finish(const Ctx&, long long r, long long s, long long cr, int rc) {
        cnt->rounds = r;
        cnt->flip_subrounds = s;
        cnt->constraint_rounds = cr;
        cnt->status |= rc;
    }
};

struct HostBackend {
    Counters* cnt;
    void launch(int k, const Ctx& c, long long n) { host_phase(k, c, n); }
    void fill(void* p, int v, size_t b) { std::memset(p, v, b); }
    void read(Counters* h) { *h = *cnt; }
    void stages(const Ctx& c0) {
        Ctx c = c0;
        HostGrid ex{cnt};
        run_stages(ex, c);
    }
    void sort(Ctx& c, int n) {
        std::vector<std::pair<unsigned long long, int>> v(n);
        for (int i = 0; i < n; ++i) v[i] = {c.keys[i], c.vals[i]};
        std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        for (int i = 0; i < n; ++i) { c.keys[i] = v[i].first; c.vals[i] = v[i].second; }
    }
};

}  // namespace

// Solve on the host.  order: 0 forward, 1 reversed, 2 shuffled (seeded);
// width: items per call in the flip passes (1: one-item bodies, 2: the
// paired bodies the GPU uses, 3-4: wider flip checks); check: mesh check
// after each fix phase.
// stats[0..4] = status, insertion rounds, flip sub-rounds, flips, constraint
// rounds; returns the status bits, or 1000+ when the mesh check failed.
extern "C" int host_triangulate(const int* xy, int n, const int* cons, int s, int* tris, int* adj,
                                unsigned char* cflags, long long* stats, int order, int width, int check) {
    g_order = order;
    g_width = width < 1 ? 1 : (width > 4 ? 4 : width);
    g_check = check != 0;
    g_bad = 0;
    g_rng.seed(12345);
    Plan p = make_plan(n, s, 0);
    std::vector<char> arena(p.L.total + 256);
    char* base = (char*)(((uintptr_t)arena.data() + 255) & ~(uintptr_t)255);
    Ctx c = bind_ctx(base, p);
    c.in_xy = (const int2*)xy;
    c.in_cons = (const int2*)cons;
    c.out_tris = tris;
    c.out_adj = adj;
    c.out_cflags = cflags;
    c.lim_rounds = g_lim[0];
    c.lim_subrounds = g_lim[1];
    c.lim_crounds = g_lim[2];
    if (g_tune[0] > 0) {
        c.nlevels = g_tune[0];
        for (int k = 0; k < 4; ++k) c.stride[k] = k < 3 && k + 1 < c.nlevels ? g_tune[1 + k] : 1;
        c.carry_q = g_tune[4];
        c.narrow_q = g_tune[5];
        c.narrow_act = g_tune[6];
    }
    HostBackend bk{c.cnt};
    SolveStats ss;
    int rc = run_solve(bk, c, ss);
    stats[0] = rc;
    stats[1] = ss.rounds;
    stats[2] = ss.flip_subrounds;
    stats[3] = ss.flips;
    stats[4] = ss.constraint_rounds;
    return g_bad ? 1000 + g_bad : rc;
}

// Loop budgets for the following host solves, as gcdt_set_limits.
extern "C" void host_set_limits(int rounds, int subrounds, int crounds) {
    g_lim[0] = rounds;
    g_lim[1] = subrounds;
    g_lim[2] = crounds;
}

// Scheduling of the following host solves, as gcdt_set_tuning (levels 0:
// the defaults).
extern "C" void host_set_tuning(int levels, int s0, int s1, int s2, int carry, int narrow_q, int narrow_act) {
    int v[7] = {levels, s0, s1, s2, carry, narrow_q, narrow_act};
    for (int k = 0; k < 7; ++k) g_tune[k] = v[k];
}

// Triangle-record accesses per phase kind since the last call (64 entries;
// entry 63 collects accesses outside any phase) and, if items is not null,
// the items each phase kind ran over; then reset both.
extern "C" void host_touch_counts(long long* out, long long* items) {
    for (int k = 0; k < 64; ++k) {
        out[k] = gcdt_host_touch[k];
        if (items) items[k] = gcdt_host_items[k];
        gcdt_host_touch[k] = 0;
        gcdt_host_items[k] = 0;
    }
}

// Flip-queue outcomes since the last call: entries checked, entries that
// found a non-locally-Delaunay edge, distinct such edges, flips; then reset.
extern "C" void host_flip_outcomes(long long* out) {
    for (int k = 0; k < 4; ++k) { out[k] = g_fq[k]; g_fq[k] = 0; }
}

// The sort keys of n points (2n int32 coordinates), as the key kernel
// computes them.
extern "C" void host_sort_keys(const int* xy, int n, unsigned long long* out) {
    for (int i = 0; i < n; ++i) out[i] = gcdt::sort_key60(make_int2(xy[2 * i], xy[2 * i + 1]));
}
