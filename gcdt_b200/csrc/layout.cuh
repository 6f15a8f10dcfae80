// layout.cuh -- carve one workspace into every array of a solve.
//
// A solve never allocates: the context owns one arena sized for its maximum
// problem, and every array below is a 256-byte aligned slice of it.
#pragma once
#include <cstddef>
#include <cstdint>
#include "mesh.cuh"

namespace gcdt {

struct Layout {
    size_t off[48];
    int count = 0;
    size_t total = 0;
    __host__ __device__ size_t take(size_t bytes) {
        size_t o = total;
        total += (bytes + 255) & ~size_t(255);
        off[count++] = o;
        return o;
    }
};

struct Plan {
    int64_t n, s, ntri, scratch_cap;
    size_t sort_temp_bytes;
    Layout L;
    size_t o_keys, o_keys_alt, o_vals, o_vals_alt, o_sort_tmp;
    size_t o_P, o_perm, o_rank, o_tri, o_loc, o_pedge, o_actA, o_actB, o_vote, o_win;
    size_t o_claim, o_cand, o_qst, o_qA, o_qB;
    size_t o_seg, o_pendA, o_pendB, o_pinfo, o_scratch, o_vt, o_lvl, o_cnt;
};

__host__ __device__ inline Plan make_plan(int64_t n, int64_t s, size_t sort_temp_bytes) {
    Plan p;
    p.n = n; p.s = s; p.ntri = 2 * n + 2;
    p.sort_temp_bytes = sort_temp_bytes;
    int64_t nn = n > 0 ? n : 1, ss = s > 0 ? s : 1, T = p.ntri;
    p.scratch_cap = 4 * T + 64;
    Layout& L = p.L;
    p.o_cnt = L.take(sizeof(Counters));
    p.o_keys = L.take(8 * nn);
    p.o_keys_alt = L.take(8 * nn);
    p.o_vals = L.take(4 * nn);
    p.o_vals_alt = L.take(4 * nn);
    p.o_sort_tmp = L.take(sort_temp_bytes);
    p.o_P = L.take(8 * (nn + 4));
    p.o_perm = L.take(4 * (nn + 4));
    p.o_rank = L.take(4 * nn);
    p.o_tri = L.take(32 * T);
    p.o_loc = L.take(4 * nn);
    p.o_pedge = L.take(nn);
    p.o_actA = L.take(4 * nn);
    p.o_actB = L.take(4 * nn);
    p.o_vote = L.take(8 * T);
    p.o_win = L.take(8 * nn);
    p.o_claim = L.take(8 * T);
    p.o_cand = L.take(8 * T);
    p.o_qst = L.take(4 * T);
    p.o_qA = L.take(4 * T);
    p.o_qB = L.take(4 * T);
    p.o_scratch = L.take(4 * p.scratch_cap);
    p.o_vt = L.take(4 * (nn + 4));
    p.o_lvl = L.take(nn);
    // the segment arrays last: every other array has the same offset for
    // any segment count
    p.o_seg = L.take(16 * ss);
    p.o_pendA = L.take(4 * ss);
    p.o_pendB = L.take(4 * ss);
    p.o_pinfo = L.take(16 * ss);
    return p;
}

}  // namespace gcdt
