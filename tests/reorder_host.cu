// reorder_host.cu -- test harness: the reference-layout export's per-item
// bodies (gcdt_b200/csrc/reorder.cuh) run on the host, one body call per
// item in a chosen order, with std::stable_sort in place of the device's
// stable radix sort on the same 30-bit keys.  Running the passes forward,
// reversed and shuffled checks that no body depends on another item's
// order.  Built by tests/test_reference_layout.py into tests/_bin/.
#include <algorithm>
#include <cstdint>
#include <numeric>
#include <random>
#include <vector>

#include "../gcdt_b200/csrc/reorder.cuh"

using namespace gcdt_reorder;

namespace {

std::vector<int> item_order(int count, int order, unsigned seed) {
    std::vector<int> ids(count > 0 ? count : 0);
    std::iota(ids.begin(), ids.end(), 0);
    if (order == 1) std::reverse(ids.begin(), ids.end());
    if (order == 2) std::shuffle(ids.begin(), ids.end(), std::mt19937(seed));
    return ids;
}

// Stable sort of (key, value) pairs by key: the values in sorted order.
std::vector<int> sorted_values(const std::vector<unsigned>& keys, const std::vector<int>& vals) {
    std::vector<int> idx(keys.size());
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return keys[a] < keys[b]; });
    std::vector<int> out(keys.size());
    for (size_t k = 0; k < idx.size(); ++k) out[k] = vals[idx[k]];
    return out;
}

}  // namespace

extern "C" int host_reference_layout(const int32_t* points, int n, const int32_t* tris, const int32_t* adj,
                                     const uint8_t* cf, int nt, int32_t* points_out, int32_t* labels,
                                     int32_t* tris_out, int32_t* adj_out, uint8_t* cf_out, int order) {
    const int2* pts = reinterpret_cast<const int2*>(points);
    const int nv = n + 4;
    int err = 0;
    std::vector<unsigned> keys(nv);
    std::vector<int> vals(nv);
    for (int i : item_order(nv, order, 1)) body_point_key(pts, n, i, keys.data(), vals.data());
    std::vector<int> perm = sorted_values(keys, vals);
    for (int j : item_order(nv, order, 2))
        body_point_scatter(pts, n, j, perm.data(), reinterpret_cast<int2*>(points_out), labels);
    if (nt > 0) {
        std::vector<unsigned> fk(nt);
        std::vector<int> fv(nt), newpos(nt, -7);
        for (int t : item_order(nt, order, 3)) err |= body_face_key(pts, n, tris, t, fk.data(), fv.data());
        std::vector<int> ord = sorted_values(fk, fv);
        if (adj)
            for (int j : item_order(nt, order, 4)) body_face_rank(ord.data(), j, newpos.data());
        for (int j : item_order(nt, order, 5))
            err |= body_face_gather(tris, adj, cf, nt, nv, j, ord.data(), labels, newpos.data(), tris_out,
                                    adj_out, cf_out);
    }
    return err;
}
