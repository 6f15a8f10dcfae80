// regions_host.cu -- test harness: the region classification's per-item
// bodies (gcdt_b200/csrc/regions.cuh) run on the host, one body call per
// item in a chosen order (forward, reversed, shuffled), with the same pass
// sequence as gcdt_classify_regions.  Built by tests/test_regions.py into
// tests/_bin/.
#include <algorithm>
#include <cstdint>
#include <numeric>
#include <random>
#include <vector>

#include "../gcdt_b200/csrc/regions.cuh"

using namespace gcdt_regions;

namespace {

std::vector<int> item_order(int count, int order, unsigned seed) {
    std::vector<int> ids(count > 0 ? count : 0);
    std::iota(ids.begin(), ids.end(), 0);
    if (order == 1) std::reverse(ids.begin(), ids.end());
    if (order == 2) std::shuffle(ids.begin(), ids.end(), std::mt19937(seed));
    return ids;
}

}  // namespace

// Returns the error bits; *max_depth and depth as gcdt_classify_regions;
// parent_out receives each triangle's component root.
extern "C" int host_classify_regions(const int32_t* adj, const uint8_t* cf, int nt, int32_t* depth,
                                     int32_t* max_depth, int32_t* parent_out, int order) {
    std::vector<int> parent(nt), level(nt);
    int err = 0;
    for (int t : item_order(nt, order, 1)) body_init(t, parent.data(), level.data());
    for (int t : item_order(nt, order, 2)) err |= body_hook(adj, cf, nt, t, parent.data());
    for (int t : item_order(nt, order, 3)) err |= body_compress(t, parent.data());
    if (err) return err;
    for (int t : item_order(nt, order, 4)) body_seed(adj, t, parent.data(), level.data());
    int L = 0;
    for (;; ++L) {
        int changed = 0;
        for (int t : item_order(nt, order, 5 + L)) changed |= body_expand(adj, cf, nt, t, L, parent.data(), level.data());
        if (!changed) break;
    }
    for (int t : item_order(nt, order, 99)) body_depth(t, parent.data(), level.data(), depth);
    std::copy(parent.begin(), parent.end(), parent_out);
    *max_depth = L;
    return 0;
}
