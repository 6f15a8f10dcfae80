// io.cpp -- input preprocessing and mesh export (host only).
//
// Reader of the reference's text format (yingtix/gCDT kernel.cu:5159-5291):
//   numPoints
//   idx x y            (numPoints lines, x y as reals)
//   numCons
//   idx a b            (numCons lines, a b point idx values)
// Steps, as the reference's readFile + transPoints (kernel.cu:171-188):
//   1. exact duplicate (x, y) pairs are merged; every idx maps to the kept point;
//   2. coordinates are normalised: (p - centre) / max(extent) * 0.99 + 0.5;
//   3. segments are mapped through the idx map; a == b and repeated segments
//      (either direction) are dropped;
//   4. coordinates are scaled by 2^30 and truncated, clamped to [0, 2^30 - 1].
// Two more steps make the result satisfy this library's input contract:
//   5. points that collide after step 4 are merged (segments remapped, then
//      step 3's filter applied again);
//   6. coordinates are clamped to [1, 2^30 - 2], off the bounding box the
//      corners span (the reference leaves a point on the box unhandled,
//      rawMesh.cu:76-131).
// The writer emits a mesh as text: numPoints, "idx x y" lines, numTriangles,
// "idx a b c n0 n1 n2 flags" lines (n_k: triangle across the edge opposite
// vertex k, -1 on the box; flags: bit k = that edge is a constraint).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <new>
#include <set>
#include <string>
#include <unordered_map>
#include <vector>

namespace {

struct TextInput {
    std::vector<int32_t> xy, cons;
};

constexpr int64_t kRes = int64_t(1) << 30;

int load(const char* path, TextInput& out) {
    std::ifstream in(path);
    if (!in) return 1;
    long long np = 0;
    if (!(in >> np) || np < 0 || np > (int64_t(1) << 30)) return 2;
    std::map<std::pair<double, double>, int> pmap;
    std::unordered_map<long long, int> idxmap;
    std::vector<double> pts;
    pts.reserve(size_t(np) * 2);
    double minx = 1e300, miny = 1e300, maxx = -1e300, maxy = -1e300;
    for (long long i = 0; i < np; ++i) {
        long long idx;
        double x, y;
        if (!(in >> idx >> x >> y)) return 2;
        auto key = std::make_pair(x, y);
        auto it = pmap.find(key);
        if (it == pmap.end()) {
            int r = int(pts.size() / 2);
            pmap.emplace(key, r);
            pts.push_back(x);
            pts.push_back(y);
            idxmap[idx] = r;
            minx = std::min(minx, x); maxx = std::max(maxx, x);
            miny = std::min(miny, y); maxy = std::max(maxy, y);
        } else {
            idxmap[idx] = it->second;
        }
    }
    int n = int(pts.size() / 2);
    double cx = (minx + maxx) / 2, cy = (miny + maxy) / 2;
    double lx = std::max(maxx - minx, maxy - miny);
    if (!(lx > 0)) lx = 1.0;
    // steps 2, 4, 6; step 5 merges integer collisions
    std::vector<int> remap(n);
    std::unordered_map<uint64_t, int> grid;
    grid.reserve(size_t(n) * 2);
    for (int i = 0; i < n; ++i) {
        double fx = (pts[2 * i] - cx) / lx * 0.99 + 0.5;
        double fy = (pts[2 * i + 1] - cy) / lx * 0.99 + 0.5;
        long long x = (long long)(fx * double(kRes)), y = (long long)(fy * double(kRes));
        x = std::min<long long>(std::max<long long>(x, 1), kRes - 2);
        y = std::min<long long>(std::max<long long>(y, 1), kRes - 2);
        uint64_t key = (uint64_t(x) << 32) | uint64_t(y);
        auto it = grid.find(key);
        if (it == grid.end()) {
            int r = int(out.xy.size() / 2);
            grid.emplace(key, r);
            out.xy.push_back(int32_t(x));
            out.xy.push_back(int32_t(y));
            remap[i] = r;
        } else {
            remap[i] = it->second;
        }
    }
    long long nc = 0;
    if (!(in >> nc)) nc = 0;
    std::set<std::pair<int, int>> seen;
    for (long long k = 0; k < nc; ++k) {
        long long idx, a, b;
        if (!(in >> idx >> a >> b)) return 2;
        auto ia = idxmap.find(a), ib = idxmap.find(b);
        if (ia == idxmap.end() || ib == idxmap.end()) return 3;
        int x = remap[ia->second], y = remap[ib->second];
        if (x == y || seen.count({x, y}) || seen.count({y, x})) continue;
        seen.insert({x, y});
        out.cons.push_back(x);
        out.cons.push_back(y);
    }
    return 0;
}

}  // namespace

extern "C" {

// Returns a handle, or NULL with *err = 1 (cannot open), 2 (malformed),
// 3 (segment refers to an unknown point).
void* gcdt_text_load(const char* path, int* err) {
    TextInput* t = new (std::nothrow) TextInput();
    if (!t) { if (err) *err = 4; return nullptr; }
    int rc = load(path, *t);
    if (err) *err = rc;
    if (rc) { delete t; return nullptr; }
    return t;
}

void gcdt_text_sizes(void* h, int64_t* n, int64_t* s) {
    TextInput* t = static_cast<TextInput*>(h);
    *n = int64_t(t->xy.size() / 2);
    *s = int64_t(t->cons.size() / 2);
}

void gcdt_text_copy(void* h, int32_t* xy, int32_t* cons) {
    TextInput* t = static_cast<TextInput*>(h);
    if (xy && !t->xy.empty()) std::memcpy(xy, t->xy.data(), t->xy.size() * 4);
    if (cons && !t->cons.empty()) std::memcpy(cons, t->cons.data(), t->cons.size() * 4);
}

void gcdt_text_free(void* h) { delete static_cast<TextInput*>(h); }

// Write a mesh (host arrays): n points (+4 corners appended), ntri triangles.
int gcdt_text_save(const char* path, const int32_t* xy, int64_t n, const int32_t* tris, const int32_t* adj,
                   const uint8_t* cflags, int64_t ntri) {
    FILE* f = fopen(path, "w");
    if (!f) return 1;
    const int64_t R = kRes - 1;
    fprintf(f, "%lld\n", (long long)(n + 4));
    for (int64_t i = 0; i < n; ++i) fprintf(f, "%lld %d %d\n", (long long)i, xy[2 * i], xy[2 * i + 1]);
    const int64_t cxy[4][2] = {{0, 0}, {R, 0}, {R, R}, {0, R}};
    for (int k = 0; k < 4; ++k) fprintf(f, "%lld %lld %lld\n", (long long)(n + k), (long long)cxy[k][0], (long long)cxy[k][1]);
    fprintf(f, "%lld\n", (long long)ntri);
    for (int64_t t = 0; t < ntri; ++t)
        fprintf(f, "%lld %d %d %d %d %d %d %d\n", (long long)t, tris[3 * t], tris[3 * t + 1], tris[3 * t + 2],
                adj ? adj[3 * t] : -1, adj ? adj[3 * t + 1] : -1, adj ? adj[3 * t + 2] : -1,
                cflags ? int(cflags[t]) : 0);
    return fclose(f) == 0 ? 0 : 1;
}

}  // extern "C"
