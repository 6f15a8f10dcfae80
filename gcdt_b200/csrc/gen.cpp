// gen.cpp -- seeded synthetic inputs for the CDT path (host only).
//
// The reference ships no data set; its driver draws random points on the host
// and scales them to the 2^30 integer grid (kernel.cu:43-58, 171-188).  These
// generators produce the five workloads the path is measured on, from a
// splitmix64 stream so that every machine produces the same bytes:
//
//   uniform points, Gaussian-mixture points, a 2^k lattice, and star-shaped
//   polygons whose boundaries are the constraint segments.
//
// All coordinates are kept in [1, 2^30-2] so that no point lies on the
// bounding box (0,0)-(2^30-1,2^30-1) the reference triangulates into
// (rawMesh.cu:5-35).  Duplicate points are removed (first occurrence kept),
// polygon vertices that coincide with an existing point reuse its index, and
// every point lying exactly on a constraint segment (orient2d == 0, inside the
// span) is dropped, as the reference's file reader does for its inputs
// (kernel.cu:5159-5291).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <unordered_map>
#include <vector>

namespace {

constexpr int64_t kBoxMax = (int64_t(1) << 30) - 1;

struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed) {}
    uint64_t next() {  // splitmix64
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return double(next() >> 11) * (1.0 / 9007199254740992.0); }
    int64_t range(int64_t lo, int64_t hi) {  // [lo, hi)
        return lo + int64_t(next() % uint64_t(hi - lo));
    }
    double gauss() {  // Box-Muller
        double u1 = uniform(), u2 = uniform();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

inline int64_t clamp_coord(int64_t v, int64_t hi) {
    if (v < 1) return 1;
    if (v > hi) return hi;
    return v;
}

inline int orient(int64_t ax, int64_t ay, int64_t bx, int64_t by, int64_t cx, int64_t cy) {
    int64_t o1 = (ax - cx) * (by - cy), o2 = (ay - cy) * (bx - cx);
    return (o1 > o2) - (o1 < o2);
}

struct Instance {
    std::vector<int32_t> xy;    // 2 per point
    std::vector<int32_t> cons;  // 2 per segment
    std::unordered_map<uint64_t, int32_t> index;
    // polygons, for the on-segment filter
    struct Poly { int64_t cx, cy; int first, count; };
    std::vector<Poly> polys;
    std::vector<int32_t> poly_vidx;  // vertex indices of all polygons, concatenated

    static uint64_t key(int64_t x, int64_t y) { return (uint64_t(x) << 32) | uint64_t(y); }

    int32_t add_point(int64_t x, int64_t y) {
        auto it = index.find(key(x, y));
        if (it != index.end()) return it->second;
        int32_t id = int32_t(xy.size() / 2);
        index.emplace(key(x, y), id);
        xy.push_back(int32_t(x));
        xy.push_back(int32_t(y));
        return id;
    }
};

// One star-shaped polygon around (cx, cy): sorted random angles with a minimum
// gap so that rounding to integers cannot reorder them, radii U[0.5R, R].
void add_star_polygon(Instance& I, Rng& rng, int64_t cx, int64_t cy, double R, int nv) {
    std::vector<double> ang(nv);
    double rmin = 0.5 * R;
    double min_gap = 32.0 / rmin;
    for (int attempt = 0;; ++attempt) {
        for (int k = 0; k < nv; ++k) ang[k] = 6.283185307179586 * rng.uniform();
        std::sort(ang.begin(), ang.end());
        bool ok = true;
        for (int k = 0; k < nv && ok; ++k) {
            double g = (k + 1 < nv) ? ang[k + 1] - ang[k] : ang[0] + 6.283185307179586 - ang[k];
            if (g < min_gap) ok = false;
        }
        if (ok) break;
        if (attempt > 64) {  // stratified fallback: one angle per equal sector
            for (int k = 0; k < nv; ++k)
                ang[k] = 6.283185307179586 * (k + 0.1 + 0.8 * rng.uniform()) / nv;
            break;
        }
    }
    Instance::Poly P{cx, cy, int(I.poly_vidx.size()), nv};
    std::vector<int32_t> vid(nv);
    for (int k = 0; k < nv; ++k) {
        double r = rmin + (R - rmin) * rng.uniform();
        int64_t x = clamp_coord(int64_t(std::llround(double(cx) + r * std::cos(ang[k]))), kBoxMax - 1);
        int64_t y = clamp_coord(int64_t(std::llround(double(cy) + r * std::sin(ang[k]))), kBoxMax - 1);
        vid[k] = I.add_point(x, y);
    }
    for (int k = 0; k < nv; ++k) {
        I.poly_vidx.push_back(vid[k]);
        int a = vid[k], b = vid[(k + 1) % nv];
        if (a != b) { I.cons.push_back(a); I.cons.push_back(b); }
    }
    I.polys.push_back(P);
}

// Drop every non-polygon point that lies exactly on a polygon edge.  `cell_of`
// maps a point to the polygon that may contain it (-1: none).
template <class CellOf>
void drop_points_on_segments(Instance& I, CellOf cell_of) {
    int n = int(I.xy.size() / 2);
    std::vector<char> is_vertex(n, 0);
    for (int32_t v : I.poly_vidx) is_vertex[v] = 1;
    std::vector<char> drop(n, 0);
    int ndrop = 0;
    for (int i = 0; i < n; ++i) {
        if (is_vertex[i]) continue;
        int64_t px = I.xy[2 * i], py = I.xy[2 * i + 1];
        int pi = cell_of(px, py);
        if (pi < 0) continue;
        const auto& P = I.polys[pi];
        const int32_t* V = I.poly_vidx.data() + P.first;
        int m = P.count;
        for (int k = 0; k < m; ++k) {  // wedge of the star containing p
            int a = V[k], b = V[(k + 1) % m];
            int64_t ax = I.xy[2 * a], ay = I.xy[2 * a + 1], bx = I.xy[2 * b], by = I.xy[2 * b + 1];
            if (orient(P.cx, P.cy, ax, ay, px, py) >= 0 && orient(P.cx, P.cy, bx, by, px, py) < 0) {
                if (orient(ax, ay, bx, by, px, py) == 0 &&
                    std::min(ax, bx) <= px && px <= std::max(ax, bx) &&
                    std::min(ay, by) <= py && py <= std::max(ay, by)) {
                    drop[i] = 1; ndrop++;
                }
                break;
            }
        }
    }
    if (!ndrop) return;
    std::vector<int32_t> remap(n, -1);
    std::vector<int32_t> xy2;
    xy2.reserve(I.xy.size());
    for (int i = 0; i < n; ++i) {
        if (drop[i]) continue;
        remap[i] = int32_t(xy2.size() / 2);
        xy2.push_back(I.xy[2 * i]);
        xy2.push_back(I.xy[2 * i + 1]);
    }
    for (auto& c : I.cons) c = remap[c];
    for (auto& v : I.poly_vidx) v = remap[v];
    I.xy.swap(xy2);
}

// Uniform / Gaussian-mixture points over [1, hi]^2 plus star polygons on a
// G x G grid over [0, span)^2, `npoly` of the G*G cells chosen at random.
void gen_mixture(Instance& I, Rng& rng, int64_t npts, int64_t hi, double frac_gauss, int ngauss,
                 double sigma, int64_t span, int G, int npoly, int vmin, int vmax, double rfrac) {
    I.index.reserve(size_t(npts * 1.3) + 1024);
    std::vector<double> gcx(ngauss), gcy(ngauss);
    for (int g = 0; g < ngauss; ++g) {
        gcx[g] = double(rng.range(1, hi + 1));
        gcy[g] = double(rng.range(1, hi + 1));
    }
    int64_t ngpts = int64_t(std::llround(frac_gauss * double(npts)));
    for (int64_t i = 0; i < npts; ++i) {
        int64_t x, y;
        if (i < ngpts && ngauss > 0) {
            int g = int(rng.next() % uint64_t(ngauss));
            x = clamp_coord(int64_t(std::llround(gcx[g] + sigma * rng.gauss())), hi);
            y = clamp_coord(int64_t(std::llround(gcy[g] + sigma * rng.gauss())), hi);
        } else {
            x = rng.range(1, hi + 1);
            y = rng.range(1, hi + 1);
        }
        I.add_point(x, y);
    }
    // polygons: choose npoly distinct cells
    int ncell = G * G;
    std::vector<int> cells(ncell);
    for (int c = 0; c < ncell; ++c) cells[c] = c;
    for (int c = ncell - 1; c > 0; --c) std::swap(cells[c], cells[int(rng.next() % uint64_t(c + 1))]);
    std::vector<int> cell_poly(ncell, -1);
    double cw = double(span) / G;
    double R = std::floor(rfrac * cw);
    for (int k = 0; k < npoly && k < ncell; ++k) {
        int c = cells[k];
        int gx = c % G, gy = c / G;
        int64_t cx = int64_t(std::llround((gx + 0.5) * cw)), cy = int64_t(std::llround((gy + 0.5) * cw));
        int nv = vmin == vmax ? vmin : int(rng.range(vmin, vmax + 1));
        cell_poly[c] = int(I.polys.size());
        add_star_polygon(I, rng, cx, cy, R, nv);
    }
    drop_points_on_segments(I, [&](int64_t x, int64_t y) {
        int gx = int(double(x) / cw), gy = int(double(y) / cw);
        if (gx < 0 || gy < 0 || gx >= G || gy >= G) return -1;
        return cell_poly[gy * G + gx];
    });
}

// 2048x2048-style lattice with axis-aligned rectangle boundaries (unit
// lattice segments) whose interiors are disjoint.
void gen_lattice(Instance& I, Rng& rng, int side, int64_t spacing, int64_t origin, int nseg, int max_rect) {
    I.xy.resize(size_t(2) * side * side);
    for (int j = 0; j < side; ++j)
        for (int i = 0; i < side; ++i) {
            size_t id = size_t(j) * side + i;
            I.xy[2 * id] = int32_t(origin + spacing * i);
            I.xy[2 * id + 1] = int32_t(origin + spacing * j);
        }
    std::vector<uint8_t> occ(size_t(side) * side, 0);  // lattice cells (i,j) covered by a rectangle interior
    std::unordered_map<uint64_t, char> seen;
    auto vid = [&](int i, int j) { return int32_t(j * side + i); };
    auto add_seg = [&](int32_t a, int32_t b) {
        if ((int)(I.cons.size() / 2) >= nseg) return;
        uint64_t k = a < b ? (uint64_t(a) << 32) | uint32_t(b) : (uint64_t(b) << 32) | uint32_t(a);
        if (seen.count(k)) return;
        seen.emplace(k, 1);
        I.cons.push_back(a); I.cons.push_back(b);
    };
    for (int attempt = 0; attempt < 50000000 && (int)(I.cons.size() / 2) < nseg; ++attempt) {
        int w = int(rng.range(1, max_rect + 1)), h = int(rng.range(1, max_rect + 1));
        int x0 = int(rng.range(0, side - w)), y0 = int(rng.range(0, side - h));
        bool free_ = true;
        for (int j = y0; j < y0 + h && free_; ++j)
            for (int i = x0; i < x0 + w; ++i)
                if (occ[size_t(j) * side + i]) { free_ = false; break; }
        if (!free_) continue;
        for (int j = y0; j < y0 + h; ++j)
            for (int i = x0; i < x0 + w; ++i) occ[size_t(j) * side + i] = 1;
        for (int i = x0; i < x0 + w; ++i) { add_seg(vid(i, y0), vid(i + 1, y0)); add_seg(vid(i, y0 + h), vid(i + 1, y0 + h)); }
        for (int j = y0; j < y0 + h; ++j) { add_seg(vid(x0, j), vid(x0, j + 1)); add_seg(vid(x0 + w, j), vid(x0 + w, j + 1)); }
    }
}

}  // namespace

extern "C" {

// Workload kinds.
//  0  uniform points in [1, 2^hi_log2) + a 4x2 grid of 64-gon stars with R = 2^16
//     (100,000 points, 512 segments at the defaults)
//  1  Gaussian mixture (90%: 64 centres, sigma 2^22) + 10% uniform over
//     [1, 2^30-2], 64-gon stars in `npoly` cells of a G x G grid, R = 0.45 cell
//  2  lattice side x side, spacing 2^14, origin (2^14, 2^14), `nseg` unit
//     segments from disjoint rectangles
//  3  one batched instance: uniform in [1, 2^24), 1-4 stars of 16-256 vertices
//     in distinct quadrants
//  4  one serving request: config-1 mix scaled to [1, 2^28), stars totalling
//     about 2% of the point count
//  5  uniform points over the whole box [1, 2^30-2]^2 (the distribution of the
//     reference driver's own randomMap, kernel.cu:43-58), no segments
// Parameters a,b,c,d are kind specific (0 = default).
void* gcdt_gen_new(int kind, uint64_t seed, int64_t a, int64_t b, int64_t c, int64_t d) {
    Instance* I = new Instance();
    Rng rng(seed * 0x100000001B3ull + 0x243F6A8885A308D3ull + uint64_t(kind));
    switch (kind) {
    case 0: {  // small plain CDT
        int64_t npts = a ? a : 100000;
        int nvert = b ? int(b) : 64;
        int64_t hi = (int64_t(1) << 20) - 1;
        I->index.reserve(size_t(npts) * 2);
        for (int64_t i = 0; i < npts; ++i) I->add_point(rng.range(1, hi + 1), rng.range(1, hi + 1));
        std::vector<int> cell_poly(8, -1);
        double cwx = double(int64_t(1) << 18), cwy = double(int64_t(1) << 19);
        for (int k = 0; k < 8; ++k) {
            int gx = k % 4, gy = k / 4;
            cell_poly[k] = int(I->polys.size());
            add_star_polygon(*I, rng, int64_t((gx + 0.5) * cwx), int64_t((gy + 0.5) * cwy),
                             double(int64_t(1) << 16), nvert);
        }
        drop_points_on_segments(*I, [&](int64_t x, int64_t y) {
            int gx = int(double(x) / cwx), gy = int(double(y) / cwy);
            if (gx < 0 || gy < 0 || gx >= 4 || gy >= 2) return -1;
            return cell_poly[gy * 4 + gx];
        });
        break;
    }
    case 1: {  // plain CDT at scale
        int64_t npts = a ? a : 10000000;
        int G = b ? int(b) : 56;
        int npoly = c ? int(c) : 3125;
        gen_mixture(*I, rng, npts, kBoxMax - 1, 0.9, 64, double(int64_t(1) << 22),
                    int64_t(1) << 30, G, npoly, 64, 64, 0.45);
        break;
    }
    case 2: {  // lattice
        int side = a ? int(a) : 2048;
        int nseg = b ? int(b) : 20000;
        gen_lattice(*I, rng, side, int64_t(1) << 14, int64_t(1) << 14, nseg, 16);
        break;
    }
    case 3: {  // one batched instance
        double lo = std::log(64.0), hiL = std::log(65536.0);
        int64_t npts = a ? a : int64_t(std::floor(std::exp(lo + (hiL - lo) * rng.uniform())));
        int npoly = int(rng.range(1, 5));
        gen_mixture(*I, rng, npts, (int64_t(1) << 24) - 1, 0.0, 0, 0.0, int64_t(1) << 24, 2, npoly,
                    16, 256, 0.45);
        break;
    }
    case 4: {  // one serving request
        double lo = std::log(1000.0), hiL = std::log(1000000.0);
        int64_t npts = a ? a : int64_t(std::floor(std::exp(lo + (hiL - lo) * rng.uniform())));
        int64_t target_seg = std::max<int64_t>(16, npts / 50);
        int npoly = int(std::max<int64_t>(1, target_seg / 64));
        int G = int(std::ceil(std::sqrt(double(npoly) * 1.0)));
        gen_mixture(*I, rng, npts, (int64_t(1) << 28) - 1, 0.9, 64, double(int64_t(1) << 20),
                    int64_t(1) << 28, G, npoly, 64, 64, 0.45);
        break;
    }
    case 5: {  // uniform points over the whole box [1, 2^30-2]^2, no segments
        int64_t npts = a ? a : 1000000;
        I->index.reserve(size_t(npts) * 2);
        for (int64_t i = 0; i < npts; ++i) I->add_point(rng.range(1, kBoxMax), rng.range(1, kBoxMax));
        break;
    }
    default:
        delete I;
        return nullptr;
    }
    return I;
}

void gcdt_gen_sizes(void* h, int64_t* npts, int64_t* nseg) {
    Instance* I = static_cast<Instance*>(h);
    *npts = int64_t(I->xy.size() / 2);
    *nseg = int64_t(I->cons.size() / 2);
}

void gcdt_gen_copy(void* h, int32_t* xy, int32_t* cons) {
    Instance* I = static_cast<Instance*>(h);
    if (xy && !I->xy.empty()) std::memcpy(xy, I->xy.data(), I->xy.size() * sizeof(int32_t));
    if (cons && !I->cons.empty()) std::memcpy(cons, I->cons.data(), I->cons.size() * sizeof(int32_t));
}

void gcdt_gen_free(void* h) { delete static_cast<Instance*>(h); }

}  // extern "C"
