// batch.cu -- many independent triangulations in one launch.
//
// The reference has no batched mode (kernel.cu:5332-5466 triangulates one
// point set per process).  Here one call triangulates thousands of
// independent instances of uneven size:
//   1. one kernel computes the Hilbert key of every point of every instance;
//   2. one segmented radix sort orders each instance's points;
//   3. one kernel with one block per instance runs the whole solve of that
//      instance -- set-up, insertion rounds, flip sub-rounds, constraint
//      rounds, output -- with the same stage driver as the single solve,
//      phases separated by block barriers.  Blocks are issued largest
//      instance first, so the hardware block scheduler acts as the
//      per-instance work queue and balances the tail.
// Every instance works in its own slice of one arena laid out on the host.
// Outputs are the single solve's, instance by instance: instance i's 2n_i+2
// triangles start at triangle 2*P_i + 2*i (P_i = its first point), with
// vertex ids and adjacency local to the instance.
#include <cuda_runtime.h>
#include <cub/device/device_segmented_radix_sort.cuh>

#include <algorithm>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "solver.cuh"
#include "exec.cuh"
#include "../../include/gcdt.h"

namespace gcdt {

struct BatchDesc {
    long long pt_off, seg_off, ws_off, tri_off;
    int n, s, status, pad;
};

struct BatchArgs {
    const int2* xy;
    const int2* cons;
    const unsigned long long* keys;   // sorted, per instance segment
    const int* vals;
    BatchDesc* desc;
    const int* order;                 // instance handled by block b
    char* ws;
    int* tris;
    int* adj;
    unsigned char* cflags;
    int stride0;
};

__global__ void gcdt_batch_keys(const int2* xy, const int* offs, int ninst, int total,
                                unsigned long long* keys, int* vals, BatchDesc* desc) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    int lo = 0, hi = ninst;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (offs[mid] <= g) lo = mid; else hi = mid;
    }
    int2 p = xy[g];
    if (p.x < 1 || p.y < 1 || p.x > kBoxMax - 1 || p.y > kBoxMax - 1) atomicOr(&desc[lo].status, ST_BAD_INPUT);
    keys[g] = sort_key60(p);
    vals[g] = g - offs[lo];
}

template <int BS>
__global__ void __launch_bounds__(BS) gcdt_batch_solve(BatchArgs a) {
    const int inst = a.order[blockIdx.x];
    BatchDesc d = a.desc[inst];
    if (d.status) return;                        // rejected by the key pass
    Plan p = make_plan(d.n, d.s, 0);
    Ctx c = bind_ctx(a.ws + d.ws_off, p);
    c.keys = const_cast<unsigned long long*>(a.keys) + d.pt_off;
    c.vals = const_cast<int*>(a.vals) + d.pt_off;
    c.in_xy = a.xy + d.pt_off;
    c.in_cons = a.cons + d.seg_off;
    c.out_tris = a.tris + 3 * d.tri_off;
    c.out_adj = a.adj + 3 * d.tri_off;
    c.out_cflags = a.cflags + d.tri_off;
    // small instances: two levels, the autotuned sample stride, then the rest
    c.nlevels = 2;
    c.stride[0] = a.stride0; c.stride[1] = 1;
    // the phases' items read the instance's context from shared memory, the
    // fields the driver changes from its own copy (42.7k vs 40.5k instances/s
    // on 4,096 instances, against a per-thread copy in local memory)
    __shared__ Ctx sc;
    if (threadIdx.x == 0) sc = c;
    __syncthreads();
    BlockExecT<true> ex{c.cnt, &sc};
    // per-solve reset: counters and the per-triangle state
    {
        int* w = reinterpret_cast<int*>(c.cnt);
        for (int k = threadIdx.x; k < (int)(sizeof(Counters) / 4); k += blockDim.x) w[k] = 0;
        __syncthreads();
    }
    ex.phase(K_CLEAR, c, c.ntri);
    ex.phase(K_GATHER, c, c.n + 4);
    ex.phase(K_ROOT, c, 1);
    if (c.n > 0) ex.phase(K_LEVEL, c, c.n);
    if (c.s > 0) {
        ex.phase(K_SEG_INIT, c, c.s);
        ex.phase(K_SEG_LEVEL0, c, c.s);
    }
    int st = ex.word(&c.cnt->err[0]) | ex.word(&c.cnt->err[1]) | ex.word(&c.cnt->status);
    if (st == 0) {
        run_stages(ex, c);
        st = ex.word(&c.cnt->err[0]) | ex.word(&c.cnt->err[1]) | ex.word(&c.cnt->status);
    }
    if (threadIdx.x == 0) {
        // run_stages' result is folded into cnt->status by BlockExec::finish
        a.desc[inst].status = st | ex.word(&c.cnt->status);
    }
}

}  // namespace gcdt

using namespace gcdt;

struct gcdt_batch {
    int device = 0;
    int64_t max_inst = 0, max_pts = 0, max_segs = 0;
    size_t ws_bytes = 0, sort_bytes = 0;
    char* ws = nullptr;
    void* sort_tmp = nullptr;
    unsigned long long* keys[2] = {nullptr, nullptr};
    int* vals[2] = {nullptr, nullptr};
    int* d_offs = nullptr;
    int* d_order = nullptr;
    BatchDesc* d_desc = nullptr;
    BatchDesc* h_desc = nullptr;     // pinned
    int* h_offs = nullptr;           // pinned
    int* h_order = nullptr;          // pinned
    gcdt_batch_config cfg{256, 64};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0;
};

namespace {

struct DevGuard {
    int prev = -1;
    explicit DevGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DevGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

// Arena bytes for a batch: the instances' solve layouts (without sort
// scratch, which is shared), each 256-byte aligned.
size_t instance_bytes(int64_t n, int64_t s) { return make_plan(n, s, 0).L.total; }

size_t arena_bound(int64_t max_inst, int64_t max_pts, int64_t max_segs) {
    // make_plan is affine in (n, s) per array plus at most 256 bytes of
    // alignment per array: bound the sum over instances by the totals plus
    // one empty instance's layout and 48 alignment pads per instance.
    return make_plan(max_pts, max_segs, 0).L.total + (size_t)max_inst * (instance_bytes(0, 0) + 48 * 256);
}

bool valid_cfg(const gcdt_batch_config& c) {
    return (c.threads_per_instance == 128 || c.threads_per_instance == 256 || c.threads_per_instance == 512) &&
           (c.sample_stride == 16 || c.sample_stride == 32 || c.sample_stride == 64 ||
            c.sample_stride == 128 || c.sample_stride == 256);
}

}  // namespace

// Launch half of a batched solve (asynchronous on `st`).  tri_off, when
// given, places instance i's triangles at tri_off[i] instead of
// 2*pt_off[i] + 2*i (the serving engine's resident output pool).
gcdt_status gcdt_batch_launch(gcdt_batch* b, int32_t ninst, const int64_t* pt_off, const int64_t* seg_off,
                              const int64_t* tri_off, const int32_t* d_points, const int32_t* d_segments,
                              int32_t* d_tris, int32_t* d_adj, uint8_t* d_cflags, cudaStream_t st,
                              const gcdt_batch_config& cfg);
// Completion half: after `st` has finished, turn the instances' status bits
// into codes; returns the first failure.
gcdt_status gcdt_batch_finalize(gcdt_batch* b, int32_t ninst, int32_t* inst_status);

namespace {

gcdt_status run_batch(gcdt_batch* b, int32_t ninst, const int64_t* pt_off, const int64_t* seg_off,
                      const int32_t* d_points, const int32_t* d_segments, int32_t* d_tris, int32_t* d_adj,
                      uint8_t* d_cflags, int32_t* inst_status, cudaStream_t st, const gcdt_batch_config& cfg) {
    if (ninst <= 0) return ninst == 0 ? GCDT_OK : GCDT_BAD_INPUT;
    gcdt_status rc = gcdt_batch_launch(b, ninst, pt_off, seg_off, nullptr, d_points, d_segments, d_tris, d_adj,
                                       d_cflags, st, cfg);
    if (rc != GCDT_OK) return rc;
    if (cudaStreamSynchronize(st) != cudaSuccess) return GCDT_CUDA_ERROR;
    return gcdt_batch_finalize(b, ninst, inst_status);
}

}  // namespace

gcdt_status gcdt_batch_launch(gcdt_batch* b, int32_t ninst, const int64_t* pt_off, const int64_t* seg_off,
                              const int64_t* tri_off, const int32_t* d_points, const int32_t* d_segments,
                              int32_t* d_tris, int32_t* d_adj, uint8_t* d_cflags, cudaStream_t st,
                              const gcdt_batch_config& cfg) {
    if (ninst <= 0) return ninst == 0 ? GCDT_OK : GCDT_BAD_INPUT;
    if (ninst > b->max_inst) return GCDT_OOM;
    int64_t total = pt_off[ninst] - pt_off[0], stotal = seg_off[ninst] - seg_off[0];
    if (pt_off[0] != 0 || seg_off[0] != 0 || total < 0 || stotal < 0) return GCDT_BAD_INPUT;
    if (total > b->max_pts || stotal > b->max_segs) return GCDT_OOM;
    size_t ws = 0;
    for (int i = 0; i < ninst; ++i) {
        int64_t n = pt_off[i + 1] - pt_off[i], s = seg_off[i + 1] - seg_off[i];
        if (n < 0 || s < 0 || n > GCDT_MAX_POINTS) return GCDT_BAD_INPUT;
        BatchDesc& d = b->h_desc[i];
        d.pt_off = pt_off[i];
        d.seg_off = seg_off[i];
        d.ws_off = (long long)ws;
        d.tri_off = tri_off ? tri_off[i] : 2 * pt_off[i] + 2 * (long long)i;
        d.n = (int)n;
        d.s = (int)s;
        d.status = 0;
        d.pad = 0;
        ws += instance_bytes(n, s);
        b->h_offs[i] = (int)pt_off[i];
        b->h_order[i] = i;
    }
    b->h_offs[ninst] = (int)total;
    if (ws > b->ws_bytes) return GCDT_OOM;
    std::stable_sort(b->h_order, b->h_order + ninst,
                     [&](int x, int y) { return b->h_desc[x].n > b->h_desc[y].n; });
    cudaMemcpyAsync(b->d_desc, b->h_desc, sizeof(BatchDesc) * ninst, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(b->d_offs, b->h_offs, sizeof(int) * (ninst + 1), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(b->d_order, b->h_order, sizeof(int) * ninst, cudaMemcpyHostToDevice, st);

    const int2* xy = reinterpret_cast<const int2*>(d_points);
    int itotal = (int)total;
    if (itotal > 0)
        gcdt_batch_keys<<<(itotal + 255) / 256, 256, 0, st>>>(xy, b->d_offs, ninst, itotal, b->keys[0],
                                                               b->vals[0], b->d_desc);
    cub::DoubleBuffer<unsigned long long> dk(b->keys[0], b->keys[1]);
    cub::DoubleBuffer<int> dv(b->vals[0], b->vals[1]);
    if (itotal > 0) {
        size_t bytes = b->sort_bytes;
        cub::DeviceSegmentedRadixSort::SortPairs(b->sort_tmp, bytes, dk, dv, itotal, ninst, b->d_offs,
                                                 b->d_offs + 1, 0, 60, st);
    }
    BatchArgs a;
    a.xy = xy;
    a.cons = reinterpret_cast<const int2*>(d_segments);
    a.keys = dk.Current();
    a.vals = dv.Current();
    a.desc = b->d_desc;
    a.order = b->d_order;
    a.ws = b->ws;
    a.tris = d_tris;
    a.adj = d_adj;
    a.cflags = d_cflags;
    a.stride0 = cfg.sample_stride;
    switch (cfg.threads_per_instance) {
    case 128: gcdt_batch_solve<128><<<ninst, 128, 0, st>>>(a); break;
    case 512: gcdt_batch_solve<512><<<ninst, 512, 0, st>>>(a); break;
    default: gcdt_batch_solve<256><<<ninst, 256, 0, st>>>(a); break;
    }
    if (cudaGetLastError() != cudaSuccess) return GCDT_CUDA_ERROR;
    cudaMemcpyAsync(b->h_desc, b->d_desc, sizeof(BatchDesc) * ninst, cudaMemcpyDeviceToHost, st);
    return GCDT_OK;
}

gcdt_status gcdt_batch_finalize(gcdt_batch* b, int32_t ninst, int32_t* inst_status) {
    gcdt_status rc = GCDT_OK;
    for (int i = 0; i < ninst; ++i) {
        int bits = b->h_desc[i].status;
        gcdt_status si = GCDT_OK;
        if (bits & ST_BAD_INPUT) si = GCDT_BAD_INPUT;
        else if (bits & ST_CONSTRAINT_FAIL) si = GCDT_CONSTRAINT_FAIL;
        else if (bits & ST_ITER_LIMIT) si = GCDT_ITER_LIMIT;
        else if (bits & ST_OOM) si = GCDT_OOM;
        else if (bits) si = GCDT_INTERNAL;
        if (inst_status) inst_status[i] = si;
        if (rc == GCDT_OK) rc = si;
    }
    return rc;
}

extern "C" gcdt_status gcdt_batch_create(gcdt_batch** out, int device, int64_t max_instances,
                                         int64_t max_total_points, int64_t max_total_segments) {
    if (!out) return GCDT_BAD_INPUT;
    *out = nullptr;
    if (max_instances < 1 || max_instances > (1 << 24) || max_total_points < 0 ||
        max_total_points > (int64_t(1) << 30) || max_total_segments < 0 || max_total_segments > (int64_t(1) << 30))
        return GCDT_BAD_INPUT;
    gcdt_batch* b = new (std::nothrow) gcdt_batch();
    if (!b) return GCDT_OOM;
    b->device = device;
    b->max_inst = max_instances;
    b->max_pts = max_total_points;
    b->max_segs = max_total_segments;
    DevGuard g(device);
    b->ws_bytes = arena_bound(max_instances, max_total_points, max_total_segments);
    {
        cub::DoubleBuffer<unsigned long long> dk(nullptr, nullptr);
        cub::DoubleBuffer<int> dv(nullptr, nullptr);
        size_t bytes = 0;
        cub::DeviceSegmentedRadixSort::SortPairs(nullptr, bytes, dk, dv, (int)std::max<int64_t>(max_total_points, 1),
                                                 (int)max_instances, (int*)nullptr, (int*)nullptr, 0, 60);
        b->sort_bytes = bytes;
    }
    size_t np = (size_t)std::max<int64_t>(max_total_points, 1);
    bool ok = cudaMalloc(&b->ws, b->ws_bytes) == cudaSuccess &&
              cudaMalloc(&b->sort_tmp, std::max<size_t>(b->sort_bytes, 256)) == cudaSuccess &&
              cudaMalloc(&b->keys[0], 8 * np) == cudaSuccess && cudaMalloc(&b->keys[1], 8 * np) == cudaSuccess &&
              cudaMalloc(&b->vals[0], 4 * np) == cudaSuccess && cudaMalloc(&b->vals[1], 4 * np) == cudaSuccess &&
              cudaMalloc(&b->d_offs, 4 * (max_instances + 1)) == cudaSuccess &&
              cudaMalloc(&b->d_order, 4 * max_instances) == cudaSuccess &&
              cudaMalloc(&b->d_desc, sizeof(BatchDesc) * max_instances) == cudaSuccess &&
              cudaMallocHost(&b->h_desc, sizeof(BatchDesc) * max_instances) == cudaSuccess &&
              cudaMallocHost(&b->h_offs, 4 * (max_instances + 1)) == cudaSuccess &&
              cudaMallocHost(&b->h_order, 4 * max_instances) == cudaSuccess &&
              cudaEventCreate(&b->ev0) == cudaSuccess && cudaEventCreate(&b->ev1) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        gcdt_batch_destroy(b);
        return GCDT_OOM;
    }
    *out = b;
    return GCDT_OK;
}

extern "C" void gcdt_batch_destroy(gcdt_batch* b) {
    if (!b) return;
    DevGuard g(b->device);
    cudaFree(b->ws);
    cudaFree(b->sort_tmp);
    for (int k = 0; k < 2; ++k) { cudaFree(b->keys[k]); cudaFree(b->vals[k]); }
    cudaFree(b->d_offs);
    cudaFree(b->d_order);
    cudaFree(b->d_desc);
    if (b->h_desc) cudaFreeHost(b->h_desc);
    if (b->h_offs) cudaFreeHost(b->h_offs);
    if (b->h_order) cudaFreeHost(b->h_order);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    delete b;
}

extern "C" gcdt_status gcdt_batch_set_config(gcdt_batch* b, const gcdt_batch_config* cfg) {
    if (!b || !cfg || !valid_cfg(*cfg)) return GCDT_BAD_INPUT;
    b->cfg = *cfg;
    return GCDT_OK;
}

extern "C" gcdt_status gcdt_batch_get_config(const gcdt_batch* b, gcdt_batch_config* cfg) {
    if (!b || !cfg) return GCDT_BAD_INPUT;
    *cfg = b->cfg;
    return GCDT_OK;
}

extern "C" gcdt_status gcdt_batch_triangulate(gcdt_batch* b, int32_t n_instances, const int64_t* point_offsets,
                                              const int64_t* segment_offsets, const int32_t* d_points,
                                              const int32_t* d_segments, int32_t* d_tris, int32_t* d_adj,
                                              uint8_t* d_cflags, int32_t* instance_status, void* stream) {
    if (!b || !point_offsets || !segment_offsets || !d_tris || !d_adj || !d_cflags) return GCDT_BAD_INPUT;
    DevGuard g(b->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaEventRecord(b->ev0, st);
    gcdt_status rc = run_batch(b, n_instances, point_offsets, segment_offsets, d_points, d_segments, d_tris,
                               d_adj, d_cflags, instance_status, st, b->cfg);
    cudaEventRecord(b->ev1, st);
    cudaEventSynchronize(b->ev1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    b->last_ms = ms;
    return rc;
}

extern "C" double gcdt_batch_last_ms(const gcdt_batch* b) { return b ? b->last_ms : -1.0; }

// Autotuner: time every (threads per instance, first-level sample stride)
// configuration on the caller's batch -- or on a sample of `sample_instances`
// instances spread over its size distribution -- and keep the fastest.
extern "C" gcdt_status gcdt_batch_autotune(gcdt_batch* b, int32_t n_instances, const int64_t* point_offsets,
                                           const int64_t* segment_offsets, const int32_t* d_points,
                                           const int32_t* d_segments, int32_t* d_tris, int32_t* d_adj,
                                           uint8_t* d_cflags, int32_t sample_instances, gcdt_batch_config* chosen,
                                           void* stream) {
    if (!b || n_instances <= 0 || !point_offsets || !segment_offsets) return GCDT_BAD_INPUT;
    DevGuard g(b->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // optional sample: every k-th instance of the size order, gathered contiguously
    std::vector<int64_t> po(point_offsets, point_offsets + n_instances + 1);
    std::vector<int64_t> so(segment_offsets, segment_offsets + n_instances + 1);
    int32_t* tp = nullptr;
    int32_t* ts = nullptr;
    const int32_t* P = d_points;
    const int32_t* S = d_segments;
    int32_t m = n_instances;
    if (sample_instances > 0 && sample_instances < n_instances) {
        std::vector<int> ord(n_instances);
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) {
            return point_offsets[x + 1] - point_offsets[x] > point_offsets[y + 1] - point_offsets[y];
        });
        std::vector<int> pick;
        for (int k = 0; k < sample_instances; ++k) pick.push_back(ord[(size_t)k * n_instances / sample_instances]);
        std::vector<int64_t> npo(1, 0), nso(1, 0);
        for (int i : pick) {
            npo.push_back(npo.back() + (point_offsets[i + 1] - point_offsets[i]));
            nso.push_back(nso.back() + (segment_offsets[i + 1] - segment_offsets[i]));
        }
        if (cudaMalloc(&tp, 8 * std::max<int64_t>(npo.back(), 1)) != cudaSuccess ||
            cudaMalloc(&ts, 8 * std::max<int64_t>(nso.back(), 1)) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(tp);
            return GCDT_OOM;
        }
        for (size_t k = 0; k < pick.size(); ++k) {
            int i = pick[k];
            cudaMemcpyAsync(tp + 2 * npo[k], d_points + 2 * point_offsets[i],
                            8 * (point_offsets[i + 1] - point_offsets[i]), cudaMemcpyDeviceToDevice, st);
            if (segment_offsets[i + 1] > segment_offsets[i])
                cudaMemcpyAsync(ts + 2 * nso[k], d_segments + 2 * segment_offsets[i],
                                8 * (segment_offsets[i + 1] - segment_offsets[i]), cudaMemcpyDeviceToDevice, st);
        }
        po = npo;
        so = nso;
        P = tp;
        S = ts;
        m = (int32_t)pick.size();
    }
    const int threads[] = {128, 256, 512};
    const int strides[] = {16, 64, 256};
    gcdt_batch_config best = b->cfg;
    float best_ms = 1e30f;
    gcdt_status rc = GCDT_OK;
    for (int ti : threads) {
        for (int si : strides) {
            gcdt_batch_config c{ti, si};
            float ms = 0.f;
            for (int rep = 0; rep < 2 && rc == GCDT_OK; ++rep) {   // warm-up, then timed
                cudaEventRecord(b->ev0, st);
                rc = run_batch(b, m, po.data(), so.data(), P, S, d_tris, d_adj, d_cflags, nullptr, st, c);
                cudaEventRecord(b->ev1, st);
                cudaEventSynchronize(b->ev1);
                cudaEventElapsedTime(&ms, b->ev0, b->ev1);
            }
            if (rc != GCDT_OK) break;
            if (ms < best_ms) { best_ms = ms; best = c; }
        }
        if (rc != GCDT_OK) break;
    }
    cudaFree(tp);
    cudaFree(ts);
    if (rc == GCDT_OK) {
        b->cfg = best;
        if (chosen) *chosen = best;
    }
    return rc;
}
