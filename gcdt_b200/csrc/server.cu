// server.cu -- continuous-batching triangulation server.
//
// The reference has no serving path (one solve per process, kernel.cu:5332).
// This engine takes a stream of triangulation requests of very different
// sizes and keeps the GPU busy with them:
//   - admission: a request's resident output (2n+2 triangles x 25 bytes)
//     must fit the output pool left after the fixed arenas inside the
//     device-memory budget, and its solve workspace (gcdt_workspace_bytes)
//     must fit the lane it is batched on; otherwise it waits until memory is
//     released;
//   - continuous batching: a scheduler thread packs queued requests into a
//     batch as soon as one of several lanes (each a stream with its own batch
//     arena) is free, so requests that arrive while others run are launched
//     next to them and their work overlaps on the device;
//   - requests of at least big_request_points points go to a second queue
//     served by big_workers worker threads, each running one request at a
//     time through the single-solve path on its own context and
//     high-priority stream, concurrently with the lanes.  One worker uses
//     the whole GPU; k workers each launch the persistent stage kernel on
//     1/k of the SMs (gcdt_set_grid_blocks), so k requests' grids fit the
//     device together and the per-phase latencies of several mid-size
//     solves overlap.  The block scheduler favours the high-priority grids,
//     lane blocks always finish, and the stage kernel's bounded grid barrier
//     turns any wait for blocks held elsewhere into an error, not a hang;
//   - results stay resident in the output pool until the client fetches
//     (copies out) or releases them.
// Latency is measured on the host from submission to the moment the
// scheduler sees the request's work complete.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/gcdt.h"

// batch.cu
gcdt_status gcdt_batch_launch(gcdt_batch* b, int32_t ninst, const int64_t* pt_off, const int64_t* seg_off,
                              const int64_t* tri_off, const int32_t* d_points, const int32_t* d_segments,
                              int32_t* d_tris, int32_t* d_adj, uint8_t* d_cflags, cudaStream_t st,
                              const gcdt_batch_config& cfg);
gcdt_status gcdt_batch_finalize(gcdt_batch* b, int32_t ninst, int32_t* inst_status);

namespace {

constexpr int64_t kTriBytes = 12 + 12 + 1;   // tris + adj + cflags per triangle

// First-fit allocator of triangle ranges in the resident output pool.
struct RangeAlloc {
    std::map<int64_t, int64_t> free_;   // offset -> length
    void init(int64_t cap) { free_.clear(); if (cap > 0) free_[0] = cap; }
    int64_t alloc(int64_t len) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= len) {
                int64_t off = it->first, rest = it->second - len;
                free_.erase(it);
                if (rest > 0) free_[off + len] = rest;
                return off;
            }
        }
        return -1;
    }
    void release(int64_t off, int64_t len) {
        auto it = free_.emplace(off, len).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

enum ReqState { QUEUED = 0, RUNNING = 1, DONE = 2 };

struct Request {
    int64_t id = 0;
    int32_t n = 0, s = 0;
    std::vector<int32_t> xy, cons;
    int64_t tri_off = -1;
    int state = QUEUED;
    gcdt_status status = GCDT_OK;
    double t_submit = 0, t_start = 0, t_done = 0;
};

struct Lane {
    gcdt_batch* batch = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    int32_t* h_pts = nullptr;    // pinned staging
    int32_t* h_segs = nullptr;
    int32_t* d_pts = nullptr;
    int32_t* d_segs = nullptr;
    std::vector<int64_t> ids, po, so, to;
    std::vector<int32_t> st;
    bool busy = false;
};

double now_ms(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

// A worker for large requests: its own solve context, input buffers and
// high-priority stream.
struct BigWorker {
    gcdt_context* ctx = nullptr;
    cudaStream_t stream = nullptr;
    int32_t* pts = nullptr;
    int32_t* segs = nullptr;
    std::thread th;
};

struct gcdt_server {
    int device = 0;
    gcdt_server_config cfg{};
    std::vector<Lane> lanes;
    std::vector<BigWorker> bigs;
    cudaStream_t fetch_stream = nullptr;
    int32_t* pool_tris = nullptr;
    int32_t* pool_adj = nullptr;
    uint8_t* pool_cf = nullptr;
    int64_t pool_tris_cap = 0, pool_used = 0, pool_peak = 0;
    RangeAlloc alloc;
    std::mutex mu;
    std::condition_variable cv, done_cv;
    std::deque<int64_t> queue;       // small requests, for the lanes
    std::deque<int64_t> big_queue;   // large requests, for the big worker
    std::unordered_map<int64_t, Request> reqs;
    int64_t next_id = 1;
    std::thread th;
    std::condition_variable big_cv;
    bool stop = false;
    gcdt_status fatal = GCDT_OK;
    std::chrono::steady_clock::time_point t0;
    int64_t submitted = 0, completed = 0, failed = 0, batches = 0, big_solves = 0;
    std::vector<double> lat;
    double first_submit = -1, last_done = 0;
    size_t fixed_bytes = 0;

    void run();
    void run_big_worker(BigWorker& W);
    bool dispatch_batch(std::unique_lock<std::mutex>& lk, Lane& L);
    bool run_big(std::unique_lock<std::mutex>& lk, BigWorker& W, int64_t id);
    void complete(Request& r, gcdt_status st) {
        r.state = DONE;
        r.status = st;
        r.t_done = now_ms(t0);
        if (st == GCDT_OK) completed++; else failed++;
        lat.push_back(r.t_done - r.t_submit);
        last_done = r.t_done;
    }
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
}  // namespace

// Pack queued small requests (FIFO) into a batch on
// lane L.  Called with the lock held; the lock is dropped while the inputs
// are staged and the batch is launched.
bool gcdt_server::dispatch_batch(std::unique_lock<std::mutex>& lk, Lane& L) {
    L.ids.clear();
    L.po.assign(1, 0);
    L.so.assign(1, 0);
    L.to.clear();
    size_t ws = 0;
    const size_t ws_cap = (size_t)cfg.lane_workspace_bytes;
    while (!queue.empty() && (int)L.ids.size() < cfg.max_batch_instances) {
        Request& r = reqs[queue.front()];
        size_t need = gcdt_workspace_bytes(r.n, r.s);
        if (L.po.back() + r.n > cfg.max_batch_points || L.so.back() + r.s > cfg.max_batch_segments ||
            ws + need > ws_cap)
            break;
        int64_t ntri = 2 * (int64_t)r.n + 2;
        int64_t off = alloc.alloc(ntri);
        if (off < 0) break;                 // output pool full: wait for releases
        pool_used += ntri;
        pool_peak = std::max(pool_peak, pool_used);
        ws += need;
        r.tri_off = off;
        r.state = RUNNING;
        r.t_start = now_ms(t0);
        L.ids.push_back(r.id);
        L.po.push_back(L.po.back() + r.n);
        L.so.push_back(L.so.back() + r.s);
        L.to.push_back(off);
        queue.pop_front();
    }
    if (L.ids.empty()) return false;
    L.busy = true;
    batches++;
    std::vector<const Request*> rs;
    for (int64_t id : L.ids) rs.push_back(&reqs[id]);
    lk.unlock();
    for (size_t k = 0; k < rs.size(); ++k) {
        if (rs[k]->n) std::memcpy(L.h_pts + 2 * L.po[k], rs[k]->xy.data(), 8 * (size_t)rs[k]->n);
        if (rs[k]->s) std::memcpy(L.h_segs + 2 * L.so[k], rs[k]->cons.data(), 8 * (size_t)rs[k]->s);
    }
    int32_t ni = (int32_t)L.ids.size();
    if (L.po.back()) cudaMemcpyAsync(L.d_pts, L.h_pts, 8 * L.po.back(), cudaMemcpyHostToDevice, L.stream);
    if (L.so.back()) cudaMemcpyAsync(L.d_segs, L.h_segs, 8 * L.so.back(), cudaMemcpyHostToDevice, L.stream);
    gcdt_batch_config bc;
    gcdt_batch_get_config(L.batch, &bc);
    gcdt_status rc = gcdt_batch_launch(L.batch, ni, L.po.data(), L.so.data(), L.to.data(), L.d_pts, L.d_segs,
                                       pool_tris, pool_adj, pool_cf, L.stream, bc);
    cudaEventRecord(L.done, L.stream);
    lk.lock();
    if (rc != GCDT_OK) {
        cudaStreamSynchronize(L.stream);
        for (int64_t id : L.ids) complete(reqs[id], rc);
        L.busy = false;
        done_cv.notify_all();
    }
    return true;
}

// A large request on worker W.  Returns false when the output pool has no
// room yet.
bool gcdt_server::run_big(std::unique_lock<std::mutex>& lk, BigWorker& W, int64_t id) {
    Request& r = reqs[id];
    int64_t ntri = 2 * (int64_t)r.n + 2;
    int64_t off = alloc.alloc(ntri);
    if (off < 0) return false;              // wait for memory
    big_queue.pop_front();
    pool_used += ntri;
    pool_peak = std::max(pool_peak, pool_used);
    r.tri_off = off;
    r.state = RUNNING;
    r.t_start = now_ms(t0);
    big_solves++;
    const int32_t* xy = r.xy.data();
    const int32_t* cons = r.cons.data();
    int32_t n = r.n, s = r.s;
    lk.unlock();
    cudaMemcpyAsync(W.pts, xy, 8 * (size_t)n, cudaMemcpyHostToDevice, W.stream);
    if (s) cudaMemcpyAsync(W.segs, cons, 8 * (size_t)s, cudaMemcpyHostToDevice, W.stream);
    int32_t nt = 0;
    gcdt_status rc = gcdt_triangulate(W.ctx, W.pts, n, s ? W.segs : nullptr, s, pool_tris + 3 * off,
                                      pool_adj + 3 * off, pool_cf + off, &nt, W.stream);
    lk.lock();
    complete(reqs[id], rc);
    done_cv.notify_all();
    return true;
}

void gcdt_server::run_big_worker(BigWorker& W) {
    DevGuard g(device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        if (stop && big_queue.empty()) break;
        if (big_queue.empty() || !run_big(lk, W, big_queue.front()))
            big_cv.wait_for(lk, std::chrono::microseconds(100));
    }
}

void gcdt_server::run() {
    DevGuard g(device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        bool any_busy = false;
        for (Lane& L : lanes) {
            if (!L.busy) continue;
            cudaError_t q = cudaEventQuery(L.done);
            if (q == cudaErrorNotReady) { any_busy = true; continue; }
            L.st.assign(L.ids.size(), 0);
            gcdt_status rc = q == cudaSuccess ? GCDT_OK : GCDT_CUDA_ERROR;
            if (q == cudaSuccess) gcdt_batch_finalize(L.batch, (int32_t)L.ids.size(), L.st.data());
            for (size_t k = 0; k < L.ids.size(); ++k)
                complete(reqs[L.ids[k]], rc != GCDT_OK ? rc : (gcdt_status)L.st[k]);
            L.busy = false;
            done_cv.notify_all();
        }
        if (stop && queue.empty() && !any_busy) break;
        bool dispatched = false;
        for (Lane& L : lanes) {
            if (L.busy || queue.empty()) continue;
            if (dispatch_batch(lk, L)) dispatched = true;
            else break;
        }
        if (!dispatched) cv.wait_for(lk, std::chrono::microseconds(50));
    }
}

extern "C" gcdt_status gcdt_server_create(gcdt_server** out, int device, const gcdt_server_config* cfg) {
    if (!out || !cfg) return GCDT_BAD_INPUT;
    *out = nullptr;
    const gcdt_server_config& c = *cfg;
    if (c.lanes < 1 || c.lanes > 16 || c.max_batch_instances < 1 || c.max_batch_points < 1 ||
        c.max_batch_segments < 0 || c.max_request_points < 1 || c.max_request_points > GCDT_MAX_POINTS ||
        c.max_request_segments < 0 || c.memory_budget_bytes <= 0 || c.big_workers < 0 || c.big_workers > 16)
        return GCDT_BAD_INPUT;
    gcdt_server* sv = new (std::nothrow) gcdt_server();
    if (!sv) return GCDT_OOM;
    sv->device = device;
    sv->cfg = c;
    if (sv->cfg.lane_workspace_bytes <= 0)
        sv->cfg.lane_workspace_bytes = (int64_t)gcdt_workspace_bytes(c.max_batch_points, c.max_batch_segments);
    DevGuard g(device);
    bool ok = true;
    size_t fixed = 0;
    int lo_prio = 0, hi_prio = 0;
    sv->lanes.resize(c.lanes);
    for (Lane& L : sv->lanes) {
        ok = ok && gcdt_batch_create(&L.batch, device, c.max_batch_instances, c.max_batch_points,
                                     c.max_batch_segments) == GCDT_OK;
        ok = ok && cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming) == cudaSuccess &&
             cudaMallocHost(&L.h_pts, 8 * (size_t)c.max_batch_points) == cudaSuccess &&
             cudaMallocHost(&L.h_segs, 8 * (size_t)std::max<int64_t>(c.max_batch_segments, 1)) == cudaSuccess &&
             cudaMalloc(&L.d_pts, 8 * (size_t)c.max_batch_points) == cudaSuccess &&
             cudaMalloc(&L.d_segs, 8 * (size_t)std::max<int64_t>(c.max_batch_segments, 1)) == cudaSuccess;
        fixed += (size_t)sv->cfg.lane_workspace_bytes + 8 * (size_t)(c.max_batch_points + c.max_batch_segments);
    }
    const int nbig = c.big_workers > 1 ? c.big_workers : 1;
    int sms = 0;
    ok = ok && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess &&
         cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio) == cudaSuccess &&
         cudaStreamCreateWithFlags(&sv->fetch_stream, cudaStreamNonBlocking) == cudaSuccess;
    sv->bigs = std::vector<BigWorker>(nbig);
    for (BigWorker& W : sv->bigs) {
        ok = ok && gcdt_create(&W.ctx, device, c.max_request_points, c.max_request_segments) == GCDT_OK &&
             (nbig == 1 || gcdt_set_grid_blocks(W.ctx, std::max(1, sms / nbig)) == GCDT_OK) &&
             cudaStreamCreateWithPriority(&W.stream, cudaStreamNonBlocking, hi_prio) == cudaSuccess &&
             cudaMalloc(&W.pts, 8 * (size_t)c.max_request_points) == cudaSuccess &&
             cudaMalloc(&W.segs, 8 * (size_t)std::max<int64_t>(c.max_request_segments, 1)) == cudaSuccess;
        fixed += gcdt_workspace_bytes(c.max_request_points, c.max_request_segments) +
                 8 * (size_t)(c.max_request_points + c.max_request_segments);
    }
    sv->fixed_bytes = fixed;
    int64_t pool_bytes = c.memory_budget_bytes - (int64_t)fixed;
    int64_t cap = pool_bytes / kTriBytes;
    if (ok && cap < 2 * c.max_request_points + 2) ok = false;     // budget too small for the largest request
    if (ok) {
        sv->pool_tris_cap = cap;
        ok = cudaMalloc(&sv->pool_tris, 12 * (size_t)cap) == cudaSuccess &&
             cudaMalloc(&sv->pool_adj, 12 * (size_t)cap) == cudaSuccess &&
             cudaMalloc(&sv->pool_cf, (size_t)cap) == cudaSuccess;
        sv->alloc.init(cap);
    }
    if (!ok) {
        cudaGetLastError();
        gcdt_server_destroy(sv);
        return GCDT_OOM;
    }
    sv->t0 = std::chrono::steady_clock::now();
    sv->th = std::thread([sv] { sv->run(); });
    for (BigWorker& W : sv->bigs) W.th = std::thread([sv, &W] { sv->run_big_worker(W); });
    *out = sv;
    return GCDT_OK;
}

extern "C" void gcdt_server_destroy(gcdt_server* sv) {
    if (!sv) return;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
        sv->queue.clear();
        sv->big_queue.clear();
    }
    sv->cv.notify_all();
    sv->big_cv.notify_all();
    if (sv->th.joinable()) sv->th.join();
    for (BigWorker& W : sv->bigs)
        if (W.th.joinable()) W.th.join();
    DevGuard g(sv->device);
    for (Lane& L : sv->lanes) {
        if (L.stream) cudaStreamSynchronize(L.stream);
        gcdt_batch_destroy(L.batch);
        if (L.stream) cudaStreamDestroy(L.stream);
        if (L.done) cudaEventDestroy(L.done);
        if (L.h_pts) cudaFreeHost(L.h_pts);
        if (L.h_segs) cudaFreeHost(L.h_segs);
        cudaFree(L.d_pts);
        cudaFree(L.d_segs);
    }
    for (BigWorker& W : sv->bigs) {
        gcdt_destroy(W.ctx);
        if (W.stream) cudaStreamDestroy(W.stream);
        cudaFree(W.pts);
        cudaFree(W.segs);
    }
    if (sv->fetch_stream) cudaStreamDestroy(sv->fetch_stream);
    cudaFree(sv->pool_tris);
    cudaFree(sv->pool_adj);
    cudaFree(sv->pool_cf);
    delete sv;
}

extern "C" gcdt_status gcdt_server_submit(gcdt_server* sv, const int32_t* points, int32_t n,
                                          const int32_t* segments, int32_t s, int64_t* request_id) {
    if (!sv || !request_id || n < 0 || s < 0 || (n > 0 && !points) || (s > 0 && !segments)) return GCDT_BAD_INPUT;
    if (n > sv->cfg.max_request_points || s > sv->cfg.max_request_segments) return GCDT_OOM;
    if (n < sv->cfg.big_request_points && (n > sv->cfg.max_batch_points || s > sv->cfg.max_batch_segments ||
                                           (int64_t)gcdt_workspace_bytes(n, s) > sv->cfg.lane_workspace_bytes))
        return GCDT_OOM;
    Request r;
    r.n = n;
    r.s = s;
    r.xy.assign(points, points + 2 * (size_t)n);
    if (s) r.cons.assign(segments, segments + 2 * (size_t)s);
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        r.id = sv->next_id++;
        r.t_submit = now_ms(sv->t0);
        if (sv->first_submit < 0) sv->first_submit = r.t_submit;
        *request_id = r.id;
        if (r.n >= sv->cfg.big_request_points) sv->big_queue.push_back(r.id);
        else sv->queue.push_back(r.id);
        sv->reqs.emplace(r.id, std::move(r));
        sv->submitted++;
    }
    sv->cv.notify_all();
    sv->big_cv.notify_all();
    return GCDT_OK;
}

extern "C" gcdt_status gcdt_server_wait(gcdt_server* sv, int64_t id, int32_t timeout_ms, int32_t* done) {
    if (!sv) return GCDT_BAD_INPUT;
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(id);
    if (it == sv->reqs.end()) return GCDT_BAD_INPUT;
    auto pred = [&] { return sv->reqs[id].state == DONE; };
    if (timeout_ms < 0) sv->done_cv.wait(lk, pred);
    else sv->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred);
    Request& r = sv->reqs[id];
    if (done) *done = r.state == DONE;
    return r.state == DONE ? r.status : GCDT_OK;
}

static gcdt_status release_locked(gcdt_server* sv, int64_t id) {
    auto it = sv->reqs.find(id);
    if (it == sv->reqs.end() || it->second.state != DONE) return GCDT_BAD_INPUT;
    if (it->second.tri_off >= 0) {
        int64_t ntri = 2 * (int64_t)it->second.n + 2;
        sv->alloc.release(it->second.tri_off, ntri);
        sv->pool_used -= ntri;
    }
    sv->reqs.erase(it);
    sv->cv.notify_all();
    sv->big_cv.notify_all();
    return GCDT_OK;
}

extern "C" gcdt_status gcdt_server_fetch(gcdt_server* sv, int64_t id, int32_t* h_tris, int32_t* h_adj,
                                         uint8_t* h_cflags, int32_t* n_tris) {
    if (!sv) return GCDT_BAD_INPUT;
    int64_t off, ntri;
    gcdt_status st;
    {
        std::unique_lock<std::mutex> lk(sv->mu);
        auto it = sv->reqs.find(id);
        if (it == sv->reqs.end()) return GCDT_BAD_INPUT;
        sv->done_cv.wait(lk, [&] { return sv->reqs[id].state == DONE; });
        Request& r = sv->reqs[id];
        off = r.tri_off;
        ntri = 2 * (int64_t)r.n + 2;
        st = r.status;
    }
    if (st == GCDT_OK && off >= 0) {
        DevGuard g(sv->device);
        if (h_tris) cudaMemcpyAsync(h_tris, sv->pool_tris + 3 * off, 12 * ntri, cudaMemcpyDeviceToHost, sv->fetch_stream);
        if (h_adj) cudaMemcpyAsync(h_adj, sv->pool_adj + 3 * off, 12 * ntri, cudaMemcpyDeviceToHost, sv->fetch_stream);
        if (h_cflags) cudaMemcpyAsync(h_cflags, sv->pool_cf + off, ntri, cudaMemcpyDeviceToHost, sv->fetch_stream);
        if (cudaStreamSynchronize(sv->fetch_stream) != cudaSuccess) st = GCDT_CUDA_ERROR;
        if (n_tris) *n_tris = (int32_t)ntri;
    }
    std::lock_guard<std::mutex> lk(sv->mu);
    release_locked(sv, id);
    return st;
}

extern "C" gcdt_status gcdt_server_release(gcdt_server* sv, int64_t id) {
    if (!sv) return GCDT_BAD_INPUT;
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(id);
    if (it == sv->reqs.end()) return GCDT_BAD_INPUT;
    sv->done_cv.wait(lk, [&] { return sv->reqs[id].state == DONE; });
    return release_locked(sv, id);
}

extern "C" gcdt_status gcdt_server_request_times(gcdt_server* sv, int64_t id, double* submit_ms, double* start_ms,
                                                 double* done_ms) {
    if (!sv) return GCDT_BAD_INPUT;
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(id);
    if (it == sv->reqs.end()) return GCDT_BAD_INPUT;
    if (submit_ms) *submit_ms = it->second.t_submit;
    if (start_ms) *start_ms = it->second.t_start;
    if (done_ms) *done_ms = it->second.t_done;
    return GCDT_OK;
}

extern "C" gcdt_status gcdt_server_get_stats(gcdt_server* sv, gcdt_server_stats* out) {
    if (!sv || !out) return GCDT_BAD_INPUT;
    std::lock_guard<std::mutex> lk(sv->mu);
    gcdt_server_stats& s = *out;
    std::memset(&s, 0, sizeof s);
    s.submitted = sv->submitted;
    s.completed = sv->completed;
    s.failed = sv->failed;
    s.batches = sv->batches;
    s.big_solves = sv->big_solves;
    s.queued = (int64_t)(sv->queue.size() + sv->big_queue.size());
    s.resident_bytes = sv->pool_used * kTriBytes;
    s.peak_resident_bytes = sv->pool_peak * kTriBytes;
    s.fixed_bytes = (int64_t)sv->fixed_bytes;
    std::vector<double> l = sv->lat;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        s.p50_ms = l[(l.size() - 1) / 2];
        s.p99_ms = l[std::min(l.size() - 1, (size_t)((l.size() - 1) * 0.99 + 0.5))];
        s.max_ms = l.back();
        double span = sv->last_done - sv->first_submit;
        s.requests_per_s = span > 0 ? 1e3 * (double)l.size() / span : 0.0;
    }
    return GCDT_OK;
}

extern "C" gcdt_status gcdt_server_reset_stats(gcdt_server* sv) {
    if (!sv) return GCDT_BAD_INPUT;
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->lat.clear();
    sv->completed = sv->failed = sv->batches = sv->big_solves = sv->submitted = 0;
    sv->first_submit = -1;
    sv->last_done = 0;
    sv->pool_peak = sv->pool_used;
    return GCDT_OK;
}
