// gcdt.cu -- CUDA kernels, the device launch backend and the C ABI.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cstdio>
#include <cstring>
#include <cstddef>
#include <new>

#include "solver.cuh"
#include "exec.cuh"
#include "../../include/gcdt.h"

namespace gcdt {

constexpr int kBlock = 256;

#define GCDT_KERNEL(name, body)                                            \
    __global__ void __launch_bounds__(kBlock) name(Ctx c, int n) {         \
        int i = blockIdx.x * kBlock + threadIdx.x;                         \
        if (i < n) body(c, i);                                             \
    }

GCDT_KERNEL(gcdt_keys, body_keys)
GCDT_KERNEL(gcdt_gather, body_gather)
GCDT_KERNEL(gcdt_root, body_root)
GCDT_KERNEL(gcdt_level, body_level)
GCDT_KERNEL(gcdt_seg_level0, body_seg_level0)
GCDT_KERNEL(gcdt_seg_init, body_seg_init)

__global__ void gcdt_predicates(const int2* q, int n, int* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int2 a = q[4 * i], b = q[4 * i + 1], cc = q[4 * i + 2], d = q[4 * i + 3];
    out[3 * i] = orient2d(a, b, cc);
    out[3 * i + 1] = incircle(a, b, cc, d);
    out[3 * i + 2] = incircle_sos(a, b, cc, d);
}

static_assert(offsetof(Counters, cur_scr) + 8 <= GridExec::kSnapWords * 8, "cursors are in the snapshot");

// kProf: the per-phase profile and balance are recorded (gcdt_set_profiling);
// the instance without them carries none of their code.
template <bool kProf>
__global__ void __launch_bounds__(kPersistBlock, kPersistMinBlocks) gcdt_stages(const __grid_constant__ Ctx c) {
    __shared__ unsigned long long snap[GridExec::kSnapWords];
    __shared__ int work;
    GridExec ex{c.cnt, gridDim.x, snap};
    ex.work = &work;
    ex.param = &c;
    ex.prof = kProf;
    if (threadIdx.x == 0) ex.take_snapshot();
    __syncthreads();
    run_stages(ex, c);
}

// Failure-detection probe of the grid barrier: every block but `absent`
// enters one barrier of the solver's executor, polling at most spin_limit
// times.  With a block absent the others' waits run out and record
// ST_BARRIER; the kernel still ends and the context stays usable.
__global__ void gcdt_barrier_probe(Counters* cnt, unsigned absent, unsigned spin_limit) {
    __shared__ unsigned long long snap[GridExec::kSnapWords];
    GridExec ex{cnt, gridDim.x, snap, spin_limit};
    if (blockIdx.x == absent) return;
    ex.barrier();
}

// Cost of the persistent kernel's grid barrier: every block of a grid
// shaped like the stage kernel's passes `rounds` barriers with no work
// between them.
__global__ void __launch_bounds__(kPersistBlock, kPersistMinBlocks) gcdt_barrier_loop(Counters* cnt, int rounds) {
    __shared__ unsigned long long snap[GridExec::kSnapWords];
    GridExec ex{cnt, gridDim.x, snap, 1u << 22};
    for (int r = 0; r < rounds; ++r) ex.barrier();
}

constexpr int ST_CUDA = 32;

struct DeviceBackend {
    cudaStream_t st = nullptr;
    Counters* dcnt = nullptr;
    Counters* hcnt = nullptr;
    void* sort_tmp = nullptr;
    size_t sort_bytes = 0;
    cudaError_t err = cudaSuccess;
    long long launches = 0;

    void note(cudaError_t e) { if (e != cudaSuccess && err == cudaSuccess) err = e; }

    void launch(int k, const Ctx& c, long long n) {
        if (n <= 0 || err != cudaSuccess) return;
        unsigned grid = (unsigned)((n + kBlock - 1) / kBlock);
        int nn = (int)n;
        switch (k) {
        case K_KEYS: gcdt_keys<<<grid, kBlock, 0, st>>>(c, nn); break;
        case K_GATHER: gcdt_gather<<<grid, kBlock, 0, st>>>(c, nn); break;
        case K_ROOT: gcdt_root<<<grid, kBlock, 0, st>>>(c, nn); break;
        case K_LEVEL: gcdt_level<<<grid, kBlock, 0, st>>>(c, nn); break;
        case K_SEG_LEVEL0: gcdt_seg_level0<<<grid, kBlock, 0, st>>>(c, nn); break;
        case K_SEG_INIT: gcdt_seg_init<<<grid, kBlock, 0, st>>>(c, nn); break;
        default: note(cudaErrorInvalidValue); return;
        }
        launches++;
        note(cudaGetLastError());
    }
    void fill(void* p, int v, size_t bytes) { note(cudaMemsetAsync(p, v, bytes, st)); }
    // All rounds run in one cooperative launch sized to the co-resident
    // block count, so every block is resident and the grid barrier is safe.
    int grid_limit = 0;   // at most this many blocks (0: no limit)
    bool profile = false; // launch the stage kernel that records the phase profile
    cudaEvent_t ev_stage0 = nullptr, ev_stage1 = nullptr;   // recorded around the stage launch when set
    void stages(const Ctx& c) {
        if (err != cudaSuccess) return;
        int dev = 0, sms = 0, per_sm = 0;
        note(cudaGetDevice(&dev));
        note(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const void* kern = profile ? (const void*)gcdt_stages<true> : (const void*)gcdt_stages<false>;
        note(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPersistBlock, 0));
        if (err != cudaSuccess || sms <= 0 || per_sm <= 0) { note(cudaErrorLaunchOutOfResources); return; }
        int blocks = sms * per_sm;
        if (grid_limit > 0 && grid_limit < blocks) blocks = grid_limit;
        Ctx cc = c;
        void* args[] = {&cc};
        if (ev_stage0) note(cudaEventRecord(ev_stage0, st));
        note(cudaLaunchCooperativeKernel(kern, dim3(blocks), dim3(kPersistBlock),
                                         args, 0, st));
        if (ev_stage1) note(cudaEventRecord(ev_stage1, st));
        launches++;
    }
    void read(Counters* h) {
        note(cudaMemcpyAsync(hcnt, dcnt, sizeof(Counters), cudaMemcpyDeviceToHost, st));
        note(cudaStreamSynchronize(st));
        *h = *hcnt;
        if (err != cudaSuccess) h->status |= ST_CUDA;
    }
    void sort(Ctx& c, int n) {
        cub::DoubleBuffer<unsigned long long> dk(c.keys, c.keys_alt);
        cub::DoubleBuffer<int> dv(c.vals, c.vals_alt);
        size_t bytes = sort_bytes;
        note(cub::DeviceRadixSort::SortPairs(sort_tmp, bytes, dk, dv, n, 0, 60, st));
        c.keys = dk.Current(); c.keys_alt = dk.Alternate();
        c.vals = dv.Current(); c.vals_alt = dv.Alternate();
    }
};

inline size_t sort_temp_bytes(int64_t n) {
    if (n <= 0) return 0;
    cub::DoubleBuffer<unsigned long long> dk(nullptr, nullptr);
    cub::DoubleBuffer<int> dv(nullptr, nullptr);
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, dk, dv, (int)n, 0, 60);
    return bytes;
}

inline gcdt_status map_status(int bits) {
    if (bits == 0) return GCDT_OK;
    if (bits & ST_CUDA) return GCDT_CUDA_ERROR;
    if (bits & ST_BAD_INPUT) return GCDT_BAD_INPUT;
    if (bits & ST_CONSTRAINT_FAIL) return GCDT_CONSTRAINT_FAIL;
    if (bits & ST_ITER_LIMIT) return GCDT_ITER_LIMIT;
    if (bits & ST_OOM) return GCDT_OOM;
    return GCDT_INTERNAL;   // ST_INTERNAL, ST_BARRIER
}

}  // namespace gcdt

using namespace gcdt;

namespace {
gcdt_tuning default_tuning() {
    gcdt_tuning t{};
    t.levels = 3;
    t.level_stride[0] = 512;
    t.level_stride[1] = 8;
    t.level_stride[2] = 1;
    t.carry_queue = (int32_t)kCarryQueue;
    t.narrow_queue = (int32_t)kNarrowQueue;
    t.narrow_active = (int32_t)kNarrowActive;
    return t;
}
}  // namespace

struct gcdt_context {
    int device = 0;
    int64_t max_n = 0, max_s = 0;
    size_t arena_bytes = 0;
    char* arena = nullptr;
    Counters* hcnt = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t evs0 = nullptr, evs1 = nullptr;   // around the stage kernel
    gcdt_stats stats{};
    // the solve enqueued by gcdt_triangulate_async, until gcdt_wait
    bool pending = false;
    int32_t pend_n = 0, pend_s = 0;
    long long pend_launches = 0;
    cudaError_t pend_err = cudaSuccess;
    // budgets of the bounded loops (gcdt_set_limits; 0 = built-in bound)
    int32_t lim_rounds = 0, lim_subrounds = 0, lim_crounds = 0;
    // scheduling (gcdt_set_tuning)
    gcdt_tuning tuning = default_tuning();
    // blocks of the persistent launch (0: all co-resident blocks)
    int32_t grid_blocks = 0;
    // per-phase profiling of the stage kernel (gcdt_set_profiling)
    int32_t profile = 0;
};

namespace {
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};
}  // namespace

extern "C" size_t gcdt_workspace_bytes(int64_t n, int64_t s) {
    if (n < 0 || s < 0 || n > GCDT_MAX_POINTS) return 0;
    return make_plan(n, s, sort_temp_bytes(n)).L.total;
}

extern "C" gcdt_status gcdt_create(gcdt_context** out, int device, int64_t max_points, int64_t max_segments) {
    if (!out) return GCDT_BAD_INPUT;
    *out = nullptr;
    if (max_points < 0 || max_points > GCDT_MAX_POINTS || max_segments < 0 || max_segments > (int64_t(1) << 30))
        return GCDT_BAD_INPUT;
    gcdt_context* ctx = new (std::nothrow) gcdt_context();
    if (!ctx) return GCDT_OOM;
    ctx->device = device;
    ctx->max_n = max_points;
    ctx->max_s = max_segments;
    DeviceGuard g(device);
    ctx->arena_bytes = gcdt_workspace_bytes(max_points, max_segments);
    if (cudaMalloc(&ctx->arena, ctx->arena_bytes) != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return GCDT_OOM;
    }
    if (cudaMallocHost(&ctx->hcnt, sizeof(Counters)) != cudaSuccess ||
        cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess ||
        cudaEventCreate(&ctx->evs0) != cudaSuccess || cudaEventCreate(&ctx->evs1) != cudaSuccess) {
        cudaGetLastError();
        gcdt_destroy(ctx);
        return GCDT_CUDA_ERROR;
    }
    *out = ctx;
    return GCDT_OK;
}

extern "C" void gcdt_destroy(gcdt_context* ctx) {
    if (!ctx) return;
    DeviceGuard g(ctx->device);
    if (ctx->pending) cudaEventSynchronize(ctx->ev1);   // a solve still writes the arena
    if (ctx->arena) cudaFree(ctx->arena);
    if (ctx->hcnt) cudaFreeHost(ctx->hcnt);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->evs0) cudaEventDestroy(ctx->evs0);
    if (ctx->evs1) cudaEventDestroy(ctx->evs1);
    delete ctx;
}

namespace {
// Enqueue a solve of (points, segments) on ctx.
gcdt_status enqueue(gcdt_context* ctx, const int32_t* d_points, int32_t n, const int32_t* d_segments, int32_t s,
                    int32_t* d_tris, int32_t* d_adj, uint8_t* d_cflags, void* stream) {
    DeviceGuard g(ctx->device);
    Plan plan = make_plan(n, s, sort_temp_bytes(n));
    if (plan.L.total > ctx->arena_bytes) return GCDT_OOM;
    Ctx c = bind_ctx(ctx->arena, plan);
    c.in_xy = reinterpret_cast<const int2*>(d_points);
    c.in_cons = reinterpret_cast<const int2*>(d_segments);
    c.out_tris = d_tris;
    c.out_adj = d_adj;
    c.out_cflags = d_cflags;
    c.lim_rounds = ctx->lim_rounds;
    c.lim_subrounds = ctx->lim_subrounds;
    c.lim_crounds = ctx->lim_crounds;
    {
        const gcdt_tuning& t = ctx->tuning;
        c.nlevels = t.levels;
        for (int k = 0; k < 4; ++k) c.stride[k] = k < 3 && k + 1 < t.levels ? t.level_stride[k] : 1;
        c.carry_q = t.carry_queue;
        c.narrow_q = t.narrow_queue;
        c.narrow_act = t.narrow_active;
    }
    DeviceBackend bk;
    bk.st = static_cast<cudaStream_t>(stream);
    bk.dcnt = c.cnt;
    bk.hcnt = ctx->hcnt;
    bk.sort_tmp = ctx->arena + plan.o_sort_tmp;
    bk.sort_bytes = plan.sort_temp_bytes;
    bk.grid_limit = ctx->grid_blocks;
    bk.profile = ctx->profile != 0;
    bk.ev_stage0 = ctx->evs0;
    bk.ev_stage1 = ctx->evs1;
    bk.note(cudaEventRecord(ctx->evs0, bk.st));   // both stage events exist even if the launch is skipped
    bk.note(cudaEventRecord(ctx->evs1, bk.st));
    bk.note(cudaEventRecord(ctx->ev0, bk.st));
    enqueue_solve(bk, c);
    bk.note(cudaMemcpyAsync(ctx->hcnt, c.cnt, sizeof(Counters), cudaMemcpyDeviceToHost, bk.st));
    bk.note(cudaEventRecord(ctx->ev1, bk.st));
    ctx->pending = true;
    ctx->pend_n = n;
    ctx->pend_s = s;
    ctx->pend_launches = bk.launches;
    ctx->pend_err = bk.err;
    return bk.err == cudaSuccess ? GCDT_OK : GCDT_CUDA_ERROR;
}
}  // namespace

extern "C" gcdt_status gcdt_triangulate_async(gcdt_context* ctx, const int32_t* d_points, int32_t n,
                                              const int32_t* d_segments, int32_t s,
                                              int32_t* d_tris, int32_t* d_adj, uint8_t* d_cflags,
                                              void* stream) {
    if (!ctx || n < 0 || s < 0 || (n > 0 && !d_points) || (s > 0 && !d_segments) ||
        !d_tris || !d_adj || !d_cflags)
        return GCDT_BAD_INPUT;
    if (n > ctx->max_n || s > ctx->max_s) return GCDT_OOM;
    if (ctx->pending) gcdt_wait(ctx, nullptr);   // one solve in flight per context
    return enqueue(ctx, d_points, n, d_segments, s, d_tris, d_adj, d_cflags, stream);
}

extern "C" gcdt_status gcdt_wait(gcdt_context* ctx, int32_t* n_tris) {
    if (!ctx) return GCDT_BAD_INPUT;
    if (!ctx->pending) return GCDT_OK;
    DeviceGuard g(ctx->device);
    ctx->pending = false;
    cudaError_t e = cudaEventSynchronize(ctx->ev1);
    SolveStats st;
    int bits = solve_result(*ctx->hcnt, st);
    if (e != cudaSuccess || ctx->pend_err != cudaSuccess) {
        cudaGetLastError();
        bits |= ST_CUDA;
    }
    float ms = 0.f, sms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    cudaEventElapsedTime(&sms, ctx->evs0, ctx->evs1);
    const int32_t n = ctx->pend_n;
    gcdt_stats& S = ctx->stats;
    S.n_points = n;
    S.n_segments = ctx->pend_s;
    S.n_triangles = 2 * (int64_t)n + 2;
    S.insertion_rounds = st.rounds;
    S.flip_subrounds = st.flip_subrounds;
    S.flips = st.flips;
    S.constraint_rounds = st.constraint_rounds;
    S.host_syncs = 1;
    S.kernel_launches = ctx->pend_launches;
    S.device_ms = ms;
    S.stage_ms = sms;
    gcdt_status rc = map_status(bits);
    if (rc == GCDT_OK && n_tris) *n_tris = 2 * n + 2;
    return rc;
}

extern "C" gcdt_status gcdt_set_grid_blocks(gcdt_context* ctx, int32_t blocks) {
    if (!ctx || blocks < 0) return GCDT_BAD_INPUT;
    if (ctx->pending) gcdt_wait(ctx, nullptr);
    ctx->grid_blocks = blocks;
    return GCDT_OK;
}

extern "C" gcdt_status gcdt_triangulate(gcdt_context* ctx, const int32_t* d_points, int32_t n,
                                        const int32_t* d_segments, int32_t s,
                                        int32_t* d_tris, int32_t* d_adj, uint8_t* d_cflags,
                                        int32_t* n_tris, void* stream) {
    if (ctx && ctx->pending) gcdt_wait(ctx, nullptr);
    gcdt_status rc = gcdt_triangulate_async(ctx, d_points, n, d_segments, s, d_tris, d_adj, d_cflags, stream);
    if (rc != GCDT_OK) {
        if (ctx && ctx->pending) gcdt_wait(ctx, nullptr);
        return rc;
    }
    return gcdt_wait(ctx, n_tris);
}

extern "C" gcdt_status gcdt_get_stats(const gcdt_context* ctx, gcdt_stats* out) {
    if (!ctx || !out) return GCDT_BAD_INPUT;
    *out = ctx->stats;
    return GCDT_OK;
}

extern "C" const char* gcdt_status_string(gcdt_status s) {
    switch (s) {
    case GCDT_OK: return "ok";
    case GCDT_BAD_INPUT: return "bad input (coordinate range, duplicate point or bad segment)";
    case GCDT_OOM: return "problem larger than the context";
    case GCDT_ITER_LIMIT: return "iteration limit reached";
    case GCDT_CONSTRAINT_FAIL: return "constraint segments cross";
    case GCDT_CUDA_ERROR: return "CUDA error";
    case GCDT_INTERNAL: return "internal error";
    }
    return "unknown status";
}

extern "C" gcdt_status gcdt_eval_predicates(const int32_t* d_quads, int32_t n_cases, int32_t* d_out, void* stream) {
    if (n_cases < 0 || (n_cases > 0 && (!d_quads || !d_out))) return GCDT_BAD_INPUT;
    if (n_cases == 0) return GCDT_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    gcdt_predicates<<<(n_cases + 255) / 256, 256, 0, st>>>(reinterpret_cast<const int2*>(d_quads), n_cases, d_out);
    if (cudaGetLastError() != cudaSuccess) return GCDT_CUDA_ERROR;
    if (cudaStreamSynchronize(st) != cudaSuccess) return GCDT_CUDA_ERROR;
    return GCDT_OK;
}

extern "C" gcdt_status gcdt_set_limits(gcdt_context* ctx, int32_t max_insertion_rounds,
                                       int32_t max_flip_subrounds, int32_t max_constraint_rounds) {
    if (!ctx || max_insertion_rounds < 0 || max_flip_subrounds < 0 || max_constraint_rounds < 0)
        return GCDT_BAD_INPUT;
    ctx->lim_rounds = max_insertion_rounds;
    ctx->lim_subrounds = max_flip_subrounds;
    ctx->lim_crounds = max_constraint_rounds;
    return GCDT_OK;
}

extern "C" gcdt_status gcdt_set_profiling(gcdt_context* ctx, int32_t on) {
    if (!ctx) return GCDT_BAD_INPUT;
    ctx->profile = on ? 1 : 0;
    return GCDT_OK;
}

extern "C" gcdt_status gcdt_set_tuning(gcdt_context* ctx, const gcdt_tuning* tuning) {
    if (!ctx) return GCDT_BAD_INPUT;
    if (!tuning) { ctx->tuning = default_tuning(); return GCDT_OK; }
    const gcdt_tuning& t = *tuning;
    if (t.levels < 1 || t.levels > 4) return GCDT_BAD_INPUT;
    for (int k = 0; k + 1 < t.levels; ++k) {
        if (t.level_stride[k] < 2) return GCDT_BAD_INPUT;
        if (k > 0 && t.level_stride[k] >= t.level_stride[k - 1]) return GCDT_BAD_INPUT;
    }
    if (t.carry_queue < 0 || t.carry_queue > (1 << 24)) return GCDT_BAD_INPUT;
    if (t.narrow_queue < 0 || t.narrow_queue > 65536 || t.narrow_active < 0 || t.narrow_active > 65536)
        return GCDT_BAD_INPUT;
    ctx->tuning = t;
    for (int k = t.levels - 1; k < 3; ++k) ctx->tuning.level_stride[k] = 1;
    return GCDT_OK;
}

// Candidate schedules of gcdt_autotune: the defaults first, then denser or
// sparser level strides, two-level schedules and smaller carries.
namespace {
gcdt_tuning candidate(int levels, int s0, int s1, int carry) {
    gcdt_tuning t = default_tuning();
    t.levels = levels;
    t.level_stride[0] = s0;
    t.level_stride[1] = levels > 2 ? s1 : 1;
    t.level_stride[2] = 1;
    t.carry_queue = carry;
    return t;
}
}  // namespace

extern "C" gcdt_status gcdt_autotune(gcdt_context* ctx, const int32_t* d_points, int32_t n,
                                     const int32_t* d_segments, int32_t s, int32_t* d_tris, int32_t* d_adj,
                                     uint8_t* d_cflags, int32_t repeats, gcdt_tuning* chosen, void* stream) {
    if (!ctx || repeats < 1 || repeats > 16) return GCDT_BAD_INPUT;
    const gcdt_tuning cands[] = {
        default_tuning(),
        candidate(3, 256, 8, (int)kCarryQueue), candidate(3, 1024, 16, (int)kCarryQueue),
        candidate(3, 512, 16, (int)kCarryQueue), candidate(3, 256, 4, (int)kCarryQueue),
        candidate(2, 64, 1, (int)kCarryQueue), candidate(2, 256, 1, (int)kCarryQueue),
        candidate(3, 512, 8, 1 << 20), candidate(3, 512, 8, 1 << 24),
    };
    const gcdt_tuning keep = ctx->tuning;
    int best = -1;
    double best_ms = 0.0;
    int32_t nt = 0;
    // one untimed solve first (module load, caches), then every candidate
    ctx->tuning = cands[0];
    gcdt_status rc = gcdt_triangulate(ctx, d_points, n, d_segments, s, d_tris, d_adj, d_cflags, &nt, stream);
    for (int k = 0; rc == GCDT_OK && k < (int)(sizeof(cands) / sizeof(cands[0])); ++k) {
        ctx->tuning = cands[k];
        double ms = 0.0;
        for (int r = 0; r < repeats && rc == GCDT_OK; ++r) {
            rc = gcdt_triangulate(ctx, d_points, n, d_segments, s, d_tris, d_adj, d_cflags, &nt, stream);
            double m = ctx->stats.device_ms;
            if (r == 0 || m < ms) ms = m;
        }
        if (rc == GCDT_OK && (best < 0 || ms < best_ms)) { best = k; best_ms = ms; }
    }
    if (rc != GCDT_OK || best < 0) {
        ctx->tuning = keep;
        return rc != GCDT_OK ? rc : GCDT_INTERNAL;
    }
    ctx->tuning = cands[best];
    if (chosen) *chosen = cands[best];
    return GCDT_OK;
}

extern "C" gcdt_status gcdt_get_tuning(const gcdt_context* ctx, gcdt_tuning* tuning) {
    if (!ctx || !tuning) return GCDT_BAD_INPUT;
    *tuning = ctx->tuning;
    return GCDT_OK;
}

extern "C" gcdt_status gcdt_time_barriers(int device, int32_t rounds, double* us_per_barrier) {
    if (!us_per_barrier || rounds < 1 || rounds > (1 << 20)) return GCDT_BAD_INPUT;
    *us_per_barrier = 0;
    DeviceGuard g(device);
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gcdt_stages<false>, kPersistBlock, 0) != cudaSuccess ||
        sms <= 0 || per_sm <= 0) {
        cudaGetLastError();
        return GCDT_CUDA_ERROR;
    }
    Counters* cnt = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    if (cudaMalloc(&cnt, sizeof(Counters)) != cudaSuccess) { cudaGetLastError(); return GCDT_CUDA_ERROR; }
    cudaError_t e = cudaMemset(cnt, 0, sizeof(Counters));
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    float ms = 0.f;
    int status = 0;
    if (e == cudaSuccess) {
        int r = rounds;
        void* args[] = {&cnt, &r};
        cudaEventRecord(a, 0);
        e = cudaLaunchCooperativeKernel((const void*)gcdt_barrier_loop, dim3(sms * per_sm), dim3(kPersistBlock), args, 0, 0);
        cudaEventRecord(b, 0);
        if (e == cudaSuccess) e = cudaEventSynchronize(b);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
        if (e == cudaSuccess) e = cudaMemcpy(&status, &cnt->status, sizeof(int), cudaMemcpyDeviceToHost);
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    cudaFree(cnt);
    if (e != cudaSuccess) { cudaGetLastError(); return GCDT_CUDA_ERROR; }
    if (status & ST_BARRIER) return GCDT_INTERNAL;
    *us_per_barrier = 1e3 * ms / rounds;
    return GCDT_OK;
}

extern "C" gcdt_status gcdt_probe_barrier(int device, int32_t blocks, int32_t absent_block, uint32_t spin_limit,
                                          int32_t* timed_out) {
    if (!timed_out || blocks < 1 || blocks > 1024 || spin_limit == 0) return GCDT_BAD_INPUT;
    *timed_out = 0;
    DeviceGuard g(device);
    Counters* cnt = nullptr;
    if (cudaMalloc(&cnt, sizeof(Counters)) != cudaSuccess) return GCDT_CUDA_ERROR;
    cudaError_t e = cudaMemset(cnt, 0, sizeof(Counters));
    if (e == cudaSuccess) {
        unsigned absent = absent_block < 0 ? 0xffffffffu : (unsigned)absent_block;
        gcdt_barrier_probe<<<blocks, 32>>>(cnt, absent, spin_limit);
        e = cudaGetLastError();
    }
    int status = 0;
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(&status, &cnt->status, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(cnt);
    if (e != cudaSuccess) return GCDT_CUDA_ERROR;
    *timed_out = (status & ST_BARRIER) ? 1 : 0;
    return GCDT_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free triangulation.
//
// Some callers cannot allocate device memory at call time: a plugin whose host
// application owns all device memory through its own caching allocator (a
// cudaMalloc there can fail even with memory free, because the host's pool
// holds it), or a latency-bound loop that cannot afford cudaMalloc/cudaFree,
// which may synchronize the whole device.  For them this entry point runs the
// same solve as gcdt_triangulate with its scratch in one file-scope device
// array instead of a context arena.  The array is part of this library's
// module, so every GPU that loads the library holds it until the process
// exits.
//
// Set-up: every call looks the array's device address up with
// cudaGetSymbolAddress on the device that is current when it is called (the
// lookup is a host-side table read, so it costs little), and checks the
// result.  Nothing is cached across calls, so the address stays right after
// a cudaDeviceReset reloads the module.  Since every call does this set-up,
// make every call before any stream capture begins on the device.  The call
// returns once the solve has finished (it reads the solve's counters back).
//
// Limits and sharing: a problem whose workspace (gcdt_workspace_bytes(n, s))
// exceeds GCDT_NOALLOC_WORKSPACE_BYTES is rejected with GCDT_OOM before any
// device work.  All calls on a device share the one array and it keeps the
// previous call's contents; the solve itself zeroes every array that must
// start at zero.  Two calls whose work overlaps on the GPU (different
// streams, or different host threads) race on the array and corrupt each
// other's results: serialize them.
// ---------------------------------------------------------------------------
namespace {
constexpr size_t kNoAllocBytes = GCDT_NOALLOC_WORKSPACE_BYTES;
__device__ __align__(256) unsigned char g_noalloc_workspace[kNoAllocBytes];
}  // namespace

extern "C" gcdt_status gcdt_triangulate_noalloc(const int32_t* d_points, int32_t n,
                                                const int32_t* d_segments, int32_t s,
                                                int32_t* d_tris, int32_t* d_adj, uint8_t* d_cflags,
                                                int32_t* n_tris, void* stream) {
    if (n < 0 || s < 0 || (n > 0 && !d_points) || (s > 0 && !d_segments) || !d_tris || !d_adj || !d_cflags)
        return GCDT_BAD_INPUT;
    Plan plan = make_plan(n, s, sort_temp_bytes(n));
    if (plan.L.total > kNoAllocBytes) return GCDT_OOM;
    // The device address of the array on the current device.  In host code
    // g_noalloc_workspace names a host-side stand-in, never a device address.
    void* sym = nullptr;
    cudaError_t se = cudaGetSymbolAddress(&sym, g_noalloc_workspace);
    if (se != cudaSuccess || !sym) {
        cudaGetLastError();
        return GCDT_CUDA_ERROR;
    }
    char* base = static_cast<char*>(sym);
    Ctx c = bind_ctx(base, plan);
    c.in_xy = reinterpret_cast<const int2*>(d_points);
    c.in_cons = reinterpret_cast<const int2*>(d_segments);
    c.out_tris = d_tris;
    c.out_adj = d_adj;
    c.out_cflags = d_cflags;
    Counters host_counters;   // pageable: counter reads go through cudaMemcpyAsync + sync
    DeviceBackend bk;
    bk.st = static_cast<cudaStream_t>(stream);
    bk.dcnt = c.cnt;
    bk.hcnt = &host_counters;
    bk.sort_tmp = base + plan.o_sort_tmp;
    bk.sort_bytes = plan.sort_temp_bytes;
    SolveStats st;
    int bits = run_solve(bk, c, st);
    bk.note(cudaStreamSynchronize(bk.st));
    if (bk.err != cudaSuccess) {
        bits |= ST_CUDA;
        cudaGetLastError();   // clear a launch error so the caller's next check does not see it
    }
    gcdt_status rc = map_status(bits);
    if (rc == GCDT_OK && n_tris) *n_tris = 2 * n + 2;
    return rc;
}

static const char* const kPhaseNames[] = {
    "keys", "gather", "root", "level", "seg_level0", "activate", "vt_reset", "vt_live",
    "reloc_vote", "split", "fix", "flip_check", "flip_do", "flip_fix", "output",
    "seg_init", "cwalk", "cclaim", "cproc", "narrow_flips", "narrow_rounds", "clear"};
static_assert(sizeof(kPhaseNames) / sizeof(kPhaseNames[0]) == K_COUNT, "one name per phase kind");

extern "C" int32_t gcdt_get_phase_profile(const gcdt_context* ctx, int64_t* cycles, int64_t* counts, int32_t max_kinds) {
    if (!ctx || !ctx->hcnt || max_kinds < 0) return -1;
    int32_t n = (int32_t)(sizeof(kPhaseNames) / sizeof(kPhaseNames[0]));
    if (n > kMaxPhaseKinds) n = kMaxPhaseKinds;
    for (int32_t k = 0; k < n && k < max_kinds; ++k) {
        if (cycles) cycles[k] = ctx->hcnt->phase_cyc[k];
        if (counts) counts[k] = ctx->hcnt->phase_cnt[k];
    }
    return n;
}

extern "C" int32_t gcdt_get_phase_balance(const gcdt_context* ctx, int64_t* wmax, int64_t* wsum, int64_t* blocks,
                                          int32_t max_kinds) {
    if (!ctx || !ctx->hcnt || max_kinds < 0) return -1;
    if (blocks) *blocks = ctx->hcnt->grid_blocks;
    int32_t n = (int32_t)(sizeof(kPhaseNames) / sizeof(kPhaseNames[0]));
    if (n > kMaxPhaseKinds) n = kMaxPhaseKinds;
    for (int32_t k = 0; k < n && k < max_kinds; ++k) {
        if (wmax) wmax[k] = ctx->hcnt->phase_wmax[k];
        if (wsum) wsum[k] = ctx->hcnt->phase_wsum[k];
    }
    return n;
}

extern "C" const char* gcdt_phase_name(int32_t kind) {
    int32_t n = (int32_t)(sizeof(kPhaseNames) / sizeof(kPhaseNames[0]));
    return (kind >= 0 && kind < n) ? kPhaseNames[kind] : "";
}
