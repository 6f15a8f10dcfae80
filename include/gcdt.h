/*
 * gcdt.h -- C ABI of the B200 constrained Delaunay triangulator.
 *
 * One entry point replaces the reference's device pipeline for the path
 *   integer points + segment index pairs -> triangles + adjacency + constraint flags.
 * In yingtix/gCDT that path is the driver sequence of kernel.cu:5395-5448:
 *   getSamplePoints (include/rawMesh.h:6), rawMeshBefore (include/rawMesh.h:4),
 *   filterTriangles (kernel.cu:5293), delaunaySample (kernel.cu:5038),
 *   getBitmap (include/boostmap.h:4), rawMeshAfter (include/rawMesh.h:5),
 *   addConstraints (include/addConstraints.h:5), delaunayNew (kernel.cu:4697).
 * The same-signature C++ symbols of that surface are declared in
 * gcdt_reference_surface.h.
 *
 * Conventions (kept from the reference):
 *   - points are int32 (x, y) pairs with 1 <= x, y <= 2^30 - 2, pairwise
 *     distinct; the four box corners (0,0), (R,0), (R,R), (0,R), R = 2^30 - 1,
 *     are added as vertices n, n+1, n+2, n+3 (rawMesh.cu:5-35);
 *   - segments are int32 index pairs into the points, non-crossing;
 *   - the output has exactly 2n + 2 triangles (hull = the box);
 *   - triangle k = (tris[3k], tris[3k+1], tris[3k+2]) is counter-clockwise;
 *     adj[3k+i] is the triangle across the edge opposite tris[3k+i], or -1 on
 *     the box (rawMesh.cu:269-276); bit i of cflags[k] is set when that edge
 *     is a constraint edge.
 * Differences from the reference, by design:
 *   - vertex ids in the output are the caller's input indices (the reference
 *     returns a Morton-permuted point array, kernel.cu:2059-2066);
 *   - a segment passing exactly through an input point is split there and
 *     recovered as two edges (the reference drops it, addConstraints.cu:962-965);
 *   - cocircular ties are broken by a fixed symbolic perturbation, so the
 *     output is unique for every input.
 * All pointers named d_* are device pointers.  Calls on one context must not
 * overlap; a call returns when its result is complete on `stream`.
 */
#ifndef GCDT_H
#define GCDT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    GCDT_OK = 0,
    GCDT_BAD_INPUT = 1,        /* range, duplicates, bad segment index */
    GCDT_OOM = 2,              /* problem larger than the context was created for */
    GCDT_ITER_LIMIT = 3,       /* a bounded device loop ran out of iterations */
    GCDT_CONSTRAINT_FAIL = 4,  /* segments cross each other */
    GCDT_CUDA_ERROR = 5,
    GCDT_INTERNAL = 6
} gcdt_status;

typedef struct gcdt_context gcdt_context;

typedef struct {
    int64_t n_points;
    int64_t n_segments;
    int64_t n_triangles;
    int64_t insertion_rounds;
    int64_t flip_subrounds;
    int64_t flips;
    int64_t constraint_rounds;
    int64_t host_syncs;
    int64_t kernel_launches;
    double device_ms;          /* CUDA-event time of the whole solve */
    double stage_ms;           /* CUDA-event time of the persistent stage kernel alone */
} gcdt_stats;

/* Largest point count a context accepts (triangle ids must fit 29 bits). */
#define GCDT_MAX_POINTS ((int64_t)((1 << 28) - 2))

/* Create a context on `device` whose arena fits max_points / max_segments.
   Replaces the reference's MemCache pre-pool (MemCache.cpp:60-76). */
gcdt_status gcdt_create(gcdt_context** ctx, int device, int64_t max_points, int64_t max_segments);
void gcdt_destroy(gcdt_context* ctx);

/* Device bytes one solve of (n, s) needs. */
size_t gcdt_workspace_bytes(int64_t n_points, int64_t n_segments);

/* Triangulate.  d_points: 2n int32, d_segments: 2s int32 (may be NULL if
   s == 0); outputs sized for 2n+2 triangles: d_tris and d_adj 3 int32 each,
   d_cflags 1 byte each.  *n_tris (host) receives 2n+2 on success. */
gcdt_status gcdt_triangulate(gcdt_context* ctx, const int32_t* d_points, int32_t n,
                             const int32_t* d_segments, int32_t s,
                             int32_t* d_tris, int32_t* d_adj, uint8_t* d_cflags,
                             int32_t* n_tris, void* stream);


/* The same solve, enqueued on `stream` without waiting for it: returns once
   the work is queued (GCDT_OK), or with the argument / capacity error.  The
   solve's own status (bad input found on the device, crossing constraints,
   iteration limits) comes from gcdt_wait, which blocks until the solve is
   done; statistics and the phase profile are those of the last waited
   solve.  A context holds one solve in flight: a further call on it first
   waits for the previous one.  With two contexts on two streams a caller
   keeps the GPU busy while one solve's input and output copies run.
   (The reference runs its stages synchronously, kernel.cu:5395-5448.) */
gcdt_status gcdt_triangulate_async(gcdt_context* ctx, const int32_t* d_points, int32_t n,
                                   const int32_t* d_segments, int32_t s,
                                   int32_t* d_tris, int32_t* d_adj, uint8_t* d_cflags,
                                   void* stream);
/* Wait for the solve enqueued by gcdt_triangulate_async and return its
   status; *n_tris (host, may be NULL) receives 2n+2 on success.  GCDT_OK at
   once when nothing is in flight. */
gcdt_status gcdt_wait(gcdt_context* ctx, int32_t* n_tris);

gcdt_status gcdt_get_stats(const gcdt_context* ctx, gcdt_stats* out);
const char* gcdt_status_string(gcdt_status s);

/* Budgets of the solve's bounded loops on ctx (0 = the built-in bound, which
   is also the ceiling): grid insertion rounds per solve, flip sub-rounds per
   flip pass, constraint-recovery rounds.  A solve that runs a budget out
   returns GCDT_ITER_LIMIT and leaves the context usable; the reference's
   counterparts are its fixed caps (multiFlipFE count > 10, kernel.cu:3667;
   locateStart 10000 steps, addConstraints.cu:769-773), after which it drops
   the work silently. */
gcdt_status gcdt_set_limits(gcdt_context* ctx, int32_t max_insertion_rounds,
                            int32_t max_flip_subrounds, int32_t max_constraint_rounds);

/* Scheduling of a context's solves (the output does not depend on it: the
   constrained Delaunay triangulation is unique under the fixed tie-break).
     levels          insertion levels, 1..4;
     level_stride    level k < levels-1 holds every level_stride[k]-th point
                     of the Hilbert order not in a lower level (plus, for
                     level 0, every segment endpoint); strictly decreasing,
                     >= 2; entries from levels-1 on are ignored;
     carry_queue     a round stops its flip sub-rounds once the queue is at
                     most this long and carries the rest into the next round
                     (0: never carry), 0..2^24;
     narrow_queue    flip queues of at most this many entries run in one
                     block with block barriers (0: never), 0..65536;
     narrow_active   insertion tails of at most this many points run in one
                     block (0: never), 0..65536.
   Defaults: 3 levels, strides 512 and 8, carry 2^22, narrow 1024 and 1024.
   The reference fixes its counterparts at compile time (logSample, the
   bitmap size, QUEUE_SIZE: math_base.cuh:24-26, kernel.cu:2827). */
typedef struct {
    int32_t levels;
    int32_t level_stride[3];
    int32_t carry_queue;
    int32_t narrow_queue;
    int32_t narrow_active;
} gcdt_tuning;
gcdt_status gcdt_set_tuning(gcdt_context* ctx, const gcdt_tuning* tuning);   /* NULL: the defaults */
/* Blocks of the persistent stage kernel's launch for ctx's solves (0, the
   default: every co-resident block, one per SM; larger values are capped
   there).  Fewer blocks leave SMs to other work, so several contexts can
   solve at once; the result does not depend on it.  No counterpart in the
   reference. */
gcdt_status gcdt_set_grid_blocks(gcdt_context* ctx, int32_t blocks);
gcdt_status gcdt_get_tuning(const gcdt_context* ctx, gcdt_tuning* tuning);
/* Solve the given problem under each of a fixed set of schedules (the
   defaults, other level strides, two-level schedules, other carries), best
   of `repeats` (1..16) device times each, keep the fastest for later solves
   on ctx and report it in *chosen (may be NULL).  The outputs hold the
   triangulation when it returns GCDT_OK; on an error the previous schedule
   is kept.  No counterpart in the reference, whose schedule is fixed at
   compile time; the batched path's counterpart is gcdt_batch_autotune. */
gcdt_status gcdt_autotune(gcdt_context* ctx, const int32_t* d_points, int32_t n,
                          const int32_t* d_segments, int32_t s, int32_t* d_tris, int32_t* d_adj,
                          uint8_t* d_cflags, int32_t repeats, gcdt_tuning* chosen, void* stream);

/* Failure-detection probe of the persistent kernel's grid barrier on
   `device`: `blocks` blocks enter one barrier, except absent_block (-1:
   none), each polling at most spin_limit times.  *timed_out = 1 when the
   waits ran out (the barrier records its timeout status and the kernel ends
   normally), 0 when the barrier completed.  Allocates and frees one small
   device buffer; synchronizes the device.  No counterpart in the reference,
   whose waits are unbounded. */
gcdt_status gcdt_probe_barrier(int device, int32_t blocks, int32_t absent_block, uint32_t spin_limit,
                               int32_t* timed_out);
/* Cost of the persistent kernel's grid barrier on `device`: a grid shaped
   like the stage kernel's (one block per co-resident slot) passes `rounds`
   barriers with no work between them; *us_per_barrier receives the
   CUDA-event time per barrier in microseconds.  Every wait is bounded.  No
   counterpart in the reference. */
gcdt_status gcdt_time_barriers(int device, int32_t rounds, double* us_per_barrier);

/* Per-phase profiling of ctx's later solves (no counterpart in the
   reference): on (nonzero), the stage kernel records the two read-outs
   below; off (the default), it records neither and their counters stay 0.
   The records cost a few atomics and counter updates per phase (0.5% of
   the 10M-point solve), so timed runs leave it off.  Returns GCDT_OK, or
   GCDT_BAD_INPUT for a null ctx. */
gcdt_status gcdt_set_profiling(gcdt_context* ctx, int32_t on);

/* Per-phase profile of the last solve on ctx, if it ran with profiling on
   (gcdt_set_profiling): SM cycles spent in each phase
   kind of the persistent stage kernel (measured by block 0, barrier wait
   included) and how often it ran.  Returns the number of phase kinds
   (names: gcdt_phase_name), or -1 on bad arguments.  Counters of the
   reference's per-stage cudaEvent printouts (e.g. rawMesh.cu:1008-1031). */
int32_t gcdt_get_phase_profile(const gcdt_context* ctx, int64_t* cycles, int64_t* counts, int32_t max_kinds);
/* Balance of the grid-wide phases of the last solve, if it ran with
   profiling on (no counterpart in the reference): per phase kind, the sum over its runs of the longest block's
   work time (wmax) and of all blocks' work times (wsum), in SM cycles, the
   work time of a block being the time from the phase's start to its arrival
   at the phase's barrier.  wmax against the phase's cycles from
   gcdt_get_phase_profile shows the barrier's share, wsum / blocks against
   wmax the imbalance; *blocks receives the block count.  Returns the number
   of kinds written (or -1). */
int32_t gcdt_get_phase_balance(const gcdt_context* ctx, int64_t* wmax, int64_t* wsum, int64_t* blocks,
                               int32_t max_kinds);
const char* gcdt_phase_name(int32_t kind);

/* Exact predicates on device, for parity tests.  d_quads: 8 int32 per case
   (a, b, c, d points); d_out: 3 int32 per case = orient2d(a,b,c),
   inCircle(a,b,c,d) (exact sign, math_base.cuh:267-328) and the perturbed
   inCircle used by the triangulator. */
gcdt_status gcdt_eval_predicates(const int32_t* d_quads, int32_t n_cases, int32_t* d_out, void* stream);

/* ---- The reference's output layout.  yingtix/gCDT returns its mesh in
   Morton order: delaunayNew (kernel.cu:4697-4701) renumbers the n+4 points
   (corners included) by a stable sort on the 30-bit Morton code of
   (x >> 15, y >> 15) (reorderPoints, kernel.cu:1966-2068) and sorts the
   triangles stably by the code of their centroid (mean of the vertices'
   (x >> 15, y >> 15), integer division; reorderFaces, kernel.cu:1886-1964).
   This call applies both orders to a triangulation given in input index
   order (gcdt_triangulate's output, or any mesh over those n+4 vertices):
     d_points_out  2(n+4) int32: sorted point j = vertex perm[j] (corners
                   n..n+3 are (0,0), (R,0), (R,R), (0,R)); identical to the
                   reference's returned point array;
     d_labels      n+4 int32: new number of vertex i;
     d_tris_out    triangle j = input triangle order[j], vertices renumbered
                   (each triangle keeps its own vertex rotation);
     d_adj_out     neighbours renumbered to their new positions, -1 kept
                   (with d_adj; NULL together with d_adj);
     d_cflags_out  flags moved with their triangle (NULL with d_cflags).
   Ties in the triangle code keep the input triangle order; the reference
   breaks them by its pre-flip slot order (it sorts before its last flips),
   so only the point array is expected to equal the reference's byte for
   byte.  d_scratch (256-byte aligned) holds at least
   gcdt_reference_layout_scratch_bytes(n, n_tris) bytes; outputs must not
   overlap inputs, scratch or each other.  Runs on the current device and
   returns when the result is complete on `stream`; GCDT_BAD_INPUT if a
   vertex id or neighbour id is out of range (those entries become -1),
   GCDT_OOM if the scratch is too small. */
size_t gcdt_reference_layout_scratch_bytes(int32_t n_points, int32_t n_tris);
gcdt_status gcdt_reference_layout(const int32_t* d_points, int32_t n,
                                  const int32_t* d_tris, const int32_t* d_adj,
                                  const uint8_t* d_cflags, int32_t n_tris,
                                  int32_t* d_points_out, int32_t* d_labels,
                                  int32_t* d_tris_out, int32_t* d_adj_out, uint8_t* d_cflags_out,
                                  void* d_scratch, size_t scratch_bytes, void* stream);

/* ---- Inside / outside (no counterpart in the reference, which returns the
   triangulation of the whole box, kernel.cu:5443-5448).  For a mesh with
   constraint flags (gcdt_triangulate's output), d_depth[t] receives the
   fewest constraint edges that a path of triangles crosses from the box
   edge to triangle t: odd = inside the constrained polygons by the even-odd
   rule, even > 0 = a hole, 0 = outside every polygon; -1 where no path from
   the box edge reaches t.  *max_depth (host, may be NULL) receives the
   greatest depth.  d_scratch (256-byte aligned) holds at least
   gcdt_classify_regions_scratch_bytes(n_tris) bytes and must not overlap
   d_depth.  Runs on the current device; returns when d_depth is complete on
   `stream` (one 4-byte read back per depth level).  GCDT_BAD_INPUT for a
   neighbour id outside -1..n_tris-1, GCDT_OOM for too little scratch. */
size_t gcdt_classify_regions_scratch_bytes(int32_t n_tris);
gcdt_status gcdt_classify_regions(const int32_t* d_adj, const uint8_t* d_cflags, int32_t n_tris,
                                  int32_t* d_depth, int32_t* max_depth, void* d_scratch,
                                  size_t scratch_bytes, void* stream);

/* ---- Batched triangulation (no counterpart in the reference, which
   triangulates one point set per process, kernel.cu:5332-5466).
   Many independent instances in one launch: one segmented Hilbert sort,
   then one block per instance running the full solve, largest first.
   Instance i owns points [point_offsets[i], point_offsets[i+1]) of d_points
   and segments [segment_offsets[i], segment_offsets[i+1]) of d_segments,
   whose indices are local to the instance (0 .. n_i-1).  Its 2n_i+2
   triangles are written at triangle 2*point_offsets[i] + 2*i of d_tris,
   d_adj and d_cflags, with local vertex ids (corners n_i .. n_i+3) and local
   adjacency: exactly the single solve's output for that instance.  The
   offset arrays are host arrays of n_instances+1 entries starting at 0. */
typedef struct gcdt_batch gcdt_batch;
typedef struct {
    int32_t threads_per_instance;   /* 128, 256 or 512 threads per instance block */
    int32_t sample_stride;          /* first insertion level: every k-th point (16..256) */
} gcdt_batch_config;

gcdt_status gcdt_batch_create(gcdt_batch** batch, int device, int64_t max_instances,
                              int64_t max_total_points, int64_t max_total_segments);
void gcdt_batch_destroy(gcdt_batch* batch);
gcdt_status gcdt_batch_triangulate(gcdt_batch* batch, int32_t n_instances,
                                   const int64_t* point_offsets, const int64_t* segment_offsets,
                                   const int32_t* d_points, const int32_t* d_segments,
                                   int32_t* d_tris, int32_t* d_adj, uint8_t* d_cflags,
                                   int32_t* instance_status, void* stream);
/* Times every configuration on the batch (or on sample_instances instances
   spread over its size distribution), keeps the fastest for later calls
   and reports it in *chosen. */
gcdt_status gcdt_batch_autotune(gcdt_batch* batch, int32_t n_instances,
                                const int64_t* point_offsets, const int64_t* segment_offsets,
                                const int32_t* d_points, const int32_t* d_segments,
                                int32_t* d_tris, int32_t* d_adj, uint8_t* d_cflags,
                                int32_t sample_instances, gcdt_batch_config* chosen, void* stream);
gcdt_status gcdt_batch_set_config(gcdt_batch* batch, const gcdt_batch_config* cfg);
gcdt_status gcdt_batch_get_config(const gcdt_batch* batch, gcdt_batch_config* cfg);
/* CUDA-event time of the last gcdt_batch_triangulate call. */
double gcdt_batch_last_ms(const gcdt_batch* batch);

/* ---- Serving (no counterpart in the reference).  A scheduler thread
   admits requests against a device-memory budget by their predicted
   footprint (resident output (2n+2) x 25 bytes from the output pool, solve
   workspace gcdt_workspace_bytes(n, s) from a lane), packs queued requests
   into batches on `lanes` concurrent streams as lanes free up (continuous
   batching: work of requests that arrive while others run overlaps theirs
   on the device), runs requests of at least big_request_points points
   through the single-solve path from big_workers worker threads on
   high-priority streams (one on the whole GPU, or several on a share of the
   SMs each), concurrently with the lanes, and keeps every result resident
   until it is fetched or released.  Submission copies the caller's host arrays; all calls are
   thread-safe. */
typedef struct gcdt_server gcdt_server;
typedef struct {
    int64_t memory_budget_bytes;    /* device bytes for arenas + resident outputs */
    int32_t lanes;                  /* concurrent batch streams (1..16) */
    int32_t max_batch_instances;    /* per lane batch */
    int64_t max_batch_points;
    int64_t max_batch_segments;
    int64_t lane_workspace_bytes;   /* 0: gcdt_workspace_bytes(max_batch_points, max_batch_segments) */
    int64_t big_request_points;     /* at least this many points: the whole-GPU single solve */
    int64_t max_request_points;
    int64_t max_request_segments;
    int32_t big_workers;            /* 0 or 1: one worker for large requests on the whole GPU; k > 1:
                                       k workers, each solving on 1/k of the SMs, so k large
                                       requests run at once */
    int32_t reserved;               /* 0 */
} gcdt_server_config;
typedef struct {
    int64_t submitted, completed, failed, batches, big_solves, queued;
    int64_t resident_bytes, peak_resident_bytes, fixed_bytes;
    double p50_ms, p99_ms, max_ms;   /* submission -> completion, host clock */
    double requests_per_s;           /* completed / (last completion - first submission) */
} gcdt_server_stats;

gcdt_status gcdt_server_create(gcdt_server** server, int device, const gcdt_server_config* cfg);
void gcdt_server_destroy(gcdt_server* server);
gcdt_status gcdt_server_submit(gcdt_server* server, const int32_t* points, int32_t n,
                               const int32_t* segments, int32_t s, int64_t* request_id);
/* Wait up to timeout_ms (-1: no limit); *done tells whether it finished;
   returns the request's status once done. */
gcdt_status gcdt_server_wait(gcdt_server* server, int64_t request_id, int32_t timeout_ms, int32_t* done);
/* Copy a finished result to host arrays sized for 2n+2 triangles, then
   release it; blocks until the request is done. */
gcdt_status gcdt_server_fetch(gcdt_server* server, int64_t request_id, int32_t* h_tris, int32_t* h_adj,
                              uint8_t* h_cflags, int32_t* n_tris);
gcdt_status gcdt_server_release(gcdt_server* server, int64_t request_id);
gcdt_status gcdt_server_request_times(gcdt_server* server, int64_t request_id, double* submit_ms,
                                      double* start_ms, double* done_ms);
gcdt_status gcdt_server_get_stats(gcdt_server* server, gcdt_server_stats* out);
gcdt_status gcdt_server_reset_stats(gcdt_server* server);

/* ---- Input preprocessing and mesh export (host only).
   gcdt_text_load reads the reference's text format (readFile,
   kernel.cu:5159-5291): numPoints, "idx x y" lines, numCons, "idx a b"
   lines; merges duplicate points, normalises the coordinates to the 2^30
   grid as readFile + transPoints (kernel.cu:171-188) do, merges points that
   collide on the grid, keeps them off the box, and drops degenerate and
   repeated segments.  Returns a handle (NULL on error; *err = 1 cannot open,
   2 malformed, 3 unknown point in a segment). */
void* gcdt_text_load(const char* path, int* err);
void gcdt_text_sizes(void* handle, int64_t* n_points, int64_t* n_segments);
void gcdt_text_copy(void* handle, int32_t* points_xy, int32_t* segments);
void gcdt_text_free(void* handle);
/* Write a mesh as text: the n points and 4 corners, then one line per
   triangle "idx a b c adj0 adj1 adj2 cflags".  Returns 0 on success. */
int gcdt_text_save(const char* path, const int32_t* points_xy, int64_t n_points, const int32_t* tris,
                   const int32_t* adj, const uint8_t* cflags, int64_t n_tris);

/* Allocation-free variant of gcdt_triangulate (no counterpart in the
   reference, whose stages all allocate from its MemCache pool).  For callers
   that cannot allocate device memory when they call in: plugins whose host
   application owns the device memory through its own caching allocator, and
   latency-bound loops that cannot pay for cudaMalloc/cudaFree (which may
   synchronize the device).  Scratch lives in one static device array of
   GCDT_NOALLOC_WORKSPACE_BYTES inside this library, held by every GPU that
   loads it until the process exits.  Every call looks up the array's
   address on the current device (nothing is cached, so a device reset does
   not leave a stale address); as that is the call's set-up, make every call
   before any stream capture starts on the device.  The call returns once the
   solve has finished.  Problems needing more workspace than the array
   (gcdt_workspace_bytes(n, s) > GCDT_NOALLOC_WORKSPACE_BYTES, about 120,000
   points) return GCDT_OOM without touching the device.  Calls share the
   array: calls that overlap on the GPU race and corrupt each other, so
   serialize them.  Inputs and outputs are as for gcdt_triangulate; the
   caller passes the device buffers, and the call allocates nothing. */
#define GCDT_NOALLOC_WORKSPACE_BYTES ((size_t)32 << 20)
gcdt_status gcdt_triangulate_noalloc(const int32_t* d_points, int32_t n,
                                     const int32_t* d_segments, int32_t s,
                                     int32_t* d_tris, int32_t* d_adj, uint8_t* d_cflags,
                                     int32_t* n_tris, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GCDT_H */
