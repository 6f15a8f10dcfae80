"""gcdt_b200 -- B200-native constrained Delaunay triangulation.

Host-side mirror of the C ABI in include/gcdt.h.  The CUDA library
(libgcdt_b200.so, built in-tree by gcdt_b200/build.py) is the only compute
path: importing the triangulator without it raises, there is no CPU fallback.

    import gcdt_b200 as g
    tri = g.Triangulator(max_points=10_000_000, max_segments=200_000)
    tris, adj, cflags = tri.triangulate(points_cuda, segments_cuda)

`points` is an (n, 2) int32 tensor of distinct coordinates in [1, 2^30-2];
`segments` an (s, 2) int32 tensor of point indices.  Outputs hold 2n+2
triangles over vertices 0..n-1 (the caller's points) and n..n+3 (the box
corners (0,0), (R,0), (R,R), (0,R), R = 2^30-1), as in the reference
(yingtix/gCDT rawMesh.cu:5-35).
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_GEN = None

STATUS = {
    0: "OK", 1: "BAD_INPUT", 2: "OOM", 3: "ITER_LIMIT",
    4: "CONSTRAINT_FAIL", 5: "CUDA_ERROR", 6: "INTERNAL",
}

# Box corner ids are n..n+3; R is the box size (reference math_base.cuh:19-29).
BOX_MAX = (1 << 30) - 1


class GcdtError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        self.status = STATUS.get(code, str(code))
        super().__init__("%s: %s" % (what or "gcdt", self.status))


class Tuning(ctypes.Structure):
    """gcdt_tuning: scheduling of a context's solves (include/gcdt.h)."""
    _fields_ = [("levels", ctypes.c_int32), ("level_stride", ctypes.c_int32 * 3),
                ("carry_queue", ctypes.c_int32), ("narrow_queue", ctypes.c_int32),
                ("narrow_active", ctypes.c_int32)]

    def as_dict(self):
        return {"levels": self.levels, "level_stride": list(self.level_stride)[:max(self.levels - 1, 0)],
                "carry_queue": self.carry_queue, "narrow_queue": self.narrow_queue,
                "narrow_active": self.narrow_active}


class Stats(ctypes.Structure):
    _fields_ = [
        ("n_points", ctypes.c_int64), ("n_segments", ctypes.c_int64),
        ("n_triangles", ctypes.c_int64), ("insertion_rounds", ctypes.c_int64),
        ("flip_subrounds", ctypes.c_int64), ("flips", ctypes.c_int64),
        ("constraint_rounds", ctypes.c_int64), ("host_syncs", ctypes.c_int64),
        ("kernel_launches", ctypes.c_int64), ("device_ms", ctypes.c_double),
        ("stage_ms", ctypes.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def lib_path():
    """The CUDA library: libgcdt_b200.so next to this file, or the build
    variant named by GCDT_B200_LIB (a path, or a variant name NAME for
    libgcdt_b200_NAME.so next to this file; see build.VARIANTS)."""
    v = os.environ.get("GCDT_B200_LIB")
    if v:
        return v if os.sep in v else os.path.join(_HERE, "libgcdt_b200_%s.so" % v)
    return os.path.join(_HERE, "libgcdt_b200.so")


def lib():
    """Load libgcdt_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = lib_path()
    if not os.path.exists(path):
        raise ImportError("%s is missing; build it with `python -m gcdt_b200.build`" % path)
    L = ctypes.CDLL(path)
    vp, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
    L.gcdt_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, i64, i64]
    L.gcdt_create.restype = ctypes.c_int
    L.gcdt_destroy.argtypes = [vp]
    L.gcdt_destroy.restype = None
    L.gcdt_workspace_bytes.argtypes = [i64, i64]
    L.gcdt_workspace_bytes.restype = ctypes.c_size_t
    L.gcdt_triangulate.argtypes = [vp, vp, i32, vp, i32, vp, vp, vp, ctypes.POINTER(i32), vp]
    L.gcdt_triangulate.restype = ctypes.c_int
    L.gcdt_set_grid_blocks.argtypes = [vp, i32]
    L.gcdt_set_grid_blocks.restype = ctypes.c_int
    L.gcdt_triangulate_async.argtypes = [vp, vp, i32, vp, i32, vp, vp, vp, vp]
    L.gcdt_triangulate_async.restype = ctypes.c_int
    L.gcdt_wait.argtypes = [vp, ctypes.POINTER(i32)]
    L.gcdt_wait.restype = ctypes.c_int
    L.gcdt_get_stats.argtypes = [vp, ctypes.POINTER(Stats)]
    L.gcdt_get_stats.restype = ctypes.c_int
    L.gcdt_status_string.argtypes = [ctypes.c_int]
    L.gcdt_status_string.restype = ctypes.c_char_p
    L.gcdt_set_profiling.argtypes = [vp, i32]
    L.gcdt_set_profiling.restype = ctypes.c_int
    L.gcdt_get_phase_profile.argtypes = [vp, vp, vp, i32]
    L.gcdt_get_phase_profile.restype = i32
    L.gcdt_get_phase_balance.argtypes = [vp, vp, vp, vp, i32]
    L.gcdt_get_phase_balance.restype = i32
    L.gcdt_phase_name.argtypes = [i32]
    L.gcdt_phase_name.restype = ctypes.c_char_p
    L.gcdt_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, i64, i64, i64]
    L.gcdt_batch_create.restype = ctypes.c_int
    L.gcdt_batch_destroy.argtypes = [vp]
    L.gcdt_batch_destroy.restype = None
    L.gcdt_batch_triangulate.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.gcdt_batch_triangulate.restype = ctypes.c_int
    L.gcdt_batch_autotune.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, vp, i32, vp, vp]
    L.gcdt_batch_autotune.restype = ctypes.c_int
    L.gcdt_batch_set_config.argtypes = [vp, vp]
    L.gcdt_batch_set_config.restype = ctypes.c_int
    L.gcdt_batch_get_config.argtypes = [vp, vp]
    L.gcdt_batch_get_config.restype = ctypes.c_int
    L.gcdt_batch_last_ms.argtypes = [vp]
    L.gcdt_batch_last_ms.restype = ctypes.c_double
    L.gcdt_server_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, vp]
    L.gcdt_server_create.restype = ctypes.c_int
    L.gcdt_server_destroy.argtypes = [vp]
    L.gcdt_server_destroy.restype = None
    L.gcdt_server_submit.argtypes = [vp, vp, i32, vp, i32, ctypes.POINTER(i64)]
    L.gcdt_server_submit.restype = ctypes.c_int
    L.gcdt_server_wait.argtypes = [vp, i64, i32, ctypes.POINTER(i32)]
    L.gcdt_server_wait.restype = ctypes.c_int
    L.gcdt_server_fetch.argtypes = [vp, i64, vp, vp, vp, ctypes.POINTER(i32)]
    L.gcdt_server_fetch.restype = ctypes.c_int
    L.gcdt_server_release.argtypes = [vp, i64]
    L.gcdt_server_release.restype = ctypes.c_int
    L.gcdt_server_request_times.argtypes = [vp, i64, vp, vp, vp]
    L.gcdt_server_request_times.restype = ctypes.c_int
    L.gcdt_server_get_stats.argtypes = [vp, vp]
    L.gcdt_server_get_stats.restype = ctypes.c_int
    L.gcdt_server_reset_stats.argtypes = [vp]
    L.gcdt_server_reset_stats.restype = ctypes.c_int
    L.gcdt_text_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
    L.gcdt_text_load.restype = vp
    L.gcdt_text_sizes.argtypes = [vp, ctypes.POINTER(i64), ctypes.POINTER(i64)]
    L.gcdt_text_sizes.restype = None
    L.gcdt_text_copy.argtypes = [vp, vp, vp]
    L.gcdt_text_copy.restype = None
    L.gcdt_text_free.argtypes = [vp]
    L.gcdt_text_free.restype = None
    L.gcdt_text_save.argtypes = [ctypes.c_char_p, vp, i64, vp, vp, vp, i64]
    L.gcdt_text_save.restype = ctypes.c_int
    L.gcdt_eval_predicates.argtypes = [vp, i32, vp, vp]
    L.gcdt_eval_predicates.restype = ctypes.c_int
    L.gcdt_reference_layout_scratch_bytes.argtypes = [i32, i32]
    L.gcdt_reference_layout_scratch_bytes.restype = ctypes.c_size_t
    L.gcdt_reference_layout.argtypes = [vp, i32, vp, vp, vp, i32, vp, vp, vp, vp, vp, vp, ctypes.c_size_t, vp]
    L.gcdt_reference_layout.restype = ctypes.c_int
    L.gcdt_set_tuning.argtypes = [vp, vp]
    L.gcdt_set_tuning.restype = ctypes.c_int
    L.gcdt_get_tuning.argtypes = [vp, vp]
    L.gcdt_get_tuning.restype = ctypes.c_int
    L.gcdt_autotune.argtypes = [vp, vp, i32, vp, i32, vp, vp, vp, i32, vp, vp]
    L.gcdt_autotune.restype = ctypes.c_int
    L.gcdt_set_limits.argtypes = [vp, i32, i32, i32]
    L.gcdt_set_limits.restype = ctypes.c_int
    L.gcdt_time_barriers.argtypes = [ctypes.c_int, i32, ctypes.POINTER(ctypes.c_double)]
    L.gcdt_time_barriers.restype = ctypes.c_int
    L.gcdt_probe_barrier.argtypes = [ctypes.c_int, i32, i32, ctypes.c_uint32, ctypes.POINTER(i32)]
    L.gcdt_probe_barrier.restype = ctypes.c_int
    L.gcdt_classify_regions_scratch_bytes.argtypes = [i32]
    L.gcdt_classify_regions_scratch_bytes.restype = ctypes.c_size_t
    L.gcdt_classify_regions.argtypes = [vp, vp, i32, vp, ctypes.POINTER(i32), vp, ctypes.c_size_t, vp]
    L.gcdt_classify_regions.restype = ctypes.c_int
    _LIB = L
    return L


def _gen_lib():
    global _GEN
    if _GEN is not None:
        return _GEN
    path = os.path.join(_HERE, "libgcdt_gen.so")
    if not os.path.exists(path):
        raise ImportError("libgcdt_gen.so is missing; build it with `python -m gcdt_b200.build`")
    G = ctypes.CDLL(path)
    G.gcdt_gen_new.restype = ctypes.c_void_p
    G.gcdt_gen_new.argtypes = [ctypes.c_int, ctypes.c_uint64] + [ctypes.c_int64] * 4
    G.gcdt_gen_sizes.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
    G.gcdt_gen_copy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    G.gcdt_gen_free.argtypes = [ctypes.c_void_p]
    _GEN = G
    return G


# Workload kinds of gcdt_gen_new (see gcdt_b200/csrc/gen.cpp).
GEN_SMALL, GEN_SCALE, GEN_LATTICE, GEN_BATCH_INSTANCE, GEN_SERVING_REQUEST, GEN_UNIFORM = 0, 1, 2, 3, 4, 5


def generate(kind, seed, a=0, b=0, c=0, d=0):
    """Seeded synthetic workload -> (points (n,2) int32, segments (s,2) int32)."""
    G = _gen_lib()
    h = G.gcdt_gen_new(int(kind), int(seed), int(a), int(b), int(c), int(d))
    if not h:
        raise ValueError("unknown workload kind %r" % (kind,))
    n = ctypes.c_int64()
    s = ctypes.c_int64()
    G.gcdt_gen_sizes(h, ctypes.byref(n), ctypes.byref(s))
    xy = np.zeros((n.value, 2), np.int32)
    cons = np.zeros((s.value, 2), np.int32)
    G.gcdt_gen_copy(h, xy.ctypes.data, cons.ctypes.data)
    G.gcdt_gen_free(h)
    return xy, cons


def canonical(tris):
    """Rotate each triangle so its smallest vertex id comes first (orientation
    kept) and sort the list: equal triangle sets give equal arrays."""
    t = np.asarray(tris, np.int64).reshape(-1, 3)
    r = np.argmin(t, axis=1)
    idx = (np.arange(3)[None, :] + r[:, None]) % 3
    c = np.take_along_axis(t, idx, axis=1)
    order = np.lexsort((c[:, 2], c[:, 1], c[:, 0]))
    return c[order]


def workspace_bytes(n_points, n_segments):
    return int(lib().gcdt_workspace_bytes(int(n_points), int(n_segments)))


class Triangulator:
    """Owns one device arena sized for (max_points, max_segments)."""

    def __init__(self, max_points, max_segments=0, device=0):
        L = lib()
        h = ctypes.c_void_p()
        rc = L.gcdt_create(ctypes.byref(h), int(device), int(max_points), int(max_segments))
        if rc != 0:
            raise GcdtError(rc, "gcdt_create")
        self._h = h
        self.device = device
        self.max_points = max_points
        self.max_segments = max_segments

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().gcdt_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def triangulate_raw(self, d_points, n, d_segments, s, d_tris, d_adj, d_cflags, stream=0):
        """Pointer-level call (device addresses as ints); returns the status code."""
        nt = ctypes.c_int32(0)
        return lib().gcdt_triangulate(self._h, ctypes.c_void_p(d_points), int(n),
                                      ctypes.c_void_p(d_segments or 0), int(s),
                                      ctypes.c_void_p(d_tris), ctypes.c_void_p(d_adj),
                                      ctypes.c_void_p(d_cflags), ctypes.byref(nt),
                                      ctypes.c_void_p(stream))

    def _args(self, points, segments, out, stream):
        import torch
        if points.dtype != torch.int32 or not points.is_cuda:
            raise TypeError("points must be a CUDA int32 tensor of shape (n, 2)")
        points = points.contiguous()
        n = points.shape[0]
        s = 0
        sp = 0
        if segments is not None and segments.numel() > 0:
            if segments.dtype != torch.int32 or not segments.is_cuda:
                raise TypeError("segments must be a CUDA int32 tensor of shape (s, 2)")
            segments = segments.contiguous()
            s = segments.shape[0]
            sp = segments.data_ptr()
        T = 2 * n + 2
        if out is None:
            tris = torch.empty((T, 3), dtype=torch.int32, device=points.device)
            adj = torch.empty((T, 3), dtype=torch.int32, device=points.device)
            cflags = torch.empty((T,), dtype=torch.uint8, device=points.device)
        else:
            tris, adj, cflags = out
        if stream is None:
            stream = torch.cuda.current_stream(points.device).cuda_stream
        return points, segments, n, sp, s, (tris, adj, cflags), stream

    def triangulate(self, points, segments=None, out=None, stream=None):
        """Device tensors in, device tensors out: (tris (T,3), adj (T,3), cflags (T,))."""
        points, segments, n, sp, s, out, stream = self._args(points, segments, out, stream)
        tris, adj, cflags = out
        rc = self.triangulate_raw(points.data_ptr() if n else 0, n, sp, s,
                                  tris.data_ptr(), adj.data_ptr(), cflags.data_ptr(), stream)
        if rc != 0:
            raise GcdtError(rc, "gcdt_triangulate")
        return tris, adj, cflags

    def set_grid_blocks(self, blocks):
        """Blocks of the persistent launch (0: one per SM), gcdt_set_grid_blocks."""
        rc = lib().gcdt_set_grid_blocks(self._h, int(blocks))
        if rc != 0:
            raise GcdtError(rc, "gcdt_set_grid_blocks")

    def set_profiling(self, on=True):
        """Record the per-phase profile and balance of later solves
        (gcdt_set_profiling; off by default: it costs a little time)."""
        rc = lib().gcdt_set_profiling(self._h, 1 if on else 0)
        if rc != 0:
            raise GcdtError(rc, "gcdt_set_profiling")

    def triangulate_async(self, points, segments=None, out=None, stream=None):
        """Enqueue a solve on `stream` (default: the current stream) and return
        the output tensors at once; wait() reports the solve's status.  The
        inputs and outputs are kept referenced until then.  One solve in
        flight per Triangulator: a further call waits for the previous one."""
        if getattr(self, "_inflight", None) is not None:
            self.wait()
        points, segments, n, sp, s, out, stream = self._args(points, segments, out, stream)
        tris, adj, cflags = out
        rc = lib().gcdt_triangulate_async(self._h, ctypes.c_void_p(points.data_ptr() if n else 0), int(n),
                                          ctypes.c_void_p(sp or 0), int(s),
                                          ctypes.c_void_p(tris.data_ptr()), ctypes.c_void_p(adj.data_ptr()),
                                          ctypes.c_void_p(cflags.data_ptr()), ctypes.c_void_p(stream))
        if rc != 0:
            self.wait()
            raise GcdtError(rc, "gcdt_triangulate_async")
        self._inflight = (points, segments, out)
        return out

    def wait(self):
        """Block until the solve enqueued by triangulate_async is done; raise
        GcdtError if it failed.  Returns the triangle count (0 if none was
        in flight)."""
        nt = ctypes.c_int32(0)
        busy = getattr(self, "_inflight", None) is not None
        rc = lib().gcdt_wait(self._h, ctypes.byref(nt))
        self._inflight = None
        if rc != 0:
            raise GcdtError(rc, "gcdt_wait")
        return int(nt.value) if busy else 0

    def triangulate_host(self, points, segments=None):
        """numpy in, numpy out (copies to and from the device)."""
        import torch
        dev = torch.device("cuda", self.device)
        p = torch.from_numpy(np.ascontiguousarray(points, dtype=np.int32)).to(dev)
        sgm = None
        if segments is not None and len(segments):
            sgm = torch.from_numpy(np.ascontiguousarray(segments, dtype=np.int32)).to(dev)
        tris, adj, cflags = self.triangulate(p, sgm)
        return tris.cpu().numpy(), adj.cpu().numpy(), cflags.cpu().numpy()

    def set_limits(self, insertion_rounds=0, flip_subrounds=0, constraint_rounds=0):
        """Budgets of the solve's bounded loops (0: the built-in bound); a
        solve that runs one out raises GcdtError ITER_LIMIT."""
        rc = lib().gcdt_set_limits(self._h, int(insertion_rounds), int(flip_subrounds), int(constraint_rounds))
        if rc != 0:
            raise GcdtError(rc, "gcdt_set_limits")

    def set_tuning(self, levels=None, level_stride=None, carry_queue=None, narrow_queue=None,
                   narrow_active=None):
        """Change the scheduling of later solves (unnamed fields keep their
        value); set_tuning() with no argument restores the defaults."""
        if all(v is None for v in (levels, level_stride, carry_queue, narrow_queue, narrow_active)):
            rc = lib().gcdt_set_tuning(self._h, None)
        else:
            t = Tuning()
            lib().gcdt_get_tuning(self._h, ctypes.byref(t))
            if levels is not None:
                t.levels = int(levels)
            if level_stride is not None:
                for k, v in enumerate(list(level_stride)[:3]):
                    t.level_stride[k] = int(v)
            if carry_queue is not None:
                t.carry_queue = int(carry_queue)
            if narrow_queue is not None:
                t.narrow_queue = int(narrow_queue)
            if narrow_active is not None:
                t.narrow_active = int(narrow_active)
            rc = lib().gcdt_set_tuning(self._h, ctypes.byref(t))
        if rc != 0:
            raise GcdtError(rc, "gcdt_set_tuning")

    def autotune(self, points, segments=None, repeats=2, out=None, stream=None):
        """Time the candidate schedules on this problem (device tensors) and
        keep the fastest; returns it as a dict."""
        points, segments, n, sp, s, out, stream = self._args(points, segments, out, stream)
        tris, adj, cflags = out
        t = Tuning()
        rc = lib().gcdt_autotune(self._h, ctypes.c_void_p(points.data_ptr() if n else 0), int(n),
                                 ctypes.c_void_p(sp or 0), int(s), ctypes.c_void_p(tris.data_ptr()),
                                 ctypes.c_void_p(adj.data_ptr()), ctypes.c_void_p(cflags.data_ptr()),
                                 int(repeats), ctypes.byref(t), ctypes.c_void_p(stream))
        if rc != 0:
            raise GcdtError(rc, "gcdt_autotune")
        return t.as_dict()

    def tuning(self):
        t = Tuning()
        rc = lib().gcdt_get_tuning(self._h, ctypes.byref(t))
        if rc != 0:
            raise GcdtError(rc, "gcdt_get_tuning")
        return t.as_dict()

    def phase_profile(self):
        """{phase name: (SM cycles, runs)} of the last solve's persistent
        kernel; empty unless that solve ran with set_profiling(True)."""
        cyc = np.zeros(32, np.int64)
        cnt = np.zeros(32, np.int64)
        k = lib().gcdt_get_phase_profile(self._h, ctypes.c_void_p(cyc.ctypes.data),
                                         ctypes.c_void_p(cnt.ctypes.data), 32)
        out = {}
        for i in range(max(k, 0)):
            if cnt[i]:
                out[lib().gcdt_phase_name(i).decode()] = (int(cyc[i]), int(cnt[i]))
        return out

    def phase_balance(self):
        """{phase name: (longest block's work cycles, mean block's work
        cycles)} summed over the runs of each grid phase of the last solve;
        against phase_profile's cycles (block 0's view, barrier included)
        they split a phase into barrier wait, imbalance and work."""
        wmax = np.zeros(32, np.int64)
        wsum = np.zeros(32, np.int64)
        blocks = ctypes.c_int64(0)
        k = lib().gcdt_get_phase_balance(self._h, ctypes.c_void_p(wmax.ctypes.data),
                                         ctypes.c_void_p(wsum.ctypes.data), ctypes.byref(blocks), 32)
        out = {}
        for i in range(max(k, 0)):
            if wmax[i]:
                out[lib().gcdt_phase_name(i).decode()] = (int(wmax[i]), float(wsum[i]) / max(1, blocks.value))
        return out

    def stats(self):
        st = Stats()
        rc = lib().gcdt_get_stats(self._h, ctypes.byref(st))
        if rc != 0:
            raise GcdtError(rc, "gcdt_get_stats")
        return st.as_dict()


def eval_predicates(quads):
    """quads: (k, 4, 2) int32 numpy -> (k, 3) int32 numpy of device signs
    [orient2d(a,b,c), inCircle(a,b,c,d), perturbed inCircle(a,b,c,d)]."""
    import torch
    q = torch.from_numpy(np.ascontiguousarray(quads, dtype=np.int32).reshape(-1, 8)).cuda()
    out = torch.empty((q.shape[0], 3), dtype=torch.int32, device=q.device)
    rc = lib().gcdt_eval_predicates(ctypes.c_void_p(q.data_ptr()), int(q.shape[0]),
                                    ctypes.c_void_p(out.data_ptr()),
                                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    if rc != 0:
        raise GcdtError(rc, "gcdt_eval_predicates")
    return out.cpu().numpy()


def reference_layout(points, tris, adj=None, cflags=None, stream=None):
    """The mesh in the reference's output layout (delaunayNew's Morton
    renumbering, yingtix/gCDT kernel.cu:1886-2068), on the device.

    points: (n, 2) int32 CUDA tensor (the caller's points, corners implied);
    tris/adj: (T, 3) int32 and cflags: (T,) uint8 CUDA tensors over vertices
    0..n+3, e.g. Triangulator.triangulate's output.  Returns (points (n+4, 2)
    in Morton order, labels (n+4,) = new number of each vertex, tris, adj or
    None, cflags or None), all sorted as gcdt_reference_layout describes."""
    import torch
    n = int(points.shape[0])
    T = int(tris.shape[0])
    dev = tris.device if T else points.device
    for t in (points, tris, adj, cflags):
        if t is not None and (not t.is_cuda or not t.is_contiguous()):
            raise ValueError("reference_layout takes contiguous CUDA tensors")
    pts_out = torch.empty((n + 4, 2), dtype=torch.int32, device=dev)
    labels = torch.empty((n + 4,), dtype=torch.int32, device=dev)
    tris_out = torch.empty((T, 3), dtype=torch.int32, device=dev)
    adj_out = torch.empty((T, 3), dtype=torch.int32, device=dev) if adj is not None else None
    cf_out = torch.empty((T,), dtype=torch.uint8, device=dev) if cflags is not None else None
    need = int(lib().gcdt_reference_layout_scratch_bytes(n, T))
    scratch = torch.empty((max(need, 256),), dtype=torch.uint8, device=dev)
    if stream is None:
        stream = torch.cuda.current_stream(dev).cuda_stream
    ptr = lambda t: ctypes.c_void_p(t.data_ptr() if t is not None and t.numel() else 0)
    with torch.cuda.device(dev):
        rc = lib().gcdt_reference_layout(ptr(points), n, ptr(tris), ptr(adj), ptr(cflags), T,
                                         ptr(pts_out), ptr(labels), ptr(tris_out), ptr(adj_out), ptr(cf_out),
                                         ptr(scratch), scratch.numel(), ctypes.c_void_p(stream))
    if rc != 0:
        raise GcdtError(rc, "gcdt_reference_layout")
    return pts_out, labels, tris_out, adj_out, cf_out


def time_barriers(device=0, rounds=4096):
    """Microseconds per grid barrier of the persistent kernel's executor
    (gcdt_time_barriers)."""
    us = ctypes.c_double(0)
    rc = lib().gcdt_time_barriers(int(device), int(rounds), ctypes.byref(us))
    if rc != 0:
        raise GcdtError(rc, "gcdt_time_barriers")
    return us.value


def probe_barrier(device=0, blocks=4, absent_block=0, spin_limit=1 << 16):
    """Run one grid barrier of the persistent kernel's executor with
    `absent_block` missing (-1: none); True if the waits ran out."""
    out = ctypes.c_int32(0)
    rc = lib().gcdt_probe_barrier(int(device), int(blocks), int(absent_block), int(spin_limit), ctypes.byref(out))
    if rc != 0:
        raise GcdtError(rc, "gcdt_probe_barrier")
    return bool(out.value)


def classify_regions(adj, cflags, stream=None):
    """Even-odd region depth of every triangle, on the device.

    adj: (T, 3) int32 and cflags: (T,) uint8 CUDA tensors (a solve's output).
    Returns (depth (T,) int32 CUDA tensor, greatest depth): depth = fewest
    constraint edges crossed from the box edge; odd = inside the polygons."""
    import torch
    T = int(adj.shape[0])
    for t in (adj, cflags):
        if not t.is_cuda or not t.is_contiguous():
            raise ValueError("classify_regions takes contiguous CUDA tensors")
    depth = torch.empty((T,), dtype=torch.int32, device=adj.device)
    need = int(lib().gcdt_classify_regions_scratch_bytes(T))
    scratch = torch.empty((max(need, 256),), dtype=torch.uint8, device=adj.device)
    if stream is None:
        stream = torch.cuda.current_stream(adj.device).cuda_stream
    md = ctypes.c_int32(0)
    with torch.cuda.device(adj.device):
        rc = lib().gcdt_classify_regions(ctypes.c_void_p(adj.data_ptr()), ctypes.c_void_p(cflags.data_ptr()), T,
                                         ctypes.c_void_p(depth.data_ptr()), ctypes.byref(md),
                                         ctypes.c_void_p(scratch.data_ptr()), scratch.numel(),
                                         ctypes.c_void_p(stream))
    if rc != 0:
        raise GcdtError(rc, "gcdt_classify_regions")
    return depth, int(md.value)


class BatchConfig(ctypes.Structure):
    _fields_ = [("threads_per_instance", ctypes.c_int32), ("sample_stride", ctypes.c_int32)]


class BatchTriangulator:
    """Many independent triangulations per call (gcdt_batch_* in include/gcdt.h).

    Instance i's output is exactly the single solve's: 2n_i+2 triangles with
    local vertex ids and local adjacency, stored at triangle 2*P_i + 2*i of
    the concatenated output (P_i = the instance's first point)."""

    def __init__(self, max_instances, max_total_points, max_total_segments=0, device=0):
        h = ctypes.c_void_p()
        rc = lib().gcdt_batch_create(ctypes.byref(h), int(device), int(max_instances),
                                     int(max_total_points), int(max_total_segments))
        if rc != 0:
            raise GcdtError(rc, "gcdt_batch_create")
        self._h = h
        self.device = device

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().gcdt_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def offsets(instances):
        po = np.zeros(len(instances) + 1, np.int64)
        so = np.zeros(len(instances) + 1, np.int64)
        for i, (xy, cons) in enumerate(instances):
            po[i + 1] = po[i] + len(xy)
            so[i + 1] = so[i] + (0 if cons is None else len(cons))
        return po, so

    def _args(self, d_points, d_segments, po, so, out):
        tris, adj, cflags = out
        return (ctypes.c_void_p(po.ctypes.data), ctypes.c_void_p(so.ctypes.data),
                ctypes.c_void_p(d_points.data_ptr() if d_points is not None and d_points.numel() else 0),
                ctypes.c_void_p(d_segments.data_ptr() if d_segments is not None and d_segments.numel() else 0),
                ctypes.c_void_p(tris.data_ptr()), ctypes.c_void_p(adj.data_ptr()), ctypes.c_void_p(cflags.data_ptr()))

    def alloc_outputs(self, po):
        import torch
        ntri = int(2 * po[-1] + 2 * (len(po) - 1))
        dev = torch.device("cuda", self.device)
        return (torch.empty((max(ntri, 1), 3), dtype=torch.int32, device=dev),
                torch.empty((max(ntri, 1), 3), dtype=torch.int32, device=dev),
                torch.empty((max(ntri, 1),), dtype=torch.uint8, device=dev))

    def triangulate_device(self, d_points, d_segments, po, so, out=None, stream=None):
        """Device inputs (concatenated) -> device outputs + per-instance status codes."""
        import torch
        po = np.ascontiguousarray(po, np.int64)
        so = np.ascontiguousarray(so, np.int64)
        if out is None:
            out = self.alloc_outputs(po)
        st = np.zeros(len(po) - 1, np.int32)
        if stream is None:
            stream = torch.cuda.current_stream(torch.device("cuda", self.device)).cuda_stream
        rc = lib().gcdt_batch_triangulate(self._h, len(po) - 1, *self._args(d_points, d_segments, po, so, out),
                                          ctypes.c_void_p(st.ctypes.data), ctypes.c_void_p(stream))
        return out, st, rc

    def triangulate(self, instances):
        """[(xy, cons), ...] host arrays -> [(tris, adj, cflags) or GcdtError] per instance."""
        import torch
        po, so = self.offsets(instances)
        dev = torch.device("cuda", self.device)
        xy = np.concatenate([np.asarray(x, np.int32).reshape(-1, 2) for x, _ in instances]) if po[-1] else np.zeros((0, 2), np.int32)
        cs = [np.asarray(c, np.int32).reshape(-1, 2) for _, c in instances if c is not None and len(c)]
        cons = np.concatenate(cs) if cs else np.zeros((0, 2), np.int32)
        d_xy = torch.from_numpy(np.ascontiguousarray(xy)).to(dev)
        d_c = torch.from_numpy(np.ascontiguousarray(cons)).to(dev) if len(cons) else None
        out, st, rc = self.triangulate_device(d_xy, d_c, po, so)
        tris, adj, cf = (o.cpu().numpy() for o in out)
        res = []
        for i in range(len(instances)):
            if st[i] != 0:
                res.append(GcdtError(int(st[i]), "instance %d" % i))
                continue
            t0 = int(2 * po[i] + 2 * i)
            t1 = t0 + int(2 * (po[i + 1] - po[i]) + 2)
            res.append((tris[t0:t1], adj[t0:t1], cf[t0:t1]))
        return res

    def autotune(self, d_points, d_segments, po, so, sample_instances=0, stream=None):
        import torch
        po = np.ascontiguousarray(po, np.int64)
        so = np.ascontiguousarray(so, np.int64)
        out = self.alloc_outputs(po)
        cfg = BatchConfig()
        if stream is None:
            stream = torch.cuda.current_stream(torch.device("cuda", self.device)).cuda_stream
        rc = lib().gcdt_batch_autotune(self._h, len(po) - 1, *self._args(d_points, d_segments, po, so, out),
                                       int(sample_instances), ctypes.byref(cfg), ctypes.c_void_p(stream))
        if rc != 0:
            raise GcdtError(rc, "gcdt_batch_autotune")
        return {"threads_per_instance": cfg.threads_per_instance, "sample_stride": cfg.sample_stride}

    def set_config(self, threads_per_instance, sample_stride):
        cfg = BatchConfig(threads_per_instance, sample_stride)
        rc = lib().gcdt_batch_set_config(self._h, ctypes.byref(cfg))
        if rc != 0:
            raise GcdtError(rc, "gcdt_batch_set_config")

    def get_config(self):
        cfg = BatchConfig()
        lib().gcdt_batch_get_config(self._h, ctypes.byref(cfg))
        return {"threads_per_instance": cfg.threads_per_instance, "sample_stride": cfg.sample_stride}

    def last_ms(self):
        return float(lib().gcdt_batch_last_ms(self._h))


class ServerConfig(ctypes.Structure):
    _fields_ = [("memory_budget_bytes", ctypes.c_int64), ("lanes", ctypes.c_int32),
                ("max_batch_instances", ctypes.c_int32), ("max_batch_points", ctypes.c_int64),
                ("max_batch_segments", ctypes.c_int64), ("lane_workspace_bytes", ctypes.c_int64),
                ("big_request_points", ctypes.c_int64), ("max_request_points", ctypes.c_int64),
                ("max_request_segments", ctypes.c_int64), ("big_workers", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
                ("batches", ctypes.c_int64), ("big_solves", ctypes.c_int64), ("queued", ctypes.c_int64),
                ("resident_bytes", ctypes.c_int64), ("peak_resident_bytes", ctypes.c_int64),
                ("fixed_bytes", ctypes.c_int64), ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("max_ms", ctypes.c_double), ("requests_per_s", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Server:
    """Continuous-batching triangulation server (gcdt_server_* in include/gcdt.h)."""

    def __init__(self, memory_budget_bytes=150 << 30, lanes=4, max_batch_instances=512,
                 max_batch_points=4_000_000, max_batch_segments=200_000, big_request_points=400_000,
                 max_request_points=1_100_000, max_request_segments=40_000, big_workers=1, device=0):
        cfg = ServerConfig(int(memory_budget_bytes), int(lanes), int(max_batch_instances), int(max_batch_points),
                           int(max_batch_segments), 0, int(big_request_points), int(max_request_points),
                           int(max_request_segments), int(big_workers), 0)
        h = ctypes.c_void_p()
        rc = lib().gcdt_server_create(ctypes.byref(h), int(device), ctypes.byref(cfg))
        if rc != 0:
            raise GcdtError(rc, "gcdt_server_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().gcdt_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, xy, cons=None):
        xy = np.ascontiguousarray(xy, np.int32).reshape(-1, 2)
        cons = np.ascontiguousarray(np.zeros((0, 2)) if cons is None else cons, np.int32).reshape(-1, 2)
        rid = ctypes.c_int64()
        rc = lib().gcdt_server_submit(self._h, ctypes.c_void_p(xy.ctypes.data), len(xy),
                                      ctypes.c_void_p(cons.ctypes.data if len(cons) else 0), len(cons),
                                      ctypes.byref(rid))
        if rc != 0:
            raise GcdtError(rc, "gcdt_server_submit")
        return rid.value

    def wait(self, rid, timeout_ms=-1):
        done = ctypes.c_int32()
        rc = lib().gcdt_server_wait(self._h, int(rid), int(timeout_ms), ctypes.byref(done))
        return bool(done.value), rc

    def fetch(self, rid, n):
        T = 2 * n + 2
        tris = np.empty((T, 3), np.int32)
        adj = np.empty((T, 3), np.int32)
        cf = np.empty(T, np.uint8)
        nt = ctypes.c_int32()
        rc = lib().gcdt_server_fetch(self._h, int(rid), ctypes.c_void_p(tris.ctypes.data),
                                     ctypes.c_void_p(adj.ctypes.data), ctypes.c_void_p(cf.ctypes.data),
                                     ctypes.byref(nt))
        if rc != 0:
            raise GcdtError(rc, "request %d" % rid)
        return tris, adj, cf

    def release(self, rid):
        return lib().gcdt_server_release(self._h, int(rid))

    def times(self, rid):
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        lib().gcdt_server_request_times(self._h, int(rid), ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return a.value, b.value, c.value

    def stats(self):
        st = ServerStats()
        lib().gcdt_server_get_stats(self._h, ctypes.byref(st))
        return st.as_dict()

    def reset_stats(self):
        lib().gcdt_server_reset_stats(self._h)


def load_text(path):
    """Read the reference's text input format -> (points (n,2) int32, segments (s,2) int32)."""
    L = lib()
    err = ctypes.c_int(0)
    h = L.gcdt_text_load(os.fsencode(path), ctypes.byref(err))
    if not h:
        raise ValueError("cannot read %s (error %d)" % (path, err.value))
    n = ctypes.c_int64()
    s = ctypes.c_int64()
    L.gcdt_text_sizes(h, ctypes.byref(n), ctypes.byref(s))
    xy = np.zeros((n.value, 2), np.int32)
    cons = np.zeros((s.value, 2), np.int32)
    L.gcdt_text_copy(h, ctypes.c_void_p(xy.ctypes.data), ctypes.c_void_p(cons.ctypes.data))
    L.gcdt_text_free(h)
    return xy, cons


def save_text(path, xy, tris, adj=None, cflags=None):
    xy = np.ascontiguousarray(xy, np.int32)
    tris = np.ascontiguousarray(tris, np.int32)
    a = np.ascontiguousarray(adj, np.int32) if adj is not None else None
    c = np.ascontiguousarray(cflags, np.uint8) if cflags is not None else None
    rc = lib().gcdt_text_save(os.fsencode(path), ctypes.c_void_p(xy.ctypes.data), len(xy),
                              ctypes.c_void_p(tris.ctypes.data),
                              ctypes.c_void_p(a.ctypes.data if a is not None else 0),
                              ctypes.c_void_p(c.ctypes.data if c is not None else 0), len(tris))
    if rc != 0:
        raise OSError("cannot write %s" % path)
