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


class Stats(ctypes.Structure):
    _fields_ = [
        ("n_points", ctypes.c_int64), ("n_segments", ctypes.c_int64),
        ("n_triangles", ctypes.c_int64), ("insertion_rounds", ctypes.c_int64),
        ("flip_subrounds", ctypes.c_int64), ("flips", ctypes.c_int64),
        ("constraint_rounds", ctypes.c_int64), ("host_syncs", ctypes.c_int64),
        ("kernel_launches", ctypes.c_int64), ("device_ms", ctypes.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def lib_path():
    return os.path.join(_HERE, "libgcdt_b200.so")


def lib():
    """Load libgcdt_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = lib_path()
    if not os.path.exists(path):
        raise ImportError("libgcdt_b200.so is missing; build it with `python -m gcdt_b200.build`")
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
    L.gcdt_get_stats.argtypes = [vp, ctypes.POINTER(Stats)]
    L.gcdt_get_stats.restype = ctypes.c_int
    L.gcdt_status_string.argtypes = [ctypes.c_int]
    L.gcdt_status_string.restype = ctypes.c_char_p
    L.gcdt_get_phase_profile.argtypes = [vp, vp, vp, i32]
    L.gcdt_get_phase_profile.restype = i32
    L.gcdt_phase_name.argtypes = [i32]
    L.gcdt_phase_name.restype = ctypes.c_char_p
    L.gcdt_eval_predicates.argtypes = [vp, i32, vp, vp]
    L.gcdt_eval_predicates.restype = ctypes.c_int
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

    def triangulate(self, points, segments=None, out=None, stream=None):
        """Device tensors in, device tensors out: (tris (T,3), adj (T,3), cflags (T,))."""
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
        rc = self.triangulate_raw(points.data_ptr() if n else 0, n, sp, s,
                                  tris.data_ptr(), adj.data_ptr(), cflags.data_ptr(), stream)
        if rc != 0:
            raise GcdtError(rc, "gcdt_triangulate")
        return tris, adj, cflags

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

    def phase_profile(self):
        """{phase name: (SM cycles, runs)} of the last solve's persistent kernel."""
        cyc = np.zeros(32, np.int64)
        cnt = np.zeros(32, np.int64)
        k = lib().gcdt_get_phase_profile(self._h, ctypes.c_void_p(cyc.ctypes.data),
                                         ctypes.c_void_p(cnt.ctypes.data), 32)
        out = {}
        for i in range(max(k, 0)):
            if cnt[i]:
                out[lib().gcdt_phase_name(i).decode()] = (int(cyc[i]), int(cnt[i]))
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
