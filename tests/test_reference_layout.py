"""The reference's output layout: Morton-renumbered points and triangles.

The CPU restatement (oracle/reference_layout.py, following
yingtix/gCDT kernel.cu:1886-2068) is checked here against hand-computed
codes, against its own definition on an oracle CDT, and, for inputs where
tests/golden/reference_fixtures.json records the point array the
reference's own build returned, against that array byte for byte.  The GPU
tests compare gcdt_reference_layout with the restatement bit for bit on the
CUDA solver's output.
"""
import ctypes
import hashlib
import json
import os
import subprocess

import numpy as np
import pytest

import gcdt_b200 as g
from oracle import oracle
from oracle import reference_layout as rl

FIX = os.path.join(os.path.dirname(__file__), "golden", "reference_fixtures.json")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST_LIB = os.path.join(ROOT, "tests", "_bin", "libreorderhost.so")


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.int64).tobytes()).hexdigest()


def _pinned_point_cases(max_n):
    with open(FIX) as f:
        cases = json.load(f)["cases"]
    return [c for c in cases if "points_sha256" in c and c["n"] <= max_n]


def test_interleave_known_answers():
    # x bits to even positions, y bits to odd positions, bits 0..14 only
    assert rl.interleave15(np.array([1]), np.array([0]))[0] == 1
    assert rl.interleave15(np.array([0]), np.array([1]))[0] == 2
    assert rl.interleave15(np.array([3]), np.array([1]))[0] == 0b111
    assert rl.interleave15(np.array([0x7fff]), np.array([0x7fff]))[0] == (1 << 30) - 1
    assert rl.interleave15(np.array([0x8000]), np.array([0]))[0] == 0     # bit 15 is not read


def test_point_order_small_known_answer():
    # codes at (x >> 15, y >> 15): p0 (2,0) -> 4, p1 (0,1) -> 2, p2 (0,1) -> 2
    # (tie: index order), corners (0,0) -> 0, (R,0) -> 0x15555555,
    # (R,R) -> 2^30-1, (0,R) -> 0x2aaaaaaa
    xy = np.array([[2 << 15, 5], [7, 1 << 15], [3, (1 << 15) + 9]], np.int32)
    perm, labels = rl.point_order(xy)
    assert perm.tolist() == [3, 1, 2, 0, 4, 6, 5]
    assert labels[perm].tolist() == list(range(7))


def test_face_code_truncates_like_c():
    xy = np.array([[1 << 15, 0], [1 << 15, 0], [0, 0]], np.int32)   # mean x = 2/3 -> 0
    assert rl.face_codes(xy, np.array([[0, 1, 2]]))[0] == 0
    xy = np.array([[1 << 15, 0], [1 << 15, 0], [1 << 15, 0]], np.int32)
    assert rl.face_codes(xy, np.array([[0, 1, 2]]))[0] == 1


def test_layout_of_an_oracle_cdt_is_the_same_mesh():
    xy, cons = g.generate(g.GEN_SMALL, 2)
    rc, tris, adj, cf, _ = oracle.cdt(xy, cons)
    assert rc == 0
    pts, labels, t2, a2, c2 = rl.reference_layout(xy, tris, adj, cf)
    n = len(xy)
    perm = np.empty(n + 4, np.int64)
    perm[labels] = np.arange(n + 4)
    # same points, codes non-decreasing, ties in index order
    assert np.array_equal(pts, rl.vertices(xy)[perm])
    code = rl.interleave15(pts[:, 0].astype(np.int64) >> 15, pts[:, 1].astype(np.int64) >> 15)
    assert np.all(np.diff(code) >= 0)
    tie = np.diff(code) == 0
    assert np.all(np.diff(perm)[tie] > 0)
    # same triangles, orientation and flags; triangles sorted by code
    assert np.array_equal(g.canonical(perm[t2]), g.canonical(tris))
    s = (pts.astype(np.int64)[t2] >> 15).sum(axis=1) // 3    # codes from the renumbered mesh itself
    assert np.all(np.diff(rl.interleave15(s[:, 0], s[:, 1])) >= 0)
    assert int(c2.astype(np.int64).sum()) == int(cf.astype(np.int64).sum())
    # adjacency still symmetric after renumbering
    T = len(t2)
    for t in range(0, T, 97):
        for k in range(3):
            u = a2[t, k]
            if u >= 0:
                assert t in a2[u]


@pytest.mark.parametrize("case", _pinned_point_cases(1_000_000), ids=lambda c: c["name"])
def test_point_order_equals_reference_build(case):
    xy, cons = g.generate(case["kind"], case["seed"], *case["args"])
    assert _sha(xy) == case["input_sha256"]
    pts, *_ = rl.reference_layout(xy, np.zeros((0, 3), np.int32))
    assert _sha(pts) == case["points_sha256"]


# ---- the export's kernel bodies, run on the host in several item orders

def build_reorder_host():
    src = os.path.join(ROOT, "tests", "reorder_host.cu")
    deps = [src, os.path.join(ROOT, "gcdt_b200", "csrc", "reorder.cuh")]
    if os.path.exists(HOST_LIB) and os.path.getmtime(HOST_LIB) > max(os.path.getmtime(d) for d in deps):
        return HOST_LIB
    os.makedirs(os.path.dirname(HOST_LIB), exist_ok=True)
    subprocess.run(["nvcc", "-O2", "-std=c++17", "-x", "cu", "-Xcompiler", "-fPIC", "-shared",
                    "-Wno-deprecated-gpu-targets", "-o", HOST_LIB, src], check=True)
    return HOST_LIB


def _host_layout(xy, tris, adj, cf, order):
    L = ctypes.CDLL(build_reorder_host())
    n, T = len(xy), len(tris)
    xy = np.ascontiguousarray(xy, np.int32)
    tris = np.ascontiguousarray(tris, np.int32)
    pts = np.zeros((n + 4, 2), np.int32)
    labels = np.zeros(n + 4, np.int32)
    t2 = np.zeros((T, 3), np.int32)
    a2 = np.zeros((T, 3), np.int32) if adj is not None else None
    c2 = np.zeros(T, np.uint8) if cf is not None else None
    if adj is not None:
        adj = np.ascontiguousarray(adj, np.int32)
    if cf is not None:
        cf = np.ascontiguousarray(cf, np.uint8)
    p = lambda a: ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else None
    L.host_reference_layout.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 5 + [ctypes.c_int]
    L.host_reference_layout.restype = ctypes.c_int
    err = L.host_reference_layout(p(xy), n, p(tris), p(adj), p(cf), T, p(pts), p(labels), p(t2), p(a2),
                                  p(c2), order)
    return err, (pts, labels, t2, a2, c2)


@pytest.mark.parametrize("order", [0, 1, 2], ids=["forward", "reversed", "shuffled"])
@pytest.mark.parametrize("kind,seed,args", [
    (g.GEN_SMALL, 3, ()),
    (g.GEN_LATTICE, 2, (128, 1000)),
    (g.GEN_BATCH_INSTANCE, 7, (5000,)),
], ids=["small", "lattice", "instance"])
def test_kernel_bodies_on_host_equal_restatement(kind, seed, args, order):
    xy, cons = g.generate(kind, seed, *args)
    rc, tris, adj, cf, _ = oracle.cdt(xy, cons)
    assert rc == 0
    err, got = _host_layout(xy, tris, adj, cf, order)
    assert err == 0
    want = rl.reference_layout(xy, tris, adj, cf)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)


def test_kernel_bodies_report_bad_ids_on_host():
    xy, cons = g.generate(g.GEN_BATCH_INSTANCE, 3, 500)
    rc, tris, adj, cf, _ = oracle.cdt(xy, cons)
    bad = tris.copy()
    bad[5, 1] = len(xy) + 4
    err, (pts, labels, t2, a2, c2) = _host_layout(xy, bad, adj, cf, 0)
    assert err == 1 and (t2 == -1).sum() == 1
    badj = adj.copy()
    badj[3, 0] = len(tris)
    err, _ = _host_layout(xy, tris, badj, cf, 0)
    assert err == 2
    err, (pts, labels, t2, a2, c2) = _host_layout(xy, tris[:0], None, None, 0)    # points only
    assert err == 0 and np.array_equal(pts, rl.reference_layout(xy, tris[:0])[0])


# ---- the CUDA export against the restatement

def _gpu_layout(xy, cons, with_adj=True):
    import torch
    tri = g.Triangulator(max_points=max(len(xy), 1), max_segments=max(len(cons), 1))
    d_xy = torch.from_numpy(np.ascontiguousarray(xy)).cuda()
    d_c = torch.from_numpy(np.ascontiguousarray(cons)).cuda() if len(cons) else None
    tris, adj, cf = tri.triangulate(d_xy, d_c)
    out = g.reference_layout(d_xy, tris, adj if with_adj else None, cf if with_adj else None)
    host = [o.cpu().numpy() if o is not None else None for o in out]
    mesh = (tris.cpu().numpy(), adj.cpu().numpy(), cf.cpu().numpy())
    tri.close()
    return host, mesh


@pytest.mark.gpu
@pytest.mark.parametrize("kind,seed,args", [
    (g.GEN_SMALL, 1, ()),
    (g.GEN_SCALE, 4, (300000, 8, 40)),
    (g.GEN_LATTICE, 1, (256, 2000)),
    (g.GEN_UNIFORM, 13159, (200000,)),
], ids=["small", "scale_300k", "lattice", "uniform_200k"])
def test_gpu_layout_equals_restatement(kind, seed, args):
    xy, cons = g.generate(kind, seed, *args)
    (pts, labels, t2, a2, c2), (tris, adj, cf) = _gpu_layout(xy, cons)
    e = rl.reference_layout(xy, tris, adj, cf)
    assert np.array_equal(pts, e[0])
    assert np.array_equal(labels, e[1])
    assert np.array_equal(t2, e[2])
    assert np.array_equal(a2, e[3])
    assert np.array_equal(c2, e[4])


@pytest.mark.gpu
@pytest.mark.parametrize("case", _pinned_point_cases(10_300_000), ids=lambda c: c["name"])
def test_gpu_point_order_equals_reference_build(case):
    import torch
    xy, _ = g.generate(case["kind"], case["seed"], *case["args"])
    d_xy = torch.from_numpy(xy).cuda()
    pts, labels, *_ = g.reference_layout(d_xy, torch.zeros((0, 3), dtype=torch.int32, device="cuda"))
    assert _sha(pts.cpu().numpy()) == case["points_sha256"]


@pytest.mark.gpu
def test_gpu_layout_edge_cases():
    import torch
    # no points: the four corners alone, two triangles
    xy = np.zeros((0, 2), np.int32)
    (pts, labels, t2, a2, c2), (tris, adj, cf) = _gpu_layout(xy, np.zeros((0, 2), np.int32))
    e = rl.reference_layout(xy, tris, adj, cf)
    assert all(np.array_equal(a, b) for a, b in zip((pts, labels, t2, a2, c2), e))
    # tris only (no adjacency, no flags)
    xy, cons = g.generate(g.GEN_BATCH_INSTANCE, 3, 2000)
    (pts, labels, t2, a2, c2), (tris, adj, cf) = _gpu_layout(xy, cons, with_adj=False)
    assert a2 is None and c2 is None
    assert np.array_equal(t2, rl.reference_layout(xy, tris)[2])
    # a vertex id out of range is reported, not read
    d_xy = torch.from_numpy(xy).cuda()
    bad = torch.from_numpy(np.array([[0, 1, len(xy) + 4]], np.int32)).cuda()
    with pytest.raises(g.GcdtError) as ei:
        g.reference_layout(d_xy, bad)
    assert ei.value.status == "BAD_INPUT"
    # a neighbour id out of range is reported
    t = torch.from_numpy(np.ascontiguousarray(tris[:4])).cuda()
    a = torch.from_numpy(np.full((4, 3), 7, np.int32)).cuda()
    with pytest.raises(g.GcdtError):
        g.reference_layout(d_xy, t, a, torch.zeros(4, dtype=torch.uint8, device="cuda"))
    # scratch smaller than required
    L = g.lib()
    n, T = len(xy), len(tris)
    need = int(L.gcdt_reference_layout_scratch_bytes(n, T))
    outs = [torch.empty(s, dtype=torch.int32, device="cuda") for s in ((n + 4) * 2, n + 4, T * 3)]
    scratch = torch.empty(need, dtype=torch.uint8, device="cuda")
    tt = torch.from_numpy(np.ascontiguousarray(tris)).cuda()
    p = lambda x: ctypes.c_void_p(x.data_ptr())
    rc = L.gcdt_reference_layout(p(d_xy), n, p(tt), None, None, T, p(outs[0]), p(outs[1]), p(outs[2]),
                                 None, None, p(scratch), need - 1, None)
    assert g.STATUS[rc] == "OOM"
    # outputs overlapping inputs are refused
    rc = L.gcdt_reference_layout(p(d_xy), n, p(tt), None, None, T, p(outs[0]), p(outs[1]), p(tt),
                                 None, None, p(scratch), need, None)
    assert g.STATUS[rc] == "BAD_INPUT"
    torch.cuda.synchronize()
