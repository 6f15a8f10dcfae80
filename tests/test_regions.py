"""Inside / outside classification of a constrained triangulation.

gcdt_classify_regions gives each triangle the fewest constraint edges a path
of triangles crosses from the box edge (odd = inside by the even-odd rule).
Its checker, oracle/regions.py, computes the same by a 0-1 breadth-first
search over triangles, a different algorithm from the CUDA path's
union-find + component rounds.  CPU tests run the CUDA path's kernel bodies
on the host in three item orders against the checker; GPU tests run the
device path against it.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import gcdt_b200 as g
from oracle import oracle
from oracle import regions

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST_LIB = os.path.join(ROOT, "tests", "_bin", "libregionshost.so")


def build_regions_host():
    src = os.path.join(ROOT, "tests", "regions_host.cu")
    deps = [src, os.path.join(ROOT, "gcdt_b200", "csrc", "regions.cuh")]
    if os.path.exists(HOST_LIB) and os.path.getmtime(HOST_LIB) > max(os.path.getmtime(d) for d in deps):
        return HOST_LIB
    os.makedirs(os.path.dirname(HOST_LIB), exist_ok=True)
    subprocess.run(["nvcc", "-O2", "-std=c++17", "-x", "cu", "-Xcompiler", "-fPIC", "-shared",
                    "-Wno-deprecated-gpu-targets", "-o", HOST_LIB, src], check=True)
    return HOST_LIB


def _host_classify(adj, cf, order):
    L = ctypes.CDLL(build_regions_host())
    adj = np.ascontiguousarray(adj, np.int32)
    cf = np.ascontiguousarray(cf, np.uint8)
    T = len(adj)
    depth = np.zeros(T, np.int32)
    parent = np.zeros(T, np.int32)
    md = ctypes.c_int32(0)
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    L.host_classify_regions.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.POINTER(ctypes.c_int32), ctypes.c_void_p, ctypes.c_int]
    L.host_classify_regions.restype = ctypes.c_int
    err = L.host_classify_regions(p(adj), p(cf), T, p(depth), ctypes.byref(md), p(parent), order)
    return err, depth, md.value, parent


def nested_rings(seed=5, rings=4, verts=48, npts=20000):
    """Concentric star-free rings (regular polygons of shrinking radius around
    the box centre) as constraints plus uniform points: depth k inside the
    k-th ring, so holes (even depth > 0) and islands occur."""
    rng = np.random.default_rng(seed)
    c = 1 << 29
    pts, segs = [], []
    for r in range(rings):
        rad = (0.8 - 0.18 * r) * (1 << 28)
        base = len(pts)
        ang = np.arange(verts) * 2 * np.pi / verts + 0.01 * r
        for a in ang:
            pts.append((int(c + rad * np.cos(a)), int(c + rad * np.sin(a))))
        for i in range(verts):
            segs.append((base + i, base + (i + 1) % verts))
    ring_set = set(pts)
    extra = rng.integers(1, (1 << 30) - 2, size=(npts, 2))
    for x, y in extra:
        if (int(x), int(y)) not in ring_set:
            pts.append((int(x), int(y)))
            ring_set.add((int(x), int(y)))
    return np.array(pts, np.int32), np.array(segs, np.int32)


def _mesh(xy, cons):
    rc, tris, adj, cf, _ = oracle.cdt(xy, cons)
    assert rc == 0
    return tris, adj, cf


def test_checker_on_nested_rings():
    xy, cons = nested_rings()
    tris, adj, cf = _mesh(xy, cons)
    depth, md = regions.region_depth(adj, cf)
    assert md == 4 and depth.min() == 0
    # a triangle's depth = how many rings enclose its centroid
    c = np.array([1 << 29, 1 << 29], np.float64)
    cen = np.concatenate([xy, [[0, 0], [(1 << 30) - 1, 0], [(1 << 30) - 1, (1 << 30) - 1], [0, (1 << 30) - 1]]])
    cen = cen.astype(np.float64)[tris].mean(axis=1)
    rad = np.hypot(cen[:, 0] - c[0], cen[:, 1] - c[1])
    inner = [(0.8 - 0.18 * r) * (1 << 28) * np.cos(np.pi / 48) for r in range(4)]
    outer = [(0.8 - 0.18 * r) * (1 << 28) for r in range(4)]
    sure = np.ones(len(tris), bool)
    want = np.zeros(len(tris), np.int64)
    for r in range(4):
        want += rad < inner[r]
        sure &= ~((rad >= inner[r]) & (rad <= outer[r]))       # skip centroids between chord and circle
    assert np.array_equal(depth[sure], want[sure])


@pytest.mark.parametrize("order", [0, 1, 2], ids=["forward", "reversed", "shuffled"])
@pytest.mark.parametrize("case", ["rings", "small", "lattice"])
def test_kernel_bodies_on_host_equal_checker(case, order):
    if case == "rings":
        xy, cons = nested_rings()
    elif case == "small":
        xy, cons = g.generate(g.GEN_SMALL, 4)
    else:
        xy, cons = g.generate(g.GEN_LATTICE, 3, 128, 1200)
    tris, adj, cf = _mesh(xy, cons)
    err, depth, md, parent = _host_classify(adj, cf, order)
    assert err == 0
    want, wmd = regions.region_depth(adj, cf)
    assert np.array_equal(depth, want) and md == wmd
    # each component's root is its smallest triangle id, whatever the order
    assert np.all(parent <= np.arange(len(parent)))
    assert np.all(parent[parent] == parent)


def test_open_chains_enclose_nothing():
    """Segments that close no loop (an open zigzag chain and a lone segment):
    both sides of each constraint edge are one component, so every depth
    is 0, in the checker and in the kernel bodies."""
    rng = np.random.default_rng(12)
    chain = np.array([[(1 << 27) * (k + 1), (1 << 28) + (1 << 26) * (k % 2)] for k in range(6)], np.int64)
    lone = np.array([[1 << 28, 3 << 28], [3 << 28, (3 << 28) + 12345]], np.int64)
    extra = rng.integers(1, (1 << 30) - 2, size=(5000, 2))
    xy = np.unique(np.concatenate([chain, lone, extra]), axis=0)
    idx = {tuple(p): i for i, p in enumerate(xy.tolist())}
    segs = [(idx[tuple(chain[k])], idx[tuple(chain[k + 1])]) for k in range(5)]
    segs.append((idx[tuple(lone[0])], idx[tuple(lone[1])]))
    tris, adj, cf = _mesh(xy.astype(np.int32), np.array(segs, np.int32))
    assert cf.any()
    want, wmd = regions.region_depth(adj, cf)
    assert wmd == 0 and not want.any()
    for order in (0, 2):
        err, depth, md, _ = _host_classify(adj, cf, order)
        assert err == 0 and md == 0 and not depth.any()


def test_kernel_bodies_report_bad_neighbours_on_host():
    xy, cons = g.generate(g.GEN_BATCH_INSTANCE, 3, 400)
    tris, adj, cf = _mesh(xy, cons)
    bad = adj.copy()
    bad[2, 1] = len(adj) + 5
    err, *_ = _host_classify(bad, cf, 0)
    assert err == 1


def test_no_constraints_is_all_outside():
    xy, _ = g.generate(g.GEN_UNIFORM, 3, 3000)
    tris, adj, cf = _mesh(xy, np.zeros((0, 2), np.int32))
    err, depth, md, _ = _host_classify(adj, cf, 2)
    assert err == 0 and md == 0 and not depth.any()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["rings", "small", "lattice", "scale_300k"])
def test_gpu_classification_equals_checker(case):
    import torch
    if case == "rings":
        xy, cons = nested_rings(npts=200000)
    elif case == "small":
        xy, cons = g.generate(g.GEN_SMALL, 4)
    elif case == "lattice":
        xy, cons = g.generate(g.GEN_LATTICE, 3, 256, 2000)
    else:
        xy, cons = g.generate(g.GEN_SCALE, 6, 300000, 8, 40)
    tri = g.Triangulator(max_points=len(xy), max_segments=max(len(cons), 1))
    tris, adj, cf = tri.triangulate(torch.from_numpy(xy).cuda(), torch.from_numpy(cons).cuda())
    depth, md = g.classify_regions(adj, cf)
    want, wmd = regions.region_depth(adj.cpu().numpy(), cf.cpu().numpy())
    tri.close()
    assert np.array_equal(depth.cpu().numpy(), want) and md == wmd


@pytest.mark.gpu
def test_gpu_classification_at_scale_equals_host_bodies():
    """The 10.2M-point scale mesh (20.4M triangles, 3,125 disjoint star
    polygons): the device's concurrent union-find must label every triangle
    as the sequential run of the same bodies does, on two calls in a row."""
    import torch
    xy, cons = g.generate(g.GEN_SCALE, 1)
    tri = g.Triangulator(max_points=len(xy), max_segments=len(cons))
    tris, adj, cf = tri.triangulate(torch.from_numpy(xy).cuda(), torch.from_numpy(cons).cuda())
    d1, md1 = g.classify_regions(adj, cf)
    d2, md2 = g.classify_regions(adj, cf)
    err, want, wmd, _ = _host_classify(adj.cpu().numpy(), cf.cpu().numpy(), 0)
    tri.close()
    assert err == 0 and wmd == 1
    assert md1 == md2 == 1
    assert np.array_equal(d1.cpu().numpy(), want) and np.array_equal(d2.cpu().numpy(), want)


@pytest.mark.gpu
def test_gpu_classification_errors():
    import torch
    xy, cons = g.generate(g.GEN_BATCH_INSTANCE, 3, 400)
    tris, adj, cf = _mesh(xy, cons)
    bad = adj.copy()
    bad[2, 1] = len(adj) + 5
    with pytest.raises(g.GcdtError) as ei:
        g.classify_regions(torch.from_numpy(bad).cuda(), torch.from_numpy(cf).cuda())
    assert ei.value.status == "BAD_INPUT"
    d_adj, d_cf = torch.from_numpy(adj).cuda(), torch.from_numpy(cf).cuda()
    L = g.lib()
    T = len(adj)
    need = int(L.gcdt_classify_regions_scratch_bytes(T))
    scratch = torch.empty(need, dtype=torch.uint8, device="cuda")
    depth = torch.empty(T, dtype=torch.int32, device="cuda")
    p = lambda x: ctypes.c_void_p(x.data_ptr())
    assert g.STATUS[L.gcdt_classify_regions(p(d_adj), p(d_cf), T, p(depth), None, p(scratch), need - 1, None)] == "OOM"
    assert g.STATUS[L.gcdt_classify_regions(p(d_adj), p(d_cf), 0, p(depth), None, p(scratch), need, None)] == "OK"
    torch.cuda.synchronize()
