"""The solver's kernel bodies and stage driver, run on the host (CPU).

tests/host_emulation.cu compiles the same bodies the GPU kernels run, with a
sequential executor that calls them one item at a time in a chosen order.
On each workload the output must be a valid CDT equal to the oracle's, the
same bytes whatever the item order (forward, reversed, shuffled: the
phases are schedule-independent), the same with the paired bodies the GPU
uses for the flip passes, and the mesh must stay consistent after every
split fix and flip fix."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import gcdt_b200 as g
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN_DIR = os.path.join(ROOT, "tests", "_bin")
LIB = os.path.join(BIN_DIR, "libhostemu.so")
CSRC = os.path.join(ROOT, "gcdt_b200", "csrc")


def build_host_emulation(defines=()):
    """Build the host harness (tests/_bin/libhostemu.so; with `defines`, a
    variant library named after them)."""
    src = os.path.join(ROOT, "tests", "host_emulation.cu")
    lib = LIB if not defines else os.path.join(BIN_DIR, "libhostemu_%s.so" % "_".join(d.lower() for d in defines))
    deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    if os.path.exists(lib) and os.path.getmtime(lib) > max(os.path.getmtime(d) for d in deps):
        return lib
    os.makedirs(BIN_DIR, exist_ok=True)
    subprocess.run(["nvcc", "-O2", "-std=c++17", "-x", "cu", "-Xcompiler", "-fPIC", "-shared",
                    "--expt-relaxed-constexpr", "-Wno-deprecated-gpu-targets"] +
                   ["-D" + d for d in defines] + ["-o", lib, src], check=True)
    return lib


@pytest.fixture(scope="module")
def emu():
    L = ctypes.CDLL(build_host_emulation())
    vp, i32 = ctypes.c_void_p, ctypes.c_int
    L.host_triangulate.argtypes = [vp, i32, vp, i32, vp, vp, vp, vp, i32, i32, i32]
    L.host_triangulate.restype = i32

    def run(xy, cons, order=0, width=1, check=True):
        xy = np.ascontiguousarray(xy, np.int32)
        cons = np.ascontiguousarray(cons, np.int32).reshape(-1, 2)
        n, s, T = len(xy), len(cons), 2 * len(xy) + 2
        tris = np.zeros((T, 3), np.int32)
        adj = np.zeros((T, 3), np.int32)
        cf = np.zeros(T, np.uint8)
        st = np.zeros(8, np.int64)
        p = lambda a: ctypes.c_void_p(a.ctypes.data)
        rc = L.host_triangulate(p(xy), n, p(cons), s, p(tris), p(adj), p(cf), p(st), order, int(width), int(check))
        return rc, tris, adj, cf, st
    return run


def _cases():
    R = (1 << 30) - 1
    rng = np.random.default_rng(3)
    xs = np.unique(rng.integers(1, R - 1, size=3000))
    diag = np.stack([xs, R - xs], 1)
    pts = np.unique(np.concatenate([diag, rng.integers(1, R - 1, size=(20000, 2))]).astype(np.int32), axis=0)
    return [
        ("diagonal+uniform", pts, np.zeros((0, 2), np.int32)),
        ("scale_200k", *g.generate(g.GEN_SCALE, 3, 200000, 8, 40)),
        ("lattice_256", *g.generate(g.GEN_LATTICE, 3, 256, 2000)),
        ("small_100k", *g.generate(g.GEN_SMALL, 3)),
        ("batch_instance", *g.generate(g.GEN_BATCH_INSTANCE, 7, 4000)),
    ]


@pytest.mark.parametrize("name,xy,cons", _cases(), ids=[c[0] for c in _cases()])
def test_host_emulation_matches_oracle_in_every_order(emu, name, xy, cons):
    runs = [emu(xy, cons, order, width) for order in (0, 1, 2) for width in (1, 2)]
    for rc, *_ in runs:
        assert rc == 0, "status %d (1000+: mesh check failed)" % rc
    ref = runs[0]
    for r in runs[1:]:
        for k in (1, 2, 3):
            assert np.array_equal(ref[k], r[k]), "output depends on item order or pairing"
        assert np.array_equal(ref[4][:5], r[4][:5])
    ok, msg = oracle.validate(xy, cons, ref[1], ref[2], ref[3])
    assert ok, msg
    orc, otris, _, _, _ = oracle.cdt(xy, cons)
    assert orc == 0
    assert np.array_equal(g.canonical(ref[1]), g.canonical(otris))


def record_accesses(npts, seed=1, defines=()):
    """Triangle records (the 32-byte vertex + adjacency row pair, read or
    written) each item touches, counted once per item, per point and phase
    kind, from the host run of the bodies on the scale workload's shape at
    `npts` generated points.  The host runs the GPU's schedule (same rounds,
    sub-rounds and flips), so this is the kernel's record-sector traffic if
    every touched record is one DRAM sector; the point, queue, claim and
    vote arrays come on top.  -> (n, {phase name: records per point},
    {phase name: items the phase ran over, per point}); the flip-queue
    outcomes per point are left in record_accesses.flip_outcomes."""
    L = ctypes.CDLL(build_host_emulation(defines))
    vp, i32 = ctypes.c_void_p, ctypes.c_int
    L.host_triangulate.argtypes = [vp, i32, vp, i32, vp, vp, vp, vp, i32, i32, i32]
    L.host_touch_counts.argtypes = [vp, vp]
    L.host_flip_outcomes.argtypes = [vp]
    gsz = max(2, int(round(56 * (npts / 10_000_000) ** 0.5)))
    xy, cons = g.generate(g.GEN_SCALE, seed, npts, gsz, int(gsz * gsz * 3125 / 3136))
    n, s, T = len(xy), len(cons), 2 * len(xy) + 2
    out = [np.zeros((T, 3), np.int32), np.zeros((T, 3), np.int32), np.zeros(T, np.uint8)]
    st = np.zeros(8, np.int64)
    cnt = np.zeros(64, np.int64)
    items = np.zeros(64, np.int64)
    fo = np.zeros(4, np.int64)
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    L.host_touch_counts(p(cnt), p(items))
    L.host_flip_outcomes(p(fo))
    rc = L.host_triangulate(p(xy), n, p(cons), s, p(out[0]), p(out[1]), p(out[2]), p(st), 0, 2, 0)
    L.host_touch_counts(p(cnt), p(items))
    L.host_flip_outcomes(p(fo))
    assert rc == 0
    names, per_item = {}, {}
    for k in range(63):
        nm = g.lib().gcdt_phase_name(k)
        if cnt[k]:
            key = nm.decode() if nm else "kind %d" % k
            names[key] = cnt[k] / n
            per_item[key] = items[k] / n
    if cnt[63]:
        names["outside phases"] = cnt[63] / n
    record_accesses.flip_outcomes = {"entries": fo[0] / n, "with_candidate": fo[1] / n,
                                     "distinct_candidates": fo[2] / n, "flips": fo[3] / n}
    return n, names, per_item


def test_record_accesses_per_point():
    """Traffic guard: the scale workload's shape at 200k points touches
    about 57 triangle records per point (1.8 KB at one 32-byte sector each;
    ncu measured 2.76 KB/point of DRAM traffic at 1.02M points, the point,
    queue, claim and vote arrays included), two thirds of them in the flip
    passes.  A change that adds re-reads shows up here first.  Run with -s
    to print the table."""
    n, acc, items = record_accesses(200000)
    total = sum(acc.values())
    for k, v in sorted(acc.items(), key=lambda kv: -kv[1]):
        it = items.get(k, 0)
        print("%-16s %6.1f accesses/point  %6.2f items/point  %5.1f accesses/item" % (
            k, v, it, v / it if it else 0))
    print("total %.1f accesses/point (%d points)" % (total, n))
    fo = record_accesses.flip_outcomes
    print("flip queue per point: %.2f entries, %.2f with a candidate edge, %.2f distinct candidate "
          "edges, %.2f flips" % (fo["entries"], fo["with_candidate"], fo["distinct_candidates"], fo["flips"]))
    assert 40 < total < 80
    assert fo["flips"] <= fo["distinct_candidates"] <= fo["with_candidate"] <= fo["entries"]
    flips = acc.get("flip_check", 0) + acc.get("flip_do", 0) + acc.get("flip_fix", 0)
    assert 0.5 < flips / total < 0.75


def _hilbert_index(x, y, n=1 << 30):
    """Hilbert index of cell (x, y) of an n x n grid by the usual quadrant
    rotation: the quadrant digit (3*rx) ^ ry per level from the top, and a
    lower quadrant (ry = 0) reflects (when rx = 1) and transposes the rest."""
    d, s = 0, n // 2
    while s > 0:
        rx, ry = int(x & s > 0), int(y & s > 0)
        d += s * s * ((3 * rx) ^ ry)
        if ry == 0:
            if rx == 1:
                x, y = n - 1 - x, n - 1 - y
            x, y = y, x
        s //= 2
    return d


def test_sort_keys_are_the_hilbert_index():
    """The key the points are sorted by equals the Hilbert index of the
    point's 30-bit coordinates, and in a 64 x 64 corner consecutive keys are
    neighbouring cells (the curve's defining property)."""
    L = ctypes.CDLL(build_host_emulation())
    L.host_sort_keys.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    rng = np.random.default_rng(3)
    xy = np.concatenate([rng.integers(0, 1 << 30, (3000, 2)),
                         rng.integers(0, 64, (200, 2)),
                         [[0, 0], [(1 << 30) - 1, (1 << 30) - 1], [0, (1 << 30) - 1], [(1 << 30) - 1, 0]]]
                        ).astype(np.int32)
    keys = np.zeros(len(xy), np.uint64)
    L.host_sort_keys(xy.ctypes.data, len(xy), keys.ctypes.data)
    want = [_hilbert_index(int(x), int(y)) for x, y in xy]
    assert keys.tolist() == want
    g64 = np.array([(x, y) for x in range(64) for y in range(64)], np.int32)
    k64 = np.zeros(len(g64), np.uint64)
    L.host_sort_keys(g64.ctypes.data, len(g64), k64.ctypes.data)
    path = g64[np.argsort(k64)]
    assert sorted(k64.tolist()) == list(range(64 * 64))
    assert (np.abs(np.diff(path, axis=0)).sum(axis=1) == 1).all()
