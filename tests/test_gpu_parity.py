"""GPU parity: the CUDA path through the C ABI against the oracle.

The bar is bit-exact: the canonical triangle set (and the constraint flags
rotated with it) must equal the oracle's, and the exact validator must pass
on the GPU output (orientation, adjacency, hull, Euler count, constraints,
local Delaunay under the shared tie-break)."""
import ctypes

import numpy as np
import pytest

import gcdt_b200 as g
from oracle import oracle

pytestmark = pytest.mark.gpu


def canonical_with_flags(tris, cflags):
    t = np.asarray(tris, np.int64).reshape(-1, 3)
    f = np.asarray(cflags, np.int64).reshape(-1)
    r = np.argmin(t, axis=1)
    idx = (np.arange(3)[None, :] + r[:, None]) % 3
    c = np.take_along_axis(t, idx, axis=1)
    bits = np.stack([(f >> k) & 1 for k in range(3)], axis=1)
    b = np.take_along_axis(bits, idx, axis=1)
    fl = b[:, 0] | (b[:, 1] << 1) | (b[:, 2] << 2)
    out = np.concatenate([c, fl[:, None]], axis=1)
    order = np.lexsort((out[:, 2], out[:, 1], out[:, 0]))
    return out[order]


def check_against_oracle(tri, xy, cons):
    tris, adj, cf = tri.triangulate_host(xy, cons)
    assert len(tris) == 2 * len(xy) + 2
    ok, msg = oracle.validate(xy, cons, tris, adj, cf)
    assert ok, msg
    rc, otris, oadj, ocf, _ = oracle.cdt(xy, cons)
    assert rc == 0
    assert np.array_equal(canonical_with_flags(tris, cf), canonical_with_flags(otris, ocf))
    return tris, adj, cf


CASES = [
    ("small_config", g.GEN_SMALL, 1, ()),
    ("small_config_seed2", g.GEN_SMALL, 2, ()),
    ("scale_mix_200k", g.GEN_SCALE, 1, (200000, 8, 40)),
    ("scale_mix_1m", g.GEN_SCALE, 2, (1000000, 18, 316)),
    ("lattice_256_2000", g.GEN_LATTICE, 1, (256, 2000)),
    ("lattice_1024_20000", g.GEN_LATTICE, 2, (1024, 20000)),
    ("serving_request_50k", g.GEN_SERVING_REQUEST, 3, (50000,)),
]


@pytest.mark.parametrize("name,kind,seed,args", CASES, ids=[c[0] for c in CASES])
def test_parity_workloads(triangulator, name, kind, seed, args):
    xy, cons = g.generate(kind, seed, *args)
    check_against_oracle(triangulator, xy, cons)


@pytest.mark.parametrize("seed", list(range(1, 9)))
def test_parity_batched_instances(triangulator, seed):
    xy, cons = g.generate(g.GEN_BATCH_INSTANCE, seed)
    check_against_oracle(triangulator, xy, cons)


def test_parity_without_constraints(triangulator):
    xy, _ = g.generate(g.GEN_SCALE, 5, 300000, 4, 0)
    check_against_oracle(triangulator, xy, np.zeros((0, 2), np.int32))


def test_golden_fixtures_on_gpu(triangulator):
    import hashlib
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "fixtures.json")) as f:
        fx = json.load(f)
    for case in fx["cases"]:
        xy, cons = g.generate(case["kind"], case["seed"], *case["args"])
        tris, adj, cf = triangulator.triangulate_host(xy, cons)
        h = hashlib.sha256(np.ascontiguousarray(g.canonical(tris), dtype=np.int64).tobytes()).hexdigest()
        assert h == case["tris_sha256"], case["name"]
    for case in fx["explicit"]:
        xy = np.array(case["points"], np.int32)
        cons = np.array(case["segments"], np.int32).reshape(-1, 2)
        tris, adj, cf = triangulator.triangulate_host(xy, cons)
        assert g.canonical(tris).tolist() == case["canonical_tris"], case["name"]


def test_deterministic_bytes(triangulator):
    xy, cons = g.generate(g.GEN_SCALE, 9, 400000, 8, 50)
    a = triangulator.triangulate_host(xy, cons)
    b = triangulator.triangulate_host(xy, cons)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_predicates_bit_equal_to_oracle():
    rng = np.random.default_rng(11)
    R = (1 << 30) - 1
    k = 200000
    q = rng.integers(0, R + 1, size=(k, 4, 2)).astype(np.int32)
    # near-degenerate: cocircular rectangles and collinear triples
    m = 20000
    base = rng.integers(0, R - 70000, size=(m, 2))
    w = rng.integers(1, 65536, size=(m, 2))
    zero = np.zeros(m, np.int64)
    rect = np.stack([base, base + np.stack([w[:, 0], zero], 1), base + w,
                     base + np.stack([zero, w[:, 1]], 1)], axis=1)
    perm = np.argsort(rng.random((m, 4)), axis=1)
    rect = np.take_along_axis(rect, perm[:, :, None], axis=1).astype(np.int32)
    t = rng.integers(1, 1000, size=(m, 1))
    d = rng.integers(-1000, 1000, size=(m, 2))
    col = np.stack([base, base + d, base + t * d, rng.integers(0, R, size=(m, 2))], axis=1)
    col = np.clip(col, 0, R).astype(np.int32)
    allq = np.concatenate([q, rect, col], axis=0)
    dev = g.eval_predicates(allq)
    sample = np.concatenate([np.arange(0, k, 37), np.arange(k, len(allq))])
    for i in sample:
        a, b, c, d4 = allq[i]
        assert dev[i, 0] == oracle.orient(a, b, c), i
        assert dev[i, 1] == oracle.incircle(a, b, c, d4), i
        assert dev[i, 2] == oracle.incircle_sos(a, b, c, d4), i


def test_predicates_bit_equal_on_1e8_cases():
    """10^8 seeded cases (uniform, tiny clusters, cocircular, collinear and
    one-unit perturbations of cocircular quads), in chunks of 10^7: the
    device's orient2d, inCircle and perturbed inCircle equal the exact
    oracle on every case."""
    from tests.predicate_cases import predicate_cases
    rng = np.random.default_rng(2026)
    zeros = 0
    for _ in range(10):
        q = predicate_cases(rng, 10_000_000)
        dev = g.eval_predicates(q)
        ref = oracle.predicates_batch(q)
        bad = np.nonzero((dev != ref).any(axis=1))[0]
        assert len(bad) == 0, (bad[:5], q[bad[:5]].tolist(), dev[bad[:5]].tolist(), ref[bad[:5]].tolist())
        zeros += int((ref[:, 1] == 0).sum())
    assert zeros > 10_000_000


@pytest.mark.gpu
@pytest.mark.parametrize("kind,seed,args", [(g.GEN_SCALE, 5, (200000, 8, 40)), (g.GEN_LATTICE, 6, (256, 2000))],
                         ids=["scale_200k", "lattice_256"])
def test_gpu_bytes_equal_host_run_of_the_same_bodies(triangulator, kind, seed, args):
    """The host run of the stage bodies (tests/host_emulation.cu) sorts the
    points with the host copy of the key function and follows the GPU's
    schedule; the output is independent of item order, so the device solve
    must give the same bytes: triangles, adjacency and flags in the same
    slots.  This pins the device's sort keys (a table in device memory) and
    every device body to the host's."""
    from tests.test_host_emulation import build_host_emulation
    L = ctypes.CDLL(build_host_emulation())
    vp, i32 = ctypes.c_void_p, ctypes.c_int
    L.host_triangulate.argtypes = [vp, i32, vp, i32, vp, vp, vp, vp, i32, i32, i32]
    L.host_triangulate.restype = i32
    xy, cons = g.generate(kind, seed, *args)
    xy = np.ascontiguousarray(xy, np.int32)
    cons = np.ascontiguousarray(cons, np.int32).reshape(-1, 2)
    T = 2 * len(xy) + 2
    host = (np.zeros((T, 3), np.int32), np.zeros((T, 3), np.int32), np.zeros(T, np.uint8))
    st = np.zeros(8, np.int64)
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    rc = L.host_triangulate(p(xy), len(xy), p(cons), len(cons), p(host[0]), p(host[1]), p(host[2]), p(st), 0, 2, 0)
    assert rc == 0
    dev = triangulator.triangulate_host(xy, cons)
    for a, b in zip(dev, host):
        assert np.array_equal(a, b)
