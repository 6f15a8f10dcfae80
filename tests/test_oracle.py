"""CPU tests of the oracle: predicates, global empty-circle property,
validator sensitivity, and the committed golden fixtures."""
import hashlib
import json
import os
import random

import numpy as np
import pytest

from oracle import oracle
from tests import bruteforce as bf
import gcdt_b200 as g

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _rand_pts(rng, n, lo=1, hi=(1 << 30) - 2):
    seen = set()
    out = []
    while len(out) < n:
        p = (rng.randint(lo, hi), rng.randint(lo, hi))
        if p not in seen:
            seen.add(p)
            out.append(p)
    return np.array(out, np.int32)


def test_predicates_match_python_ints():
    rng = random.Random(1)
    for _ in range(20000):
        pts = [(rng.randint(0, (1 << 30) - 1), rng.randint(0, (1 << 30) - 1)) for _ in range(4)]
        a, b, c, d = pts
        assert oracle.orient(a, b, c) == bf.orient(a, b, c)
        assert oracle.incircle(a, b, c, d) == bf.incircle(a, b, c, d)
        assert oracle.incircle_sos(a, b, c, d) == bf.incircle_sos(a, b, c, d)


def test_predicates_degenerate():
    rng = random.Random(2)
    R = (1 << 30) - 1
    cases = []
    # cocircular: lattice squares and rectangles, the box itself
    for _ in range(2000):
        x, y = rng.randint(0, R - 4096), rng.randint(0, R - 4096)
        w, h = rng.randint(1, 4095), rng.randint(1, 4095)
        sq = [(x, y), (x + w, y), (x + w, y + h), (x, y + h)]
        rng.shuffle(sq)
        cases.append(sq)
    cases.append([(0, 0), (R, 0), (R, R), (0, R)])
    # collinear triples with extreme coordinates
    for _ in range(2000):
        x, y = rng.randint(0, R // 2), rng.randint(0, R // 2)
        dx, dy = rng.randint(-1000, 1000), rng.randint(-1000, 1000)
        k = rng.randint(1, 1000)
        cases.append([(x, y), (x + dx, y + dy), (x + k * dx, y + k * dy), (rng.randint(0, R), rng.randint(0, R))])
    for a, b, c, d in cases:
        assert oracle.orient(a, b, c) == bf.orient(a, b, c)
        assert oracle.incircle(a, b, c, d) == bf.incircle(a, b, c, d)
        s = oracle.incircle_sos(a, b, c, d)
        assert s == bf.incircle_sos(a, b, c, d)
        if bf.orient(a, b, c) != 0:
            assert s != 0


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_unconstrained_bruteforce(seed):
    rng = random.Random(seed)
    xy = _rand_pts(rng, 120)
    rc, tris, adj, cf, _ = oracle.cdt(xy)
    assert rc == 0
    assert len(tris) == 2 * len(xy) + 2
    assert bf.check_empty_circles(xy, tris.tolist()) == []
    ok, msg = oracle.validate(xy, None, tris, adj, cf)
    assert ok, msg


def test_oracle_lattice_bruteforce():
    # maximal cocircularity: every unit square is cocircular
    side = 9
    xy = np.array([(1000 + 7 * i, 5000 + 7 * j) for j in range(side) for i in range(side)], np.int32)
    rc, tris, adj, cf, _ = oracle.cdt(xy)
    assert rc == 0
    assert bf.check_empty_circles(xy, tris.tolist()) == []
    ok, msg = oracle.validate(xy, None, tris, adj, cf)
    assert ok, msg


@pytest.mark.parametrize("seed", [4, 5])
def test_oracle_constrained_bruteforce(seed):
    xy, cons = g.generate(g.GEN_BATCH_INSTANCE, seed, 100)
    rc, tris, adj, cf, _ = oracle.cdt(xy, cons)
    assert rc == 0
    assert bf.check_empty_circles(xy, tris.tolist(), cons.tolist()) == []
    ok, msg = oracle.validate(xy, cons, tris, adj, cf)
    assert ok, msg


def test_validator_catches_planted_mistakes():
    xy, cons = g.generate(g.GEN_SMALL, 3, 3000)
    rc, tris, adj, cf, _ = oracle.cdt(xy, cons)
    assert rc == 0
    ok, _ = oracle.validate(xy, cons, tris, adj, cf)
    assert ok
    # 1. flip one unconstrained interior edge by hand: not locally Delaunay
    t2, a2 = tris.copy(), adj.copy()
    for t in range(len(t2)):
        i = 0
        n = a2[t, i]
        if n < 0 or cf[t] & 1:
            continue
        j = list(a2[n]).index(t)
        A, B, C = t2[t, 0], t2[t, 1], t2[t, 2]
        D = t2[n, j]
        if bf.orient(*(bf.with_corners(xy)[v] for v in (A, B, D))) <= 0:
            continue
        if bf.orient(*(bf.with_corners(xy)[v] for v in (A, D, C))) <= 0:
            continue
        nCA, nAB = a2[t, 1], a2[t, 2]
        nBD, nDC = a2[n, (j + 1) % 3], a2[n, (j + 2) % 3]
        t2[t] = (A, B, D); a2[t] = (nBD, n, nAB)
        t2[n] = (A, D, C); a2[n] = (nDC, nCA, t)
        for m, old, new in ((nBD, n, t), (nCA, t, n)):
            if m >= 0:
                a2[m][list(a2[m]).index(old)] = new
        break
    ok, msg = oracle.validate(xy, cons, t2, a2, np.zeros_like(cf))
    assert not ok
    # 2. drop one constraint flag pair
    cf2 = cf.copy()
    t = int(np.nonzero(cf2)[0][0])
    bit = int(cf2[t]) & -int(cf2[t])
    cf2[t] = int(cf2[t]) & ~bit & 0xFF
    ok, msg = oracle.validate(xy, cons, tris, adj, cf2)
    assert not ok
    # 3. reverse one triangle
    t3 = tris.copy()
    t3[5] = t3[5][::-1]
    ok, msg = oracle.validate(xy, cons, t3, adj, cf)
    assert not ok


def test_oracle_rejects_bad_input():
    xy = np.array([[10, 10], [20, 20], [10, 10]], np.int32)
    assert oracle.cdt(xy)[0] == 1
    xy = np.array([[0, 10], [20, 20]], np.int32)
    assert oracle.cdt(xy)[0] == 1
    xy = np.array([[10, 10], [20, 20], [30, 10], [20, 5]], np.int32)
    assert oracle.cdt(xy, np.array([[0, 4]], np.int32))[0] == 1
    # crossing segments
    xy = np.array([[10, 10], [30, 30], [10, 30], [30, 10]], np.int32)
    assert oracle.cdt(xy, np.array([[0, 1], [2, 3]], np.int32))[0] == 4


def test_oracle_splits_segment_at_collinear_vertex():
    xy = np.array([[100, 100], [200, 200], [300, 300], [150, 400], [250, 50]], np.int32)
    cons = np.array([[0, 2]], np.int32)
    rc, tris, adj, cf, _ = oracle.cdt(xy, cons)
    assert rc == 0
    ok, msg = oracle.validate(xy, cons, tris, adj, cf)
    assert ok, msg
    assert int(sum(bin(int(f)).count("1") for f in cf)) == 4   # edges (0,1),(1,2), both sides


def _sha(arr):
    return hashlib.sha256(np.ascontiguousarray(arr, dtype=np.int64).tobytes()).hexdigest()


def test_golden_fixtures():
    with open(os.path.join(GOLDEN, "fixtures.json")) as f:
        fx = json.load(f)
    for case in fx["cases"]:
        xy, cons = g.generate(case["kind"], case["seed"], *case["args"])
        assert len(xy) == case["n"] and len(cons) == case["s"], case["name"]
        assert _sha(xy) == case["input_sha256"], case["name"]
        rc, tris, adj, cf, _ = oracle.cdt(xy, cons)
        assert rc == 0
        assert _sha(g.canonical(tris)) == case["tris_sha256"], case["name"]
    for case in fx["explicit"]:
        xy = np.array(case["points"], np.int32)
        cons = np.array(case["segments"], np.int32).reshape(-1, 2)
        rc, tris, adj, cf, _ = oracle.cdt(xy, cons)
        assert rc == 0
        assert g.canonical(tris).tolist() == case["canonical_tris"], case["name"]


def test_batched_predicates_equal_python_ints():
    """oracle.predicates_batch (the checker of the device predicates on
    10^8 cases) against independent Python-integer arithmetic."""
    from tests.predicate_cases import predicate_cases
    q = predicate_cases(np.random.default_rng(5), 6000)
    out = oracle.predicates_batch(q)
    for i in range(len(q)):
        a, b, c, d = (tuple(int(v) for v in p) for p in q[i])
        assert out[i, 0] == bf.orient(a, b, c)
        assert out[i, 1] == bf.incircle(a, b, c, d)
        assert out[i, 2] == bf.incircle_sos(a, b, c, d)
    assert (out[:, 1] == 0).sum() > 1000          # the degenerate shapes are present
