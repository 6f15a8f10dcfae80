"""Regenerate tests/golden/fixtures.json.

The reference (yingtix/gCDT) ships no tests, fixtures or data, so these
fixtures are produced here: seeded inputs from gcdt_b200's generators, and
the canonical triangle set the oracle computes for them.  Every explicit
(small) case is accepted only after the independent brute-force
empty-circumcircle check in tests/bruteforce.py passes on it, and every
case only after the exact validator passes.  The input hash guards the
generators; the triangle hash guards the oracle and, through the GPU
parity tests, the CUDA path.

    python tests/golden/make_fixtures.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import gcdt_b200 as g  # noqa: E402
from oracle import oracle  # noqa: E402
from tests import bruteforce as bf  # noqa: E402


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.int64).tobytes()).hexdigest()


CASES = [
    ("small_config_default", g.GEN_SMALL, 1, [0]),
    ("small_config_seed2", g.GEN_SMALL, 2, [0]),
    ("scale_mix_200k", g.GEN_SCALE, 1, [200000, 8, 40]),
    ("lattice_256", g.GEN_LATTICE, 1, [256, 2000]),
    ("batch_instance_5000", g.GEN_BATCH_INSTANCE, 1, [5000]),
    ("serving_request_20000", g.GEN_SERVING_REQUEST, 1, [20000]),
]


def explicit_cases():
    out = []
    rng = np.random.default_rng(7)
    # tiny general-position set
    xy = rng.integers(1, (1 << 30) - 2, size=(40, 2)).astype(np.int32)
    out.append(("random_40", xy, np.zeros((0, 2), np.int32)))
    # lattice 6x6 (cocircular everywhere) with a 2x1 rectangle boundary
    xy = np.array([(5000 + 16 * i, 9000 + 16 * j) for j in range(6) for i in range(6)], np.int32)
    cons = np.array([[7, 8], [8, 9], [9, 15], [15, 14], [14, 13], [13, 7]], np.int32)
    out.append(("lattice_6x6_rect", xy, cons))
    # a segment through collinear points (split into a chain)
    xy = np.array([[100, 100], [200, 200], [300, 300], [400, 400], [150, 420], [260, 40], [90, 310]], np.int32)
    out.append(("collinear_chain", xy, np.array([[0, 3]], np.int32)))
    # batched-style instance with two star polygons
    xy, cons = g.generate(g.GEN_BATCH_INSTANCE, 11, 80)
    out.append(("stars_80", xy, cons))
    return out


def main():
    fx = {"generator": "gcdt_b200/csrc/gen.cpp", "oracle": "oracle/cdt_oracle.c", "cases": [], "explicit": []}
    for name, kind, seed, args in CASES:
        xy, cons = g.generate(kind, seed, *args)
        rc, tris, adj, cf, _ = oracle.cdt(xy, cons)
        assert rc == 0, name
        ok, msg = oracle.validate(xy, cons, tris, adj, cf)
        assert ok, (name, msg)
        fx["cases"].append({"name": name, "kind": kind, "seed": seed, "args": args,
                            "n": int(len(xy)), "s": int(len(cons)),
                            "input_sha256": sha(xy), "tris_sha256": sha(g.canonical(tris))})
    for name, xy, cons in explicit_cases():
        rc, tris, adj, cf, _ = oracle.cdt(xy, cons)
        assert rc == 0, name
        ok, msg = oracle.validate(xy, cons, tris, adj, cf)
        assert ok, (name, msg)
        assert bf.check_empty_circles(xy, tris.tolist(), cons.tolist()) == [], name
        fx["explicit"].append({"name": name, "points": xy.tolist(), "segments": cons.tolist(),
                               "canonical_tris": g.canonical(tris).tolist()})
    with open(os.path.join(HERE, "fixtures.json"), "w") as f:
        json.dump(fx, f, indent=1)
    print("wrote", len(fx["cases"]), "cases and", len(fx["explicit"]), "explicit cases")


if __name__ == "__main__":
    main()
