"""Parity against the reference's own CUDA build.

tests/golden/reference_fixtures.json was produced by running the reference's
device pipeline (yingtix/gCDT, kernel.cu:5398-5443, built for sm_100a by
oracle/build_ref.sh; script oracle/make_reference_fixtures.py) on seeded
inputs.  Cases where the reference's output is complete (final Delaunay
self-check mark == 0, no ignored constraint, 2n+2 triangles) are "pinned":
the canonical triangle set must be identical, bit for bit, for the oracle
(CPU test) and for the CUDA path (GPU test).  The other cases record where
the reference drops constraints; they are not parity targets.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import gcdt_b200 as g
from oracle import oracle

FIX = os.path.join(os.path.dirname(__file__), "golden", "reference_fixtures.json")


def _cases(pinned=True, max_n=None):
    with open(FIX) as f:
        fx = json.load(f)
    out = []
    for c in fx["cases"]:
        if c["pinned"] != pinned:
            continue
        if max_n is not None and c["n"] > max_n:
            continue
        out.append(c)
    return out


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.int64).tobytes()).hexdigest()


def _input(c):
    xy, cons = g.generate(c["kind"], c["seed"], *c["args"])
    if c["drop_segments"]:
        cons = cons[:0]
    assert len(xy) == c["n"] and len(cons) == c["s"]
    assert _sha(xy) == c["input_sha256"], "generator drifted from the fixture"
    return xy, cons


def test_fixture_file_is_consistent():
    pinned = _cases(True)
    assert len(pinned) >= 4
    for c in pinned:
        assert c["ref_mark"] == 0 and c["ref_ignored"] == 0 and c["ref_ntri"] == 2 * c["n"] + 2


@pytest.mark.parametrize("case", _cases(True, max_n=1_000_000), ids=lambda c: c["name"])
def test_oracle_equals_reference(case):
    xy, cons = _input(case)
    rc, tris, adj, cf, _ = oracle.cdt(xy, cons)
    assert rc == 0
    assert _sha(g.canonical(tris)) == case["tris_sha256"]


@pytest.mark.gpu
@pytest.mark.parametrize("case", _cases(True), ids=lambda c: c["name"])
def test_gpu_equals_reference(case):
    xy, cons = _input(case)
    tri = g.Triangulator(max_points=len(xy), max_segments=max(len(cons), 1))
    tris, adj, cf = tri.triangulate_host(xy, cons)
    tri.close()
    assert _sha(g.canonical(tris)) == case["tris_sha256"]
