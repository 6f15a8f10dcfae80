"""GPU edge cases: empty and tiny inputs, degenerate geometry, error codes,
and the full-size workload through size-independent properties."""
import numpy as np
import pytest

import gcdt_b200 as g
from oracle import oracle
from tests.test_gpu_parity import canonical_with_flags, check_against_oracle

pytestmark = pytest.mark.gpu


def test_empty_input(triangulator):
    tris, adj, cf = triangulator.triangulate_host(np.zeros((0, 2), np.int32), None)
    assert len(tris) == 2
    ok, msg = oracle.validate(np.zeros((0, 2), np.int32), None, tris, adj, cf)
    assert ok, msg


@pytest.mark.parametrize("n", [1, 2, 3, 5])
def test_tiny_inputs(triangulator, n):
    rng = np.random.default_rng(n)
    xy = rng.choice(1 << 20, size=(n, 2), replace=False).astype(np.int32) + 1
    check_against_oracle(triangulator, xy, np.zeros((0, 2), np.int32))


def test_collinear_points(triangulator):
    xy = np.array([(1000 + 37 * i, 2000 + 11 * i) for i in range(500)], np.int32)
    check_against_oracle(triangulator, xy, np.zeros((0, 2), np.int32))


def test_points_on_root_diagonal(triangulator):
    R = (1 << 30) - 1
    xs = np.unique(np.random.default_rng(3).integers(1, R - 1, size=2000))
    xy = np.stack([xs, R - xs], axis=1).astype(np.int32)
    xy = np.concatenate([xy, np.random.default_rng(4).integers(1, R - 1, size=(2000, 2)).astype(np.int32)])
    xy = np.unique(xy, axis=0)
    check_against_oracle(triangulator, xy, np.zeros((0, 2), np.int32))


def test_segment_through_collinear_points(triangulator):
    rng = np.random.default_rng(5)
    line = np.array([(100000 + 1000 * i, 200000 + 700 * i) for i in range(50)], np.int32)
    other = rng.integers(1, 1 << 22, size=(3000, 2)).astype(np.int32)
    xy = np.unique(np.concatenate([line, other]), axis=0)
    idx = {tuple(p): i for i, p in enumerate(xy.tolist())}
    cons = np.array([[idx[tuple(line[0])], idx[tuple(line[-1])]],
                     [idx[tuple(line[3])], idx[tuple(line[20])]]], np.int32)
    check_against_oracle(triangulator, xy, cons)


def test_lattice_with_unit_segments(triangulator):
    xy, cons = g.generate(g.GEN_LATTICE, 3, 128, 1500)
    check_against_oracle(triangulator, xy, cons)


def test_duplicate_segments_are_harmless(triangulator):
    xy, cons = g.generate(g.GEN_BATCH_INSTANCE, 21, 2000)
    cons2 = np.concatenate([cons, cons[:, ::-1], cons[:10]])
    tris, adj, cf = triangulator.triangulate_host(xy, cons2)
    rc, otris, oadj, ocf, _ = oracle.cdt(xy, cons)
    assert np.array_equal(canonical_with_flags(tris, cf), canonical_with_flags(otris, ocf))


def _status(tri, xy, cons):
    try:
        tri.triangulate_host(xy, cons)
    except g.GcdtError as e:
        return e.status
    return "OK"


def test_error_codes(triangulator):
    ok = np.array([[10, 10], [20, 20], [30, 10], [20, 5]], np.int32)
    assert _status(triangulator, ok, None) == "OK"
    assert _status(triangulator, np.array([[10, 10], [10, 10]], np.int32), None) == "BAD_INPUT"
    assert _status(triangulator, np.array([[0, 10], [20, 20]], np.int32), None) == "BAD_INPUT"
    assert _status(triangulator, np.array([[(1 << 30) - 1, 10]], np.int32), None) == "BAD_INPUT"
    assert _status(triangulator, ok, np.array([[0, 4]], np.int32)) == "BAD_INPUT"
    assert _status(triangulator, ok, np.array([[2, 2]], np.int32)) == "BAD_INPUT"
    crossing = np.array([[10, 10], [30, 30], [10, 30], [30, 10]], np.int32)
    assert _status(triangulator, crossing, np.array([[0, 1], [2, 3]], np.int32)) == "CONSTRAINT_FAIL"
    # the context keeps working after errors
    check_against_oracle(triangulator, *g.generate(g.GEN_BATCH_INSTANCE, 2, 500))


def test_problem_larger_than_context():
    tri = g.Triangulator(max_points=100, max_segments=4)
    xy = np.random.default_rng(1).choice(1 << 20, size=(101, 2), replace=False).astype(np.int32) + 1
    assert _status(tri, xy, None) == "OOM"
    tri.close()


def test_full_scale_workload_properties():
    """10M points + 200k segments: the exact validator (size independent)
    plus determinism across two runs."""
    xy, cons = g.generate(g.GEN_SCALE, 1)
    tri = g.Triangulator(max_points=len(xy), max_segments=len(cons))
    tris, adj, cf = tri.triangulate_host(xy, cons)
    assert len(tris) == 2 * len(xy) + 2
    ok, msg = oracle.validate(xy, cons, tris, adj, cf)
    assert ok, msg
    st = tri.stats()
    assert st["n_triangles"] == 2 * len(xy) + 2
    tris2, adj2, cf2 = tri.triangulate_host(xy, cons)
    assert np.array_equal(tris, tris2) and np.array_equal(adj, adj2) and np.array_equal(cf, cf2)
    tri.close()
    # the oracle's own CDT of the same 10.2M + 200k instance (about 8 s on
    # one core): canonical triangle set with the flags rotated along
    rc, otris, _, ocf, _ = oracle.cdt(xy, cons)
    assert rc == 0
    assert np.array_equal(canonical_with_flags(tris, cf), canonical_with_flags(otris, ocf))


def test_full_size_lattice_config():
    """The degenerate lattice workload at full size: a 2048 x 2048 lattice of
    spacing 2^14 offset by (2^14, 2^14), N = 4,194,304, with 20,000 unit
    constraint segments on the sides of disjoint lattice rectangles.  Every
    empty circle through four lattice neighbours is a tie, which the shared
    symbolic perturbation resolves; the reference keeps whatever diagonal it
    had (strict inCircle > 0, kernel.cu:2218-2219), so its count 2N+2 and
    the exact validator are what it pins, and the oracle pins the set."""
    xy, cons = g.generate(g.GEN_LATTICE, 1)
    assert len(xy) == 2048 * 2048 and len(cons) == 20000
    tri = g.Triangulator(max_points=len(xy), max_segments=len(cons))
    tris, adj, cf = tri.triangulate_host(xy, cons)
    tri.close()
    assert len(tris) == 2 * len(xy) + 2
    ok, msg = oracle.validate(xy, cons, tris, adj, cf)
    assert ok, msg
    rc, otris, _, ocf, _ = oracle.cdt(xy, cons)
    assert rc == 0
    assert np.array_equal(canonical_with_flags(tris, cf), canonical_with_flags(otris, ocf))
