"""Failure detection without a GPU fault.

Every device loop of a solve is bounded, and a bound that runs out ends the
solve with a status the host reads (GCDT_ITER_LIMIT) instead of hanging or
dropping work silently, as the reference does with its fixed caps
(kernel.cu:3667, addConstraints.cu:769-773).  The tests shrink the budgets
(gcdt_set_limits) below what a solve needs and check that the solve stops
with that status, and that the same context then solves correctly with the
budgets restored.  The grid barrier's own wait is bounded too: a probe runs
one barrier with a block that never arrives and checks that the waits run
out, record their status and end.  No test faults, traps or hangs a GPU.
"""
import ctypes

import numpy as np
import pytest

import gcdt_b200 as g
from oracle import oracle

ST_ITER_LIMIT = 4       # status bit of the stage driver (mesh.cuh)


@pytest.fixture(scope="module")
def host():
    from tests.test_host_emulation import build_host_emulation
    L = ctypes.CDLL(build_host_emulation())
    vp, i32 = ctypes.c_void_p, ctypes.c_int
    L.host_triangulate.argtypes = [vp, i32, vp, i32, vp, vp, vp, vp, i32, i32, i32]
    L.host_triangulate.restype = i32
    L.host_set_limits.argtypes = [i32, i32, i32]
    L.host_set_limits.restype = None

    def run(xy, cons, limits=(0, 0, 0)):
        L.host_set_limits(*limits)
        n, s, T = len(xy), len(cons), 2 * len(xy) + 2
        xy = np.ascontiguousarray(xy, np.int32)
        cons = np.ascontiguousarray(cons, np.int32).reshape(-1, 2)
        tris = np.zeros((T, 3), np.int32)
        adj = np.zeros((T, 3), np.int32)
        cf = np.zeros(T, np.uint8)
        st = np.zeros(8, np.int64)
        p = lambda a: ctypes.c_void_p(a.ctypes.data)
        rc = L.host_triangulate(p(xy), n, p(cons), s, p(tris), p(adj), p(cf), p(st), 0, 2, 0)
        L.host_set_limits(0, 0, 0)
        return rc, (tris, adj, cf), st
    return run


def _workload():
    return g.generate(g.GEN_SMALL, 6, 30000)


def test_budgets_on_host_stop_the_solve_and_restore(host):
    xy, cons = _workload()
    rc, mesh, st = host(xy, cons)
    assert rc == 0
    rounds, crounds = int(st[1]), int(st[4])
    assert rounds > 2 and crounds >= 1
    # each budget just below what the solve needs ends it with ITER_LIMIT
    for lim in [(rounds - 1, 0, 0), (0, 1, 0)] + ([(0, 0, crounds - 1)] if crounds > 1 else []):
        rc, _, _ = host(xy, cons, lim)
        assert rc == ST_ITER_LIMIT, lim
    # a budget that suffices changes nothing
    rc2, mesh2, _ = host(xy, cons, (rounds + 8, 0, crounds))
    assert rc2 == 0 and all(np.array_equal(a, b) for a, b in zip(mesh, mesh2))
    ok, msg = oracle.validate(xy, cons, *mesh)
    assert ok, msg


@pytest.mark.gpu
def test_budgets_on_gpu_stop_the_solve_and_context_stays_usable():
    xy, cons = _workload()
    tri = g.Triangulator(max_points=len(xy), max_segments=len(cons))
    tris, adj, cf = tri.triangulate_host(xy, cons)
    st = tri.stats()
    for lim in [dict(insertion_rounds=1), dict(flip_subrounds=1)]:
        tri.set_limits(**lim)
        with pytest.raises(g.GcdtError) as ei:
            tri.triangulate_host(xy, cons)
        assert ei.value.status == "ITER_LIMIT", lim
    tri.set_limits()
    t2, a2, c2 = tri.triangulate_host(xy, cons)
    tri.close()
    assert np.array_equal(t2, tris) and np.array_equal(a2, adj) and np.array_equal(c2, cf)
    rc, otris, _, _, _ = oracle.cdt(xy, cons)
    assert rc == 0 and np.array_equal(g.canonical(t2), g.canonical(otris))
    assert st["insertion_rounds"] > 1


@pytest.mark.gpu
def test_grid_barrier_wait_runs_out_and_the_device_stays_usable():
    # one block never arrives: the others' bounded waits run out
    assert g.probe_barrier(blocks=4, absent_block=0, spin_limit=1 << 14) is True
    assert g.probe_barrier(blocks=8, absent_block=5, spin_limit=1 << 14) is True
    # every block arrives: the barrier completes
    assert g.probe_barrier(blocks=8, absent_block=-1, spin_limit=1 << 20) is False
    # the device still solves
    xy, cons = g.generate(g.GEN_BATCH_INSTANCE, 9, 3000)
    tri = g.Triangulator(max_points=len(xy), max_segments=max(len(cons), 1))
    tris, adj, cf = tri.triangulate_host(xy, cons)
    tri.close()
    ok, msg = oracle.validate(xy, cons, tris, adj, cf)
    assert ok, msg


def test_limit_arguments_are_checked_without_a_device():
    L = g.lib()
    assert g.STATUS[L.gcdt_set_limits(None, 1, 1, 1)] == "BAD_INPUT"
    out = ctypes.c_int32(0)
    assert g.STATUS[L.gcdt_probe_barrier(0, 0, 0, 16, ctypes.byref(out))] == "BAD_INPUT"
    assert g.STATUS[L.gcdt_probe_barrier(0, 4, 0, 0, ctypes.byref(out))] == "BAD_INPUT"


@pytest.mark.gpu
def test_grid_barrier_cost_is_measured_and_bounded():
    """The persistent kernel's grid barrier, alone in a loop on a grid shaped
    like the stage kernel's: every wait completes (bounded polls) and one
    barrier costs a few microseconds, so a flip sub-round's three barriers
    are a small part of its time."""
    us = g.time_barriers(rounds=4096)
    print("grid barrier: %.2f us" % us)
    assert 0 < us < 50
