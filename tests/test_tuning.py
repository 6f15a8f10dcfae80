"""Scheduling of the solve (gcdt_set_tuning): insertion levels and their
strides, the flip-queue carry threshold and the single-block thresholds.
The constrained Delaunay triangulation is unique under the fixed tie-break,
so every valid schedule must give the same triangle set as the oracle.  CPU
tests run the stage driver on the host (tests/host_emulation.cu) under
several schedules; GPU tests do the same through the C ABI."""
import ctypes

import numpy as np
import pytest

import gcdt_b200 as g
from oracle import oracle

SCHEDULES = [
    # levels, strides, carry, narrow queue, narrow active
    (3, (512, 8, 1), 1 << 22, 1024, 1024),      # the defaults
    (1, (1, 1, 1), 0, 0, 0),                    # one level, no carry, never one block
    (2, (64, 1, 1), 256, 64, 4096),
    (4, (1024, 128, 16), 1 << 24, 65536, 0),
]


@pytest.fixture(scope="module")
def host():
    from tests.test_host_emulation import build_host_emulation
    L = ctypes.CDLL(build_host_emulation())
    vp, i32 = ctypes.c_void_p, ctypes.c_int
    L.host_triangulate.argtypes = [vp, i32, vp, i32, vp, vp, vp, vp, i32, i32, i32]
    L.host_triangulate.restype = i32
    L.host_set_tuning.argtypes = [i32] * 7
    L.host_set_tuning.restype = None

    def run(xy, cons, sched):
        lv, st, carry, nq, na = sched
        L.host_set_tuning(lv, st[0], st[1], st[2], carry, nq, na)
        n, s, T = len(xy), len(cons), 2 * len(xy) + 2
        xy = np.ascontiguousarray(xy, np.int32)
        cons = np.ascontiguousarray(cons, np.int32).reshape(-1, 2)
        out = (np.zeros((T, 3), np.int32), np.zeros((T, 3), np.int32), np.zeros(T, np.uint8))
        stats = np.zeros(8, np.int64)
        p = lambda a: ctypes.c_void_p(a.ctypes.data)
        rc = L.host_triangulate(p(xy), n, p(cons), s, p(out[0]), p(out[1]), p(out[2]), p(stats), 2, 2, 1)
        L.host_set_tuning(0, 0, 0, 0, 0, 0, 0)
        return rc, out
    return run


@pytest.mark.parametrize("sched", SCHEDULES, ids=["default", "flat", "two_level", "four_level"])
@pytest.mark.parametrize("case", ["small", "lattice"])
def test_schedules_on_host_give_the_oracle_cdt(host, case, sched):
    xy, cons = g.generate(g.GEN_SMALL, 8, 20000) if case == "small" else g.generate(g.GEN_LATTICE, 4, 96, 800)
    rc, (tris, adj, cf) = host(xy, cons, sched)
    assert rc == 0
    ok, msg = oracle.validate(xy, cons, tris, adj, cf)
    assert ok, msg
    orc, otris, _, _, _ = oracle.cdt(xy, cons)
    assert orc == 0 and np.array_equal(g.canonical(tris), g.canonical(otris))


@pytest.mark.gpu
def test_schedules_on_gpu_give_the_same_cdt():
    xy, cons = g.generate(g.GEN_SCALE, 7, 400000, 8, 50)
    tri = g.Triangulator(max_points=len(xy), max_segments=len(cons))
    assert tri.tuning() == {"levels": 3, "level_stride": [512, 8], "carry_queue": 1 << 22,
                            "narrow_queue": 1024, "narrow_active": 1024}
    ref = g.canonical(tri.triangulate_host(xy, cons)[0])
    for lv, st, carry, nq, na in SCHEDULES[1:]:
        tri.set_tuning(levels=lv, level_stride=st, carry_queue=carry, narrow_queue=nq, narrow_active=na)
        tris, adj, cf = tri.triangulate_host(xy, cons)
        assert np.array_equal(g.canonical(tris), ref), (lv, st)
    tri.set_tuning()
    assert tri.tuning()["levels"] == 3
    tri.close()


@pytest.mark.gpu
def test_autotune_keeps_a_candidate_and_the_cdt():
    import torch
    xy, cons = g.generate(g.GEN_SCALE, 8, 300000, 8, 40)
    tri = g.Triangulator(max_points=len(xy), max_segments=len(cons))
    d_xy, d_c = torch.from_numpy(xy).cuda(), torch.from_numpy(cons).cuda()
    ref = g.canonical(tri.triangulate(d_xy, d_c)[0].cpu().numpy())
    chosen = tri.autotune(d_xy, d_c, repeats=1)
    assert chosen == tri.tuning() and 2 <= chosen["levels"] <= 3
    tris = tri.triangulate(d_xy, d_c)[0].cpu().numpy()
    assert np.array_equal(g.canonical(tris), ref)
    tri.close()


def test_tuning_is_validated_without_a_device():
    L = g.lib()
    assert g.STATUS[L.gcdt_set_tuning(None, None)] == "BAD_INPUT"
    assert g.STATUS[L.gcdt_get_tuning(None, None)] == "BAD_INPUT"
    assert g.STATUS[L.gcdt_autotune(None, None, 0, None, 0, None, None, None, 1, None, None)] == "BAD_INPUT"


@pytest.mark.gpu
@pytest.mark.parametrize("blocks", [1, 37, 100])
def test_grid_share_gives_the_same_bytes(blocks):
    """gcdt_set_grid_blocks: a context whose persistent kernel runs on a
    share of the SMs (as the server's large-request workers do) returns the
    same bytes as one on the whole GPU: the phases' results do not depend
    on how their items are spread over blocks."""
    xy, cons = g.generate(g.GEN_SCALE, 6, 200000, 8, 40)
    full = g.Triangulator(max_points=len(xy), max_segments=len(cons))
    part = g.Triangulator(max_points=len(xy), max_segments=len(cons))
    part.set_grid_blocks(blocks)
    a = full.triangulate_host(xy, cons)
    b = part.triangulate_host(xy, cons)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    full.close()
    part.close()
