"""Serving: every result is the same alone and in a concurrent mix, equal to
the single solve; admission waits for memory instead of failing."""
import threading

import numpy as np
import pytest

import gcdt_b200 as g
from tests.test_gpu_parity import canonical_with_flags

pytestmark = pytest.mark.gpu


def _requests(k, seed0, cap):
    out = []
    for i in range(k):
        xy, cons = g.generate(g.GEN_SERVING_REQUEST, seed0 + i, 0)
        if len(xy) > cap:
            xy, cons = g.generate(g.GEN_SERVING_REQUEST, seed0 + i, cap)
        out.append((xy, cons))
    return out


def test_same_alone_and_in_the_mix():
    reqs = _requests(40, 700, cap=120_000)
    probe = reqs[7]
    sv = g.Server(memory_budget_bytes=24 << 30, lanes=3, max_batch_instances=64, max_batch_points=600_000,
                  max_batch_segments=30_000, big_request_points=90_000, max_request_points=130_000,
                  max_request_segments=10_000)
    rid = sv.submit(*probe)
    alone = sv.fetch(rid, len(probe[0]))
    # the mix: three client threads submit concurrently, the probe among them
    ids = [None] * len(reqs)

    def client(part):
        for i in part:
            ids[i] = sv.submit(*reqs[i])

    th = [threading.Thread(target=client, args=(range(k, len(reqs), 3),)) for k in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    results = [sv.fetch(ids[i], len(reqs[i][0])) for i in range(len(reqs))]
    for a, b in zip(alone, results[7]):
        assert np.array_equal(a, b)                      # byte for byte, alone vs in the mix
    single = g.Triangulator(max(len(x) for x, _ in reqs), max(len(c) for _, c in reqs))
    for (xy, cons), (t, a, c) in zip(reqs, results):
        st, sa, sc = single.triangulate_host(xy, cons)
        assert np.array_equal(canonical_with_flags(t, c), canonical_with_flags(st, sc))
    st = sv.stats()
    assert st["completed"] == len(reqs) + 1 and st["failed"] == 0
    assert st["batches"] >= 1 and st["big_solves"] >= 1
    single.close()
    sv.close()


def test_admission_waits_for_memory():
    reqs = _requests(12, 900, cap=40_000)
    # output pool sized for about three resident results at a time
    fixed = (g.workspace_bytes(90_000, 4_000) + g.workspace_bytes(45_000, 2_000) +
             8 * (90_000 + 4_000 + 45_000 + 2_000))
    budget = fixed + 3 * (2 * 45_000 + 2) * 25 + (1 << 20)
    sv = g.Server(memory_budget_bytes=budget, lanes=1, max_batch_instances=8, max_batch_points=90_000,
                  max_batch_segments=4_000, big_request_points=1 << 30, max_request_points=45_000,
                  max_request_segments=2_000)
    ids = [sv.submit(*r) for r in reqs]
    for i, rid in enumerate(ids):          # fetch in order; later requests get memory as earlier ones leave
        t, a, c = sv.fetch(rid, len(reqs[i][0]))
        assert len(t) == 2 * len(reqs[i][0]) + 2
    assert sv.stats()["completed"] == len(reqs)
    sv.close()


def _overlap(a, b):
    return max(a[0], b[0]) < min(a[1], b[1])


def test_work_of_different_requests_overlaps_on_the_device():
    """Continuous batching runs requests' work side by side: two small
    requests in different batches (so on two lanes), a small request and a
    large one (a lane and a single-solve worker), and two large requests
    (two workers, each on half of the SMs) are in flight at the same time,
    by the server's own start/completion times; every result equals the
    single solve."""
    small = _requests(36, 1300, cap=20_000)
    big = [g.generate(g.GEN_SERVING_REQUEST, 1400 + i, 150_000) for i in range(4)]
    sv = g.Server(memory_budget_bytes=24 << 30, lanes=3, max_batch_instances=4, max_batch_points=80_000,
                  max_batch_segments=8_000, big_request_points=100_000, max_request_points=200_000,
                  max_request_segments=10_000, big_workers=2)
    order = []
    for i in range(len(small)):
        order.append(("s", i))
        if i % 9 == 0:
            order.append(("b", i // 9))
    ids = {}
    for kind, i in order:
        ids[(kind, i)] = sv.submit(*(small[i] if kind == "s" else big[i]))
    times = {}
    for key, rid in ids.items():
        done, rc = sv.wait(rid)
        assert done and rc == 0
        sub, start, end = sv.times(rid)
        times[key] = (start, end)
    smalls = [times[("s", i)] for i in range(len(small))]
    bigs = [times[("b", i)] for i in range(len(big))]
    assert any(_overlap(a, b) for k, a in enumerate(smalls) for b in smalls[k + 1:] if a[0] != b[0])
    assert any(_overlap(a, b) for a in smalls for b in bigs)
    assert any(_overlap(a, b) for k, a in enumerate(bigs) for b in bigs[k + 1:])
    single = g.Triangulator(200_000, 10_000)
    for (kind, i), rid in ids.items():
        xy, cons = small[i] if kind == "s" else big[i]
        t, a, c = sv.fetch(rid, len(xy))
        st, sa, sc = single.triangulate_host(xy, cons)
        assert np.array_equal(canonical_with_flags(t, c), canonical_with_flags(st, sc))
    st = sv.stats()
    assert st["big_solves"] == len(big) and st["batches"] >= 3 and st["failed"] == 0
    single.close()
    sv.close()
