"""Batched triangulation: every instance's output equals the single solve's
(same canonical triangle set with constraint flags, valid CDT), errors stay
confined to their instance, and the autotuner picks a valid configuration."""
import numpy as np
import pytest

import gcdt_b200 as g
from oracle import oracle
from tests.test_gpu_parity import canonical_with_flags

pytestmark = pytest.mark.gpu


def _instances(k, seed0=100, cap=20000):
    out = []
    for i in range(k):
        xy, cons = g.generate(g.GEN_BATCH_INSTANCE, seed0 + i)
        if len(xy) > cap:
            xy, cons = g.generate(g.GEN_BATCH_INSTANCE, seed0 + i, cap)
        out.append((xy, cons))
    return out


@pytest.mark.parametrize("cfg", [(256, 64), (128, 16), (512, 256)])
def test_batch_equals_single_solves(cfg):
    inst = _instances(48)
    po, so = g.BatchTriangulator.offsets(inst)
    bt = g.BatchTriangulator(len(inst), int(po[-1]), int(so[-1]))
    bt.set_config(*cfg)
    res = bt.triangulate(inst)
    single = g.Triangulator(max(len(x) for x, _ in inst), max(len(c) for _, c in inst))
    for i, ((xy, cons), r) in enumerate(zip(inst, res)):
        assert not isinstance(r, Exception), (i, r)
        tris, adj, cf = r
        ok, msg = oracle.validate(xy, cons, tris, adj, cf)
        assert ok, (i, msg)
        st, sa, sc = single.triangulate_host(xy, cons)
        assert np.array_equal(canonical_with_flags(tris, cf), canonical_with_flags(st, sc)), i
    single.close()
    bt.close()


def test_batch_matches_oracle_and_isolates_errors():
    inst = _instances(12, seed0=300)
    bad_xy = np.array([[10, 10], [20, 20], [10, 10]], np.int32)          # duplicate point
    cross = (np.array([[10, 10], [30, 30], [10, 30], [30, 10]], np.int32),
             np.array([[0, 1], [2, 3]], np.int32))                         # crossing segments
    inst = inst[:5] + [(bad_xy, np.zeros((0, 2), np.int32))] + inst[5:9] + [cross] + inst[9:]
    po, so = g.BatchTriangulator.offsets(inst)
    bt = g.BatchTriangulator(len(inst), int(po[-1]), int(so[-1]))
    res = bt.triangulate(inst)
    for i, ((xy, cons), r) in enumerate(zip(inst, res)):
        if i == 5:
            assert isinstance(r, g.GcdtError) and r.status == "BAD_INPUT"
            continue
        if i == 10:
            assert isinstance(r, g.GcdtError) and r.status == "CONSTRAINT_FAIL"
            continue
        assert not isinstance(r, Exception), (i, r)
        rc, ot, oa, oc, _ = oracle.cdt(xy, cons)
        assert np.array_equal(canonical_with_flags(r[0], r[2]), canonical_with_flags(ot, oc)), i
    bt.close()


def test_batch_autotune_and_empty_instances():
    import torch
    inst = _instances(32, seed0=500, cap=8000) + [(np.zeros((0, 2), np.int32), np.zeros((0, 2), np.int32))]
    po, so = g.BatchTriangulator.offsets(inst)
    bt = g.BatchTriangulator(len(inst), int(po[-1]), int(so[-1]))
    xy = torch.from_numpy(np.concatenate([x for x, _ in inst])).cuda()
    cons = torch.from_numpy(np.concatenate([c for _, c in inst if len(c)])).cuda()
    cfg = bt.autotune(xy, cons, po, so, sample_instances=8)
    assert cfg["threads_per_instance"] in (128, 256, 512) and cfg["sample_stride"] in (16, 64, 256)
    assert bt.get_config() == cfg
    res = bt.triangulate(inst)
    assert len(res[-1][0]) == 2                                   # empty instance: the two box triangles
    for (xy_i, c_i), r in zip(inst[:-1], res[:-1]):
        ok, msg = oracle.validate(xy_i, c_i, *r)
        assert ok, msg
    bt.close()
