"""Per-phase profiling of the stage kernel (gcdt_set_profiling).

Off by default: a solve then records no phase profile and no phase balance.
On, it records both, and the mesh is byte-identical to the unprofiled
solve's (profiling only adds counter updates beside the phases)."""
import numpy as np
import pytest

import gcdt_b200 as g

pytestmark = pytest.mark.gpu


def test_profiling_is_off_by_default_and_changes_no_output():
    import torch
    xy, cons = g.generate(g.GEN_SCALE, 7, 200_000, 8, 40)
    tri = g.Triangulator(len(xy), len(cons), device=0)
    p = torch.from_numpy(xy).cuda()
    c = torch.from_numpy(cons).cuda()
    ref = [t.cpu().numpy() for t in tri.triangulate(p, c)]
    assert tri.phase_profile() == {}
    assert tri.phase_balance() == {}

    tri.set_profiling(True)
    got = [t.cpu().numpy() for t in tri.triangulate(p, c)]
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)
    prof = tri.phase_profile()
    bal = tri.phase_balance()
    for name in ("activate", "reloc_vote", "split", "fix", "flip_check", "flip_do", "flip_fix", "output"):
        cyc, runs = prof[name]
        assert cyc > 0 and runs >= 1, name
    assert bal, "no phase balance recorded"
    for name, (wmax, wmean) in bal.items():
        assert 0 < wmean <= wmax, name
        assert wmax <= prof[name][0] * 1.05 + 1e5, name   # work ends before the phase does

    tri.set_profiling(False)
    again = [t.cpu().numpy() for t in tri.triangulate(p, c)]
    for a, b in zip(ref, again):
        assert np.array_equal(a, b)
    assert tri.phase_profile() == {}
    tri.close()
