"""The asynchronous entry point (gcdt_triangulate_async + gcdt_wait).

Its output must be byte-identical to the blocking call's on the same input
(the solve is deterministic), also when two contexts run a stream of inputs
double-buffered on two streams, and a bad input found on the device must
come back from wait() as the same status the blocking call reports."""
import numpy as np
import pytest

import gcdt_b200 as g
from oracle import oracle

pytestmark = pytest.mark.gpu


def _inputs():
    return [g.generate(g.GEN_SCALE, seed, 200_000, 8, 40) for seed in (11, 12)] + \
           [g.generate(g.GEN_LATTICE, 5, 256, 2000), g.generate(g.GEN_SMALL, 4)]


def test_async_matches_blocking_call():
    import torch
    xy, cons = g.generate(g.GEN_SCALE, 3, 200_000, 8, 40)
    tri = g.Triangulator(len(xy), len(cons), device=0)
    p = torch.from_numpy(xy).cuda()
    c = torch.from_numpy(cons).cuda()
    ref = [t.cpu().numpy() for t in tri.triangulate(p, c)]
    out = tri.triangulate_async(p, c)
    assert tri.wait() == 2 * len(xy) + 2
    got = [t.cpu().numpy() for t in out]
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)
    assert tri.wait() == 0          # nothing in flight any more
    tri.close()


def test_two_contexts_double_buffered_on_two_streams():
    import torch
    inputs = _inputs()
    nmax = max(len(x) for x, _ in inputs)
    smax = max(len(c) for _, c in inputs)
    ref_tri = g.Triangulator(nmax, smax, device=0)
    refs = [ref_tri.triangulate_host(x, c) for x, c in inputs]
    ref_tri.close()
    ctxs = [g.Triangulator(nmax, smax, device=0) for _ in range(2)]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    solved = [torch.cuda.Event() for _ in inputs]
    host = []
    for k, (x, c) in enumerate(inputs):
        j = k & 1
        with torch.cuda.stream(streams[j]):
            p = torch.from_numpy(x).pin_memory().cuda(non_blocking=True)
            s = torch.from_numpy(c).pin_memory().cuda(non_blocking=True)
            if k > 0:
                streams[j].wait_event(solved[k - 1])
            out = ctxs[j].triangulate_async(p, s)
            solved[k].record(streams[j])
            host.append([t.to("cpu", non_blocking=True) for t in out])
    for t in ctxs:
        t.wait()
    torch.cuda.synchronize()
    for (x, c), ref, got in zip(inputs, refs, host):
        for a, b in zip(ref, got):
            assert np.array_equal(a, b.numpy())
    ok, msg = oracle.validate(inputs[0][0], inputs[0][1], *[t.numpy() for t in host[0]])
    assert ok, msg
    for t in ctxs:
        t.close()


def test_async_bad_input_is_reported_by_wait():
    import torch
    tri = g.Triangulator(16, 4, device=0)
    dup = torch.tensor([[10, 10], [10, 10], [30, 40]], dtype=torch.int32, device="cuda")
    tri.triangulate_async(dup)
    with pytest.raises(g.GcdtError) as e:
        tri.wait()
    assert e.value.status == "BAD_INPUT"
    # the context stays usable
    ok = torch.tensor([[10, 10], [20, 30], [30, 12]], dtype=torch.int32, device="cuda")
    tris, adj, cf = tri.triangulate(ok)
    assert tris.shape[0] == 8
    tri.close()
