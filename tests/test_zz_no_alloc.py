"""The allocation-free entry point against the context entry point.

gcdt_triangulate_noalloc serves callers that cannot allocate device memory
when they call in (a plugin whose host application owns the device memory
through its own allocator, or a loop that cannot pay for cudaMalloc's
device-wide synchronization): it keeps its scratch in a static device array
of the library instead of a context arena.  This test drives it through the
C ABI with buffers the test allocates, twice in a row on different inputs,
and requires the output to equal gcdt_triangulate's byte for byte (the
path's tolerance is exact).  The file name makes pytest collect it last.
"""
import ctypes

import numpy as np
import pytest

import gcdt_b200 as g


def _noalloc():
    L = g.lib()
    f = L.gcdt_triangulate_noalloc
    vp = ctypes.c_void_p
    f.argtypes = [vp, ctypes.c_int32, vp, ctypes.c_int32, vp, vp, vp, ctypes.POINTER(ctypes.c_int32), vp]
    f.restype = ctypes.c_int
    return f


def _run_noalloc(xy, cons, poison):
    import torch
    f = _noalloc()
    dev = torch.device("cuda", 0)
    p = torch.from_numpy(np.ascontiguousarray(xy, np.int32)).to(dev)
    sgm = torch.from_numpy(np.ascontiguousarray(cons, np.int32)).to(dev) if len(cons) else None
    T = 2 * len(xy) + 2
    tris = torch.full((T, 3), poison, dtype=torch.int32, device=dev)
    adj = torch.full((T, 3), poison, dtype=torch.int32, device=dev)
    cf = torch.full((T,), poison & 0xFF, dtype=torch.uint8, device=dev)
    nt = ctypes.c_int32(0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    torch.cuda.synchronize()
    rc = f(ctypes.c_void_p(p.data_ptr()), len(xy), ctypes.c_void_p(sgm.data_ptr() if sgm is not None else 0),
           len(cons), ctypes.c_void_p(tris.data_ptr()), ctypes.c_void_p(adj.data_ptr()),
           ctypes.c_void_p(cf.data_ptr()), ctypes.byref(nt), ctypes.c_void_p(stream))
    assert rc == 0, g.STATUS.get(rc, rc)
    assert nt.value == T
    return tris.cpu().numpy(), adj.cpu().numpy(), cf.cpu().numpy()


@pytest.mark.gpu
def test_noalloc_equals_context_entry_point_twice_in_a_row():
    inputs = [g.generate(g.GEN_SMALL, 1),                     # 100,512 points + 512 segments
              g.generate(g.GEN_BATCH_INSTANCE, 3, 20000)]     # a different, smaller instance
    for xy, cons in inputs:
        assert g.workspace_bytes(len(xy), len(cons)) <= (32 << 20)
    tri = g.Triangulator(max_points=max(len(x) for x, _ in inputs),
                         max_segments=max(len(c) for _, c in inputs))
    expected = [tri.triangulate_host(xy, cons) for xy, cons in inputs]
    tri.close()
    for call, ((xy, cons), want) in enumerate(zip(inputs, expected)):
        got = _run_noalloc(xy, cons, poison=-7 - call)
        for a, b in zip(got, want):
            assert np.array_equal(a, b), "call %d differs from gcdt_triangulate" % call


@pytest.mark.gpu
def test_noalloc_rejects_problems_beyond_the_static_workspace():
    import torch
    f = _noalloc()
    n = 400000          # needs ~110 MB of workspace, more than the 32 MiB array
    assert g.workspace_bytes(n, 0) > (32 << 20)
    dummy = torch.zeros(16, dtype=torch.int32, device="cuda")
    nt = ctypes.c_int32(0)
    ptr = ctypes.c_void_p(dummy.data_ptr())
    rc = f(ptr, n, None, 0, ptr, ptr, ptr, ctypes.byref(nt), None)
    assert g.STATUS[rc] == "OOM"
