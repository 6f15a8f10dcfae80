"""CPU tests of the C-ABI library and the host-side plumbing (no GPU calls)."""
import ctypes
import os
import re

import numpy as np
import pytest

import gcdt_b200 as g

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(inc, fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        if 'extern "C"' not in src:
            continue
        for m in re.finditer(r"\b(gcdt_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_builds_and_loads():
    assert os.path.exists(g.lib_path())
    g.lib()


def test_every_declared_symbol_is_exported():
    names = _declared_functions()
    assert {"gcdt_create", "gcdt_destroy", "gcdt_triangulate", "gcdt_get_stats",
            "gcdt_status_string", "gcdt_workspace_bytes", "gcdt_eval_predicates"} <= names
    L = ctypes.CDLL(g.lib_path())
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert missing == []


def test_status_strings_and_workspace_size():
    L = g.lib()
    for code in range(7):
        assert L.gcdt_status_string(code)
    a = g.workspace_bytes(1000, 10)
    b = g.workspace_bytes(100000, 10)
    c = g.workspace_bytes(100000, 5000)
    assert 0 < a < b <= c
    # bytes per point of the arena at scale: a fixed layout, ~200 B/point
    big = g.workspace_bytes(10_000_000, 200_000)
    assert 100 * 10_000_000 < big < 400 * 10_000_000
    assert g.workspace_bytes(-1, 0) == 0


def test_create_rejects_bad_sizes_without_touching_the_device():
    L = g.lib()
    h = ctypes.c_void_p()
    assert L.gcdt_create(ctypes.byref(h), 0, -5, 0) == 1
    assert L.gcdt_create(ctypes.byref(h), 0, 1 << 40, 0) == 1


def test_generators_are_deterministic_and_clean():
    for kind, args in [(g.GEN_SMALL, (5000,)), (g.GEN_SCALE, (40000, 6, 20)),
                       (g.GEN_LATTICE, (64, 400)), (g.GEN_BATCH_INSTANCE, (3000,)),
                       (g.GEN_SERVING_REQUEST, (5000,))]:
        xy, cons = g.generate(kind, 3, *args)
        xy2, cons2 = g.generate(kind, 3, *args)
        assert np.array_equal(xy, xy2) and np.array_equal(cons, cons2)
        assert xy.min() >= 1 and xy.max() <= (1 << 30) - 2
        assert len(np.unique(xy.view(np.int64))) == len(xy)
        if len(cons):
            assert cons.min() >= 0 and cons.max() < len(xy)
            assert np.all(cons[:, 0] != cons[:, 1])


def test_config_shapes():
    xy, cons = g.generate(g.GEN_SMALL, 1)
    assert len(cons) == 512 and 100000 <= len(xy) <= 100512
    xy, cons = g.generate(g.GEN_LATTICE, 1)
    assert len(xy) == 2048 * 2048 and len(cons) == 20000


def test_canonical_is_rotation_invariant():
    t = np.array([[3, 1, 2], [5, 4, 6]])
    r = np.array([[4, 6, 5], [1, 2, 3]])
    assert np.array_equal(g.canonical(t), g.canonical(r))
    assert not np.array_equal(g.canonical(t), g.canonical(t[:, ::-1]))


def test_variant_library_selection(monkeypatch):
    """GCDT_B200_LIB names a build variant (or a path); unset, the default
    library is used.  A missing variant fails loudly at load."""
    import importlib
    monkeypatch.delenv("GCDT_B200_LIB", raising=False)
    assert g.lib_path().endswith(os.path.join("gcdt_b200", "libgcdt_b200.so"))
    monkeypatch.setenv("GCDT_B200_LIB", "probe")
    assert g.lib_path().endswith(os.path.join("gcdt_b200", "libgcdt_b200_probe.so"))
    monkeypatch.setenv("GCDT_B200_LIB", "/nonexistent/libx.so")
    assert g.lib_path() == "/nonexistent/libx.so"
    saved = g._LIB
    try:
        g._LIB = None
        with pytest.raises(ImportError):
            g.lib()
    finally:
        g._LIB = saved
