"""ctypes wrapper of the CPU oracle (oracle/cdt_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py, as the checker.  The product path never
imports this module.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "liboracle.so")
_O = None


def build(force=False):
    src = os.path.join(HERE, "cdt_oracle.c")
    if force or not os.path.exists(SO) or os.path.getmtime(SO) < os.path.getmtime(src):
        subprocess.run(["gcc", "-O2", "-std=gnu11", "-shared", "-fPIC", "-o", SO, src], check=True)
    return SO


def _lib():
    global _O
    if _O is None:
        if not os.path.exists(SO):
            build()
        O = ctypes.CDLL(SO)
        vp = ctypes.c_void_p
        O.oracle_cdt.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, vp, vp, vp, ctypes.POINTER(ctypes.c_int), vp]
        O.oracle_cdt.restype = ctypes.c_int
        O.oracle_validate.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, vp, vp, vp, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        O.oracle_validate.restype = ctypes.c_int
        O.oracle_orient.argtypes = [ctypes.c_int64] * 6
        O.oracle_orient.restype = ctypes.c_int
        O.oracle_incircle.argtypes = [ctypes.c_int64] * 8
        O.oracle_incircle.restype = ctypes.c_int
        O.oracle_incircle_sos.argtypes = [vp]
        O.oracle_incircle_sos.restype = ctypes.c_int
        O.oracle_predicates_batch.argtypes = [vp, ctypes.c_int64, vp]
        O.oracle_predicates_batch.restype = None
        _O = O
    return _O


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def cdt(xy, cons=None):
    """Sequential exact CDT -> (status, tris (T,3), adj (T,3), cflags (T,), flips)."""
    xy = np.ascontiguousarray(xy, dtype=np.int32).reshape(-1, 2)
    cons = np.ascontiguousarray(np.zeros((0, 2)) if cons is None else cons, dtype=np.int32).reshape(-1, 2)
    n, s = len(xy), len(cons)
    T = 2 * n + 2
    tris = np.zeros((T, 3), np.int32)
    adj = np.zeros((T, 3), np.int32)
    cf = np.zeros(T, np.uint8)
    nt = ctypes.c_int(0)
    st = np.zeros(4, np.int64)
    rc = _lib().oracle_cdt(_p(xy), n, _p(cons), s, _p(tris), _p(adj), _p(cf), ctypes.byref(nt), _p(st))
    return rc, tris[:nt.value], adj[:nt.value], cf[:nt.value], int(st[0])


def validate(xy, cons, tris, adj, cflags):
    """Exact CDT validator -> (ok, message)."""
    xy = np.ascontiguousarray(xy, dtype=np.int32).reshape(-1, 2)
    cons = np.ascontiguousarray(np.zeros((0, 2)) if cons is None else cons, dtype=np.int32).reshape(-1, 2)
    tris = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1, 3)
    adj = np.ascontiguousarray(adj, dtype=np.int32).reshape(-1, 3)
    cflags = np.ascontiguousarray(cflags, dtype=np.uint8).reshape(-1)
    msg = ctypes.create_string_buffer(512)
    rc = _lib().oracle_validate(_p(xy), len(xy), _p(cons), len(cons), _p(tris), _p(adj), _p(cflags),
                                len(tris), msg, 512)
    return rc == 0, msg.value.decode()


def orient(a, b, c):
    return _lib().oracle_orient(int(a[0]), int(a[1]), int(b[0]), int(b[1]), int(c[0]), int(c[1]))


def incircle(a, b, c, d):
    return _lib().oracle_incircle(*[int(v) for p in (a, b, c, d) for v in p])


def incircle_sos(a, b, c, d):
    q = np.array([a, b, c, d], dtype=np.int64).reshape(8)
    return _lib().oracle_incircle_sos(_p(q))


def predicates_batch(quads):
    """quads: (k, 4, 2) int32 -> (k, 3) int32 of [orient2d(a,b,c),
    incircle(a,b,c,d), perturbed incircle(a,b,c,d)], exact."""
    q = np.ascontiguousarray(quads, dtype=np.int32).reshape(-1, 8)
    out = np.zeros((len(q), 3), np.int32)
    _lib().oracle_predicates_batch(_p(q), len(q), _p(out))
    return out
