"""The reference's stage functions (include/gcdt_reference_surface.h):
exported with the reference's C++ signatures (CPU), and the reference
driver's stage sequence run against them yields the oracle's CDT (GPU)."""
import os
import re
import struct
import subprocess
import tempfile

import numpy as np
import pytest

import gcdt_b200 as g
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN_DIR = os.path.join(ROOT, "tests", "_bin")
DRIVER = os.path.join(BIN_DIR, "surface_driver")


def build_driver():
    src = os.path.join(ROOT, "tests", "surface_driver.cu")
    lib = g.lib_path()
    if os.path.exists(DRIVER) and os.path.getmtime(DRIVER) > max(os.path.getmtime(src), os.path.getmtime(lib)):
        return DRIVER
    os.makedirs(BIN_DIR, exist_ok=True)
    subprocess.run(["nvcc", "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-o", DRIVER, src, "-L" + os.path.dirname(lib), "-lgcdt_b200",
                    "-Xlinker", "-rpath," + os.path.dirname(lib)], check=True)
    return DRIVER


def test_surface_symbols_exported():
    hdr = open(os.path.join(ROOT, "include", "gcdt_reference_surface.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    names = set(re.findall(r"^\s*(?:double|void)\s+(\w+)\s*\(", hdr, flags=re.M))
    assert {"rawMesh", "rawMeshBefore", "rawMeshAfter", "getSamplePoints", "getBitmap", "addConstraints",
            "tryFastDelaunay", "delaunayNew", "filterTriangles", "delaunaySample"} <= names
    out = subprocess.run(["nm", "-DC", "--defined-only", g.lib_path()], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (\w+)\(", out))
    assert names <= exported, names - exported
    # the reference's own parameter lists, e.g. rawMesh.h:5 and addConstraints.h:5
    assert "rawMeshAfter(void*, unsigned long, int2*, int3*, int3*, int*, int*, int*, int&, int)" in out
    assert ("addConstraints(void*, unsigned long, int2*, int3*, int3*, int*, int*, int*, int2*, int3*&, "
            "int, int, int, int&)") in out
    assert "delaunayNew(void*, unsigned long, int2*&, int3*&, int2*, int, int, int)" in out


def _run_driver(xy, cons):
    exe = build_driver()
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as f:
            f.write(struct.pack("<ii", len(xy), len(cons)))
            f.write(np.ascontiguousarray(xy, np.int32).tobytes())
            f.write(np.ascontiguousarray(cons, np.int32).tobytes())
        p = subprocess.run([exe, fin, fout], capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stdout + p.stderr
        raw = open(fout, "rb").read()
    nt = struct.unpack_from("<i", raw)[0]
    return np.frombuffer(raw, np.int32, 3 * nt, 4).reshape(-1, 3)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,seed,args", [(g.GEN_BATCH_INSTANCE, 31, (6000,)),
                                            (g.GEN_SCALE, 4, (300000, 8, 50)),
                                            (g.GEN_UNIFORM, 13159, (200000,))])
def test_reference_driver_sequence_gives_the_cdt(kind, seed, args):
    xy, cons = g.generate(kind, seed, *args)
    tris = _run_driver(xy, cons)
    rc, ot, oa, oc, _ = oracle.cdt(xy, cons)
    assert rc == 0
    assert len(tris) == 2 * len(xy) + 2
    assert np.array_equal(g.canonical(tris), g.canonical(ot))
