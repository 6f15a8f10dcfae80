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


def _run_driver(xy, cons, runs=3):
    """Run the reference's stage sequence; -> {tag: bytes} of the last run's
    stage outputs (see tests/surface_driver.cu) and its stdout."""
    exe = build_driver()
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as f:
            f.write(struct.pack("<ii", len(xy), len(cons)))
            f.write(np.ascontiguousarray(xy, np.int32).tobytes())
            f.write(np.ascontiguousarray(cons, np.int32).tobytes())
        p = subprocess.run([exe, fin, fout, str(runs)], capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stdout + p.stderr
        raw = open(fout, "rb").read()
    out, off = {}, 0
    while off < len(raw):
        tag, nb = struct.unpack_from("<iq", raw, off)
        off += 12
        out[tag] = raw[off:off + nb]
        off += nb
    return out, p.stdout


def _i32(buf, cols):
    a = np.frombuffer(buf, np.int32)
    return a.reshape(-1, cols) if cols > 1 else a


def _canon_mapped(tris, ids):
    return g.canonical(np.asarray(ids)[np.asarray(tris, np.int64)])


CASES = [(g.GEN_BATCH_INSTANCE, 31, (6000,)), (g.GEN_SCALE, 4, (300000, 8, 50)), (g.GEN_UNIFORM, 13159, (200000,))]


@pytest.mark.gpu
@pytest.mark.parametrize("kind,seed,args", CASES)
def test_reference_driver_sequence_stage_by_stage(kind, seed, args):
    """Every stage of the reference's driver sequence against its checker:
    getSamplePoints and getBitmap against host restatements of the
    reference's kernels (oracle/surface_stages.py), the meshing stages
    against the oracle's (C)DT, filterTriangles against a numpy compaction,
    delaunayNew's swapped-in point array against the reference's Morton
    layout (oracle/reference_layout.py) with its triangles and renumbered
    segments, and tryFastDelaunay and rawMesh against the oracle's DT."""
    from oracle import reference_layout as rl
    from oracle import surface_stages as ss
    xy, cons = g.generate(kind, seed, *args)
    n = len(xy)
    out, _ = _run_driver(xy, cons)
    # getSamplePoints
    sid, spts = ss.sample_points(xy)
    ns = len(sid)
    assert np.array_equal(_i32(out[1], 1), sid)
    got_sp = _i32(out[2], 2)
    assert np.array_equal(got_sp[:ns], spts)
    assert got_sp[ns:].tolist() == [[0, 0], [(1 << 30) - 1, 0], [(1 << 30) - 1, (1 << 30) - 1], [0, (1 << 30) - 1]]
    # rawMeshBefore + filterTriangles + delaunaySample: the samples' DT
    stris, sadj = _i32(out[3], 3), _i32(out[4], 3)
    ok, msg = oracle.validate(spts, None, stris, sadj, np.zeros(len(stris), np.uint8))
    assert ok, msg
    rc, ot, _, _, _ = oracle.cdt(spts, None)
    assert rc == 0 and np.array_equal(g.canonical(stris), g.canonical(ot))
    # getBitmap over the sample mesh
    off, lst = ss.bitmap(got_sp, stris)
    assert np.array_equal(_i32(out[5], 1), off)
    assert np.array_equal(_i32(out[6], 1), lst)
    # rawMeshAfter: the DT of all points
    rtris, radj = _i32(out[7], 3), _i32(out[8], 3)
    ok, msg = oracle.validate(xy, None, rtris, radj, np.zeros(len(rtris), np.uint8))
    assert ok, msg
    rc, odt, _, _, _ = oracle.cdt(xy, None)
    assert rc == 0 and np.array_equal(g.canonical(rtris), g.canonical(odt))
    # addConstraints: the CDT
    rc, ocdt, _, _, _ = oracle.cdt(xy, cons)
    assert rc == 0
    ctris, cadj = _i32(out[9], 3), _i32(out[10], 3)
    assert np.array_equal(g.canonical(ctris), g.canonical(ocdt))
    # filterTriangles with every triangle live: the same arrays
    ftris, fadj = ss.filter_triangles(ctris, cadj, -np.ones(len(ctris), np.int32))
    assert np.array_equal(_i32(out[11], 3), ftris) and np.array_equal(_i32(out[12], 3), fadj)
    # delaunayNew: the reference's point layout, triangles over it, segments renumbered
    perm, labels = rl.point_order(xy)
    assert np.array_equal(_i32(out[13], 2), rl.vertices(xy)[perm].astype(np.int32))
    dtris = _i32(out[14], 3)
    assert len(dtris) == 2 * n + 2
    assert np.array_equal(_canon_mapped(dtris, perm), g.canonical(ocdt))
    if len(cons):
        assert np.array_equal(_i32(out[15], 2), labels[np.asarray(cons, np.int64)].astype(np.int32))
    # tryFastDelaunay and rawMesh
    assert np.array_equal(g.canonical(_i32(out[16], 3)), g.canonical(odt))
    ok, msg = oracle.validate(xy, None, _i32(out[16], 3), _i32(out[17], 3), np.zeros(2 * n + 2, np.uint8))
    assert ok, msg
    assert np.array_equal(g.canonical(_i32(out[18], 3)), g.canonical(odt))


@pytest.mark.gpu
def test_reference_driver_sequence_time_against_one_solve():
    """The reference's whole stage sequence on 1M points + 20k segments,
    timed by the driver (second of three runs), against gcdt_triangulate on
    the same input.  The stages reuse one another's triangulations
    (delaunaySample copies rawMeshBefore's, delaunayNew addConstraints'), so
    the sequence costs the unconstrained solve its rawMeshAfter stage asks
    for, the constrained solve, the sample stages and the layout export."""
    import torch
    xy, cons = g.generate(g.GEN_SCALE, 2, 1000000, 18, 316)
    out, stdout = _run_driver(xy, cons)
    times = np.frombuffer(out[19], np.float64)
    seq_ms = times[0]
    tri = g.Triangulator(max_points=len(xy), max_segments=len(cons))
    d_xy, d_c = torch.from_numpy(xy).cuda(), torch.from_numpy(cons).cuda()
    for _ in range(3):
        tri.triangulate(d_xy, d_c)
    ms = []
    for _ in range(5):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        tri.triangulate(d_xy, d_c)
        b.record()
        b.synchronize()
        ms.append(a.elapsed_time(b))
    tri.close()
    one = float(np.median(ms))
    names = ["getSamplePoints", "rawMeshBefore", "filterTriangles", "delaunaySample", "getBitmap",
             "rawMeshAfter", "addConstraints", "filterTriangles", "delaunayNew"]
    print("sequence %.2f ms, one solve %.2f ms, ratio %.2f; stages: %s" % (
        seq_ms, one, seq_ms / one, ", ".join("%s %.2f" % (k, v) for k, v in zip(names, times[2:]))))
    assert seq_ms < 3.5 * one
