"""Run the reference's own CUDA pipeline (oracle/_ref/gcdt_ref, built by
oracle/build_ref.sh) on one input and map its output to input indices.

TEST INFRASTRUCTURE ONLY: a checker and a comparison point for the CUDA path.
The reference returns its triangles over a Morton-permuted copy of the points
(kernel.cu:2059-2066 frees the permutation), so vertices are mapped back to
input indices by their coordinates, which are distinct.
"""
import os
import re
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "_ref", "gcdt_ref")
R = (1 << 30) - 1


def available():
    return os.path.exists(BIN)


def run(xy, cons=None, repeat=1, timeout=600):
    """-> dict(tris (T,3) in input ids with corners n..n+3, points (n+4,2) =
    the reference's returned (Morton-permuted) point array, event_ms,
    sum_time, marks [final Delaunay self-check counts], ignored [constraints
    the reference dropped], stdout)."""
    xy = np.ascontiguousarray(xy, dtype=np.int32).reshape(-1, 2)
    cons = np.ascontiguousarray(np.zeros((0, 2)) if cons is None else cons, dtype=np.int32).reshape(-1, 2)
    n, s = len(xy), len(cons)
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as f:
            f.write(struct.pack("<ii", n, s))
            f.write(xy.tobytes())
            f.write(cons.tobytes())
        p = subprocess.run([BIN, fin, fout, str(repeat)], capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError("reference run failed (%d): %s" % (p.returncode, (p.stdout + p.stderr)[-2000:]))
        raw = open(fout, "rb").read()
    ntri = struct.unpack_from("<i", raw, 0)[0]
    off = 4
    tris = np.frombuffer(raw, np.int32, 3 * ntri, off).reshape(-1, 3)
    off += 12 * ntri
    pts = np.frombuffer(raw, np.int32, 2 * (n + 4), off).reshape(-1, 2)
    off += 8 * (n + 4)
    event_ms, sum_time = struct.unpack_from("<dd", raw, off)
    # map the reference's point order to input ids by coordinates
    corners = np.array([[0, 0], [R, 0], [R, R], [0, R]], np.int64)
    allpts = np.concatenate([xy.astype(np.int64), corners])
    key_in = (allpts[:, 0] << 32) | allpts[:, 1]
    order = np.argsort(key_in)
    key_ref = (pts[:, 0].astype(np.int64) << 32) | pts[:, 1].astype(np.int64)
    pos = np.searchsorted(key_in[order], key_ref)
    if np.any(pos >= len(order)) or np.any(key_in[order][np.minimum(pos, len(order) - 1)] != key_ref):
        raise RuntimeError("reference output holds points that are not in the input")
    ref_to_in = order[pos]
    mapped = ref_to_in[tris]
    out = p.stdout
    marks = [int(m) for m in re.findall(r"^mark (-?\d+)", out, re.M)]
    ignored = [int(m) for m in re.findall(r"^sum ig: (-?\d+)", out, re.M)]
    reps = [float(m) for m in re.findall(r"^harness rep \d+ event_ms ([0-9.]+)", out, re.M)]
    return {"tris": mapped, "points": pts.copy(), "event_ms": event_ms, "rep_ms": reps, "sum_time": sum_time,
            "marks": marks, "ignored": ignored, "stdout": out}
