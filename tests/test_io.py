"""Reader of the reference's text format and the mesh writer (CPU)."""
import os

import numpy as np

import gcdt_b200 as g
from oracle import oracle


def _restated_reader(text):
    """readFile (kernel.cu:5159-5291) + transPoints (kernel.cu:171-188) in
    Python, plus the two grid clean-ups of gcdt_text_load."""
    tok = text.split()
    p = 0
    n = int(tok[p]); p += 1
    pmap, idxmap, pts = {}, {}, []
    for _ in range(n):
        idx, x, y = int(tok[p]), float(tok[p + 1]), float(tok[p + 2]); p += 3
        if (x, y) not in pmap:
            pmap[(x, y)] = len(pts)
            pts.append((x, y))
        idxmap[idx] = pmap[(x, y)]
    xs = [q[0] for q in pts]; ys = [q[1] for q in pts]
    cx, cy = (min(xs) + max(xs)) / 2, (min(ys) + max(ys)) / 2
    lx = max(max(xs) - min(xs), max(ys) - min(ys))
    res = 1 << 30
    grid, remap, out = {}, [], []
    for x, y in pts:
        fx = (x - cx) / lx * 0.99 + 0.5
        fy = (y - cy) / lx * 0.99 + 0.5
        ix = min(max(int(fx * res), 1), res - 2)
        iy = min(max(int(fy * res), 1), res - 2)
        if (ix, iy) not in grid:
            grid[(ix, iy)] = len(out)
            out.append((ix, iy))
        remap.append(grid[(ix, iy)])
    m = int(tok[p]); p += 1
    seen, cons = set(), []
    for _ in range(m):
        a, b = remap[idxmap[int(tok[p + 1])]], remap[idxmap[int(tok[p + 2])]]; p += 3
        if a == b or (a, b) in seen or (b, a) in seen:
            continue
        seen.add((a, b))
        cons.append((a, b))
    return np.array(out, np.int32), np.array(cons, np.int32).reshape(-1, 2)


def test_reader_matches_the_restated_reference_reader(tmp_path):
    rng = np.random.default_rng(4)
    pts = rng.uniform(-3.5, 12.25, size=(400, 2))
    pts[50] = pts[10]                        # exact duplicate
    pts[51] = pts[10] + 1e-13                # collides on the integer grid
    lines = [str(len(pts))] + ["%d %.17g %.17g" % (i + 100, x, y) for i, (x, y) in enumerate(pts)]
    segs = [(100, 101), (101, 102), (102, 100), (101, 100), (150, 110), (103, 103), (151, 104)]
    lines += [str(len(segs))] + ["%d %d %d" % (k, a, b) for k, (a, b) in enumerate(segs)]
    path = tmp_path / "in.txt"
    path.write_text("\n".join(lines) + "\n")
    xy, cons = g.load_text(str(path))
    exy, econs = _restated_reader(path.read_text())
    assert np.array_equal(xy, exy)
    assert np.array_equal(cons, econs)
    assert len(xy) == 398                    # two merges
    assert len(np.unique(xy.view(np.int64))) == len(xy)
    rc, tris, adj, cf, _ = oracle.cdt(xy, cons)
    assert rc == 0


def test_writer_round_trip(tmp_path):
    xy, cons = g.generate(g.GEN_BATCH_INSTANCE, 3, 300)
    rc, tris, adj, cf, _ = oracle.cdt(xy, cons)
    path = tmp_path / "mesh.txt"
    g.save_text(str(path), xy, tris, adj, cf)
    tok = path.read_text().split()
    n = int(tok[0])
    assert n == len(xy) + 4
    pts = np.array(tok[1:1 + 3 * n], np.int64).reshape(-1, 3)
    assert np.array_equal(pts[:len(xy), 1:], xy)
    k = 1 + 3 * n
    nt = int(tok[k])
    rows = np.array(tok[k + 1:k + 1 + 8 * nt], np.int64).reshape(-1, 8)
    assert np.array_equal(rows[:, 1:4], tris) and np.array_equal(rows[:, 4:7], adj)
    assert np.array_equal(rows[:, 7], cf)


def test_reader_errors(tmp_path):
    import pytest
    with pytest.raises(ValueError):
        g.load_text(str(tmp_path / "missing.txt"))
    bad = tmp_path / "bad.txt"
    bad.write_text("3\n0 1 2\n1 3 4\n")
    with pytest.raises(ValueError):
        g.load_text(str(bad))
