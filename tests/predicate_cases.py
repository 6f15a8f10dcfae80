"""Seeded predicate test cases: (k, 4, 2) int32 quads (a, b, c, d) in
[0, 2^30 - 1]^2, mixing uniform points with the degenerate and
near-degenerate shapes where a floating-point filter must defer to exact
arithmetic:
  - uniform over the whole 30-bit box;
  - tiny clusters (offsets in [-8, 8] around a random base): many exact
    zeros and repeated points;
  - axis-aligned rectangles' corners in random order (cocircular);
  - four of the eight points (+-u, +-v), (+-v, +-u) around a centre
    (cocircular, not a rectangle in general);
  - three collinear points and a fourth anywhere;
  - a cocircular quad with its last point moved by one unit (the sign is
    decided by a tiny determinant next to large terms).
"""
import numpy as np

R = (1 << 30) - 1


def predicate_cases(rng, k):
    parts = []
    sizes = [int(k * f) for f in (0.4, 0.15, 0.1, 0.15, 0.1)]
    sizes.append(k - sum(sizes))
    n_uni, n_tiny, n_rect, n_circ, n_col, n_near = sizes
    parts.append(rng.integers(0, R + 1, size=(n_uni, 4, 2), dtype=np.int64))
    base = rng.integers(8, R - 8, size=(n_tiny, 1, 2), dtype=np.int64)
    parts.append(base + rng.integers(-8, 9, size=(n_tiny, 4, 2), dtype=np.int64))
    parts.append(_rects(rng, n_rect))
    parts.append(_circle_quads(rng, n_circ))
    b = rng.integers(0, R - (1 << 21), size=(n_col, 1, 2), dtype=np.int64)
    d = rng.integers(-1024, 1025, size=(n_col, 1, 2), dtype=np.int64)
    t = rng.integers(-1000, 1001, size=(n_col, 3, 1), dtype=np.int64)
    col = np.clip(b + t * d, 0, R)
    parts.append(np.concatenate([col, rng.integers(0, R + 1, size=(n_col, 1, 2), dtype=np.int64)], axis=1))
    near = np.concatenate([_rects(rng, n_near // 2), _circle_quads(rng, n_near - n_near // 2)])
    near[:, 3, :] += rng.integers(-1, 2, size=(len(near), 2))
    parts.append(np.clip(near, 0, R))
    q = np.concatenate(parts)
    return q[rng.permutation(len(q))].astype(np.int32)


def _rects(rng, m):
    base = rng.integers(0, R - (1 << 29), size=(m, 2), dtype=np.int64)
    w = rng.integers(1, 1 << 29, size=(m, 2), dtype=np.int64)
    z = np.zeros(m, np.int64)
    rect = np.stack([base, base + np.stack([w[:, 0], z], 1), base + w, base + np.stack([z, w[:, 1]], 1)], axis=1)
    perm = np.argsort(rng.random((m, 4)), axis=1)
    return np.take_along_axis(rect, perm[:, :, None], axis=1)


def _circle_quads(rng, m):
    u = rng.integers(1, 1 << 27, size=m, dtype=np.int64)
    v = rng.integers(1, 1 << 27, size=m, dtype=np.int64)
    c = rng.integers(1 << 28, R - (1 << 28), size=(m, 2), dtype=np.int64)
    pts = np.stack([np.stack([u, v], 1), np.stack([-u, v], 1), np.stack([-u, -v], 1), np.stack([u, -v], 1),
                    np.stack([v, u], 1), np.stack([-v, u], 1), np.stack([-v, -u], 1), np.stack([v, -u], 1)],
                   axis=1)                                        # (m, 8, 2), all on one circle
    pick = np.argsort(rng.random((m, 8)), axis=1)[:, :4]
    return c[:, None, :] + np.take_along_axis(pts, pick[:, :, None], axis=1)
