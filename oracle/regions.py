"""Region depth of a constrained triangulation by 0-1 breadth-first search.

TEST INFRASTRUCTURE ONLY: the checker for gcdt_classify_regions; imported by
tests/ alone.  The reference has no such step (it returns the whole box
triangulation, kernel.cu:5443-5448), so this restates the definition
directly, by a different algorithm from the CUDA path's union-find +
component rounds: a deque search over triangles where crossing an
unconstrained edge costs 0 and crossing a constrained edge costs 1,
starting from every triangle on the box edge.
"""
from collections import deque

import numpy as np


def region_depth(adj, cflags):
    """-> (depth (T,) int32, greatest depth): fewest constraint edges crossed
    from the box edge; -1 where the box edge does not reach."""
    adj = np.asarray(adj, np.int64).reshape(-1, 3)
    cf = np.asarray(cflags, np.int64).reshape(-1)
    T = len(adj)
    inf = 1 << 40
    depth = np.full(T, inf, np.int64)
    dq = deque()
    for t in np.nonzero((adj == -1).any(axis=1))[0]:
        depth[t] = 0
        dq.append(int(t))
    a = adj.tolist()
    c = cf.tolist()
    d = depth.tolist()
    while dq:
        t = dq.popleft()
        dt = d[t]
        for k in range(3):
            u = a[t][k]
            if u < 0:
                continue
            w = (c[t] >> k) & 1
            if dt + w < d[u]:
                d[u] = dt + w
                if w:
                    dq.append(u)
                else:
                    dq.appendleft(u)
    out = np.array(d, np.int64)
    out[out == inf] = -1
    return out.astype(np.int32), int(out.max()) if T else 0
