"""The oracle's fewest-hop temporal paths against a brute-force definition on small random graphs
(CPU only): the fewest edges on a time-respecting path, by breadth-first search over
(vertex, arrival time) states."""
from __future__ import annotations

from collections import deque

import numpy as np
import pytest

import compresstemporalgraph_b200 as tga
import pyoracle

INF32 = np.iinfo(np.int32).max


def brute(off, dst, ts, n, src, lo, hi):
    """BFS over states (v, t): from (x, a) every kept edge (x->y, t) with a <= t leads to (y, t);
    the kept edges are the first in-window occurrence of each run of equal successors."""
    kept = [[] for _ in range(n)]
    for x in range(n):
        prev = -1
        for e in range(off[x], off[x + 1]):
            t = int(ts[e])
            if t < lo or t >= hi:
                continue
            y = int(dst[e])
            if y == prev:
                continue
            prev = y
            kept[x].append((y, t))
    start = max(lo, 0)
    best = {}
    hops = np.full(n, INF32, np.int64)
    hops[src] = 0
    seen = {(src, start)}
    q = deque([(src, start, 0)])
    while q:
        x, a, k = q.popleft()
        for y, t in kept[x]:
            if a > t or (y, t) in seen:
                continue
            seen.add((y, t))
            hops[y] = min(hops[y], k + 1)
            q.append((y, t, k + 1))
    return hops.astype(np.int32)


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_shortest_equals_state_bfs(tmp_path, seed):
    n = 60
    p = tga.GenParams(n=n, m=400, deg_exponent=2.0, repeat_frac=0.4, local_frac=0.3, local_radius=4, ts_kind=0,
                      ts_span=50, seed=seed)
    tga.generate(p, tmp_path, "g")
    o = pyoracle.Oracle(tmp_path, "g", n)
    off, dst, ts = o.csr()
    deg = np.diff(off)
    for src in (int(deg.argmax()), 1, 7):
        for lo, hi in ((0, 1 << 40), (10, 40)):
            hops, _ = o.shortest(n - 1, n, 0, src, lo, hi)
            assert np.array_equal(hops, brute(off, dst, ts, n, src, lo, hi)), (src, lo, hi)
    o.close()
