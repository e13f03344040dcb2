"""Fastest temporal paths (tga_fastest) on the CPU: the composition the engine computes equals the
definition.

The engine takes, for every distinct in-window departure time d of the source's out-edges, the
earliest arrivals over the window [d, hi) and keeps min over d of (arrival - d), the earliest d on
ties.  The definition is the least (last-edge time - first-edge time) over time-respecting paths
from the source, the first edge leaving the source inside the window.  Both are evaluated here with
the oracle: the composition through its BFS (the same rows the engine's multi-source traversal
produces), the definition by a search per first edge.  The graphs have unique (source, successor)
pairs, so tga_bfs's rule for runs of repeated successors (only the first in-window one counts)
plays no part; the GPU parity test compares the engine with the same composition on the generated
shapes, repeated successors included.
"""
from __future__ import annotations

import heapq

import numpy as np
import pytest

import compresstemporalgraph_b200 as tga
import pyoracle

INF32 = np.iinfo(np.int32).max


def fastest_by_departures(o, n, ml, mv, act, src, lo, hi):
    """The composition, with the oracle's BFS: (duration, departure) per vertex, -1 unreachable."""
    dur = np.full(mv, -1, np.int64)
    dep = np.full(mv, -1, np.int64)
    dur[src] = 0
    if src < n:
        _, ts = o.neighbors(src)
        for d in np.unique(ts[(ts >= lo) & (ts < hi)]):
            arr, _ = o.bfs(ml, mv, act, src, int(d), hi)
            reach = arr != INF32
            reach[src] = False
            cand = arr.astype(np.int64) - int(d)
            better = reach & ((dur < 0) | (cand < dur))
            dur[better] = cand[better]
            dep[better] = int(d)
    return dur, dep


def fastest_by_definition(out, n, ml, mv, act, src, lo, hi):
    """Least last-edge minus first-edge time, by one earliest-arrival search per first edge.  A
    vertex's edges are followed when act <= x <= ml and x < n, to successors in [act, mv), as the
    oracle's BFS does."""
    dur = [-1] * mv
    dep = [-1] * mv
    dur[src] = 0
    expands = lambda x: act <= x <= ml and x < n  # noqa: E731
    if not expands(src):
        return np.array(dur, np.int64), np.array(dep, np.int64)
    firsts = sorted({t for y, t in out[src] if lo <= t < hi and act <= y < mv})
    for d in firsts:
        arr = {}
        heap = []
        for y, t in out[src]:
            if t == d and act <= y < mv and arr.get(y, INF32) > d:
                arr[y] = d
                heapq.heappush(heap, (d, y))
        while heap:
            a, x = heapq.heappop(heap)
            if a != arr[x] or not expands(x):
                continue
            for y, t in out[x]:
                if a <= t < hi and act <= y < mv and t < arr.get(y, INF32):
                    arr[y] = t
                    heapq.heappush(heap, (t, y))
        for v, a in arr.items():
            if v != src and (dur[v] < 0 or a - d < dur[v]):
                dur[v] = a - d
                dep[v] = d
    return np.array(dur, np.int64), np.array(dep, np.int64)


def _graph(tmp_path, seed, nv, m, span):
    rng = np.random.default_rng(seed)
    pairs = set()
    while len(pairs) < m:
        x, y = (int(v) for v in rng.integers(0, nv, 2))
        if x != y:
            pairs.add((x, y))
    out = {}
    lines = []
    for x, y in sorted(pairs):
        t = int(rng.integers(0, span))
        out.setdefault(x, []).append((y, t))
        lines.append(f"{x} {y} 1 {t}\n")
    raw = tmp_path / f"p{seed}.txt"
    raw.write_text("".join(lines))
    s = tga.encode_raw(raw, tmp_path, f"p{seed}")
    n = s["n"]
    for v in range(n):
        out.setdefault(v, [])
    return pyoracle.Oracle(tmp_path, f"p{seed}", n), out, n


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("view", ["plain", "narrowed"])
def test_composition_equals_definition(tmp_path, seed, view):
    # A small time span makes many edges share a timestamp, so paths chain at one instant.
    o, out, n = _graph(tmp_path, seed, 40, 220, 30)
    if view == "plain":
        ml, mv, act = n - 1, n, 0
    else:  # inactive low ids, unexpanded high ids, result arrays longer than the id space
        ml, mv, act = n - 4, n + 5, 3
    for lo, hi in [(0, tga.T_MAX), (8, 22)]:
        for src in range(n):
            got = fastest_by_departures(o, n, ml, mv, act, src, lo, hi)
            want = fastest_by_definition(out, n, ml, mv, act, src, lo, hi)
            assert np.array_equal(got[0], want[0]), (src, lo, hi)
            assert np.array_equal(got[1], want[1]), (src, lo, hi)


def test_hand_made_case(tmp_path):
    """0 -> 1 at 1 and at 5, 0 -> 2 at 9, 1 -> 2 at 6, 2 -> 3 at 6.  The earliest arrival at 2 is 6
    (leaving at 1 or 5), but the one-edge path at 9 takes no time; 3 is reached only through
    0 -> 1 -> 2 -> 3 at 5, 6, 6 (1 unit), since 2 -> 3 at 6 is gone by 9."""
    raw = tmp_path / "h.txt"
    raw.write_text("0 1 1 1\n0 1 1 5\n0 2 1 9\n1 2 1 6\n2 3 1 6\n")
    tga.encode_raw(raw, tmp_path, "h")
    o = pyoracle.Oracle(tmp_path, "h", 4)
    dur, dep = fastest_by_departures(o, 4, 3, 4, 0, 0, 0, tga.T_MAX)
    assert dur.tolist() == [0, 0, 0, 1]
    assert dep.tolist() == [-1, 1, 9, 5]
    # The window [2, 9) drops the departures at 1 and 9.
    dur, dep = fastest_by_departures(o, 4, 3, 4, 0, 0, 2, 9)
    assert dur.tolist() == [0, 0, 1, 1]
    assert dep.tolist() == [-1, 5, 5, 5]


# ---- latest departure through the time-reversed copy -------------------------------------------

def latest_by_reversal(orev, n, ml, mv, act, pivot, target, lo, hi):
    """tga_latest_departure's mapping, with the oracle's BFS on the reversed copy."""
    out = np.full(mv, -1, np.int64)
    if lo > pivot:
        out[target] = min(hi - 1, pivot)
        return out
    rlo = 0 if hi > pivot else pivot - hi + 1
    arr, _ = orev.bfs(ml, mv, act, target, rlo, pivot - lo + 1)
    reach = arr != INF32
    out[reach] = pivot - arr[reach].astype(np.int64)
    return out


def latest_by_definition(out, n, mv, pivot, target, lo, hi):
    """Latest first-edge time of a time-respecting path v -> target inside [lo, hi), trying each
    vertex's out-edges from the latest (plain view: every vertex's edges are followed)."""
    res = np.full(mv, -1, np.int64)
    res[target] = min(hi - 1, pivot)

    def reaches(y, d):
        arr = {y: d}
        heap = [(d, y)]
        while heap:
            a, x = heapq.heappop(heap)
            if x == target:
                return True
            if a != arr[x]:
                continue
            for z, t in out[x]:
                if a <= t < hi and t < arr.get(z, INF32):
                    arr[z] = t
                    heapq.heappush(heap, (t, z))
        return False

    for v in range(n):
        if v == target:
            continue
        for y, d in sorted(out[v], key=lambda e: -e[1]):
            if lo <= d < hi and (y == target or reaches(y, d)):
                res[v] = d
                break
    return res


def test_reversed_copy_is_the_transposition(tmp_path, datasets):
    d = datasets["chains"]  # reference chains, intervals and repeated successors
    n = d["summary"]["n"]
    off, dst, ts = pyoracle.Oracle(d["dir"], d["base"], n).csr()
    pivot = int(ts.max()) + 3
    tga.write_reversed(off, dst, ts, pivot, tmp_path, "rev")
    roff, rdst, rts = pyoracle.Oracle(tmp_path, "rev", n).csr()
    src = np.repeat(np.arange(n), np.diff(off))
    order = np.lexsort((pivot - ts, src, dst))  # by new source, then successor, then reversed time
    assert np.array_equal(roff, np.concatenate([[0], np.cumsum(np.bincount(dst, minlength=n))]))
    assert np.array_equal(rdst, src[order])
    assert np.array_equal(rts, (pivot - ts)[order])


def test_write_reversed_rejects_bad_input(tmp_path):
    off = np.array([0, 1, 2])
    with pytest.raises(tga.TgaError):
        tga.write_reversed(off, np.array([1, 0]), np.array([5, 9]), 8, tmp_path, "x")  # 9 > pivot
    with pytest.raises(tga.TgaError):
        tga.write_reversed(off, np.array([1, 2]), np.array([5, 6]), 8, tmp_path, "x")  # successor 2 >= n
    with pytest.raises(tga.TgaError):
        tga.write_reversed(np.array([0, 2, 1]), np.array([1, 0]), np.array([5, 6]), 8, tmp_path, "x")


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_latest_departure_by_reversal_equals_definition(tmp_path, seed):
    o, out, n = _graph(tmp_path, seed, 40, 220, 30)
    off, dst, ts = o.csr()
    pivot = int(ts.max())
    tga.write_reversed(off, dst, ts, pivot, tmp_path, f"r{seed}")
    orev = pyoracle.Oracle(tmp_path, f"r{seed}", n)
    for lo, hi in [(0, tga.T_MAX), (8, 22), (0, 15), (pivot + 1, pivot + 5)]:
        for target in range(n):
            got = latest_by_reversal(orev, n, n - 1, n, 0, pivot, target, lo, hi)
            want = latest_by_definition(out, n, n, pivot, target, lo, hi)
            assert np.array_equal(got, want), (target, lo, hi)


def test_reversal_edge_cases(tmp_path):
    # No edges at all: an empty copy that still opens in the oracle.
    tga.write_reversed(np.array([0, 0, 0]), np.array([], np.int32), np.array([], np.int64), 0, tmp_path, "e")
    off, dst, ts = pyoracle.Oracle(tmp_path, "e", 2).csr()
    assert off.tolist() == [0, 0, 0] and len(dst) == 0 and len(ts) == 0
    summary, depth = tga.reference_depths(tmp_path, "e")
    assert summary["depth_counts"][0] == 2 and depth.tolist() == [0, 0]
    # One edge 0 -> 1 at 5, reflected about pivot 5: 1 -> 0 at 0.
    tga.write_reversed(np.array([0, 1, 1]), np.array([1], np.int32), np.array([5], np.int64), 5, tmp_path, "o")
    off, dst, ts = pyoracle.Oracle(tmp_path, "o", 2).csr()
    assert off.tolist() == [0, 0, 1] and dst.tolist() == [0] and ts.tolist() == [0]
