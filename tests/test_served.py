"""Served form: a request loop over two resident graphs.  Every result must equal the plain
single-query call (BFS arrivals, CC labels and point queries bit-exact, PageRank within the
batched-vs-single tolerance), and a query gives the same result alone and inside a mix of
concurrent queries."""
from __future__ import annotations

import numpy as np
import pytest

import compresstemporalgraph_b200 as tga

pytestmark = pytest.mark.gpu

T_MAX = tga.T_MAX


def _open(d):
    n = d["summary"]["n"]
    return tga.Graph.open_dir(d["dir"], d["base"], tga.DatasetConfig(name=d["base"], max_label=n - 1, max_vertex=n))


def _mix(rng, gid, d, count):
    n = d["summary"]["n"]
    lo0, span = d["params"].min_timestamp, d["params"].ts_span
    out = []
    for _ in range(count):
        lo = int(lo0 + rng.integers(0, span // 2))
        hi = int(lo + rng.integers(span // 20, span // 2))
        if rng.random() < 0.2:
            lo, hi = 0, T_MAX
        r = rng.random()
        if r < 0.1:
            out.append(dict(kind=tga.Q_NEIGHBOR, graph=gid, src=int(rng.integers(0, n)), dst=int(rng.integers(0, n)),
                            t_lo=lo, t_hi=hi))
        elif r < 0.6:
            out.append(dict(kind=tga.Q_BFS, graph=gid, src=int(rng.integers(0, n)), t_lo=lo, t_hi=hi))
        elif r < 0.85:
            out.append(dict(kind=tga.Q_PAGERANK, graph=gid, iters=int(rng.integers(3, 7)), t_lo=lo, t_hi=hi))
        else:
            out.append(dict(kind=tga.Q_CC, graph=gid, t_lo=lo, t_hi=hi))
    return out


def _plain(g, q):
    if q["kind"] == tga.Q_NEIGHBOR:
        return np.array([g.is_neighbor([q["src"]], [q["dst"]], q["t_lo"], q["t_hi"])[0]], np.uint8)
    if q["kind"] == tga.Q_BFS:
        return g.bfs(q["src"], q["t_lo"], q["t_hi"])[0]
    if q["kind"] == tga.Q_PAGERANK:
        return g.pagerank(q["iters"], 0.85, 0.1, q["t_lo"], q["t_hi"])
    return g.connected_components(q["t_lo"], q["t_hi"])[0]


def _same(q, a, b):
    if q["kind"] == tga.Q_PAGERANK:
        # Same tolerance as test_batched_pagerank_equals_single: both are FP32, summed in other orders.
        return np.allclose(a, b, rtol=1e-4, atol=1e-9)
    return np.array_equal(a, b)


def test_served_mix_equals_plain_and_alone(datasets):
    rng = np.random.default_rng(12)
    graphs = [_open(datasets["chains"]), _open(datasets["hubs"])]
    try:
        with tga.Server(budget_bytes=1 << 30) as srv:
            gids = [srv.add_graph(g) for g in graphs]
            queries = _mix(rng, gids[0], datasets["chains"], 50) + _mix(rng, gids[1], datasets["hubs"], 50)
            order = rng.permutation(len(queries))
            queries = [queries[i] for i in order]
            queries.append(dict(queries[0]))  # the same query twice in the mix
            tickets = [srv.submit(**q) for q in queries]
            srv.drain()
            results = []
            for t in tickets:
                r = srv.poll(t)
                assert r is not None
                results.append(r[0])
            st = srv.stats()
            assert st["completed"] == len(queries) and st["failed"] == 0
            assert 0 < st["p50_ms"] <= st["p99_ms"] and st["queries_per_s"] > 0
            assert _same(queries[0], results[0], results[-1])
        # Alone: a fresh server with one query at a time.
        with tga.Server(budget_bytes=1 << 30) as srv:
            gids = [srv.add_graph(g) for g in graphs]
            for k in (0, 1, 2, 3):
                t = srv.submit(**queries[k])
                srv.drain()
                alone, _ = srv.poll(t)
                assert _same(queries[k], alone, results[k]), k
        # Plain single-query calls (the server no longer holds the handles).
        for q, r in zip(queries, results):
            assert _same(q, _plain(graphs[q["graph"]], q), r), q
    finally:
        for g in graphs:
            g.close()


def test_served_rejects_queries_beyond_budget(datasets):
    g = _open(datasets["small"])
    try:
        with tga.Server(budget_bytes=1000) as srv:
            gid = srv.add_graph(g)
            with pytest.raises(tga.TgaError) as e:
                srv.submit(tga.Q_BFS, gid, src=0)
            assert e.value.code == tga.TGA_E_OOM
    finally:
        g.close()


def test_served_live_arrivals_equal_plain(datasets):
    """Queries keep arriving while earlier rounds run on the device (a CC window first, then batches
    of BFS and PageRank joined by queries submitted while they are in flight): every result equals
    the plain single-query call, and the server ran many rounds rather than one batch."""
    import time

    rng = np.random.default_rng(31)
    graphs = [_open(datasets["chains"]), _open(datasets["hubs"])]
    try:
        with tga.Server(budget_bytes=1 << 30) as srv:
            gids = [srv.add_graph(g) for g in graphs]
            queries = [dict(kind=tga.Q_CC, graph=gids[1], t_lo=0, t_hi=T_MAX)]
            queries += _mix(rng, gids[0], datasets["chains"], 40) + _mix(rng, gids[1], datasets["hubs"], 40)
            tickets = []
            for k, q in enumerate(queries):
                tickets.append(srv.submit(**q))
                if k % 5 == 4:
                    time.sleep(0.003)  # the next queries arrive while the last round runs
            srv.drain()
            results = [srv.poll(t)[0] for t in tickets]
            st = srv.stats()
            assert st["completed"] == len(queries) and st["failed"] == 0
            assert st["rounds"] >= 8, st["rounds"]
        for q, r in zip(queries, results):
            assert _same(q, _plain(graphs[q["graph"]], q), r), q
    finally:
        for g in graphs:
            g.close()
