"""GPU parity: every fused decode kernel against the CPU oracle on the same seeded datasets.

Integer results (decoded lists, timestamps, checksums, arrivals, hop counts, components, degrees,
colours) must be bit-exact.  PageRank and HITS run in FP32 on the GPU and in FP64 in the oracle;
their tolerances are stated next to each assertion.
"""
from __future__ import annotations

import numpy as np
import pytest

import compresstemporalgraph_b200 as tga
import pyoracle
from conftest import SHAPES
from test_temporal_paths import fastest_by_departures, latest_by_reversal

pytestmark = pytest.mark.gpu

T_MAX = tga.T_MAX


class Pair:
    def __init__(self, d, **cfg_kw):
        n = d["summary"]["n"]
        kw = dict(name=d["base"], max_label=n - 1, max_vertex=n)
        kw.update(cfg_kw)
        self.cfg = tga.DatasetConfig(**kw)
        self.g = tga.Graph.open_dir(d["dir"], d["base"], self.cfg)
        self.o = pyoracle.Oracle(d["dir"], d["base"], n)
        self.d = d
        self.n = n
        self.ml, self.mv, self.act = self.cfg.max_label, self.cfg.max_vertex, self.cfg.active_vertex_begin


@pytest.fixture(scope="module")
def pairs(datasets):
    out = {name: Pair(d) for name, d in datasets.items()}
    # Non-default configuration: inactive low ids and result arrays longer than the id space.
    out["small_view"] = Pair(datasets["chains"], active_vertex_begin=100, max_vertex=datasets["chains"]["summary"]["n"] + 37)
    yield out
    for p in out.values():
        p.g.close()


ALL = list(SHAPES) + ["small_view"]


@pytest.mark.parametrize("shape", list(SHAPES))
def test_decode_all_bit_exact(pairs, shape):
    p = pairs[shape]
    off, dst, ts = p.g.decode_all()
    ooff, odst, ots = p.o.csr()
    assert np.array_equal(off, ooff)
    assert np.array_equal(dst, odst)
    assert np.array_equal(ts, ots)


@pytest.mark.parametrize("shape", ALL)
def test_neighbor_access_checksums(pairs, shape):
    p = pairs[shape]
    small, csum, deg = p.g.neighbor_access()
    end = min(p.ml, p.n)
    osmall, ocs = p.o.checksums(p.act, end, p.mv)
    assert np.array_equal(csum[p.act:end], ocs[p.act:end])
    assert np.array_equal(small[p.act:end], osmall[p.act:end])
    t = p.g.timing()
    assert t["edges_decoded"] == int(deg[p.act:end].sum())


@pytest.mark.parametrize("shape", ["chains", "hubs", "small"])
def test_neighbors_single_vertex(pairs, shape):
    p = pairs[shape]
    off, _, _ = p.o.csr()
    degs = np.diff(off)
    picks = [0, int(np.argmax(degs)), p.n - 1] + list(np.random.default_rng(1).integers(0, p.n, 20))
    for v in picks:
        dst, ts = p.g.neighbors(int(v))
        odst, ots = p.o.neighbors(int(v))
        assert np.array_equal(dst, odst) and np.array_equal(ts, ots), v


def _windows(p):
    lo = p.d["params"].min_timestamp
    span = p.d["params"].ts_span
    return [(0, T_MAX), (lo + span // 4, lo + 3 * span // 4), (lo + span // 2, lo + span // 2 + span // 20)]


@pytest.mark.parametrize("shape", ALL)
def test_bfs_arrival_and_hops(pairs, shape):
    p = pairs[shape]
    off, _, _ = p.o.csr()
    degs = np.diff(off)
    srcs = [int(np.argmax(degs)), max(p.act, 1), p.act + 7]
    for src in srcs:
        for lo, hi in _windows(p):
            arr, hops = p.g.bfs(src, lo, hi)
            oarr, ohops = p.o.bfs(p.ml, p.mv, p.act, src, lo, hi)
            assert np.array_equal(arr, oarr), (src, lo, hi)
            assert np.array_equal(hops, ohops), (src, lo, hi)


@pytest.mark.parametrize("shape", ALL)
@pytest.mark.parametrize("early", [True, False])
@pytest.mark.parametrize("one_seed", [False, True])
def test_connected_components(pairs, shape, early, one_seed):
    p = pairs[shape]
    for lo, hi in _windows(p)[:2]:
        lab, k = p.g.connected_components(lo, hi, early_exit=early, one_seed=one_seed)
        olab, ok = p.o.cc(p.ml, p.mv, p.act, p.cfg.connected_components_vertex_begin, lo, hi, early)
        assert k == ok
        assert np.array_equal(lab, olab)


@pytest.mark.parametrize("shape", ["hubs", "chains"])
def test_cc_batch_equals_single_windows(pairs, shape):
    """Several CC windows in one launch (slots shared between the windows, each with its own
    candidates, early exits and labels) give every window the oracle's labels."""
    p = pairs[shape]
    lo0, span = p.d["params"].min_timestamp, p.d["params"].ts_span
    rng = np.random.default_rng(21)
    lo = lo0 + rng.integers(0, span // 2, 6)
    hi = lo + rng.integers(span // 20, span // 2, 6)
    lo[0], hi[0] = 0, T_MAX
    lo[3], hi[3] = lo[2], hi[2]  # the same window twice
    for early in (True, False):
        lab, comps = p.g.cc_batch(lo, hi, early_exit=early)
        for i in range(len(lo)):
            olab, ok = p.o.cc(p.ml, p.mv, p.act, p.cfg.connected_components_vertex_begin, int(lo[i]), int(hi[i]), early)
            assert comps[i] == ok, (i, early)
            assert np.array_equal(lab[i], olab), (i, early)


def test_cc_batch_more_windows_than_one_launch(pairs):
    """35 windows run as two launches (32 + 3); each row equals the single-window call."""
    p = pairs["hubs"]
    lo0, span = p.d["params"].min_timestamp, p.d["params"].ts_span
    rng = np.random.default_rng(22)
    lo = lo0 + rng.integers(0, span // 2, 35)
    hi = lo + rng.integers(span // 20, span // 2, 35)
    lab, comps = p.g.cc_batch(lo, hi)
    for i in (0, 5, 31, 32, 34):
        one, k = p.g.connected_components(int(lo[i]), int(hi[i]))
        assert comps[i] == k and np.array_equal(lab[i], one), i


@pytest.mark.parametrize("shape", ["hubs", "chains"])
def test_pagerank_batch_mixed_iteration_counts(pairs, shape):
    """One batch with a different iteration count per query (1, 3, 8, ...): row i equals the
    single-query PageRank with iters[i] within the FP32 tolerance of the other batched tests."""
    p = pairs[shape]
    lo0, span = p.d["params"].min_timestamp, p.d["params"].ts_span
    rng = np.random.default_rng(24)
    nq = 7
    lo = lo0 + rng.integers(0, span // 2, nq)
    hi = lo + rng.integers(span // 20, span // 2, nq)
    lo[0], hi[0] = 0, T_MAX
    iters = np.array([1, 3, 8, 3, 5, 2, 8], np.int32)
    out = p.g.pagerank_batch(lo, hi, iters=iters)
    for i in range(nq):
        one = p.g.pagerank(int(iters[i]), 0.85, 0.1, int(lo[i]), int(hi[i]))
        assert np.allclose(out[i], one, rtol=1e-4, atol=1e-9), i
        o = p.o.pagerank(p.ml, p.mv, p.act, int(iters[i]), 0.85, 0.1, int(lo[i]), int(hi[i]))
        assert float(np.abs(out[i].astype(np.float64) - o).sum()) <= 1e-5, i


@pytest.mark.parametrize("shape", ["hubs", "chains", "small"])
def test_is_neighbor_vs_oracle(pairs, shape):
    """Windowed point queries against the oracle's decoded lists: pairs taken from real edges (the
    window exactly one edge's timestamp, both ends inclusive, as the reference) and random pairs,
    hub lists entered through their checkpoints."""
    p = pairs[shape]
    off, dst, ts = p.o.csr()
    rng = np.random.default_rng(25)
    m = len(dst)
    deg = np.diff(off)
    hub = int(np.argmax(deg))
    k = rng.integers(0, m, 300)
    srcv = np.searchsorted(off, k, side="right") - 1
    hub_k = off[hub] + rng.integers(0, deg[hub], 100)
    x = np.concatenate([srcv, np.full(100, hub), rng.integers(0, p.n, 200)]).astype(np.int32)
    y = np.concatenate([dst[k], dst[hub_k], rng.integers(0, p.mv, 200)]).astype(np.int32)
    t_at = np.concatenate([ts[k], ts[hub_k], rng.integers(0, 10**8, 200)]).astype(np.int64)
    lo = t_at - rng.integers(0, 3, len(x))
    hi = t_at + rng.integers(-1, 3, len(x))  # hi < t_at in some rows: the edge itself is outside
    got = p.g.is_neighbor(x, y, lo, hi)
    any_t = p.g.is_neighbor(x, y)
    for i in range(len(x)):
        a, b = off[x[i]], off[x[i] + 1]
        sel = dst[a:b] == y[i]
        assert got[i] == bool(np.any(sel & (ts[a:b] >= lo[i]) & (ts[a:b] <= hi[i]))), i
        assert any_t[i] == bool(np.any(sel)), i


def test_cc_job_resumes_across_steps_and_reuses_slots(pairs):
    """A CC job stepped with a tiny budget (one batch per step), with batched BFS and a plain CC
    run on the handle between steps and windows added as slots free up, gives each window the
    single-call result."""
    p = pairs["hubs"]
    lo0, span = p.d["params"].min_timestamp, p.d["params"].ts_span
    rng = np.random.default_rng(23)
    lo = [int(x) for x in lo0 + rng.integers(0, span // 2, 5)]
    hi = [int(l + w) for l, w in zip(lo, rng.integers(span // 20, span // 2, 5))]
    lo[0], hi[0] = 0, T_MAX
    want = [p.g.connected_components(lo[i], hi[i], early_exit=False) for i in range(5)]
    got, steps = {}, 0
    with tga.CcJob(p.g, capacity=2, early_exit=False) as job:
        slot_of = {job.add(lo[0], hi[0]): 0, job.add(lo[1], hi[1]): 1}
        nxt = 2
        while slot_of:
            fin = job.step(budget_ms=1e-6)
            steps += 1
            p.g.bfs_batch(np.array([0, 5], np.int32), np.array([lo[2], 0], np.int64), np.array([hi[2], T_MAX], np.int64))
            if steps == 2:
                p.g.connected_components(lo[3], hi[3])
            for s in fin:
                got[slot_of.pop(s)] = job.take(s)
                if nxt < 5:
                    slot_of[job.add(lo[nxt], hi[nxt])] = nxt
                    nxt += 1
            assert steps < 100000
    assert steps > 5  # the budget really split the work (no early exit: every window runs to the end)
    for i in range(5):
        assert got[i][1] == want[i][1] and np.array_equal(got[i][0], want[i][0]), i


def test_cc_after_work_decomposition_change(pairs):
    """The cached CC job (and a caller's job) hold a per-run table sized for the decomposition they
    were made under: after set_work_params the cached one is rebuilt (results still exact) and a
    caller's job refuses to run instead of using the stale table."""
    p = pairs["hubs"]
    lo, hi = _windows(p)[1]
    olab, ok = p.o.cc(p.ml, p.mv, p.act, p.cfg.connected_components_vertex_begin, lo, hi, True)
    default = p.g.work_params()
    job = tga.CcJob(p.g, capacity=2)
    try:
        lab, k = p.g.connected_components(lo, hi)  # makes the cached job
        assert k == ok and np.array_equal(lab, olab)
        for sl in (16, 4096):
            p.g.set_work_params(sl, default["item_edges"])
            lab, k = p.g.connected_components(lo, hi)
            assert k == ok and np.array_equal(lab, olab), sl
        with pytest.raises(tga.TgaError) as e:
            job.add(lo, hi)
        assert e.value.code == tga.TGA_E_ARG
    finally:
        job.close()
        p.g.set_work_params(default["slice_edges"], default["item_edges"])


def test_autotune_keeps_results(pairs):
    """The autotuner picks a configuration from its candidate sets, no slower than the starting
    one on its own probe, and every result stays equal to the oracle under it."""
    p = pairs["hubs"]
    default = p.g.work_params()
    try:
        r = p.g.autotune()
        assert r["slice_edges"] in (16, 24, 32, 48) and r["item_edges"] in (128, 256, 512)
        # the starting configuration is timed once (one fewer grid point when it lies on the grid)
        assert r["dense_div"] in (1, 2, 4) and r["candidates"] in (14, 15)
        assert 0 < r["best_ms"] <= r["default_ms"]
        assert p.g.work_params()["slice_edges"] == r["slice_edges"]
        off, dst, ts = p.g.decode_all()
        ooff, odst, ots = p.o.csr()
        assert np.array_equal(dst, odst) and np.array_equal(ts, ots)
        lo, hi = _windows(p)[1]
        lab, k = p.g.connected_components(lo, hi)
        olab, ok = p.o.cc(p.ml, p.mv, p.act, p.cfg.connected_components_vertex_begin, lo, hi, True)
        assert k == ok and np.array_equal(lab, olab)
    finally:
        p.g.set_work_params(default["slice_edges"], default["item_edges"])


def test_bounded_barrier_wait_reports_timeout(pairs):
    """A grid-barrier wait that nothing ends (a block that never arrives) runs out after its limit
    and reports the timeout status; the context stays usable for the next traversal."""
    import time as _time

    t = _time.perf_counter()
    assert tga.barrier_selftest(200.0)
    assert _time.perf_counter() - t >= 0.2
    p = pairs["chains"]
    arr, _ = p.g.bfs(0)
    assert np.array_equal(arr, p.o.bfs(p.ml, p.mv, p.act, 0)[0])


def test_multi_source_state_survives_other_calls(pairs):
    """The batched traversal keeps its per-source arrays between calls and resets only the
    vertices the previous traversal touched; single-source traversals, batched CC and batched
    BFS interleaved on one handle must each still match the oracle."""
    p = pairs["hubs"]
    lo, hi = _windows(p)[1]
    n = p.n
    srcs = np.array([0, n // 3, n - 1, 7], np.int32)
    blo = np.array([lo, 0, lo, lo], np.int64)
    bhi = np.array([hi, T_MAX, T_MAX, hi], np.int64)
    for _ in range(2):
        out = p.g.bfs_batch(srcs, blo, bhi)
        for i in range(len(srcs)):
            oarr, _ = p.o.bfs(p.ml, p.mv, p.act, int(srcs[i]), int(blo[i]), int(bhi[i]))
            assert np.array_equal(out[i], oarr), i
        arr, _ = p.g.bfs(int(srcs[1]), lo, hi)
        assert np.array_equal(arr, p.o.bfs(p.ml, p.mv, p.act, int(srcs[1]), lo, hi)[0])
        lab, k = p.g.connected_components(lo, hi)
        olab, ok = p.o.cc(p.ml, p.mv, p.act, p.cfg.connected_components_vertex_begin, lo, hi, True)
        assert k == ok and np.array_equal(lab, olab)


@pytest.mark.parametrize("shape", ALL)
@pytest.mark.parametrize("iters", [1, 20])
def test_pagerank_fp32_vs_fp64(pairs, shape, iters):
    p = pairs[shape]
    for lo, hi in _windows(p)[:2]:
        r = p.g.pagerank(iters, 0.85, 0.1, lo, hi)
        o = p.o.pagerank(p.ml, p.mv, p.act, iters, 0.85, 0.1, lo, hi)
        # Stated tolerance: L1 distance to the FP64 oracle <= 1e-5 of the total rank mass (1.0),
        # and every entry within 1e-4 relative + 1e-9 absolute.
        l1 = float(np.abs(r.astype(np.float64) - o).sum())
        assert l1 <= 1e-5, l1
        assert np.allclose(r, o, rtol=1e-4, atol=1e-9)


@pytest.mark.parametrize("shape", ALL)
@pytest.mark.parametrize("mode", [tga.HITS_GPU, tga.HITS_JAVA])
def test_hits_fp32_vs_fp64(pairs, shape, mode):
    p = pairs[shape]
    iters = 10
    for lo, hi in _windows(p)[:2]:
        hub, auth = p.g.hits(iters, mode, lo, hi)
        ohub, oauth = p.o.hits(p.ml, p.mv, p.act, iters, mode == tga.HITS_JAVA, lo, hi)
        # Stated tolerance: unit-L2 vectors; L1 distance to FP64 <= 1e-4 and max error <= 1e-5.
        for a, b in ((hub, ohub), (auth, oauth)):
            assert float(np.abs(a.astype(np.float64) - b).sum()) <= 1e-4
            assert float(np.abs(a.astype(np.float64) - b).max()) <= 1e-5


@pytest.mark.parametrize("shape", ALL)
def test_degree_centrality(pairs, shape):
    p = pairs[shape]
    lo = p.d["params"].min_timestamp
    span = p.d["params"].ts_span
    for s, e in [(0, 0), (lo + span // 3, lo + 2 * span // 3), (lo, lo)]:
        deg, avg = p.g.degree_centrality(s, e)
        odeg, oavg = p.o.degree(p.ml, p.mv, p.act, s, e)
        assert np.array_equal(deg, odeg), (s, e)
        assert np.array_equal(avg, oavg), (s, e)


@pytest.mark.parametrize("shape", ALL)
@pytest.mark.parametrize("java_isolated", [False, True])
def test_coloring_curand_priorities(pairs, shape, java_isolated):
    p = pairs[shape]
    col, prio, rounds = p.g.color(0, java_isolated=java_isolated)
    assert prio.max() < 256
    ocol, orounds = p.o.color(p.ml, p.mv, p.act, prio, java_isolated)
    assert rounds == orounds
    assert np.array_equal(col, ocol)


def test_coloring_java_priorities(pairs):
    p = pairs["small"]
    col, prio, rounds = p.g.color(1)
    assert np.array_equal(prio, pyoracle.java_random256(123, p.mv))
    ocol, _ = p.o.color(p.ml, p.mv, p.act, prio)
    assert np.array_equal(col, ocol)


def test_coloring_given_priorities(pairs):
    p = pairs["hubs"]
    prio = np.random.default_rng(5).integers(0, 4, p.mv).astype(np.uint32)  # many ties
    col, pout, _ = p.g.color(2, prio)
    assert np.array_equal(pout, prio)
    ocol, _ = p.o.color(p.ml, p.mv, p.act, prio)
    assert np.array_equal(col, ocol)


def test_batched_bfs_equals_single(pairs):
    p = pairs["chains"]
    rng = np.random.default_rng(2)
    srcs = rng.integers(0, p.n, 70).astype(np.int32)
    span = p.d["params"].ts_span
    lo = rng.integers(0, span // 2, 70)
    hi = lo + rng.integers(span // 20, span // 2, 70)
    out = p.g.bfs_batch(srcs, lo, hi)
    for i in range(0, 70, 9):
        arr, _ = p.g.bfs(int(srcs[i]), int(lo[i]), int(hi[i]))
        assert np.array_equal(out[i], arr)


@pytest.mark.parametrize("shape", ["hubs", "intervals"])
def test_batched_bfs_many_sources_vs_oracle(pairs, shape):
    """300 sources (two launches of at most 256), each with its own window, duplicates included."""
    p = pairs[shape]
    rng = np.random.default_rng(4)
    lo0, span = p.d["params"].min_timestamp, p.d["params"].ts_span
    srcs = rng.integers(0, p.n, 300).astype(np.int32)
    srcs[10] = srcs[11]
    lo = lo0 + rng.integers(0, span // 2, 300)
    hi = lo + rng.integers(span // 20, span // 2, 300)
    lo[:5], hi[:5] = 0, T_MAX
    out = p.g.bfs_batch(srcs, lo, hi)
    for i in list(range(0, 300, 7)) + [10, 11, 255, 256, 299]:
        oarr, _ = p.o.bfs(p.ml, p.mv, p.act, int(srcs[i]), int(lo[i]), int(hi[i]))
        assert np.array_equal(out[i], oarr), i


def test_batched_pagerank_equals_single(pairs):
    p = pairs["small"]
    span = p.d["params"].ts_span
    lo = np.array([0, span // 4, span // 2], np.int64)
    hi = np.array([T_MAX, span // 2, span], np.int64)
    out = p.g.pagerank_batch(lo, hi, iters=5)
    for i in range(3):
        r = p.g.pagerank(5, 0.85, 0.1, int(lo[i]), int(hi[i]))
        assert np.allclose(out[i], r, rtol=1e-4, atol=1e-9)


@pytest.mark.parametrize("shape", ["hubs", "chains"])
def test_batched_pagerank_many_queries_vs_oracle(pairs, shape):
    """40 queries (two launches of at most 32), full and windowed, against the FP64 oracle with the
    tolerance of test_pagerank_fp32_vs_fp64."""
    p = pairs[shape]
    rng = np.random.default_rng(6)
    lo0, span = p.d["params"].min_timestamp, p.d["params"].ts_span
    lo = lo0 + rng.integers(0, span // 2, 40)
    hi = lo + rng.integers(span // 20, span // 2, 40)
    lo[:3], hi[:3] = 0, T_MAX
    out = p.g.pagerank_batch(lo, hi, iters=8)
    for i in list(range(0, 40, 6)) + [1, 31, 32, 39]:
        o = p.o.pagerank(p.ml, p.mv, p.act, 8, 0.85, 0.1, int(lo[i]), int(hi[i]))
        assert float(np.abs(out[i].astype(np.float64) - o).sum()) <= 1e-5, i
        assert np.allclose(out[i], o, rtol=1e-4, atol=1e-9), i


def test_timing_reports_device_time(pairs):
    p = pairs["small"]
    for _ in range(2):  # the first call captures the iteration loop as a CUDA graph, the second replays it
        p.g.pagerank(3)
        t = p.g.timing()
        assert t["total_ms"] > 0 and t["decode_ms"] > 0 and t["decode_launches"] == 3
        assert t["decode_ms"] <= t["total_ms"] * 1.01
    assert t["edges_decoded"] == 3 * p.o.m - 3 * int(np.diff(p.o.csr()[0])[p.ml:].sum())


@pytest.mark.parametrize("shape", ["hubs", "chains", "small"])
@pytest.mark.parametrize("slice_edges,item_edges", [(16, 8), (64, 300), (4096, 2048)])
def test_work_decomposition_does_not_change_results(pairs, shape, slice_edges, item_edges):
    """Tiny slices force checkpoint restores (including seeks over long skip blocks of a
    referenced list); results must not depend on the decomposition."""
    p = pairs[shape]
    g = p.g
    default = g.work_params()
    g.set_work_params(slice_edges, item_edges)
    try:
        wp = g.work_params()
        assert wp["slice_edges"] == slice_edges and wp["items"] > 0
        off, dst, ts = g.decode_all()
        ooff, odst, ots = p.o.csr()
        assert np.array_equal(dst, odst) and np.array_equal(ts, ots)
        _, csum, _ = g.neighbor_access()
        end = min(p.ml, p.n)
        _, ocs = p.o.checksums(p.act, end, p.mv)
        assert np.array_equal(csum[p.act:end], ocs[p.act:end])
        src = int(np.argmax(np.diff(ooff)))
        arr, hops = g.bfs(src)
        oarr, ohops = p.o.bfs(p.ml, p.mv, p.act, src)
        assert np.array_equal(arr, oarr) and np.array_equal(hops, ohops)
        r = g.pagerank(5)
        assert float(np.abs(r - p.o.pagerank(p.ml, p.mv, p.act, 5)).sum()) <= 1e-5
        col, prio, _ = g.color(0)
        ocol, _ = p.o.color(p.ml, p.mv, p.act, prio)
        assert np.array_equal(col, ocol)
        deg, avg = g.degree_centrality(0, 0)
        odeg, oavg = p.o.degree(p.ml, p.mv, p.act, 0, 0)
        assert np.array_equal(deg, odeg) and np.array_equal(avg, oavg)
        # Windowed calls: slices that start inside a run of equal successors must keep exactly the
        # run's first in-window edge, whose position depends on the window.
        lo, hi = _windows(p)[1]
        arr, hops = g.bfs(src, lo, hi)
        oarr, ohops = p.o.bfs(p.ml, p.mv, p.act, src, lo, hi)
        assert np.array_equal(arr, oarr) and np.array_equal(hops, ohops)
        lab, k = g.connected_components(lo, hi)
        olab, ok = p.o.cc(p.ml, p.mv, p.act, p.cfg.connected_components_vertex_begin, lo, hi, True)
        assert k == ok and np.array_equal(lab, olab)
        r = g.pagerank(5, 0.85, 0.1, lo, hi)
        assert float(np.abs(r - p.o.pagerank(p.ml, p.mv, p.act, 5, 0.85, 0.1, lo, hi)).sum()) <= 1e-5
        srcs = np.array([src, src, 0, p.n - 1, src], np.int32)
        blo = np.array([lo, 0, lo, 0, lo + (hi - lo) // 2], np.int64)
        bhi = np.array([hi, T_MAX, hi, hi, hi], np.int64)
        bout = g.bfs_batch(srcs, blo, bhi)
        for i in range(len(srcs)):
            oarr, _ = p.o.bfs(p.ml, p.mv, p.act, int(srcs[i]), int(blo[i]), int(bhi[i]))
            assert np.array_equal(bout[i], oarr), i
        rb = g.pagerank_batch(np.array([lo, 0], np.int64), np.array([hi, T_MAX], np.int64), iters=5)
        assert float(np.abs(rb[0] - p.o.pagerank(p.ml, p.mv, p.act, 5, 0.85, 0.1, lo, hi)).sum()) <= 1e-5
        assert float(np.abs(rb[1] - p.o.pagerank(p.ml, p.mv, p.act, 5)).sum()) <= 1e-5
        hub, auth = g.hits(5, tga.HITS_JAVA, lo, hi)
        ohub, oauth = p.o.hits(p.ml, p.mv, p.act, 5, True, lo, hi)
        assert float(np.abs(hub.astype(np.float64) - ohub).max()) <= 1e-5
        assert float(np.abs(auth.astype(np.float64) - oauth).max()) <= 1e-5
    finally:
        g.set_work_params(default["slice_edges"], default["item_edges"])


# ---- fastest temporal paths --------------------------------------------------------------------

def _fastest_oracle(p, src, lo, hi):
    return fastest_by_departures(p.o, p.n, p.ml, p.mv, p.act, src, lo, hi)


def _path_sources(p, lo, hi, count=3, most=40):
    off, _, ts = p.o.csr()
    out = []
    for v in np.random.default_rng(5).permutation(min(p.n, p.ml)):
        t = ts[off[v]:off[v + 1]]
        if 2 <= len(np.unique(t[(t >= lo) & (t < hi)])) <= most:
            out.append(int(v))
            if len(out) == count:
                break
    return out


# widespan is left out: arrivals are 32-bit times, so the path queries need timestamps below 2^31.
@pytest.mark.parametrize("shape", ["small", "chains", "hubs", "intervals", "sparse", "small_view"])
def test_fastest_paths(pairs, shape):
    p = pairs[shape]
    for lo, hi in _windows(p)[:2]:
        lo = max(lo, 0)
        for src in _path_sources(p, lo, hi):
            dur, dep = p.g.fastest(src, lo, hi)
            odur, odep = _fastest_oracle(p, src, lo, hi)
            assert np.array_equal(dur, odur), (src, lo, hi)
            assert np.array_equal(dep, odep), (src, lo, hi)
            assert (dur >= -1).all() and dur[src] == 0
            # A fastest path departs no earlier than the window and takes no longer than arriving early.
            arr, _ = p.g.bfs(src, lo, hi)
            r = dur > 0
            assert (dep[r] >= lo).all()
            assert (dur[r] <= arr[r].astype(np.int64) - lo).all()


def test_fastest_paths_from_a_hub(pairs):
    """400 departures of the largest hub: two traversal batches (256 + 144 rows of 2,000 vertices),
    each large enough for the minimum to be taken on several host threads."""
    p = pairs["hubs"]
    off, _, _ = p.o.csr()
    hub = int(np.argmax(np.diff(off)))
    _, ts = p.o.neighbors(hub)
    uts = np.unique(ts)
    assert len(uts) > 500
    lo, hi = int(uts[len(uts) // 4]), int(uts[len(uts) // 4 + 400])
    dur, dep = p.g.fastest(hub, lo, hi)
    odur, odep = _fastest_oracle(p, hub, lo, hi)
    assert np.array_equal(dur, odur)
    assert np.array_equal(dep, odep)


def test_fastest_paths_edge_cases(pairs):
    p = pairs["small_view"]  # max_vertex exceeds the vertices in the files
    dur, dep = p.g.fastest(p.mv - 1)
    assert dur[p.mv - 1] == 0 and (np.delete(dur, p.mv - 1) == -1).all() and (dep == -1).all()
    off, _, _ = p.o.csr()
    for sink in np.flatnonzero(np.diff(off) == 0)[:1]:  # a vertex without out-edges, if there is one
        dur, dep = p.g.fastest(int(sink))
        assert dur[sink] == 0 and (np.delete(dur, sink) == -1).all() and (dep == -1).all()
    with pytest.raises(tga.TgaError):
        p.g.fastest(0, 10, 10)
    with pytest.raises(tga.TgaError):
        p.g.fastest(p.mv)


# ---- latest departure on the time-reversed copy -----------------------------------------------

@pytest.mark.parametrize("shape", ["small", "chains", "hubs", "intervals", "sparse"])
def test_latest_departure(pairs, shape, tmp_path):
    p = pairs[shape]
    off, dst, ts = p.o.csr()
    pivot = p.g.reverse(tmp_path / "dev", "rev")
    assert pivot == int(ts.max())
    # The copy written from the device decode equals the one written from the oracle's lists.
    tga.write_reversed(off, dst, ts, pivot, tmp_path / "cpu", "rev")
    for f in sorted((tmp_path / "cpu").iterdir()):
        assert (tmp_path / "dev" / f.name).read_bytes() == f.read_bytes(), f.name
    orev = pyoracle.Oracle(tmp_path / "cpu", "rev", p.n)
    with tga.Graph.open_dir(tmp_path / "dev", "rev", p.cfg) as grev:
        targets = [int(np.argmax(np.bincount(dst, minlength=p.n))), 1, p.n // 2]
        lo0, span = p.d["params"].min_timestamp, p.d["params"].ts_span
        for target in targets:
            for lo, hi in [(0, T_MAX), (lo0 + span // 4, lo0 + 3 * span // 4), (pivot + 1, T_MAX)]:
                got = grev.latest_departure(pivot, target, lo, hi)
                want = latest_by_reversal(orev, p.n, p.ml, p.mv, p.act, pivot, target, lo, hi)
                assert np.array_equal(got, want), (target, lo, hi)
        with pytest.raises(tga.TgaError):
            grev.latest_departure(pivot, 0, 5, 5)


# ---- fewest-hop temporal paths --------------------------------------------------------------

# widespan is left out: arrivals are 32-bit times, as in tga_bfs.
@pytest.mark.parametrize("shape", ["small", "chains", "hubs", "intervals", "sparse", "refsafe", "small_view"])
def test_shortest_paths(pairs, shape):
    p = pairs[shape]
    off, _, _ = p.o.csr()
    degs = np.diff(off)
    srcs = [int(np.argmax(degs)), max(p.act, 1), p.act + 7]
    for src in srcs:
        for lo, hi in _windows(p):
            hops, arr = p.g.shortest(src, lo, hi)
            ohops, oarr = p.o.shortest(p.ml, p.mv, p.act, src, lo, hi)
            assert np.array_equal(hops, ohops), (src, lo, hi)
            assert np.array_equal(arr, oarr), (src, lo, hi)
            # The earliest arrival is tga_bfs's, and no path is longer than the one along earliest arrivals.
            barr, bhops = p.g.bfs(src, lo, hi)
            assert np.array_equal(arr, barr)
            r = hops != np.iinfo(np.int32).max
            assert (hops[r] <= bhops[r]).all()


def test_shortest_paths_rejects_bad_input(pairs):
    p = pairs["small"]
    with pytest.raises(tga.TgaError):
        p.g.shortest(0, 10, 10)
    with pytest.raises(tga.TgaError):
        p.g.shortest(p.mv)


@pytest.mark.parametrize("shape", ["hubs", "chains"])
def test_dense_levels_equal_queue_levels(datasets, shape, monkeypatch):
    """With the default divisor a level sweeps the whole schedule only when every entry is in its
    frontier; TGA_DENSE_DIV=64 (read at open) makes every level with 1/64 of the entries a sweep,
    so the dense paths of BFS (phase 1 and hops), the one-seed and batched CC and the multi-source
    BFS give the oracle's results as well."""
    monkeypatch.setenv("TGA_DENSE_DIV", "64")
    p = Pair(datasets[shape])
    try:
        off, _, _ = p.o.csr()
        src = int(np.argmax(np.diff(off)))
        for lo, hi in _windows(p)[:2]:
            arr, hops = p.g.bfs(src, lo, hi)
            oarr, ohops = p.o.bfs(p.ml, p.mv, p.act, src, lo, hi)
            assert np.array_equal(arr, oarr) and np.array_equal(hops, ohops), (lo, hi)
            for one_seed in (False, True):
                lab, k = p.g.connected_components(lo, hi, early_exit=False, one_seed=one_seed)
                olab, ok = p.o.cc(p.ml, p.mv, p.act, p.cfg.connected_components_vertex_begin, lo, hi, False)
                assert k == ok and np.array_equal(lab, olab), (lo, hi, one_seed)
        srcs = np.arange(0, p.n, max(1, p.n // 40), dtype=np.int32)[:40]
        lo = np.zeros(len(srcs), np.int64)
        hi = np.full(len(srcs), T_MAX, np.int64)
        out = p.g.bfs_batch(srcs, lo, hi)
        for i in range(0, len(srcs), 5):
            oarr, _ = p.o.bfs(p.ml, p.mv, p.act, int(srcs[i]), 0, T_MAX)
            assert np.array_equal(out[i], oarr), i
    finally:
        p.g.close()
