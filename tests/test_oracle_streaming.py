"""The oracle's streaming workloads (lists decoded from the compressed streams at every visit, the
form bench.py's CPU arm times) give the same results as its materialised workloads, and count
the edges they decode.  CPU only."""
from __future__ import annotations

import numpy as np
import pytest

import pyoracle
from conftest import SHAPES


@pytest.fixture(scope="module")
def oracles(datasets):
    out = {}
    for name, d in datasets.items():
        n = d["summary"]["n"]
        out[name] = (pyoracle.Oracle(d["dir"], d["base"], n), n, d)
    yield out
    for o, _, _ in out.values():
        o.close()


@pytest.mark.parametrize("shape", list(SHAPES))
def test_streaming_equals_materialised(oracles, shape):
    o, n, d = oracles[shape]
    ml, mv, act = n - 1, n, 0
    off, _, _ = o.csr()
    deg = np.diff(off)
    src = int(deg.argmax())
    m_active = int(deg[act:ml].sum())

    (arr, hops), e = o.stream_bfs(ml, mv, act, src)
    oarr, ohops = o.bfs(ml, mv, act, src)
    assert np.array_equal(arr, oarr) and np.array_equal(hops, ohops)
    assert e > 0

    (lab, k), e = o.stream_cc(ml, mv, act, 0)
    olab, ok = o.cc(ml, mv, act, 0)
    assert k == ok and np.array_equal(lab, olab)

    (hub, auth), e = o.stream_hits(ml, mv, act, 5, threads=2)
    ohub, oauth = o.hits(ml, mv, act, 5)
    assert np.allclose(hub, ohub, rtol=1e-12, atol=1e-15) and np.allclose(auth, oauth, rtol=1e-12, atol=1e-15)
    assert e == 2 * 5 * m_active  # every list of [active, max_label) twice per iteration

    lo = d["params"].min_timestamp + d["params"].ts_span // 3
    for s, t in [(0, 0), (lo, lo + d["params"].ts_span // 3)]:
        (dg, avg), e = o.stream_degree(ml, mv, act, s, t, threads=2)
        odg, oavg = o.degree(ml, mv, act, s, t)
        assert np.array_equal(dg, odg) and np.array_equal(avg, oavg)
        assert e == int(deg[act:ml + 1].sum())

    prio = pyoracle.java_random256(123, mv)
    (col, r), e = o.stream_color(ml, mv, act, prio, threads=2)
    ocol, orr = o.color(ml, mv, act, prio)
    assert r == orr and np.array_equal(col, ocol)

    r1, e1 = o.stream_pagerank(ml, mv, act, 3, threads=2)
    assert np.allclose(r1, o.pagerank(ml, mv, act, 3), rtol=1e-9, atol=1e-15)
