"""Host logic of the drop-in executables without a GPU: the tool's own source linked against a fake of
the C ABI (tests/fakes/fake_tga.cpp) whose calls return fixed arrays.  Checks the reference's stdout
lines, the JSON result line, the --out layouts, the PageRank summary line (pagerank.cu:2012-2042),
--repeat and the mapping of library failures to exit statuses."""
from __future__ import annotations

import json
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
NV = 10000  # the Comm preset's MAX_Vertex


@pytest.fixture(scope="module")
def fake_tool(tmp_path_factory):
    d = tmp_path_factory.mktemp("fake_tool")
    inc = f"-I{ROOT / 'include'}"
    subprocess.run(["g++", "-O1", "-std=c++17", inc, "-shared", "-fPIC", str(ROOT / "tests" / "fakes" / "fake_tga.cpp"),
                    "-o", str(d / "libtgafake.so")], check=True)
    subprocess.run(["g++", "-O1", "-std=c++17", inc, str(ROOT / "compresstemporalgraph_b200" / "csrc" / "tools" / "tga_tool.cpp"),
                    "-o", str(d / "tga_tool"), f"-L{d}", "-ltgafake", f"-Wl,-rpath,{d}"], check=True)
    return d / "tga_tool"


def run(tool, *args, fail=None):
    env = {k: v for k, v in os.environ.items() if k not in ("FAKE_TGA_FAIL", "TGA_DUMP_RANK_SUMMARY")}
    if fail is not None:
        env["FAKE_TGA_FAIL"] = str(fail)
    return subprocess.run([str(tool), *map(str, args)], capture_output=True, text=True, env=env)


def out_of(tool, tmp_path, alg, *extra):
    out = tmp_path / f"{alg}.bin"
    r = run(tool, alg, "--dataset", "Comm", "--json", "--out", out, *extra)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    return lines, json.loads(lines[-1]), out.read_bytes()


def test_bfs(fake_tool, tmp_path):
    lines, js, raw = out_of(fake_tool, tmp_path, "bfs", "--repeat", 3, "--autotune")
    assert lines[:6] == ["Starting simple parallel bfs.", "BFS Elapsed time in milliseconds : 12 ms."] * 3
    i = np.arange(NV)
    arr = np.where(i % 3 != 0, i, 2**31 - 1).astype(np.int32)
    got = np.frombuffer(raw, np.int32)
    assert np.array_equal(got[:NV], arr) and np.array_equal(got[NV:], (i % 7).astype(np.int32))
    assert js["reached"] == int((i % 3 != 0).sum()) and js["max_hops"] == 6 and js["repeat"] == 3
    assert js["device_ms"] == 12.75 and js["edges_decoded"] == 1000 and js["window"] == [0, 2**63 - 1]
    assert js["tuned"] == {"slice_edges": 16, "item_edges": 128, "dense_div": 8}
    assert js["max_vertex"] == NV and js["max_label"] == NV - 1 and js["dataset"] == "Comm"


def test_connected_components(fake_tool, tmp_path):
    lines, js, raw = out_of(fake_tool, tmp_path, "connected_components")
    assert lines[0] == "Elapsed time in milliseconds : 12 ms."
    lab = np.arange(NV) % 4 - 1
    assert np.array_equal(np.frombuffer(raw, np.int32), lab)
    assert js["components"] == 3 and js["labelled"] == int((lab != -1).sum())


def test_degree_centrality(fake_tool, tmp_path):
    lines, js, raw = out_of(fake_tool, tmp_path, "degree_centrality")
    assert lines[:2] == ["Starting simple parallel Degree Centre.", "Elapsed time in milliseconds : 12 ms."]
    assert np.array_equal(np.frombuffer(raw[:4 * NV], np.int32), np.arange(NV))
    assert np.array_equal(np.frombuffer(raw[4 * NV:], np.int64), -np.arange(NV))
    assert js["degree_sum"] == NV * (NV - 1) // 2 and js["window"] == [0, 0]


def test_graph_coloring(fake_tool, tmp_path):
    lines, js, raw = out_of(fake_tool, tmp_path, "graph_coloring")
    assert lines[:2] == ["Starting simple parallel Graph Color.", "Elapsed time in milliseconds : 12 ms."]
    i = np.arange(NV)
    col = np.where(i % 5 != 0, i % 5, 2**32 - 1).astype(np.uint32)
    assert np.array_equal(np.frombuffer(raw[:4 * NV], np.uint32), col)
    assert np.array_equal(np.frombuffer(raw[4 * NV:], np.uint32), (i * 7 % 256).astype(np.uint32))
    assert js["rounds"] == 5 and js["coloured"] == int((i % 5 != 0).sum())


def test_hits_non_finite_is_null(fake_tool, tmp_path):
    lines, js, raw = out_of(fake_tool, tmp_path, "hits")
    assert lines[:2] == ["Starting simple parallel HITS.", "Elapsed time in milliseconds : 12 ms."]
    assert js["hub_l2sq"] is None and js["auth_l2sq"] == pytest.approx(NV * 0.0625)
    got = np.frombuffer(raw, np.float32)
    assert np.isnan(got[0]) and (got[1:NV] == 0.5).all() and (got[NV:] == 0.25).all()


def test_neighbor_access(fake_tool, tmp_path):
    lines, js, raw = out_of(fake_tool, tmp_path, "neighbor_access")
    assert lines[0] == "Time = 12.75 ms."
    i = np.arange(NV)
    assert np.array_equal(np.frombuffer(raw[:4 * NV], np.int32), 2 * i)
    assert np.array_equal(np.frombuffer(raw[4 * NV:12 * NV], np.uint64), np.uint64(2**64 - 1) - i.astype(np.uint64))
    assert np.array_equal(np.frombuffer(raw[12 * NV:], np.uint8), (i & 1).astype(np.uint8))
    assert js["edges"] == NV * (NV - 1) and js["small"] == NV // 2
    assert js["checksum_sum"] == f"{int((np.uint64(2**64 - 1) - i.astype(np.uint64)).sum(dtype=np.uint64)):016x}"


@pytest.mark.parametrize("how", ["flag", "env"])
def test_pagerank_summary_line(fake_tool, tmp_path, how):
    out = tmp_path / "pr.bin"
    args = ["pagerank", "--dataset", "Comm", "--out", out]
    if how == "flag":
        r = run(fake_tool, *args, "--rank-summary")
    else:
        env = dict(os.environ, TGA_DUMP_RANK_SUMMARY="1")
        r = subprocess.run([str(fake_tool), *map(str, args)], capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert lines[:2] == ["Starting simple parallel PageRank.", "PageRank Elapsed time in milliseconds : 12 ms."]
    rank = np.frombuffer(out.read_bytes(), np.float32).astype(np.float64)
    head, top = lines[2].split(" top10=")
    assert head.startswith("PageRank alpha=0.1 rank_sum=")
    assert float(head.split("rank_sum=")[1]) == pytest.approx(rank.sum(), rel=1e-11)
    # Ten equal largest values: the lowest ids first, as the reference's insertion keeps them.
    order = np.lexsort((np.arange(NV), -rank))[:10]
    assert [int(p.split(":")[0]) for p in top.split(",")] == order.tolist()
    assert len(lines) == 3


def test_library_failures_map_to_exit_statuses(fake_tool):
    r = run(fake_tool, "bfs", "--dataset", "Comm", fail=5)  # TGA_E_TIMEOUT
    assert r.returncode == 1
    assert "bfs failed (status 5): fake failure" in r.stderr
    assert "BFS Elapsed" not in r.stdout
    r = run(fake_tool, "hits", "--dataset", "Comm", fail=6)  # TGA_E_ARG
    assert r.returncode == 2
    r = run(fake_tool, "neighbor_access", "--dataset", "Comm", "--out", "/nonexistent-dir/x.bin")
    assert r.returncode == 1 and "cannot write /nonexistent-dir/x.bin" in r.stderr
