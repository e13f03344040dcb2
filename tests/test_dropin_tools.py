"""The seven drop-in executables (bfs, connected_components, degree_centrality, graph_coloring,
hits, neighbor_access, pagerank; gpu_cuda/<DS>/<alg>.cu in the reference).

CPU: names, usage, argument errors (exit 2) and the reference's missing-file line and exit status
(shared/path_config.cuh:26-36).  GPU: each executable's result arrays (--out) equal the library's
for the same dataset and settings, its stdout carries the reference's lines, and --json summarises
the same result.
"""
import json
import os
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import REFERENCE_ROOT, has_gpu

import compresstemporalgraph_b200 as tga

BIN = Path(tga.__file__).resolve().parent / "bin"
ALGS = ["bfs", "connected_components", "degree_centrality", "graph_coloring", "hits", "neighbor_access", "pagerank"]
INT32_MAX = 2**31 - 1


def run(name, *args, env=None, cwd=None, timeout=300):
    e = dict(os.environ)
    e.pop("TGA_COMPRESS_ROOT", None)
    e.pop("TGA_DUMP_RANK_SUMMARY", None)
    e.update(env or {})
    return subprocess.run([str(BIN / name), *map(str, args)], capture_output=True, text=True, env=e, cwd=cwd,
                          timeout=timeout)


# ---- CPU ----------------------------------------------------------------------------------------

def test_seven_names_link_to_one_tool():
    assert (BIN / "tga_tool").is_file()
    for a in ALGS:
        p = BIN / a
        assert p.is_symlink() and os.readlink(p) == "tga_tool", a


@pytest.mark.parametrize("name", ALGS)
def test_help(name):
    r = run(name, "--help")
    assert r.returncode == 0
    assert r.stdout.startswith(f"usage: {name} ")


def test_missing_file_is_the_reference_line(tmp_path):
    # Default root ../.. relative to the working directory (dataset_config_base.cuh:39-41).
    work = tmp_path / "a" / "b"
    work.mkdir(parents=True)
    r = run("bfs", "--dataset", "Comm", cwd=work)
    assert r.returncode == 1
    assert r.stderr.strip() == ("Cannot open required file: ../../data/compressed/Comm/Comm.graph "
                                "(set TGA_COMPRESS_ROOT if needed)")
    assert r.stdout == ""
    # $TGA_COMPRESS_ROOT, trailing slashes dropped (path_config.cuh:10-19).
    r = run("pagerank", "--dataset", "Wiki", env={"TGA_COMPRESS_ROOT": str(tmp_path) + "//"})
    assert r.returncode == 1
    assert f"Cannot open required file: {tmp_path}/data/compressed/Wiki/Wiki.graph" in r.stderr
    # --root wins over the environment; Yahoo-sub reads Yahoo's files (DATASET_STORAGE_NAME).
    r = run("hits", "--dataset", "Yahoo-sub", "--root", tmp_path / "x", env={"TGA_COMPRESS_ROOT": str(tmp_path)})
    assert r.returncode == 1
    assert f"{tmp_path}/x/data/compressed/Yahoo/Yahoo.graph" in r.stderr


def test_dir_and_base_missing_file(tmp_path):
    r = run("neighbor_access", "--dir", tmp_path, "--base", "g", "--max-label", 9)
    assert r.returncode == 1
    assert f"Cannot open required file: {tmp_path}/g.graph" in r.stderr


@pytest.mark.parametrize("args, msg", [
    (["--dataset", "other"], "--max-label is required"),
    ([], "--dataset (or --dir with --base) is required"),
    (["--dataset", "Comm", "--bogus"], "unknown option: --bogus"),
    (["--dataset", "Comm", "--window", "5:3"], "bad --window"),
    (["--dataset", "Comm", "--window", "x"], "bad --window"),
    (["--dataset", "Comm", "--src", "-4"], "bad value for --src"),
    (["--dataset", "Comm", "--max-label", "10", "--max-vertex", "10"], "--max-vertex must exceed --max-label"),
    (["--dir", "/tmp"], "--dir and --base go together"),
    (["--dir", "/tmp", "--base", "g", "--root", "/tmp", "--max-label", "9"], "--root and --dir exclude each other"),
    (["--dataset", "Comm", "--repeat"], "missing value for --repeat"),
])
def test_bad_arguments_exit_2(args, msg):
    r = run("bfs", *args)
    assert r.returncode == 2
    assert msg in r.stderr


def test_window_refused_where_the_workload_has_none():
    for name in ("graph_coloring", "neighbor_access"):
        r = run(name, "--dataset", "Comm", "--window", "0:10")
        assert r.returncode == 2 and "takes no --window" in r.stderr


def test_tool_name_as_first_argument():
    r = run("tga_tool", "nosuch")
    assert r.returncode == 2 and "unknown algorithm: nosuch" in r.stderr
    r = run("tga_tool", "connected_components", "--help")
    assert r.returncode == 0 and r.stdout.startswith("usage: tga_tool connected_components ")


REF_GPU = (REFERENCE_ROOT / "gpu_cuda") if REFERENCE_ROOT else Path("/nonexistent")  # read when given


def _macros(path: Path) -> dict:
    out = {}
    for m in re.finditer(r'^\s*#define\s+(\w+)\s+("[^"]*"|-?\d+)', path.read_text(), flags=re.M):
        out.setdefault(m.group(1), m.group(2).strip('"') if m.group(2).startswith('"') else int(m.group(2)))
    return out


@pytest.mark.skipif(not REF_GPU.exists(), reason="reference tree not present")
@pytest.mark.parametrize("ds", ["Comm", "MyD", "Flickr", "Wiki", "Yahoo", "Yahoo-sub"])
def test_presets_equal_the_reference_dataset_configs(ds):
    """Each preset resolves to the reference's macros: gpu_cuda/<DS>/dataset_config.cuh over the
    #ifndef defaults of shared/dataset_config_base.cuh."""
    base = _macros(REF_GPU / "shared" / "dataset_config_base.cuh")
    want = {**base, **_macros(REF_GPU / ds / "dataset_config.cuh")}
    want.setdefault("DATASET_STORAGE_NAME", want["DATASET_NAME"])
    r = run("bfs", "--dataset", ds, "--show-config")
    assert r.returncode == 0, r.stderr
    got = json.loads(r.stdout)
    for k, v in got.items():
        assert want[k] == v, (ds, k)


@pytest.mark.parametrize("ds", list(tga.PRESETS))
def test_python_presets_equal_the_tool_presets(ds):
    got = json.loads(run("bfs", "--dataset", ds, "--show-config").stdout)
    c = tga.DatasetConfig.preset(ds).to_c()
    assert got["DATASET_STORAGE_NAME"] == c.storage_name.decode() and got["MAX_LABEL"] == c.max_label
    assert got["MAX_Vertex"] == c.max_vertex and got["minTimestamp"] == c.min_timestamp
    assert got["MIN_GRAPH_VERTEX"] == c.min_graph_vertex and got["ACTIVE_VERTEX_BEGIN"] == c.active_vertex_begin
    assert got["BFS_START_VERTEX"] == c.bfs_start_vertex and got["CONNECTED_COMPONENTS_VERTEX_BEGIN"] == c.cc_vertex_begin
    assert got["MULTIPLE_INITIAL_VALUE"] == c.multiple_initial_value
    assert got["PAGERANK_ITERATIONS"] == c.pr_iters and got["HITS_ITERATIONS"] == c.hits_iters
    assert tga.DatasetConfig.preset(ds, pagerank_iterations=3).pagerank_iterations == 3


def test_show_config_for_other_datasets():
    r = run("hits", "--dataset", "x", "--max-label", 5, "--hits-iters", 3, "--show-config")
    got = json.loads(r.stdout)
    assert got["MAX_Vertex"] == 6 and got["HITS_ITERATIONS"] == 3 and got["minTimestamp"] is None
    # Options after a preset override it.
    r = run("bfs", "--dataset", "Wiki", "--pr-iters", 7, "--bfs-start", 3, "--show-config")
    got = json.loads(r.stdout)
    assert got["PAGERANK_ITERATIONS"] == 7 and got["BFS_START_VERTEX"] == 3 and got["HITS_ITERATIONS"] == 100


@pytest.mark.skipif(has_gpu(), reason="checks the failure without a GPU")
def test_without_a_gpu_it_fails_loudly(datasets):
    d = datasets["sparse"]
    n = d["summary"]["n"]
    r = run("bfs", "--dir", d["dir"], "--base", d["base"], "--max-label", n - 1)
    assert r.returncode == 1
    assert "status 7" in r.stderr  # TGA_E_CUDA, no CPU fallback
    assert "BFS Elapsed" not in r.stdout


# ---- GPU ----------------------------------------------------------------------------------------

def fnv1a(b: bytes) -> str:
    h = 0xCBF29CE484222325
    for x in b:
        h = ((h ^ x) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return f"{h:016x}"


TOOL_ARGS = {
    "bfs": ["--repeat", "2"],
    "connected_components": [],
    "degree_centrality": [],
    "graph_coloring": [],
    "hits": [],
    "neighbor_access": [],
    "pagerank": ["--rank-summary"],
}


@pytest.fixture(scope="module")
def tool_runs(datasets, tmp_path_factory):
    """Runs every executable on the small dataset before this process touches the GPU, so each
    child has the device to itself whatever the compute mode."""
    d = datasets["small"]
    n = d["summary"]["n"]
    tmp = tmp_path_factory.mktemp("tools")
    runs = {}
    for name, extra in TOOL_ARGS.items():
        out = tmp / f"{name}.bin"
        runs[name] = (run(name, "--dir", d["dir"], "--base", d["base"], "--max-label", n - 1, "--max-vertex", n,
                          "--json", "--out", out, *extra), out)
    # The reference's layout: <root>/data/compressed/<STORAGE>/<STORAGE>.*, root from the environment.
    root = tmp / "root"
    (root / "data" / "compressed").mkdir(parents=True)
    (root / "data" / "compressed" / d["base"]).symlink_to(d["dir"], target_is_directory=True)
    runs["layout"] = (run("bfs", "--dataset", d["base"], "--max-label", n - 1, "--src", 7, "--window", "0:1000000",
                          "--json", env={"TGA_COMPRESS_ROOT": str(root)}), None)
    return d, n, runs


@pytest.fixture(scope="module")
def small(tool_runs):
    d, n, runs = tool_runs
    g = tga.Graph.open_dir(d["dir"], d["base"], tga.DatasetConfig(name=d["base"], max_label=n - 1, max_vertex=n))
    yield d, n, g, runs
    g.close()


def tool(small, name):
    r, out = small[3][name]
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    return lines, json.loads(lines[-1]), out.read_bytes() if out else None


@pytest.mark.gpu
def test_bfs_tool(small):
    d, n, g, _ = small
    lines, js, raw = tool(small, "bfs")
    assert lines[:4:2] == ["Starting simple parallel bfs."] * 2
    assert all(s.startswith("BFS Elapsed time in milliseconds : ") and s.endswith(" ms.") for s in lines[1:4:2])
    arr, hops = g.bfs()
    got = np.frombuffer(raw, np.int32)
    np.testing.assert_array_equal(got[:n], arr)
    np.testing.assert_array_equal(got[n:], hops)
    assert js["tool"] == "bfs" and js["repeat"] == 2
    assert js["reached"] == int((arr != INT32_MAX).sum())
    assert js["arrival_fnv1a"] == fnv1a(arr.tobytes())
    assert js["edges_decoded"] > 0 and js["device_ms"] > 0


@pytest.mark.gpu
def test_bfs_tool_reads_the_reference_layout(small):
    d, n, g, _ = small
    _, js, _ = tool(small, "layout")
    arr, _ = g.bfs(src=7, t_lo=0, t_hi=1_000_000)
    assert js["reached"] == int((arr != INT32_MAX).sum())
    assert js["arrival_fnv1a"] == fnv1a(arr.tobytes())


@pytest.mark.gpu
def test_connected_components_tool(small):
    d, n, g, _ = small
    lines, js, raw = tool(small, "connected_components")
    assert lines[0].startswith("Elapsed time in milliseconds : ")
    lab, comps = g.connected_components()
    np.testing.assert_array_equal(np.frombuffer(raw, np.int32), lab)
    assert js["components"] == comps


@pytest.mark.gpu
def test_degree_centrality_tool(small):
    d, n, g, _ = small
    lines, js, raw = tool(small, "degree_centrality")
    assert lines[0] == "Starting simple parallel Degree Centre."
    assert lines[1].startswith("Elapsed time in milliseconds : ")
    deg, avg = g.degree_centrality()
    np.testing.assert_array_equal(np.frombuffer(raw[:4 * n], np.int32), deg)
    np.testing.assert_array_equal(np.frombuffer(raw[4 * n:], np.int64), avg)
    assert js["degree_sum"] == int(deg.astype(np.int64).sum())


@pytest.mark.gpu
def test_graph_coloring_tool(small):
    d, n, g, _ = small
    lines, js, raw = tool(small, "graph_coloring")
    assert lines[0] == "Starting simple parallel Graph Color."
    col, prio, rounds = g.color()
    np.testing.assert_array_equal(np.frombuffer(raw[:4 * n], np.uint32), col)
    np.testing.assert_array_equal(np.frombuffer(raw[4 * n:], np.uint32), prio)
    assert js["rounds"] == rounds


@pytest.mark.gpu
def test_hits_tool(small):
    d, n, g, _ = small
    lines, js, raw = tool(small, "hits")
    assert lines[0] == "Starting simple parallel HITS."
    hub, auth = g.hits()
    got = np.frombuffer(raw, np.float32)
    np.testing.assert_allclose(got[:n], hub, rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(got[n:], auth, rtol=1e-6, atol=1e-9)


@pytest.mark.gpu
def test_neighbor_access_tool(small):
    d, n, g, _ = small
    lines, js, raw = tool(small, "neighbor_access")
    assert lines[0].startswith("Time = ") and lines[0].endswith(" ms.")
    small_, csum, deg = g.neighbor_access()
    np.testing.assert_array_equal(np.frombuffer(raw[:4 * n], np.int32), deg)
    np.testing.assert_array_equal(np.frombuffer(raw[4 * n:12 * n], np.uint64), csum)
    np.testing.assert_array_equal(np.frombuffer(raw[12 * n:], np.uint8), small_)
    assert js["edges"] == int(deg.astype(np.int64).sum())


@pytest.mark.gpu
def test_pagerank_tool_and_rank_summary(small):
    d, n, g, _ = small
    lines, js, raw = tool(small, "pagerank")
    assert lines[0] == "Starting simple parallel PageRank."
    assert lines[1].startswith("PageRank Elapsed time in milliseconds : ")
    rank = g.pagerank()
    got = np.frombuffer(raw, np.float32)
    np.testing.assert_allclose(got, rank, rtol=1e-6, atol=1e-12)
    # pagerank.cu:2012-2042: "PageRank alpha=0.1 rank_sum=S top10=i:v,..." (ties to the lower id).
    head, top = lines[2].split(" top10=")
    assert head.startswith("PageRank alpha=0.1 rank_sum=")
    assert float(head.split("rank_sum=")[1]) == pytest.approx(float(got.astype(np.float64).sum()), rel=1e-9)
    order = np.lexsort((np.arange(n), -got.astype(np.float64)))[:10]
    pairs = [p.split(":") for p in top.split(",")]
    assert [int(i) for i, _ in pairs] == order.tolist()
    np.testing.assert_allclose([float(v) for _, v in pairs], got[order], rtol=1e-9)


# ---- dataset preparation ------------------------------------------------------------------------

def test_prepare_plain_and_gzipped_inputs_give_the_same_files(datasets, tmp_path):
    import gzip

    raw = Path(datasets["chains"]["raw"])
    gz = tmp_path / "chains.raw.txt.gz"
    gz.write_bytes(gzip.compress(raw.read_bytes()))
    outs = {}
    for name, src in (("plain", raw), ("gz", gz)):
        bn = tmp_path / name / "chains"
        r = run("tga_tool", "prepare", src, bn)
        assert r.returncode == 0, r.stderr
        assert r.stdout.startswith(f"PREPARED basename={bn} nodes={datasets['chains']['summary']['n']} ")
        outs[name] = {f.name: f.read_bytes() for f in (tmp_path / name).iterdir()}
    assert outs["plain"] == outs["gz"]
    # The generator's own files for the same edges.
    gen = {f.name: f.read_bytes() for f in Path(datasets["chains"]["dir"]).iterdir() if f.name.startswith("chains.")}
    for k in ("chains.graph", "chains.timestamps", "chains.offsets"):
        assert outs["gz"][k] == gen[k], k
    for k in ("graph_lower_bits.bin", "graph_upper_bits.bin", "timestamp_lower_bits.bin", "timestamp_upper_bits.bin"):
        assert k in outs["gz"]


def test_prepare_errors(tmp_path, datasets):
    import gzip

    # A truncated gzip stream is refused; a file named .gz that is not gzip at all is read as text
    # (zlib's transparent mode) and fails as text.
    whole = gzip.compress(Path(datasets["sparse"]["raw"]).read_bytes())
    cut = tmp_path / "cut.txt.gz"
    cut.write_bytes(whole[: len(whole) // 2])
    r = run("tga_tool", "prepare", cut, tmp_path / "o" / "x")
    assert r.returncode == 1 and "Cannot open required file" in r.stderr
    bad = tmp_path / "bad.txt.gz"
    bad.write_bytes(b"not gzip at all")
    r = run("tga_tool", "prepare", bad, tmp_path / "o" / "x")
    assert r.returncode == 1 and "invalid number at line 1" in r.stderr
    r = run("tga_tool", "prepare", tmp_path / "missing.txt", tmp_path / "o" / "x")
    assert r.returncode == 1
    r = run("tga_tool", "prepare", tmp_path / "missing.txt")
    assert r.returncode == 2 and "Usage: tga_tool prepare" in r.stderr
