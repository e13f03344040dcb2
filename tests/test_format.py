"""Format layer on CPU: encoder round trips through the oracle's independent decoder, the GPU
Elias-Fano files against the .offsets stream, raw-text semantics and host-side fault handling."""
from __future__ import annotations

import os
import re
import shutil
from pathlib import Path

import numpy as np
import pytest

import compresstemporalgraph_b200 as tga
import pyoracle
from conftest import SHAPES


def _raw(path):
    a = np.loadtxt(path, dtype=np.int64, ndmin=2)
    return a[:, 0], a[:, 1], a[:, 3]


@pytest.mark.parametrize("shape", list(SHAPES))
def test_round_trip_oracle(datasets, shape):
    d = datasets[shape]
    o = pyoracle.Oracle(d["dir"], d["base"], d["summary"]["n"])
    off, dst, ts = o.csr()
    src_raw, dst_raw, ts_raw = _raw(d["raw"])
    assert o.m == len(dst_raw) == d["summary"]["m"]
    assert np.array_equal(np.repeat(np.arange(o.n), np.diff(off)), src_raw)
    assert np.array_equal(dst, dst_raw)
    assert np.array_equal(ts, ts_raw)
    assert o.min_ts == d["params"].min_timestamp


@pytest.mark.parametrize("shape", list(SHAPES))
def test_ef_index_files_match_offsets(datasets, shape):
    d = datasets[shape]
    n = d["summary"]["n"]
    o = pyoracle.Oracle(d["dir"], d["base"], n, materialize=False)
    gbytes = (d["dir"] / f"{d['base']}.graph").stat().st_size
    tbytes = (d["dir"] / f"{d['base']}.timestamps").stat().st_size
    # l = (int)log2(fileBytes * 8 / MAX_LABEL) as the reference reader computes it (bfs.cu:1785-1786)
    gl = int(np.log2(gbytes * 8 // (n - 1))) if gbytes * 8 // (n - 1) else 0
    tl = int(np.log2(tbytes * 8 // (n - 1))) if tbytes * 8 // (n - 1) else 0
    rd = lambda f: (d["dir"] / f).read_bytes()
    idx = np.linspace(0, n, num=min(n + 1, 400), dtype=np.int64)
    gv = pyoracle.ef_values(rd("graph_lower_bits.bin"), rd("graph_upper_bits.bin"), gl, n + 1)
    tv = pyoracle.ef_values(rd("timestamp_lower_bits.bin"), rd("timestamp_upper_bits.bin"), tl, n + 1)
    assert np.array_equal(gv[idx], o.graph_offsets()[idx])
    assert np.array_equal(tv[idx], o.ts_offsets()[idx])
    assert len(rd("graph_upper_bits.bin")) % 8 == 0 and len(rd("timestamp_upper_bits.bin")) % 8 == 0


class Bits:
    def __init__(self, data: bytes):
        self.bits = "".join(f"{b:08b}" for b in data)
        self.p = 0

    def unary(self):
        z = self.bits.index("1", self.p) - self.p
        self.p += z + 1
        return z

    def gamma(self):
        m = self.unary()
        v = int("1" + self.bits[self.p:self.p + m], 2) if m else 1
        self.p += m
        return v - 1

    def zeta(self, k):
        h = self.unary()
        left = 1 << (h * k)
        nb = h * k + k - 1
        v = int(self.bits[self.p:self.p + nb], 2)
        if v < left:
            self.p += nb
            return v + left - 1
        v = int(self.bits[self.p:self.p + nb + 1], 2)
        self.p += nb + 1
        return v - 1


def test_intervalize_multiples_known_answer(tmp_path):
    """BVMultiGraphTest.testIntervalizeMultiples: {4,4,4,6,7,8,8} -> multiples (4,3),(8,2), residuals 6,7."""
    raw = tmp_path / "kat.txt"
    raw.write_text("".join(f"0 {y} 1 {t}\n" for t, y in enumerate([4, 4, 4, 6, 7, 8, 8])))
    tga.encode_raw(raw, tmp_path, "kat")
    b = Bits((tmp_path / "kat.graph").read_bytes())
    assert b.gamma() == 7          # outdegree
    assert b.unary() == 0          # no reference
    assert b.gamma() == 2          # multiples count
    assert b.gamma() == 2 * 4      # int2nat(4 - 0)
    assert b.gamma() == 3 - 2      # run length - 2
    assert b.gamma() == 8 - 4 - 1  # gap to the next run
    assert b.gamma() == 2 - 2
    assert b.gamma() == 0          # intervals
    assert b.zeta(3) == 2 * 6      # first residual int2nat(6 - 0)
    assert b.zeta(3) == 7 - 6 - 1
    o = pyoracle.Oracle(tmp_path, "kat", 9)
    dst, ts = o.neighbors(0)
    assert list(dst) == [4, 4, 4, 6, 7, 8, 8] and list(ts) == list(range(7))


def test_multiples_iterator_known_answer(tmp_path):
    """IntMultiplesSequenceIteratorTest: values {3,7} lengths {2,3} -> 3,3,7,7,7."""
    raw = tmp_path / "m.txt"
    raw.write_text("".join(f"1 {y} 1 {5 + i}\n" for i, y in enumerate([3, 3, 7, 7, 7])))
    tga.encode_raw(raw, tmp_path, "m")
    o = pyoracle.Oracle(tmp_path, "m", 8)
    dst, ts = o.neighbors(1)
    assert list(dst) == [3, 3, 7, 7, 7]
    assert list(ts) == [5, 6, 7, 8, 9]


def test_timestamps_keep_line_order(tmp_path):
    """Successors are sorted by value, timestamps keep input-line order (ArcListASCIIEvolvingGraph.java:359
    vs EvolvingMultiGraph.java:258)."""
    raw = tmp_path / "o.txt"
    raw.write_text("0 5 1 10\n0 3 1 20\n1 0 1 7\n")
    tga.encode_raw(raw, tmp_path, "o")
    o = pyoracle.Oracle(tmp_path, "o", 6)
    dst, ts = o.neighbors(0)
    assert list(dst) == [3, 5] and list(ts) == [10, 20]
    assert o.min_ts == 7


@pytest.mark.parametrize("text,msg", [
    ("1 2 1 5\n0 3 1 6\n", "sorted"),
    ("0 2 5\n", "four columns"),
    ("0 -2 1 5\n", "range"),
    ("", "no edges"),
])
def test_raw_parse_errors(tmp_path, text, msg):
    raw = tmp_path / "bad.txt"
    raw.write_text(text)
    with pytest.raises(tga.TgaError, match=msg):
        tga.encode_raw(raw, tmp_path, "bad")


def test_reference_chain_depth_bounded(datasets):
    s = datasets["chains"]["summary"]
    assert 1 <= s["max_chain"] <= 3
    assert s["copied_arcs"] > 0 and s["intervalised_arcs"] > 0 and s["multiples_arcs"] > 0


def test_generator_is_seeded(tmp_path):
    p = tga.GenParams(n=500, m=4000, seed=42, copy_frac=0.2)
    a = tga.generate(p, tmp_path / "a", "g")
    b = tga.generate(p, tmp_path / "b", "g")
    assert a == b
    for f in ("g.graph", "g.timestamps", "graph_upper_bits.bin", "timestamp_lower_bits.bin"):
        assert (tmp_path / "a" / f).read_bytes() == (tmp_path / "b" / f).read_bytes()


def test_properties_written(datasets):
    d = datasets["small"]
    props = dict(line.split("=", 1) for line in (d["dir"] / "small.properties").read_text().splitlines()
                 if "=" in line and not line.startswith("#"))
    assert props["nodes"] == "10000" and props["arcs"] == "200000"
    assert props["windowsize"] == "7" and props["maxrefcount"] == "3" and props["zetak"] == "3"


# ---- host-side fault handling (detected before any device work) -----------------------------

def _cfg(n, **kw):
    return tga.DatasetConfig(name="x", max_label=n - 1, max_vertex=n, **kw)


def test_open_missing_file_is_io_error(datasets, tmp_path):
    d = datasets["sparse"]
    work = tmp_path / "w"
    shutil.copytree(d["dir"], work)
    # An index file alone is rebuilt from <base>.offsets (test_index_rebuild.py); without both the
    # open fails before any device work, naming the missing files.
    (work / "timestamp_upper_bits.bin").unlink()
    (work / f"{d['base']}.offsets").unlink()
    with pytest.raises(tga.TgaError) as e:
        tga.Graph.open_dir(work, d["base"], _cfg(d["summary"]["n"]))
    assert e.value.code == tga.TGA_E_IO and "timestamp_upper_bits.bin" in str(e.value) and ".offsets" in str(e.value)


def test_open_wrong_min_timestamp_is_format_error(datasets):
    d = datasets["intervals"]
    with pytest.raises(tga.TgaError) as e:
        tga.Graph.open_dir(d["dir"], d["base"], _cfg(d["summary"]["n"], min_timestamp=0))
    assert e.value.code == tga.TGA_E_FORMAT and "minTimestamp" in str(e.value)


def test_open_unsupported_properties(datasets, tmp_path):
    d = datasets["sparse"]
    work = tmp_path / "p"
    shutil.copytree(d["dir"], work)
    pf = work / f"{d['base']}.properties"
    pf.write_text(pf.read_text().replace("zetak=3", "zetak=4"))
    with pytest.raises(tga.TgaError) as e:
        tga.Graph.open_dir(work, d["base"], _cfg(d["summary"]["n"]))
    assert e.value.code == tga.TGA_E_FORMAT


def test_open_truncated_index(datasets, tmp_path):
    d = datasets["sparse"]
    work = tmp_path / "t"
    shutil.copytree(d["dir"], work)
    up = work / "graph_upper_bits.bin"
    up.write_bytes(up.read_bytes()[: len(up.read_bytes()) // 3])
    with pytest.raises(tga.TgaError) as e:
        tga.Graph.open_dir(work, d["base"], _cfg(d["summary"]["n"]))
    assert e.value.code == tga.TGA_E_FORMAT


def test_open_bad_config(datasets):
    d = datasets["sparse"]
    with pytest.raises(tga.TgaError) as e:
        tga.Graph.open_dir(d["dir"], d["base"], tga.DatasetConfig(name="x", max_label=10, max_vertex=5))
    assert e.value.code == tga.TGA_E_ARG


def test_drop_in_path_convention(datasets, tmp_path, monkeypatch):
    """tga_open resolves <root>/data/compressed/<STORAGE>/<STORAGE>.* like dataset_config_base.cuh:46-67."""
    d = datasets["sparse"]
    root = tmp_path / "root"
    dst = root / "data" / "compressed" / "Sparse"
    dst.mkdir(parents=True)
    for f in d["dir"].iterdir():
        name = f.name.replace(d["base"] + ".", "Sparse.")
        shutil.copy(f, dst / name)
    (dst / "graph_upper_bits.bin").unlink()
    (dst / "Sparse.offsets").unlink()  # else the index is rebuilt from it
    monkeypatch.setenv("TGA_COMPRESS_ROOT", str(root) + "/")
    with pytest.raises(tga.TgaError) as e:
        tga.Graph.open(_cfg(d["summary"]["n"], storage_name="Sparse"))
    assert e.value.code == tga.TGA_E_IO and str(dst / "graph_upper_bits.bin") in str(e.value)
