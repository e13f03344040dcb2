"""Realised reference-chain depth (cpu_java ReferenceDepthScanner.java): the library's scan against a
record-by-record reading of the outdegree and reference fields in Python, the encoder's own chain
statistic, and the scanner's RESULT line from the tool."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

import compresstemporalgraph_b200 as tga
import pyoracle
from test_format import Bits

TOOL = Path(tga.__file__).resolve().parent / "bin" / "tga_tool"


def _depths_by_hand(d):
    n = d["summary"]["n"]
    goff = pyoracle.Oracle(d["dir"], d["base"], n).graph_offsets()
    b = Bits((Path(d["dir"]) / f"{d['base']}.graph").read_bytes())
    depth = np.zeros(n, np.int32)
    for v in range(n):
        b.p = int(goff[v])
        if b.gamma() > 0:
            ref = b.unary()
            if ref:
                depth[v] = depth[v - ref] + 1
    return depth


@pytest.mark.parametrize("shape", ["chains", "small", "hubs", "sparse"])
def test_depths_match_a_reading_of_the_records(datasets, shape):
    d = datasets[shape]
    summary, depth = tga.reference_depths(d["dir"], d["base"])
    want = _depths_by_hand(d)
    assert np.array_equal(depth, want)
    assert summary["nodes"] == d["summary"]["n"]
    assert summary["maximum_depth"] == int(want.max()) == d["summary"]["max_chain"]
    assert summary["referenced_nodes"] == int((want > 0).sum())
    assert summary["depth_counts"][:4] == [int((want == k).sum()) for k in range(4)]
    assert summary["truncated_nodes"] == 0 and summary["configured_max_ref_count"] == 3


def test_tool_prints_the_scanner_line(datasets):
    d = datasets["chains"]
    s, _ = tga.reference_depths(d["dir"], d["base"])
    bn = f"{d['dir']}/{d['base']}"
    r = subprocess.run([str(TOOL), "reference_depths", bn], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    c = s["depth_counts"]
    assert r.stdout == (f"RESULT basename={bn} maximum_depth={s['maximum_depth']} configured_max_ref_count=3 "
                        f"referenced_nodes={s['referenced_nodes']} truncated_nodes=0 "
                        f"depth_counts=0:{c[0]},1:{c[1]},2:{c[2]},3:{c[3]}\n")


def test_tool_errors(tmp_path):
    r = subprocess.run([str(TOOL), "reference_depths", str(tmp_path / "none")], capture_output=True, text=True)
    assert r.returncode == 1 and "Cannot open required file" in r.stderr
    r = subprocess.run([str(TOOL), "reference_depths"], capture_output=True, text=True)
    assert r.returncode == 2 and "Usage: tga_tool reference_depths" in r.stderr
