"""The GPU index files rebuilt from the webgraph offsets (what a directory written by the Java
encoder holds instead of them): byte-identical to the files the encoder writes, whether the walks
run on the host (tga_build_index) or on the GPU (tga_build_index_device, speculative chunked
decoding), and a graph opened without them decodes the same lists."""
from __future__ import annotations

import shutil

import numpy as np
import pytest

import compresstemporalgraph_b200 as tga

INDEX_FILES = ("graph_lower_bits.bin", "graph_upper_bits.bin", "timestamp_lower_bits.bin", "timestamp_upper_bits.bin")


def _strip(d, tmp_path, name):
    out = tmp_path / name
    shutil.copytree(d["dir"], out)
    for f in INDEX_FILES:
        (out / f).unlink()
    return out


@pytest.mark.parametrize("shape", ["small", "chains", "hubs", "intervals", "sparse"])
def test_rebuilt_index_files_equal_encoder_output(datasets, tmp_path, shape):
    d = datasets[shape]
    out = _strip(d, tmp_path, shape)
    tga.build_index(out, d["base"], d["summary"]["n"] - 1)
    for f in INDEX_FILES:
        assert (out / f).read_bytes() == (d["dir"] / f).read_bytes(), f


def test_rebuild_needs_offsets_and_nodes(datasets, tmp_path):
    d = datasets["small"]
    out = _strip(d, tmp_path, "small")
    (out / "small.offsets").unlink()
    with pytest.raises(tga.TgaError) as e:
        tga.build_index(out, "small", d["summary"]["n"] - 1)
    assert e.value.code == tga.TGA_E_IO


@pytest.mark.gpu
@pytest.mark.parametrize("shape", ["chains", "hubs"])
def test_open_without_index_files(datasets, tmp_path, shape):
    d = datasets[shape]
    n = d["summary"]["n"]
    cfg = tga.DatasetConfig(name=d["base"], max_label=n - 1, max_vertex=n)
    out = _strip(d, tmp_path, shape)
    with tga.Graph.open_dir(d["dir"], d["base"], cfg) as a, tga.Graph.open_dir(out, d["base"], cfg) as b:
        ca, cb = a.decode_all(), b.decode_all()
        for x, y in zip(ca, cb):
            assert np.array_equal(x, y)
        assert np.array_equal(a.bfs(0)[0], b.bfs(0)[0])


@pytest.mark.gpu
@pytest.mark.parametrize("shape", ["small", "chains", "hubs", "intervals", "sparse"])
def test_device_rebuilt_index_files_equal_encoder_output(datasets, tmp_path, shape):
    d = datasets[shape]
    out = _strip(d, tmp_path, shape)
    tga.build_index(out, d["base"], d["summary"]["n"] - 1, device=True)
    for f in INDEX_FILES:
        assert (out / f).read_bytes() == (d["dir"] / f).read_bytes(), f


@pytest.mark.gpu
def test_device_rebuilt_index_at_bench_size(tmp_path):
    # 2M vertices / 40M edges: 46K chunks of the timestamp stream, most entered mid-code at first.
    name = "all7"
    src = tmp_path / "src"
    tga.generate(tga.CONFIGS[name], src, name)
    out = tmp_path / "out"
    shutil.copytree(src, out)
    for f in INDEX_FILES:
        (out / f).unlink()
    tga.build_index(out, name, tga.CONFIGS[name].n - 1, device=True)
    for f in INDEX_FILES:
        assert (out / f).read_bytes() == (src / f).read_bytes(), f
