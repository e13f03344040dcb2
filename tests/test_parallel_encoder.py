"""The block-parallel encoder (reference costs on threads, choices in order, records joined bit by
bit) writes the same files and statistics as the node-by-node encoder, whatever the thread count;
with blocks, the generator encodes each block on its own thread while it generates the next."""
from __future__ import annotations

import os

import pytest

import compresstemporalgraph_b200 as tga
from conftest import SHAPES

FILES = ("{b}.graph", "{b}.offsets", "{b}.timestamps", "{b}.properties", "graph_lower_bits.bin",
         "graph_upper_bits.bin", "timestamp_lower_bits.bin", "timestamp_upper_bits.bin")


def _gen(params, d, threads):
    old = os.environ.get("TGA_ENCODE_THREADS")
    os.environ["TGA_ENCODE_THREADS"] = str(threads)
    try:
        return tga.generate(params, d, "g")
    finally:
        if old is None:
            del os.environ["TGA_ENCODE_THREADS"]
        else:
            os.environ["TGA_ENCODE_THREADS"] = old


@pytest.mark.parametrize("shape", ["chains", "hubs", "sparse", "intervals", "widespan"])
def test_block_encoder_equals_node_encoder(tmp_path, shape):
    p = SHAPES[shape]
    ref = _gen(p, tmp_path / "seq", 0)
    for threads in (1, 5):
        got = _gen(p, tmp_path / f"t{threads}", threads)
        assert got == ref, threads
        for f in FILES:
            name = f.format(b="g")
            assert (tmp_path / f"t{threads}" / name).read_bytes() == (tmp_path / "seq" / name).read_bytes(), (threads, name)


def test_block_encoder_across_block_boundaries(tmp_path):
    """More than one block of nodes (65,536 per block): the reference window and chain depths carry
    over from one block to the next."""
    p = tga.GenParams(n=150_000, m=900_000, deg_exponent=2.2, repeat_frac=0.3, local_frac=0.8, local_radius=8,
                      copy_frac=0.5, ts_kind=0, ts_span=1_000_000, seed=31)
    ref = _gen(p, tmp_path / "seq", 0)
    got = _gen(p, tmp_path / "par", 7)
    assert got == ref
    for f in FILES:
        name = f.format(b="g")
        assert (tmp_path / "par" / name).read_bytes() == (tmp_path / "seq" / name).read_bytes(), name


@pytest.mark.parametrize("shape", ["chains", "intervals"])
def test_raw_encoder_block_equals_node(datasets, tmp_path, shape):
    """tga_encode_raw through the block encoders writes the node-by-node bytes."""
    d = datasets[shape]
    outs = {}
    for threads in (0, 3):
        old = os.environ.get("TGA_ENCODE_THREADS")
        os.environ["TGA_ENCODE_THREADS"] = str(threads)
        try:
            outs[threads] = tga.encode_raw(d["raw"], tmp_path / f"t{threads}", "r")
        finally:
            if old is None:
                del os.environ["TGA_ENCODE_THREADS"]
            else:
                os.environ["TGA_ENCODE_THREADS"] = old
    assert outs[0] == outs[3]
    for f in FILES:
        name = f.format(b="r")
        assert (tmp_path / "t3" / name).read_bytes() == (tmp_path / "t0" / name).read_bytes(), name
