"""Code-level parity: the engine's codes against the reference's golden decode tables and the
reference's known-answer tests (restated in tests/golden/golden.json, see make_golden.py)."""
from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import compresstemporalgraph_b200 as tga
import pyoracle
from conftest import REFERENCE_ROOT

GOLD = json.loads((Path(__file__).parent / "golden" / "golden.json").read_text())
REF_TABLES = (REFERENCE_ROOT / "gpu_cuda" / "decode_tables") if REFERENCE_ROOT else Path("/nonexistent")


@pytest.mark.parametrize("kind,key", [(0, "gamma"), (3, "zeta3")])
def test_decode_tables_match_reference(kind, key):
    a = tga.decode_table(kind)
    g = GOLD["decode_tables"][key]
    assert hashlib.sha256(a.tobytes()).hexdigest() == g["sha256"]
    assert int((a != 0).sum()) == g["nonzero"]
    for i, v in g["samples"].items():
        assert a[int(i)] == v


@pytest.mark.skipif(not REF_TABLES.exists(), reason="reference checkout not present")
def test_decode_tables_against_files_when_present():
    for kind, fname in ((0, "gammaInA.txt"), (3, "zetaInA.txt")):
        vals = np.array([int(x) for x in (REF_TABLES / fname).read_text().replace("\n", "").split(",") if x.strip()],
                        np.int32)
        assert np.array_equal(tga.decode_table(kind), vals)


def test_write_long_zeta_known_answer():
    kat = GOLD["known_answers"]["write_long_zeta"]
    head, hb = tga.encode_codes(tga.CODE_LONG64, [kat["header"]])
    assert hb == 64
    body, nb = tga.encode_codes(tga.CODE_ZETA, kat["values"], k=kat["zeta_k"])
    v, used = pyoracle.read_codes(head, 3, 1)
    assert v[0] == kat["header"]
    v, used = pyoracle.read_codes(body, 1, len(kat["values"]), k=kat["zeta_k"])
    assert list(v) == kat["values"] and used == nb


@pytest.mark.parametrize("kind,k", [(0, 0), (1, 2), (1, 3), (1, 5), (2, 0)])
def test_code_round_trip_random(kind, k):
    rng = np.random.default_rng(kind * 10 + k)
    vals = np.concatenate([np.arange(300), rng.integers(0, 1 << 30, 500), [0, 1, 2, (1 << 31) - 1]])
    if kind == 2:
        vals = vals % 97
    data, nbits = tga.encode_codes(kind, vals, k=k)
    back, used = pyoracle.read_codes(data, kind, len(vals), k=k)
    assert used == nbits
    assert np.array_equal(back, vals.astype(np.uint64))


def test_zeta2_lengths_match_definition():
    # zeta_2 of x: unary(h) + (2h+1 or 2h+2) bits, h = floor(log2(x+1)) / 2
    for x in [0, 1, 2, 3, 10, 1000, 123456, 10**8]:
        _, nb = tga.encode_codes(tga.CODE_ZETA, [x], k=2)
        h = (x + 1).bit_length() // 2 if False else ((x + 1).bit_length() - 1) // 2
        assert nb in (h + 1 + 2 * h + 1, h + 1 + 2 * h + 2)


def test_elias_fano_known_answer():
    vals = GOLD["known_answers"]["ef_roundtrip"]["values"]
    for l in range(0, 5):
        lo, up = tga.ef_encode(vals, l)
        assert list(pyoracle.ef_values(lo, up, l, len(vals))) == vals


def test_elias_fano_random_monotone():
    rng = np.random.default_rng(3)
    vals = np.cumsum(rng.integers(0, 500, 3000)).astype(np.uint64)
    l = 7
    lo, up = tga.ef_encode(vals, l)
    assert len(up) % 8 == 0  # whole 64-bit words, as the reference select reads them
    assert np.array_equal(pyoracle.ef_values(lo, up, l, len(vals)), vals)


def test_ef_rejects_decreasing():
    with pytest.raises(tga.TgaError):
        tga.ef_encode([5, 3], 2)


def test_aggregator_known_answers():
    from compresstemporalgraph_b200 import timestamps as agg

    k = GOLD["known_answers"]["aggregator"]
    for m, f, out in k["aggregate_min"]:
        assert agg.aggregate_min_timestamp(m, f) == out
    for a, b, f, out in k["difference"]:
        assert agg.timestamps_difference(a, b, f) == out
    for p, d, f, out in k["reverse"]:
        assert agg.reverse(p, d, f) == out
    with pytest.raises(ValueError):
        agg.aggregate_min_timestamp(100, k["rejects_factor"])
