"""Round trip of the reference's own format fixture, third_party/ChronoGraph/src/test/resources/
cbtComm-sample.txt (1000 raw edges "src dst w ts", unsorted; ChronoGraph's TestStore stores the
(src, dst)-sorted form).  Read where it lies when the reference tree is present, skipped otherwise:
sorted stably by (src, dst), compressed by the engine's encoder, decoded by the oracle's independent
decoder, every list and timestamp must come back; the GPU index rebuilt from .offsets must equal the
one the encoder wrote."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import compresstemporalgraph_b200 as tga
import pyoracle
from conftest import REFERENCE_ROOT

FIXTURE = ((REFERENCE_ROOT / "third_party/ChronoGraph/src/test/resources/cbtComm-sample.txt") if REFERENCE_ROOT
           else Path("/nonexistent"))
INDEX = ("graph_lower_bits.bin", "graph_upper_bits.bin", "timestamp_lower_bits.bin", "timestamp_upper_bits.bin")

pytestmark = pytest.mark.skipif(not FIXTURE.exists(), reason="reference tree not present")


def _edges():
    rows = [tuple(int(x) for x in line.split()) for line in FIXTURE.read_text().splitlines() if line.strip()]
    assert len(rows) == 1000 and all(len(r) == 4 for r in rows)
    return sorted(rows, key=lambda r: (r[0], r[1]))  # stable: equal (src, dst) keep line order


def test_fixture_round_trip(tmp_path):
    rows = _edges()
    raw = tmp_path / "cbt.txt"
    raw.write_text("".join(f"{s} {d} {w} {t}\n" for s, d, w, t in rows))
    n = max(max(r[0], r[1]) for r in rows) + 1
    summary = tga.encode_raw(raw, tmp_path / "enc", "cbt", n - 1)
    assert summary["m"] == 1000
    o = pyoracle.Oracle(tmp_path / "enc", "cbt", summary["n"])
    off, dst, ts = o.csr()
    src = np.repeat(np.arange(len(off) - 1), np.diff(off))
    assert np.array_equal(src, [r[0] for r in rows])
    assert np.array_equal(dst, [r[1] for r in rows])
    assert np.array_equal(ts, [r[3] for r in rows])
    assert o.min_ts == min(r[3] for r in rows)


def test_fixture_index_rebuild(tmp_path):
    rows = _edges()
    raw = tmp_path / "cbt.txt"
    raw.write_text("".join(f"{s} {d} {w} {t}\n" for s, d, w, t in rows))
    n = max(max(r[0], r[1]) for r in rows) + 1
    d = tmp_path / "enc"
    tga.encode_raw(raw, d, "cbt", n - 1)
    written = {f: (d / f).read_bytes() for f in INDEX}
    for f in INDEX:
        (d / f).unlink()
    tga.build_index(d, "cbt", n - 1)
    for f in INDEX:
        assert (d / f).read_bytes() == written[f], f
