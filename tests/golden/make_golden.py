"""Generates tests/golden/golden.json from the reference checkout (run once in a container that
has it; the fixture is committed so the tests never read the reference at run time).

  python tests/golden/make_golden.py <reference checkout>     (or set TGA_REFERENCE_ROOT)

Contents:
  * decode_tables: for gpu_cuda/decode_tables/gammaInA.txt and zetaInA.txt (65,536 entries of
    (code length << 16) | value) the sha256 of the int32 array, the number of non-zero entries and
    every 257th entry, so the engine's regenerated tables can be compared without the files;
  * known-answer vectors restated from the reference's unit tests (file:line cited per entry).
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

import os

if len(sys.argv) < 2 and not os.environ.get("TGA_REFERENCE_ROOT"):
    sys.exit("usage: make_golden.py <reference checkout>  (or set TGA_REFERENCE_ROOT)")
REF = Path(sys.argv[1] if len(sys.argv) > 1 else os.environ["TGA_REFERENCE_ROOT"])
OUT = Path(__file__).resolve().parent / "golden.json"


def table(path: Path) -> np.ndarray:
    vals = [int(x) for x in path.read_text().replace("\n", "").split(",") if x.strip()]
    a = np.array(vals, np.int32)
    assert a.shape == (65536,), a.shape
    return a


def main() -> None:
    tables = {}
    for key, fname in (("gamma", "gammaInA.txt"), ("zeta3", "zetaInA.txt")):
        a = table(REF / "gpu_cuda" / "decode_tables" / fname)
        tables[key] = {
            "source": f"gpu_cuda/decode_tables/{fname}",
            "sha256": hashlib.sha256(a.tobytes()).hexdigest(),
            "nonzero": int((a != 0).sum()),
            "samples": {str(i): int(a[i]) for i in range(0, 65536, 257)},
        }
    kats = {
        "ef_roundtrip": {
            "source": "cpu_java/src/test/java/gr/uoa/di/networkanalysis/EliasFanoDsiTest.java:18-41",
            "values": [10, 11, 11, 25],
        },
        "multiples_iterator": {
            "source": "cpu_java/src/test/java/gr/uoa/di/networkanalysis/IntMultiplesSequenceIteratorTest.java:10-31",
            "values": [3, 7], "lengths": [2, 3], "expected": [3, 3, 7, 7, 7], "skip3_then": [7, 7],
        },
        "intervalize_multiples": {
            "source": "third_party/ChronoGraph/src/test/java/gr/uoa/di/networkanalysis/BVMultiGraphTest.java:98-122",
            "extras": [4, 4, 4, 6, 7, 8, 8], "left": [4, 8], "len": [3, 2], "residuals": [6, 7],
        },
        "aggregator": {
            "source": "cpu_java/src/test/java/gr/uoa/di/networkanalysis/TimestampComparerAggregatorTest.java:10-20",
            "aggregate_min": [[109, 10, 100]], "difference": [[100, 115, 10, 1]], "reverse": [[100, 1, 10, 110]],
            "rejects_factor": 0,
        },
        "write_long_zeta": {
            "source": "third_party/ChronoGraph/src/test/java/gr/uoa/di/networkanalysis/WriteLongZetaTest.java:16-86",
            "header": 124, "zeta_k": 3, "values": [1, 2, 1, 198765],
        },
    }
    OUT.write_text(json.dumps({"decode_tables": tables, "known_answers": kats}, indent=1, sort_keys=True) + "\n")
    print(OUT)


if __name__ == "__main__":
    main()
