"""Shared fixtures: in-tree build of the engine and the oracle, seeded synthetic datasets.

Marker ``gpu``: the test needs a CUDA GPU (run with ``-m gpu`` on a B200); everything else runs
on CPU only.

``TGA_REFERENCE_ROOT``: a checkout of the reference project (Yukun-Cui/CompressTemporalGraph).  The
few tests that read its files in place (decode tables, dataset configs, the ChronoGraph format
fixture) run only when it is set; every other test uses the committed fixtures under golden/.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
REFERENCE_ROOT = Path(os.environ["TGA_REFERENCE_ROOT"]) if os.environ.get("TGA_REFERENCE_ROOT") else None
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def _build():
    import importlib.util

    spec = importlib.util.spec_from_file_location("tga_build", ROOT / "compresstemporalgraph_b200" / "build.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)  # the package itself refuses to import before libtga.so exists

    b.build()
    import pyoracle

    pyoracle.build()


_build()

import compresstemporalgraph_b200 as tga  # noqa: E402

# Small datasets for exhaustive parity (each decodes in well under a second on the oracle).
SHAPES = {
    # The small benchmark configuration: 10K vertices, 200K temporal edges.
    "small": tga.CONFIGS["small"],
    # Reference chains, copy blocks, intervals and multiples all at once.
    "chains": tga.GenParams(n=3000, m=60000, deg_exponent=2.3, repeat_frac=0.3, local_frac=0.9, local_radius=3,
                            copy_frac=0.6, ts_kind=0, ts_span=10_000, seed=11),
    # Vertex 0 and the largest id receive no edges; minimum timestamp 0 (reference-safe layout).
    "refsafe": tga.GenParams(n=4000, m=50000, deg_exponent=2.1, repeat_frac=0.3, local_frac=0.6, local_radius=32,
                             copy_frac=0.3, ts_kind=0, ts_span=1_000_000, seed=7, ref_safe=True),
    # Mostly isolated vertices and degree-1 lists.
    "sparse": tga.GenParams(n=5000, m=6000, deg_exponent=3.0, repeat_frac=0.1, local_frac=0.5, ts_kind=0,
                            ts_span=1000, seed=5),
    # A few hubs holding most edges; bursty timestamps over a 1e8 span.
    "hubs": tga.GenParams(n=2000, m=100000, deg_exponent=1.5, max_degree=50000, repeat_frac=0.3, local_frac=0.7,
                          local_radius=64, pref_frac=0.5, copy_frac=0.2, ts_kind=2, ts_span=100_000_000, seed=9),
    # Timestamps spread over 6e9 (more than 2^31): the 64-bit paths (degree-centrality mean).
    "widespan": tga.GenParams(n=2000, m=60000, deg_exponent=1.6, max_degree=20000, repeat_frac=0.3, local_frac=0.7,
                              local_radius=64, pref_frac=0.3, copy_frac=0.2, ts_kind=0, ts_span=6_000_000_000, seed=17),
    # Long runs of consecutive successors (intervals) and a non-zero minimum timestamp.
    "intervals": tga.GenParams(n=4000, m=80000, deg_exponent=2.2, repeat_frac=0.05, local_frac=1.0, local_radius=1,
                               copy_frac=0.1, ts_kind=1, ts_span=5_000_000, min_timestamp=1_206_214_540 - 5_000_000,
                               seed=13),
}


@pytest.fixture(scope="session")
def datasets(tmp_path_factory):
    base = tmp_path_factory.mktemp("tga_data")
    out = {}
    for name, p in SHAPES.items():
        d = base / name
        raw = str(d / f"{name}.raw.txt")
        d.mkdir(parents=True, exist_ok=True)
        s = tga.generate(p, d, name, raw_path=raw)
        out[name] = {"dir": d, "base": name, "summary": s, "raw": raw, "params": p}
    return out


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
