"""The C-ABI library loads on a CPU-only host and exports every function include/tga.h declares."""
from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path

import compresstemporalgraph_b200 as tga

ROOT = Path(__file__).resolve().parents[1]


def declared():
    text = (ROOT / "include" / "tga.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tga_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared()
    for must in ("tga_open", "tga_bfs", "tga_cc", "tga_pagerank", "tga_hits", "tga_degree", "tga_color",
                 "tga_neighbor_access", "tga_neighbors", "tga_bfs_batch", "tga_pagerank_batch"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(tga.LIB_PATH))
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_exports_are_c_linkage():
    out = subprocess.run(["nm", "-D", "--defined-only", str(tga.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (tga_\w+)$", out, flags=re.M))
    assert set(declared()) <= exported


def test_header_compiles_as_c(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "tga.h"\nint main(void){tga_dataset_cfg c; tga_cfg_default(&c); return c.bfs_start_vertex-1;}\n')
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", f"-I{ROOT / 'include'}", "-c", str(src), "-o",
                        str(tmp_path / "t.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_cfg_defaults_match_reference_macros():
    c = tga.DatasetConfig(name="x", max_label=9, max_vertex=10).to_c()
    # shared/dataset_config_base.cuh:11-37 defaults
    assert c.active_vertex_begin == 0 and c.min_graph_vertex == 0 and c.bfs_start_vertex == 1
    assert c.cc_vertex_begin == 1 and c.multiple_initial_value == -1 and c.pr_iters == 10 and c.hits_iters == 10


def test_python_mirror_declares_every_entry_point():
    """Every function of include/tga.h has a ctypes signature in the Python mirror."""
    src = (ROOT / "compresstemporalgraph_b200" / "__init__.py").read_text()
    mirrored = set(re.findall(r'"(tga_[a-z0-9_]+)":\s*\(', src))
    missing = [n for n in declared() if n not in mirrored]
    assert not missing, missing
