"""Builds the engine in-tree: compresstemporalgraph_b200/libtga.so (sm_100a) and the drop-in
executables under compresstemporalgraph_b200/bin/.

Run ``python compresstemporalgraph_b200/build.py`` (or call ``build()``); objects go to
compresstemporalgraph_b200/_build/ and are rebuilt when a source or header is newer.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "_build"
LIB = PKG / "libtga.so"
BIN = PKG / "bin"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function"]

CU_SOURCES = ["engine.cu", "algos.cu", "traverse.cu", "batch.cu", "noalloc.cu", "paths.cu", "indexbuild.cu"]
CPP_SOURCES = ["format.cpp", "gen.cpp", "hostapi.cpp", "server.cpp"]
TOOLS = {"tga_tool": "tools/tga_tool.cpp"}
DROPIN_NAMES = ["bfs", "connected_components", "degree_centrality", "graph_coloring", "hits",
                "neighbor_access", "pagerank"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.hpp")) + sorted(CSRC.glob("*.cuh")) + [INCLUDE / "tga.h"]


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        sys.stdout.write(r.stdout + r.stderr)


def build(verbose: bool = False, force: bool = False) -> Path:
    nvcc = _nvcc()
    OUT.mkdir(exist_ok=True)
    headers = _headers()
    objs: list[Path] = []
    steps: list[list[str]] = []
    for src in CU_SOURCES:
        s = CSRC / src
        o = OUT / (s.stem + ".cu.o")
        if force or _stale(o, [s] + headers):
            steps.append([nvcc, *ARCH, *NVCC_FLAGS, f"-I{INCLUDE}", "-c", str(s), "-o", str(o)])
        objs.append(o)
    for src in CPP_SOURCES:
        s = CSRC / src
        o = OUT / (s.stem + ".cpp.o")
        if force or _stale(o, [s] + headers):
            steps.append(["g++", *CXX_FLAGS, f"-I{INCLUDE}", "-c", str(s), "-o", str(o)])
        objs.append(o)
    # The translation units are independent: compile them side by side.
    with ThreadPoolExecutor(max_workers=max(1, min(len(steps), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(_run, cmd, verbose) for cmd in steps]:
            f.result()
    if force or _stale(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        _run([nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart_static", "-lrt", "-lpthread",
              "-ldl", "-lz"], verbose)
        os.replace(tmp, LIB)
    BIN.mkdir(exist_ok=True)
    for name, src in TOOLS.items():
        s = CSRC / src
        exe = BIN / name
        if force or _stale(exe, [s, LIB] + headers):
            _run(["g++", *CXX_FLAGS, f"-I{INCLUDE}", str(s), "-o", str(exe), f"-L{PKG}", "-ltga",
                  f"-Wl,-rpath,$ORIGIN/..", "-lpthread"], verbose)
        if exe.exists():
            for alias in DROPIN_NAMES:
                link = BIN / alias
                if not link.exists():
                    link.symlink_to(name)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
