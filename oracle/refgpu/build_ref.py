"""Builds the reference's own GPU programs for the second oracle (TEST INFRASTRUCTURE ONLY).

For each program of config.PROGRAMS it writes a translation unit that defines the dataset macros of
config.py (as a gpu_cuda/<DS>/dataset_config.cuh does) and includes the reference's
gpu_cuda/shared/dataset_config_base.cuh and gpu_cuda/shared/<program>.cu from the checkout, unchanged;
nvcc compiles it for sm_100a with harness_pre.h force-included and links harness_main.cu against the
shared CUDA runtime (the harness brackets each kernel launch with events, harness_main.cu).  Outputs go
only to oracle/_ref/: the executables and manifest.json (for each compared buffer, the source line of
its allocation).

  python oracle/refgpu/build_ref.py [reference checkout]    (default: $TGA_REFERENCE_ROOT, else
                                                               /root/reference)
Skips (exit 0, nothing written) when the checkout is absent.
"""
from __future__ import annotations

import json
import os
import re
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE.parent / "_ref"
sys.path.insert(0, str(HERE))
import config  # noqa: E402


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def alloc_line(src: Path, name: str) -> int:
    pat = re.compile(r"cudaMalloc\(\s*\(void\s*\*\*\)\s*&" + re.escape(name) + r"\s*,")
    for i, line in enumerate(src.read_text(encoding="utf-8-sig").splitlines(), 1):
        if pat.search(line) and not line.strip().startswith("//"):
            return i
    raise RuntimeError(f"no allocation of {name} in {src}")


def main() -> int:
    ref = Path(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TGA_REFERENCE_ROOT", "/root/reference"))
    shared = ref / "gpu_cuda" / "shared"
    if not shared.exists():
        print(f"reference checkout not found at {ref}; reference GPU programs not built")
        return 0
    OUT.mkdir(exist_ok=True)
    manifest = {"name": config.NAME, "n": config.N, "bfs_source": config.BFS_SOURCE, "programs": {}}
    arch = [nvcc(), "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a"]
    harness = OUT / "harness_main.o"
    jobs = []
    for prog, bufs in config.PROGRAMS.items():
        src = shared / f"{prog}.cu"
        tu = OUT / f"{prog}_tu.cu"
        tu.write_text(
            f'#define DATASET_NAME "{config.NAME}"\n'
            f"#define MAX_LABEL {config.N - 1}\n"
            f"#define MAX_Vertex {config.N}\n"
            f"#define minTimestamp 0\n"
            f"#define BFS_START_VERTEX {config.BFS_SOURCE}\n"
            f'#include "{shared / "dataset_config_base.cuh"}"\n'
            f'#include "{src}"\n')
        exe = OUT / prog
        manifest["programs"][prog] = {b: alloc_line(src, b) for b in bufs}
        stale = not exe.exists() or any(p.stat().st_mtime > exe.stat().st_mtime
                                        for p in (src, HERE / "harness_pre.h", HERE / "harness_main.cu", HERE / "config.py",
                                                  HERE / "build_ref.py"))
        if stale:
            obj = OUT / f"{prog}_tu.o"
            jobs.append([[*arch, "-w", "-Xcompiler", "-fpermissive", "-include", str(HERE / "harness_pre.h"), "-c", str(tu), "-o", str(obj)],
                         [*arch, "-cudart", "shared", str(obj), str(harness), "-o", str(exe), "-ldl"]])

    def run(steps):
        for cmd in steps:
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError("reference program build failed: " + cmd[-1])

    # The harness main is compiled on its own: the force-included header renames `main`.
    arch = [nvcc(), "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a"]
    harness = OUT / "harness_main.o"
    if jobs or not harness.exists():
        run([[*arch, "-c", str(HERE / "harness_main.cu"), "-o", str(harness)]])

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(run, j) for j in jobs]:
            f.result()
    (OUT / "manifest.json").write_text(json.dumps(manifest, indent=1))
    print(f"reference GPU programs in {OUT}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
