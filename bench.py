"""Benchmark: GTEPS of the fused decode kernels on the compressed temporal graph.

A step is one pass of the seven reference workloads (RA/neighbour access, BFS, CC, PageRank x30,
HITS x30, degree centrality, JP colouring) over the configuration "2M vertices, 40M temporal
edges" -- seeded synthetic data with that shape, compressed in the reference's format and held
in HBM.  value = temporal edges decoded by all workloads / device time (GTEPS, whole job over
all ranks); e2e = the same through the public C-ABI calls with host result buffers (device-to-
host copies inside the timed region); roofline = the PageRank iteration kernel's compressed bytes
per launch / its average launch time against the measured HBM copy bandwidth.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
  python bench.py --batched-graph batched      # batched form alone on the 20M/500M graph
  python bench.py --skew-graph skew            # HITS x30 + colouring on the 100M/2B skew graph

The line also carries the batched form at its own size (256 windowed BFS + 32 windowed PageRanks
against one query per call on the 20M-vertex / 500M-edge graph, generated on the machine on first
use), the served form (open-loop queries through the server against plain calls), a second
GTEPS figure over the workloads that read the timestamp stream, the FP32 PageRank/HITS error
against the FP64 oracle at this configuration (computed after the timed regions), and the
reference's own GPU programs timed beside the engine on the small graph they are built for.

--impl reference is the CPU arm: the same graph (generated in a child process, so the engine's
library is never loaded there) and the same seven-workload step, run by the C port of the
reference's algorithms on the host cores with every list decoded at each visit; PageRank and HITS
run a sample of their 30 iterations and the step's time is projected from it.
Multi-GPU runs are independent replicas (every graph fits one GPU; nothing is exchanged): time is
the slowest rank's, edges are summed over ranks; the forms, the CPU baseline and the FP64 check
run only at N = 1.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CONFIG_NAME = "all7"
WORKLOAD = ("all7: 2,000,000 vertices, 40,000,000 temporal edges, power-law out-degree alpha 2.0 with "
            "preferential in-degree, 70% of successors within +-64, 20% of each list copied from a vertex "
            "in the window of 7, Poisson timestamps over a 1e8 span; RA, BFS, CC, PR x30, HITS x30, DC, GC")
METRIC = "GTEPS on compressed graph (all seven workloads)"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def replica_totals(ms: float, edges: int, world: int, device: str = "cuda") -> tuple[float, int]:
    """Whole-job figures of N independent replicas: the slowest rank's time (max over ranks) and the
    edges all ranks decoded (sum).  Every rank calls it at the same point (two collectives)."""
    if world == 1:
        return ms, edges
    import torch
    import torch.distributed as dist

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e = torch.tensor([edges], dtype=torch.int64, device=device)
    dist.all_reduce(e, op=dist.ReduceOp.SUM)
    return float(t.item()), int(e.item())


def dataset_dir() -> Path:
    return Path(os.environ.get("TGA_BENCH_DATA", Path(tempfile.gettempdir()) / "tga_bench_all7"))


def ensure_dataset(tga, rank: int, world: int, barrier):
    d = dataset_dir()
    marker = d / "summary.json"
    if rank == 0 and not marker.exists():
        t = time.time()
        s = tga.generate(tga.CONFIGS[CONFIG_NAME], d, CONFIG_NAME)
        s["gen_seconds"] = time.time() - t
        marker.write_text(json.dumps(s))
        log(f"generated {CONFIG_NAME} in {s['gen_seconds']:.1f}s: {s}")
    if world > 1:
        barrier()
    return d, json.loads(marker.read_text())


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = Path(tempfile.gettempdir()) / f"tga_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        self.path.unlink(missing_ok=True)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


ONLY = None  # --only: run a single workload per step (profiling runs; not a bench line)


def suite(g, outputs: bool):
    """One step: the seven workloads; returns (edges decoded, launches, per-workload timing)."""
    cfg = g.cfg
    per = {}
    edges = launches = 0

    def rec(name):
        nonlocal edges, launches
        t = g.timing()
        per[name] = t
        edges += t["edges_decoded"]
        launches += t["launches"]

    runs = {
        "RA": lambda: g.neighbor_access(outputs=outputs),
        "BFS": lambda: g.bfs(cfg.bfs_start_vertex, outputs=outputs),
        "CC": lambda: g.connected_components(outputs=outputs),
        "PR": lambda: g.pagerank(30, outputs=outputs),
        "HITS": lambda: g.hits(30, outputs=outputs),
        "DC": lambda: g.degree_centrality(0, 0, outputs=outputs),
        "GC": lambda: g.color(0, outputs=outputs),
    }
    for name, fn in runs.items():
        if ONLY and name != ONLY:
            continue
        fn()
        rec(name)
    return edges, launches, per


def d2h_bytes_per_step(nv: int) -> int:
    # RA: uint8 + uint64 + int32; BFS: 2x int32; CC: int32; PR: f32; HITS: 2x f32; DC: int32 + int64; GC: 2x u32
    return nv * ((1 + 8 + 4) + 8 + 4 + 4 + 8 + 12 + 8)


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        j = json.loads(p.read_text())
        return float(j["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def kernel_traffic():
    """DRAM bytes per launch of the PageRank kernel from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get("k_pr_iter_all7_bytes_per_launch")
        except Exception:
            return None
    return None


def cpu_baseline(ddir: Path, summary: dict, threads: int):
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle

    n = int(summary["n"])
    o = pyoracle.Oracle(ddir, CONFIG_NAME, n, materialize=False)
    iters = 1
    # A thread count given to the oracle stays set for its later calls, so both passes name theirs.
    cores = threads or pyoracle.max_threads()
    t = time.time()
    _, edges = o.stream_pagerank(n - 1, n, 0, iters, threads=cores)
    dt = time.time() - t
    # The same pass on one core: the like-for-like figure against a single-threaded CPU runner.
    t = time.time()
    _, edges1 = o.stream_pagerank(n - 1, n, 0, iters, threads=1)
    dt1 = time.time() - t
    o.close()
    return {"value": edges / dt / 1e9, "unit": "GTEPS", "cores": cores, "kind": "port",
            "sample": f"{iters} temporal-PageRank iteration over the full {CONFIG_NAME} graph, every list decoded "
                      f"from the compressed streams by the C oracle port ({edges} edges, {dt:.2f}s)",
            "one_core": {"value": edges1 / dt1 / 1e9, "unit": "GTEPS", "cores": 1,
                         "sample": f"the same pass on one thread ({edges1} edges, {dt1:.2f}s)"}}


def fp64_check(ddir: Path, summary: dict, pr, hub, auth, bfs_src: int) -> dict:
    """Error of the engine's FP32 PageRank x30 and HITS x30 at the benchmarked configuration against
    the FP64 oracle (computed after the timed regions; the oracle is the checker here)."""
    import numpy as np

    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle

    n = int(summary["n"])
    t = time.time()
    o = pyoracle.Oracle(ddir, CONFIG_NAME, n)
    opr = o.pagerank(n - 1, n, 0, 30)
    ohub, oauth = o.hits(n - 1, n, 0, 30)
    o.close()

    def err(a, b):
        d = np.abs(np.asarray(a, np.float64) - b)
        return {"l1": float(d.sum()), "max": float(d.max()), "l1_rel": float(d.sum() / max(np.abs(b).sum(), 1e-300))}

    return {"pagerank_x30": err(pr, opr), "hits_x30_hub": err(hub, ohub), "hits_x30_auth": err(auth, oauth),
            "tolerance": "PageRank L1 <= 1e-5 of the rank mass; HITS max <= 1e-5 per entry (tests)",
            "oracle_s": round(time.time() - t, 1)}


REF_GPU_PROGRAMS = {  # reference program -> the engine's call for the same workload on the same graph
    "neighbor_access": ("RA", lambda g, c: g.neighbor_access(outputs=False)),
    "bfs": ("BFS", lambda g, c: g.bfs(c.BFS_SOURCE, outputs=False)),
    "connected_components": ("CC", lambda g, c: g.connected_components(outputs=False)),
    "pagerank": ("PR", lambda g, c: g.pagerank(c.PR_ITERS, outputs=False)),
    "hits": ("HITS", lambda g, c: g.hits(c.HITS_ITERS, outputs=False)),
    "graph_coloring": ("GC", lambda g, c: g.color(0, outputs=False)),
}


def ref_gpu_section(tga) -> dict:
    """The reference's own GPU programs beside the engine, on one GPU and one graph (a baseline leg,
    like cpu_baseline; their results are compared with the engine's in tests/test_reference_gpu.py).

    The programs (gpu_cuda/shared/<algorithm>.cu, built unchanged into oracle/_ref/ with sizes
    compiled in) run on the 6,000-vertex / 120,000-edge dataset they were built for; their harness
    brackets every kernel launch with events and reports the device time per kernel.  The engine's
    figure is the device time of the same workload through its public call, best of 5 after a
    warm-up.  Skipped when oracle/_ref/ holds no programs."""
    ref = ROOT / "oracle" / "_ref"
    if not (ref / "manifest.json").exists():
        return {"skipped": "reference GPU programs not built (oracle/_ref/manifest.json absent)"}
    sys.path.insert(0, str(ROOT / "oracle" / "refgpu"))
    import config as refcfg

    root = Path(tempfile.mkdtemp(prefix="tga_refgpu_"))
    ddir = root / "data" / "compressed" / refcfg.NAME
    tga.generate(tga.GenParams(**refcfg.PARAMS), ddir, refcfg.NAME)
    tables = root / "gpu_cuda" / "decode_tables"
    tables.mkdir(parents=True)
    for kind, fname in ((0, "gammaInA.txt"), (3, "zetaInA.txt")):
        (tables / fname).write_text(",".join(str(int(v)) for v in tga.decode_table(kind)) + ",")
    n = refcfg.N
    cfg = tga.DatasetConfig(name=refcfg.NAME, max_label=n - 1, max_vertex=n, bfs_start_vertex=refcfg.BFS_SOURCE,
                            connected_components_vertex_begin=refcfg.CC_BEGIN)
    g = tga.Graph.open_dir(ddir, refcfg.NAME, cfg)
    out = {"workload": f"reference GPU programs vs the engine on the {n:,}-vertex / "
                       f"{refcfg.PARAMS['m']:,}-edge graph they are built for (PR and HITS x{refcfg.PR_ITERS})",
           "programs": {}}
    try:
        for prog, (name, call) in REF_GPU_PROGRAMS.items():
            exe = ref / prog
            if not exe.exists():
                continue
            times = root / f"{prog}.times"
            env = dict(os.environ, TGA_COMPRESS_ROOT=str(root), TGA_REF_DUMP=str(root / f"{prog}.dump"),
                       TGA_REF_TIMES=str(times))
            r = subprocess.run([str(exe)], cwd=root, env=env, capture_output=True, text=True, timeout=600)
            if r.returncode != 0 or not times.exists():
                out["programs"][prog] = {"error": f"exit {r.returncode}: {(r.stderr or r.stdout)[-200:]}"}
                continue
            kernels = {}
            for line in times.read_text().splitlines():
                cnt, ms, kname = line.split(" ", 2)
                kernels[kname] = {"launches": int(cnt), "ms": float(ms)}
            ref_ms = sum(k["ms"] for k in kernels.values())
            call(g, refcfg)  # warm-up
            eng = []
            for _ in range(5):
                call(g, refcfg)
                eng.append(g.timing()["total_ms"])
            top = max(kernels.items(), key=lambda kv: kv[1]["ms"]) if kernels else ("", {"ms": 0.0})
            out["programs"][prog] = {
                "engine_workload": name, "ref_kernel_ms": round(ref_ms, 4),
                "ref_launches": sum(k["launches"] for k in kernels.values()),
                "ref_top_kernel": {"name": top[0], "ms": round(top[1]["ms"], 4)},
                "engine_ms": round(min(eng), 4), "speedup": round(ref_ms / min(eng), 2) if min(eng) > 0 else None}
    finally:
        g.close()
    return out


def random_windows(rng, k, span, lo_frac=0.05, hi_frac=0.5):
    """Windows of 5-50% of the timestamp span at random positions (the batched/served query mix)."""
    import numpy as np

    w = rng.uniform(lo_frac, hi_frac, k) * span
    lo = rng.uniform(0, 1, k) * (span - w)
    return lo.astype(np.int64), (lo + w).astype(np.int64)


def batched_section(tga, g, n, span, tune=True, plain_bfs=256, plain_pr=32):
    """256 windowed BFS sources as one batched traversal and 32 windowed PageRanks (20 iterations)
    as one strided vector, against the same queries one call each.  Results stay on the device
    (NULL outputs) on both sides, so the comparison is the device work of the two forms."""
    import ctypes as C

    import numpy as np

    L = tga.lib()
    # The batched form runs under the project autotuner's choice of slice length, item size and
    # dense-level divisor (tga_autotune; its probe and choice are reported).
    if tune:
        t0 = time.perf_counter()
        tune = g.autotune()
        tune["wall_s"] = time.perf_counter() - t0
    else:
        tune = None
    rng = np.random.default_rng(3)
    src = rng.integers(0, n, 256).astype(np.int32)
    blo, bhi = random_windows(rng, 256, span)
    plo, phi = random_windows(rng, 32, span)
    d, a = C.c_float(0.85), C.c_float(0.1)
    _check = tga._check
    _check(L.tga_bfs_batch(g.handle, 16, src.ctypes.data, blo.ctypes.data, bhi.ctypes.data, None))  # warm-up
    _check(L.tga_bfs_batch(g.handle, 256, src.ctypes.data, blo.ctypes.data, bhi.ctypes.data, None))
    bfs_batch_ms = g.timing()["total_ms"]
    _check(L.tga_pagerank_batch(g.handle, 32, 20, d, a, plo.ctypes.data, phi.ctypes.data, None))
    pr_batch_ms = g.timing()["total_ms"]
    # Plain calls: every query, or the first plain_bfs / plain_pr of them scaled to all (large graphs).
    bfs_plain_ms = pr_plain_ms = 0.0
    for i in range(plain_bfs):
        _check(L.tga_bfs(g.handle, int(src[i]), int(blo[i]), int(bhi[i]), None, None))
        bfs_plain_ms += g.timing()["total_ms"]
    for i in range(plain_pr):
        _check(L.tga_pagerank(g.handle, 20, d, a, int(plo[i]), int(phi[i]), None))
        pr_plain_ms += g.timing()["total_ms"]
    bfs_plain_ms *= 256 / plain_bfs
    pr_plain_ms *= 32 / plain_pr
    qs = 256 + 32
    return {"workload": f"256 BFS (random sources, windows 5-50% of span) + 32 windowed PageRank x20 on the "
                        f"{n // 1_000_000}M-vertex graph",
            "queries_per_s": qs / ((bfs_batch_ms + pr_batch_ms) / 1e3),
            "plain_queries_per_s": qs / ((bfs_plain_ms + pr_plain_ms) / 1e3),
            "bfs_batch_ms": bfs_batch_ms, "bfs_plain_ms": bfs_plain_ms, "pr_batch_ms": pr_batch_ms,
            "pr_plain_ms": pr_plain_ms, "timing": "device time (CUDA events), results left on the device",
            "plain_sample": {"bfs": plain_bfs, "pagerank": plain_pr}, "autotune": tune}


def served_section(tga, graphs, spans, load, count):
    """Served form against plain one-query calls on the same query sequence: 60% BFS, 25% PageRank
    (10-50 iterations), 15% CC, random windows (5-50% of the span) over the resident graphs.

    1. Plain service times: each query alone through its single-query call, back to back; the
       plain capacity is count / total service time.
    2. Open loop: Poisson arrivals at `load` x the plain capacity, taken live twice -- by a serial
       client that runs each query with its single-query call once it has arrived and the previous
       one is done (the plain path as a caller would run it), and by the server (tga_submit /
       tga_poll).  Latency = result in the caller's buffer minus arrival.
    3. Burst: all queries submitted at once; served capacity = count / time to drain."""
    import numpy as np

    rng = np.random.default_rng(4)
    queries = []
    for _ in range(count):
        gi = int(rng.integers(0, len(graphs)))
        lo, hi = random_windows(rng, 1, spans[gi])
        r = rng.random()
        if r < 0.6:
            queries.append(dict(kind=tga.Q_BFS, graph=gi, src=int(rng.integers(0, graphs[gi].max_vertex)),
                                t_lo=int(lo[0]), t_hi=int(hi[0])))
        elif r < 0.85:
            queries.append(dict(kind=tga.Q_PAGERANK, graph=gi, iters=int(rng.integers(10, 51)), t_lo=int(lo[0]),
                                t_hi=int(hi[0])))
        else:
            queries.append(dict(kind=tga.Q_CC, graph=gi, t_lo=int(lo[0]), t_hi=int(hi[0])))

    def plain_call(q):
        g = graphs[q["graph"]]
        if q["kind"] == tga.Q_BFS:
            g.bfs(q["src"], q["t_lo"], q["t_hi"])
        elif q["kind"] == tga.Q_PAGERANK:
            g.pagerank(q["iters"], 0.85, 0.1, q["t_lo"], q["t_hi"])
        else:
            g.connected_components(q["t_lo"], q["t_hi"])

    # 1. plain service times (results to host buffers, as the served queries get)
    service = []
    for q in queries:
        t = time.perf_counter()
        plain_call(q)
        service.append(time.perf_counter() - t)
    plain_capacity = count / sum(service)
    rate = load * plain_capacity
    arrivals = np.cumsum(np.random.default_rng(5).exponential(1.0 / rate, count))

    def pct(x, p):
        x = np.sort(np.asarray(x))
        return float(x[min(len(x) - 1, int(p * (len(x) - 1) + 0.5))])

    kinds = {tga.Q_BFS: "bfs", tga.Q_PAGERANK: "pagerank", tga.Q_CC: "cc"}

    def by_kind(lat_ms):
        out = {}
        for k, name in kinds.items():
            x = [l for l, q in zip(lat_ms, queries) if q["kind"] == k]
            if x:
                out[name] = {"n": len(x), "p50_ms": pct(x, 0.5), "p99_ms": pct(x, 0.99)}
        return out

    # 2a. open loop, plain: a serial client
    plain_lat = []
    t0 = time.perf_counter()
    for q, at in zip(queries, arrivals):
        wait = at - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        plain_call(q)
        plain_lat.append((time.perf_counter() - t0 - at) * 1e3)
    plain_span = time.perf_counter() - t0
    # 2b. open loop through the server
    with tga.Server(budget_bytes=120 << 30) as srv:
        for g in graphs:
            srv.add_graph(g)
        t0 = time.perf_counter()
        tickets = []
        for q, at in zip(queries, arrivals):
            wait = at - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
            tickets.append(srv.submit(**q))
        srv.drain()
        served_span = time.perf_counter() - t0
        st = srv.stats()
        served_lat = [srv.poll(t)[1] for t in tickets]
    # 3. burst
    with tga.Server(budget_bytes=120 << 30) as srv:
        for g in graphs:
            srv.add_graph(g)
        t0 = time.perf_counter()
        for q in queries:
            srv.submit(**q)
        srv.drain()
        burst_s = time.perf_counter() - t0
        bst = srv.stats()
    return {"workload": f"{count} queries over resident graphs of {[gg.max_vertex for gg in graphs]} vertices; "
                        "60% BFS, 25% PageRank x10-50, 15% CC; windows 5-50% of span; results to host buffers; "
                        f"open-loop Poisson arrivals at {load:.2f} x the plain capacity, taken live by a serial "
                        "plain client and by the server",
            "offered_queries_per_s": rate,
            "served": {"p50_ms": pct(served_lat, 0.5), "p99_ms": pct(served_lat, 0.99),
                       "mean_ms": float(np.mean(served_lat)), "rounds": st["rounds"],
                       "queries_per_s": count / served_span, "burst_queries_per_s": count / burst_s,
                       "burst_p50_ms": bst["p50_ms"], "burst_p99_ms": bst["p99_ms"], "by_kind": by_kind(served_lat)},
            "plain": {"p50_ms": pct(plain_lat, 0.5), "p99_ms": pct(plain_lat, 0.99),
                      "mean_ms": float(np.mean(plain_lat)), "queries_per_s": count / plain_span,
                      "capacity_queries_per_s": plain_capacity, "by_kind": by_kind(plain_lat),
                      "service_ms_by_kind": {name: float(np.mean([sv for sv, q in zip(service, queries)
                                                                  if q["kind"] == k]) * 1e3)
                                             for k, name in kinds.items()}}}


def batched_at_size(tga, g_tune, name: str) -> dict:
    """The batched form on its named configuration (20M vertices / 500M temporal edges by default),
    generated on this machine if absent: the project autotuner runs on the benchmark graph g_tune
    (the 2M/40M one; tuning the 20M graph itself would take minutes) and its slice length and item
    size are applied to the large graph, whose batched section then runs with plain calls timed on
    a sample (16 BFS, 4 PageRanks) and scaled."""
    p = tga.CONFIGS[name]
    ddir = Path(tempfile.gettempdir()) / f"tga_bench_{name}"
    t0 = time.perf_counter()
    if not (ddir / f"{name}.graph").exists():
        tga.generate(p, ddir, name)
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    tune = g_tune.autotune()
    tune["wall_s"] = time.perf_counter() - t0
    n = int(p.n)
    t0 = time.perf_counter()
    big = tga.Graph.open_dir(ddir, name, tga.DatasetConfig(name=name, max_label=n - 1, max_vertex=n))
    load_s = time.perf_counter() - t0
    try:
        big.set_work_params(tune["slice_edges"], tune["item_edges"])
        sec = batched_section(tga, big, n, int(p.ts_span), tune=False, plain_bfs=16, plain_pr=4)
    finally:
        big.close()
    sec["autotune"] = dict(tune, applied="slice length and item size, tuned on the benchmark graph")
    sec["config"] = {"workload": name, "vertices": n, "temporal_edges": int(p.m)}
    sec["generate_s"], sec["load_s"] = gen_s, load_s
    return sec


def run_batched_scale(args):
    """Batched form alone on a named configuration (the 20M/500M one by default): generated here,
    loaded, one batched section with plain calls timed on a sample.  Prints one JSON line."""
    import compresstemporalgraph_b200 as tga

    name = args.batched_graph
    p = tga.CONFIGS[name]
    ddir = Path(tempfile.gettempdir()) / f"tga_bench_{name}"
    t0 = time.perf_counter()
    if not (ddir / f"{name}.graph").exists():
        summary = tga.generate(p, ddir, name)
    else:
        summary = None
    gen_s = time.perf_counter() - t0
    n = int(p.n)
    t0 = time.perf_counter()
    g = tga.Graph.open_dir(ddir, name, tga.DatasetConfig(name=name, max_label=n - 1, max_vertex=n))
    load_s = time.perf_counter() - t0
    import ctypes as C

    sec = batched_section(tga, g, n, int(p.ts_span), tune=False, plain_bfs=16, plain_pr=4)
    info = tga._Info()
    tga._check(tga.lib().tga_get_info(g.handle, C.byref(info)))  # device bytes now include the scratch
    info = {k: getattr(info, k) for k, _ in tga._Info._fields_}
    g.close()
    line = {"metric": "batched queries/s (256 windowed BFS + 32 windowed PageRank x20)", "value": sec["queries_per_s"],
            "unit": "queries/s", "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
            "config": {"workload": name, "vertices": n, "temporal_edges": int(p.m)}, "batched": sec,
            "generate_s": gen_s, "load_s": load_s, "summary": summary, "info": info}
    print(json.dumps(line), flush=True)
    return 0


def generate_in_subprocess(name: str, ddir: Path) -> dict:
    """Generates a configuration's dataset in a child process, so that the calling process never
    maps the engine's library (the reference arm times the CPU port alone)."""
    marker = ddir / "summary.json"
    if not marker.exists():
        code = ("import json, sys, time; sys.path.insert(0, %r); import compresstemporalgraph_b200 as tga; "
                "t = time.time(); s = tga.generate(tga.CONFIGS[%r], %r, %r); s['gen_seconds'] = time.time() - t; "
                "open(%r, 'w').write(json.dumps(s))") % (str(ROOT), name, str(ddir), name, str(marker))
        subprocess.run([sys.executable, "-c", code], check=True)
    return json.loads(marker.read_text())


# PageRank and HITS iterations the CPU arm runs per step (of the 30 each that the step holds);
# every iteration decodes the same lists, so the full step's time is the sample's scaled up.
REF_ITER_SAMPLE = 3


def reference_step(o, n: int, deg, src: int, prio, threads: int) -> dict:
    """One sampled step of the seven workloads on the CPU port, every list decoded from the
    compressed streams at each visit.  Returns {workload: (edges, seconds)}."""
    ml, mv, act = n - 1, n, 0
    out = {}

    def timed(name, fn):
        t = time.perf_counter()
        e = fn()
        out[name] = (int(e), time.perf_counter() - t)

    timed("RA", lambda: o.stream_decode(act, ml, threads=threads, max_vertex=mv)[1])
    timed("BFS", lambda: o.stream_bfs(ml, mv, act, src)[1])
    timed("CC", lambda: o.stream_cc(ml, mv, act, 0)[1])
    timed("PR", lambda: o.stream_pagerank(ml, mv, act, REF_ITER_SAMPLE, threads=threads)[1])
    timed("HITS", lambda: o.stream_hits(ml, mv, act, REF_ITER_SAMPLE, threads=threads)[1])
    timed("DC", lambda: o.stream_degree(ml, mv, act, 0, 0, threads=threads)[1])
    timed("GC", lambda: o.stream_color(ml, mv, act, prio, threads=threads)[1])
    return out


def run_skew(args):
    """Skew stress on its named configuration (100M vertices / 2B temporal edges, Zipf 1.6, 16 hubs of
    5M out-edges, bursty timestamps): generated on this machine if absent, loaded, then HITS x30 and
    Jones-Plassmann colouring (cuRAND priorities) timed as the benchmark times its steps (device
    time, W warm-up and K timed runs).  Prints one JSON line.  Parity at this shape, scaled down 100x,
    is tests/test_gpu_bench_config.py's skew1m case."""
    import compresstemporalgraph_b200 as tga

    name = args.skew_graph
    p = tga.CONFIGS[name]
    ddir = Path(tempfile.gettempdir()) / f"tga_bench_{name}"
    t0 = time.perf_counter()
    summary = None
    if not (ddir / f"{name}.graph").exists():
        summary = tga.generate(p, ddir, name)
    gen_s = time.perf_counter() - t0
    n = int(p.n)
    t0 = time.perf_counter()
    g = tga.Graph.open_dir(ddir, name, tga.DatasetConfig(name=name, max_label=n - 1, max_vertex=n))
    load_s = time.perf_counter() - t0
    info = g.info
    out = {}
    for wl, fn in (("HITS", lambda: g.hits(30, outputs=False)), ("GC", lambda: g.color(0, outputs=False))):
        for _ in range(args.warmup):
            fn()
        ms = edges = 0.0
        iters = 0
        for _ in range(args.steps):
            fn()
            t = g.timing()
            ms += t["total_ms"]
            edges += t["edges_decoded"]
            iters = t["iterations"]
        out[wl] = {"ms": ms / args.steps, "edges": int(edges / args.steps), "gteps": edges / (ms / 1e3) / 1e9,
                   "iterations": iters}
    _, _, deg = g.neighbor_access()
    g.close()
    tot_edges = sum(v["edges"] for v in out.values())
    tot_ms = sum(v["ms"] for v in out.values())
    line = {"metric": "GTEPS on compressed graph (skew stress: HITS x30 + JP colouring)", "value": tot_edges / tot_ms / 1e6,
            "unit": "GTEPS", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "data": "synthetic", "config": {"workload": name, "vertices": n, "temporal_edges": int(p.m),
                                            "hubs": int(p.hub_count), "hub_degree": int(p.hub_degree),
                                            "largest_list": int(deg.max()), "compressed_bytes": info["graph_bytes"] +
                                            info["timestamp_bytes"] + info["index_bytes"]},
            "workloads": out, "generate_s": gen_s, "load_s": load_s, "summary": summary, "info": info}
    print(json.dumps(line), flush=True)
    return 0


def run_reference(args):
    """CPU arm: the reference's algorithms as restated by the C port (the reference's own CPU code
    is Java, and no JDK exists on either machine), timed on the host cores over the same graph and
    the same seven-workload step, every list decoded from the compressed streams at each visit.
    The engine's library is never loaded in this process.

    Each timed step runs RA, BFS, CC, DC and GC once, and REF_ITER_SAMPLE of the 30 PageRank and
    30 HITS iterations; value = the full step's edges over its projected time (PageRank and HITS
    scaled by 30 / REF_ITER_SAMPLE), so it is the same GTEPS definition as the engine's line."""
    rank, local, world = dist_env()
    if rank != 0:
        return 0
    sys.path.insert(0, str(ROOT / "oracle"))
    import numpy as np

    import pyoracle

    ddir = dataset_dir()
    summary = generate_in_subprocess(CONFIG_NAME, ddir)
    n = int(summary["n"])
    threads = pyoracle.max_threads()
    o = pyoracle.Oracle(ddir, CONFIG_NAME, n, materialize=False)
    deg = o.outdegrees()
    src = int(deg.argmax())  # the engine arm's BFS source
    # Colouring priorities: java.util.Random(123).nextInt(256) per vertex (the Java runner's); the
    # engine's line uses cuRAND's, which only the GPU produces.
    prio = pyoracle.java_random256(123, n)
    for _ in range(args.warmup):
        o.stream_decode(0, n - 1, threads=threads)
    steps = [reference_step(o, n, deg, src, prio, threads) for _ in range(args.steps)]
    o.close()
    scale = {"PR": 30 / REF_ITER_SAMPLE, "HITS": 30 / REF_ITER_SAMPLE}
    per, edges_full, secs_full, secs_sampled = {}, 0.0, 0.0, 0.0
    for name in steps[0]:
        e = sum(st[name][0] for st in steps) / len(steps)
        t = sum(st[name][1] for st in steps) / len(steps)
        k = scale.get(name, 1.0)
        per[name] = {"edges": int(e), "s": round(t, 4), "gteps": e / t / 1e9 if t else None,
                     "iterations_sampled": REF_ITER_SAMPLE if name in scale else None}
        edges_full += e * k
        secs_full += t * k
        secs_sampled += t
    v = edges_full / secs_full / 1e9
    sample = (f"per step: RA, BFS (source {src}), CC, DC and GC once, {REF_ITER_SAMPLE} of the 30 PageRank and "
              f"30 HITS iterations, over the full {CONFIG_NAME} graph with every list decoded from the compressed "
              f"streams at each visit by the C oracle port on {threads} threads (BFS/CC one thread); value = full "
              f"step's edges / its projected time (PageRank and HITS x{30 // REF_ITER_SAMPLE}); colouring with "
              "java.util.Random(123) priorities")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "GTEPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": secs_full * 1000, "sampled_ms_per_step": secs_sampled * 1000,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "vertices": n, "temporal_edges": int(summary["m"])},
            "workloads": per,
            "cpu_baseline": {"value": v, "unit": "GTEPS", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the batched and served measurements")
    ap.add_argument("--served-load", type=float, default=0.8,
                    help="offered load of the served open loop, as a fraction of the plain path's capacity")
    ap.add_argument("--served-count", type=int, default=300)
    ap.add_argument("--served-graphs", default="small,served1m",
                    help="resident graphs of the served section besides the benchmark graph (configuration names)")
    ap.add_argument("--batched-config", default="batched",
                    help="configuration of the line's batched section (default: batched, 20M/500M; '' skips it)")
    ap.add_argument("--batched-graph", default=None,
                    help="run only the batched section on this generated configuration (e.g. batched: 20M/500M)")
    ap.add_argument("--skew-graph", default=None,
                    help="run only the skew-stress section on this generated configuration (e.g. skew: 100M/2B)")
    ap.add_argument("--only", choices=["RA", "BFS", "CC", "PR", "HITS", "DC", "GC"],
                    help="run one workload per step (for profiling; the line is not the benchmark)")
    args = ap.parse_args()
    global ONLY
    ONLY = args.only
    if args.impl == "reference":
        return run_reference(args)
    if args.batched_graph:
        return run_batched_scale(args)
    if args.skew_graph:
        return run_skew(args)

    import torch

    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    barrier = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        barrier = lambda: dist.barrier(device_ids=[local])
    import compresstemporalgraph_b200 as tga

    ddir, summary = ensure_dataset(tga, rank, world, barrier)
    n = int(summary["n"])
    cfg = tga.DatasetConfig(name=CONFIG_NAME, max_label=n - 1, max_vertex=n, bfs_start_vertex=1)
    g = tga.Graph.open_dir(ddir, CONFIG_NAME, cfg)
    # BFS starts at the vertex with the largest out-list (vertex 1, the reference default, has a
    # handful of edges in this graph and would time an empty traversal).
    _, _, deg = g.neighbor_access()
    cfg.bfs_start_vertex = int(deg.argmax())
    stream = torch.cuda.ExternalStream(g.stream)

    for _ in range(args.warmup):
        suite(g, outputs=False)

    def timed(outputs: bool):
        if barrier:
            barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        edges = launches = 0
        per_all = []
        for _ in range(args.steps):
            e, l, per = suite(g, outputs)
            edges += e
            launches += l
            per_all.append(per)
        ev1.record(stream)
        torch.cuda.synchronize()
        if barrier:
            barrier()
        ms, total = replica_totals(ev0.elapsed_time(ev1), edges, world)
        return ms, edges, total, launches, per_all

    with Clocks(local) as clk:
        ms, edges, total_edges, launches, per_all = timed(outputs=False)
    clocks = clk.summary()
    e2e_ms, _, e2e_total, _, _ = timed(outputs=True)

    value = total_edges / (ms / 1e3) / 1e9
    e2e_value = e2e_total / (e2e_ms / 1e3) / 1e9

    if ONLY:
        print(json.dumps({"only": ONLY, "ms": ms, "edges": edges, "workloads": {k: v for k, v in per_all[0].items()}}))
        g.close()
        return 0
    # Roofline of the PageRank iteration kernel (30 launches per step, one full decode pass each).
    pr = [p["PR"] for p in per_all]
    pr_launch_ms = sum(p["decode_ms"] for p in pr) / max(1, sum(p["decode_launches"] for p in pr))
    info = g.info
    active_bytes = info["graph_bytes"] + info["timestamp_bytes"] + info["index_bytes"]
    achieved = active_bytes / (pr_launch_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    traffic = kernel_traffic()
    breakdown = {}
    for name in per_all[0]:
        ms_w = sum(p[name]["total_ms"] for p in per_all) / len(per_all)
        ed = sum(p[name]["edges_decoded"] for p in per_all) / len(per_all)
        breakdown[name] = {"ms": round(ms_w, 3), "edges": int(ed), "gteps": round(ed / (ms_w / 1e3) / 1e9, 3) if ms_w else None,
                           "iterations": per_all[0][name]["iterations"]}

    # Workloads that read the timestamp stream (81% of the compressed bytes): HITS over the full
    # window and colouring depend only on the successor order and skip it, so this figure counts
    # only the workloads that decode every byte of every list they visit.
    ts_names = [nm for nm in ("RA", "BFS", "CC", "PR", "DC") if nm in breakdown]
    ts_edges = sum(breakdown[nm]["edges"] for nm in ts_names)
    ts_ms = sum(breakdown[nm]["ms"] for nm in ts_names)
    all_edges = sum(b["edges"] for b in breakdown.values())
    timestamp_reading = {"workloads": ts_names, "gteps": ts_edges / (ts_ms / 1e3) / 1e9 if ts_ms else None,
                         "edges_share": ts_edges / all_edges if all_edges else None}
    line = {
        "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "vertices": n, "temporal_edges": int(summary["m"]),
                   "compressed_bytes": active_bytes, "l2": "inputs larger than L2 (compressed graph "
                   f"{active_bytes / 1e6:.0f} MB > 126 MB L2), no flush", "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": "GTEPS", "h2d_bytes_per_step": 64,
                "d2h_bytes_per_step": d2h_bytes_per_step(n)},
        "roofline": {"bound": "hbm", "kernel": "k_pr_iter", "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "bytes_per_launch": active_bytes, "launch_ms": pr_launch_ms},
        "bfs_source": cfg.bfs_start_vertex,
        "clocks": clocks,
        "gpu_launches": launches,
        "workloads": breakdown,
        "timestamp_reading": timestamp_reading,
    }
    # The forms, the CPU baseline and the FP64 check describe the one-GPU line; a replica run
    # (N > 1) reports the replicas' figures only, so its GPUs are held for the timed work alone.
    if rank == 0 and world == 1 and not args.no_forms and not ONLY:
        try:
            extra = []
            names = [nm for nm in args.served_graphs.split(",") if nm and nm != CONFIG_NAME]
            for name in names:
                dd = Path(tempfile.gettempdir()) / f"tga_bench_{name}"
                if not (dd / f"{name}.graph").exists():
                    tga.generate(tga.CONFIGS[name], dd, name)
                nn = tga.CONFIGS[name].n
                extra.append(tga.Graph.open_dir(dd, name, tga.DatasetConfig(name=name, max_label=nn - 1, max_vertex=nn)))
            spans = [int(tga.CONFIGS[nm].ts_span) for nm in names + [CONFIG_NAME]]
            line["served"] = served_section(tga, extra + [g], spans, args.served_load, args.served_count)
            for gg in extra:
                gg.close()
        except Exception as e:  # reported, not fatal
            line["served_error"] = str(e)
        if args.batched_config:
            try:
                line["batched"] = batched_at_size(tga, g, args.batched_config)
            except Exception as e:  # reported, not fatal
                line["batched_error"] = str(e)
        try:
            line["ref_gpu"] = ref_gpu_section(tga)
        except Exception as e:  # reported, not fatal
            line["ref_gpu"] = {"error": str(e)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(ddir, summary, 0)
        except Exception as e:  # reported, not fatal
            line["cpu_baseline"] = {"value": None, "error": str(e)}
        try:
            pr_out = g.pagerank(30)
            hub_out, auth_out = g.hits(30)
            line["fp64_error"] = fp64_check(ddir, summary, pr_out, hub_out, auth_out, cfg.bfs_start_vertex)
        except Exception as e:  # reported, not fatal
            line["fp64_error"] = {"error": str(e)}
    g.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
