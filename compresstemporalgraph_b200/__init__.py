"""Python mirror of the engine's C ABI (include/tga.h).

The reference exposes its workloads as one CUDA executable per (dataset, algorithm), configured
by the macros of gpu_cuda/shared/dataset_config_base.cuh.  This module exposes the same
workloads over the in-tree native library ``libtga.so``: a :class:`DatasetConfig` with the
macro names, :class:`Graph` (one resident compressed graph) with one method per executable,
and the format-layer helpers (:func:`generate`, :func:`encode_raw`, :func:`decode_table`).

There is no fallback: if ``libtga.so`` is missing, importing raises ImportError, and every
workload runs on the GPU through the native library.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libtga.so"

TGA_OK, TGA_E_IO, TGA_E_FORMAT, TGA_E_OOM, TGA_E_DECODE, TGA_E_TIMEOUT, TGA_E_ARG, TGA_E_CUDA, TGA_E_AGAIN = range(9)
TGA_UNSET_TS = -(1 << 63)
T_MAX = (1 << 63) - 1
HITS_GPU, HITS_JAVA = 0, 1
CC_EARLY_EXIT = 1
CC_ONE_SEED = 2
GC_JAVA_ISOLATED = 1
UINT32_INF = 0xFFFFFFFF
INT32_INF = 0x7FFFFFFF


class TgaError(RuntimeError):
    """A non-zero tga_status with the library's message."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"tga error {code}: {msg}")
        self.code = code


class _Cfg(C.Structure):
    _fields_ = [("name", C.c_char_p), ("storage_name", C.c_char_p), ("max_label", C.c_int32),
                ("max_vertex", C.c_int32), ("min_timestamp", C.c_int64), ("min_graph_vertex", C.c_int32),
                ("active_vertex_begin", C.c_int32), ("bfs_start_vertex", C.c_int32),
                ("cc_vertex_begin", C.c_int32), ("multiple_initial_value", C.c_int32),
                ("pr_iters", C.c_int32), ("hits_iters", C.c_int32)]


class _Info(C.Structure):
    _fields_ = [("n", C.c_int32), ("max_label", C.c_int32), ("max_vertex", C.c_int32),
                ("active_vertex_begin", C.c_int32), ("min_timestamp", C.c_int64), ("graph_bytes", C.c_uint64),
                ("timestamp_bytes", C.c_uint64), ("index_bytes", C.c_uint64), ("device_bytes", C.c_uint64),
                ("graph_ef_low_bits", C.c_int32), ("timestamp_ef_low_bits", C.c_int32)]


class _Timing(C.Structure):
    _fields_ = [("total_ms", C.c_double), ("decode_ms", C.c_double), ("decode_launches", C.c_int64),
                ("edges_decoded", C.c_int64), ("compressed_bytes", C.c_uint64), ("iterations", C.c_int32), ("launches", C.c_int64)]


class _Query(C.Structure):
    _fields_ = [("kind", C.c_int32), ("graph", C.c_int32), ("src", C.c_int32), ("iters", C.c_int32),
                ("dst", C.c_int32), ("reserved", C.c_int32), ("t_lo", C.c_int64), ("t_hi", C.c_int64),
                ("out", C.c_void_p)]


class _TuneResult(C.Structure):
    _fields_ = [("slice_edges", C.c_int32), ("item_edges", C.c_int32), ("dense_div", C.c_int32),
                ("candidates", C.c_int32), ("best_ms", C.c_double), ("default_ms", C.c_double)]


class _ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64), ("rounds", C.c_int64),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double), ("queries_per_s", C.c_double)]


class _GenParams(C.Structure):
    _fields_ = [("n", C.c_int64), ("m", C.c_int64), ("deg_exponent", C.c_double), ("max_degree", C.c_int64),
                ("repeat_frac", C.c_double), ("local_frac", C.c_double), ("local_radius", C.c_int32),
                ("pref_frac", C.c_double), ("copy_frac", C.c_double), ("ts_kind", C.c_int32),
                ("ts_span", C.c_int64), ("min_timestamp", C.c_int64), ("seed", C.c_uint64), ("ref_safe", C.c_int32),
                ("hub_count", C.c_int32), ("hub_degree", C.c_int64)]


class _RefDepths(C.Structure):
    _fields_ = [("nodes", C.c_int64), ("referenced_nodes", C.c_int64), ("truncated_nodes", C.c_int64),
                ("maximum_depth", C.c_int32), ("configured_max_ref_count", C.c_int32),
                ("depth_counts", C.c_int64 * 16)]


class _GenSummary(C.Structure):
    _fields_ = [("n", C.c_int64), ("m", C.c_int64), ("max_degree", C.c_int64), ("graph_bytes", C.c_uint64),
                ("timestamp_bytes", C.c_uint64), ("index_bytes", C.c_uint64), ("copied_arcs", C.c_int64),
                ("intervalised_arcs", C.c_int64), ("residual_arcs", C.c_int64), ("multiples_arcs", C.c_int64),
                ("max_chain", C.c_int64)]


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python compresstemporalgraph_b200/build.py`")
    lib = C.CDLL(str(LIB_PATH))
    P = C.c_void_p
    sig = {
        "tga_cfg_default": (None, [C.POINTER(_Cfg)]),
        "tga_last_error": (C.c_char_p, []),
        "tga_open": (C.c_int, [C.c_char_p, C.POINTER(_Cfg), C.POINTER(P)]),
        "tga_open_dir": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(_Cfg), C.POINTER(P)]),
        "tga_close": (C.c_int, [P]),
        "tga_get_info": (C.c_int, [P, C.POINTER(_Info)]),
        "tga_get_timing": (C.c_int, [P, C.POINTER(_Timing)]),
        "tga_stream": (P, [P]),
        "tga_set_work_params": (C.c_int, [P, C.c_int32, C.c_int32]),
        "tga_get_work_params": (C.c_int, [P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                          C.POINTER(C.c_int32)]),
        "tga_neighbor_access": (C.c_int, [P, P, P, P]),
        "tga_neighbors": (C.c_int, [P, C.c_int32, P, P, C.c_int32, C.POINTER(C.c_int32)]),
        "tga_decode_all": (C.c_int, [P, P, P, P, C.c_int64]),
        "tga_bfs": (C.c_int, [P, C.c_int32, C.c_int64, C.c_int64, P, P]),
        "tga_cc": (C.c_int, [P, C.c_int64, C.c_int64, C.c_int32, P, C.POINTER(C.c_int32)]),
        "tga_pagerank": (C.c_int, [P, C.c_int32, C.c_float, C.c_float, C.c_int64, C.c_int64, P]),
        "tga_shortest": (C.c_int, [P, C.c_int32, C.c_int64, C.c_int64, P, P]),
        "tga_pagerank_noalloc": (C.c_int, [P, C.c_int32, C.c_float, C.c_float, C.c_int64, C.c_int64, P]),
        "tga_hits": (C.c_int, [P, C.c_int32, C.c_int32, C.c_int64, C.c_int64, P, P]),
        "tga_degree": (C.c_int, [P, C.c_int64, C.c_int64, P, P]),
        "tga_color": (C.c_int, [P, C.c_int32, P, C.c_int32, P, P, C.POINTER(C.c_int32)]),
        "tga_bfs_batch": (C.c_int, [P, C.c_int32, P, P, P, P]),
        "tga_fastest": (C.c_int, [P, C.c_int32, C.c_int64, C.c_int64, P, P]),
        "tga_reverse": (C.c_int, [P, C.c_int64, C.c_char_p, C.c_char_p, C.POINTER(C.c_int64)]),
        "tga_latest_departure": (C.c_int, [P, C.c_int64, C.c_int32, C.c_int64, C.c_int64, P]),
        "tga_cc_batch": (C.c_int, [P, C.c_int32, P, P, C.c_int32, P, P]),
        "tga_is_neighbor": (C.c_int, [P, C.c_int32, P, P, P, P, P]),
        "tga_pagerank_batch_iters": (C.c_int, [P, C.c_int32, P, C.c_float, C.c_float, P, P, P]),
        "tga_cc_job_create": (C.c_int, [P, C.c_int32, C.c_int32, P]),
        "tga_cc_job_add": (C.c_int, [P, C.c_int64, C.c_int64, P]),
        "tga_cc_job_step": (C.c_int, [P, C.c_double, P]),
        "tga_cc_job_take": (C.c_int, [P, C.c_int32, P, P]),
        "tga_cc_job_destroy": (C.c_int, [P]),
        "tga_pagerank_batch": (C.c_int, [P, C.c_int32, C.c_int32, C.c_float, C.c_float, P, P, P]),
        "tga_server_create": (C.c_int, [C.c_int64, C.POINTER(P)]),
        "tga_server_add_graph": (C.c_int, [P, P, C.POINTER(C.c_int32)]),
        "tga_submit": (C.c_int, [P, C.POINTER(_Query), C.POINTER(C.c_int64)]),
        "tga_poll": (C.c_int, [P, C.c_int64, C.POINTER(C.c_double)]),
        "tga_server_drain": (C.c_int, [P]),
        "tga_server_get_stats": (C.c_int, [P, C.POINTER(_ServerStats)]),
        "tga_server_destroy": (C.c_int, [P]),
        "tga_generate": (C.c_int, [C.POINTER(_GenParams), C.c_char_p, C.c_char_p, C.c_char_p,
                                   C.POINTER(_GenSummary)]),
        "tga_encode_raw": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int64, C.POINTER(_GenSummary)]),
        "tga_build_index": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int64]),
        "tga_build_index_device": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int64]),
        "tga_write_reversed": (C.c_int, [P, P, P, C.c_int64, C.c_int64, C.c_char_p, C.c_char_p,
                                          C.POINTER(_GenSummary)]),
        "tga_reference_depths": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(_RefDepths), P]),
        "tga_autotune": (C.c_int, [P, P]),
        "tga_barrier_selftest": (C.c_int, [C.c_double, P]),
        "tga_decode_table": (C.c_int, [C.c_int32, P]),
        "tga_encode_codes": (C.c_int, [C.c_int32, C.c_int32, P, C.c_int64, P, C.c_int64, C.POINTER(C.c_int64)]),
        "tga_ef_encode": (C.c_int, [P, C.c_int64, C.c_int32, P, C.c_int64, P, C.c_int64, C.POINTER(C.c_int64),
                                    C.POINTER(C.c_int64)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = _load()


def lib() -> C.CDLL:
    return _lib


def _check(rc: int) -> None:
    if rc != TGA_OK:
        raise TgaError(rc, (_lib.tga_last_error() or b"").decode(errors="replace"))


def _ptr(a: np.ndarray | None):
    return None if a is None else C.c_void_p(a.ctypes.data)


# The per-dataset macros of gpu_cuda/<DS>/dataset_config.cuh; other fields keep the defaults of
# gpu_cuda/shared/dataset_config_base.cuh.
PRESETS = {
    "Comm": dict(max_label=9999, max_vertex=10000, min_timestamp=0),
    "MyD": dict(max_label=999967, max_vertex=1000001, min_timestamp=0),
    "Flickr": dict(max_label=2585568, max_vertex=2585570, min_timestamp=0),
    "Wiki": dict(max_label=42640545, max_vertex=42640546, min_timestamp=979675713, min_graph_vertex=1,
                 multiple_initial_value=0, pagerank_iterations=100, hits_iterations=100),
    "Yahoo": dict(max_label=102867214, max_vertex=102867263, min_timestamp=1206214540),
    "Yahoo-sub": dict(max_label=102867214, max_vertex=102867263, min_timestamp=1206214540, storage_name="Yahoo",
                      active_vertex_begin=2000, bfs_start_vertex=2001, connected_components_vertex_begin=2000),
}


@dataclass
class DatasetConfig:
    """Runtime form of gpu_cuda/shared/dataset_config_base.cuh (same names and defaults)."""

    name: str
    max_label: int
    max_vertex: int
    storage_name: str | None = None
    min_timestamp: int = TGA_UNSET_TS
    min_graph_vertex: int = 0
    active_vertex_begin: int = 0
    bfs_start_vertex: int = 1
    connected_components_vertex_begin: int = 1
    multiple_initial_value: int = -1
    pagerank_iterations: int = 10
    hits_iterations: int = 10
    _keep: list = field(default_factory=list, repr=False)

    @classmethod
    def preset(cls, name: str, **overrides) -> "DatasetConfig":
        """One of the six datasets the reference ships (gpu_cuda/<DS>/dataset_config.cuh), with
        keyword overrides: Comm, MyD, Flickr, Wiki, Yahoo, Yahoo-sub."""
        if name not in PRESETS:
            raise KeyError(f"no preset {name!r}; presets: {', '.join(PRESETS)}")
        kw = dict(PRESETS[name])
        kw.update(overrides)
        return cls(name=name, **kw)

    def to_c(self) -> _Cfg:
        c = _Cfg()
        _lib.tga_cfg_default(C.byref(c))
        nm = self.name.encode()
        st = (self.storage_name or self.name).encode()
        self._keep = [nm, st]
        c.name, c.storage_name = nm, st
        c.max_label, c.max_vertex = self.max_label, self.max_vertex
        c.min_timestamp = self.min_timestamp
        c.min_graph_vertex = self.min_graph_vertex
        c.active_vertex_begin = self.active_vertex_begin
        c.bfs_start_vertex = self.bfs_start_vertex
        c.cc_vertex_begin = self.connected_components_vertex_begin
        c.multiple_initial_value = self.multiple_initial_value
        c.pr_iters, c.hits_iters = self.pagerank_iterations, self.hits_iterations
        return c


class Graph:
    """One compressed temporal graph resident on the current GPU."""

    def __init__(self, handle: C.c_void_p, cfg: DatasetConfig):
        self._h = handle
        self.cfg = cfg
        info = _Info()
        _check(_lib.tga_get_info(self._h, C.byref(info)))
        self.info = {k: getattr(info, k) for k, _ in _Info._fields_}
        self.n = info.n
        self.max_vertex = info.max_vertex

    @classmethod
    def open(cls, cfg: DatasetConfig, root: str | None = None) -> "Graph":
        """Drop-in loader: <root>/data/compressed/<STORAGE>/... (root None -> $TGA_COMPRESS_ROOT or ../..)."""
        h = C.c_void_p()
        c = cfg.to_c()
        _check(_lib.tga_open(root.encode() if root else None, C.byref(c), C.byref(h)))
        return cls(h, cfg)

    @classmethod
    def open_dir(cls, directory: str | os.PathLike, basename: str, cfg: DatasetConfig) -> "Graph":
        h = C.c_void_p()
        c = cfg.to_c()
        _check(_lib.tga_open_dir(str(directory).encode(), basename.encode(), C.byref(c), C.byref(h)))
        return cls(h, cfg)

    def close(self) -> None:
        if self._h:
            _lib.tga_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        return _lib.tga_stream(self._h) or 0

    def set_work_params(self, slice_edges: int, item_edges: int) -> None:
        _check(_lib.tga_set_work_params(self._h, slice_edges, item_edges))

    def autotune(self) -> dict:
        """Picks slice length, item size and dense-level divisor by timing (tga_autotune)."""
        r = _TuneResult()
        _check(_lib.tga_autotune(self._h, C.byref(r)))
        return {k: getattr(r, k) for k, _ in _TuneResult._fields_}

    def work_params(self) -> dict:
        a, b, c, d = C.c_int32(), C.c_int32(), C.c_int64(), C.c_int32()
        _check(_lib.tga_get_work_params(self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)))
        return {"slice_edges": a.value, "item_edges": b.value, "slices": c.value, "items": d.value}

    def timing(self) -> dict:
        t = _Timing()
        _check(_lib.tga_get_timing(self._h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in _Timing._fields_}

    # ---- workloads ------------------------------------------------------------------------
    def neighbor_access(self, outputs: bool = True):
        nv = self.max_vertex
        if not outputs:
            _check(_lib.tga_neighbor_access(self._h, None, None, None))
            return None
        small = np.zeros(nv, np.uint8)
        csum = np.zeros(nv, np.uint64)
        deg = np.zeros(nv, np.int32)
        _check(_lib.tga_neighbor_access(self._h, _ptr(small), _ptr(csum), _ptr(deg)))
        return small, csum, deg

    def neighbors(self, v: int):
        cnt = C.c_int32()
        _check(_lib.tga_neighbors(self._h, v, None, None, 0, C.byref(cnt)))
        dst = np.zeros(cnt.value, np.int32)
        ts = np.zeros(cnt.value, np.int64)
        _check(_lib.tga_neighbors(self._h, v, _ptr(dst), _ptr(ts), cnt.value, C.byref(cnt)))
        return dst, ts

    def decode_all(self):
        off = np.zeros(self.n + 1, np.int64)
        _check(_lib.tga_decode_all(self._h, _ptr(off), None, None, 0))
        m = int(off[-1])
        dst = np.zeros(max(m, 1), np.int32)
        ts = np.zeros(max(m, 1), np.int64)
        _check(_lib.tga_decode_all(self._h, _ptr(off), _ptr(dst), _ptr(ts), m))
        return off, dst[:m], ts[:m]

    def bfs(self, src: int = -1, t_lo: int = 0, t_hi: int = T_MAX, outputs: bool = True):
        if not outputs:
            _check(_lib.tga_bfs(self._h, src, t_lo, t_hi, None, None))
            return None
        arr = np.zeros(self.max_vertex, np.int32)
        hops = np.zeros(self.max_vertex, np.int32)
        _check(_lib.tga_bfs(self._h, src, t_lo, t_hi, _ptr(arr), _ptr(hops)))
        return arr, hops

    def connected_components(self, t_lo: int = 0, t_hi: int = T_MAX, early_exit: bool = True, outputs: bool = True,
                             one_seed: bool = False):
        """Labels by temporal reach (tga_cc).  Seeds run as validated batches of a multi-source
        traversal; one_seed=True runs one seed per traversal (same labels)."""
        comps = C.c_int32()
        lab = np.zeros(self.max_vertex, np.int32) if outputs else None
        flags = (CC_EARLY_EXIT if early_exit else 0) | (CC_ONE_SEED if one_seed else 0)
        _check(_lib.tga_cc(self._h, t_lo, t_hi, flags, _ptr(lab), C.byref(comps)))
        return lab, comps.value

    def pagerank(self, iters: int = 0, damping: float = 0.85, alpha: float = 0.1, t_lo: int = 0, t_hi: int = T_MAX,
                 outputs: bool = True):
        out = np.zeros(self.max_vertex, np.float32) if outputs else None
        _check(_lib.tga_pagerank(self._h, iters, damping, alpha, t_lo, t_hi, _ptr(out)))
        return out

    def hits(self, iters: int = 0, mode: int = HITS_GPU, t_lo: int = 0, t_hi: int = T_MAX, outputs: bool = True):
        hub = np.zeros(self.max_vertex, np.float32) if outputs else None
        auth = np.zeros(self.max_vertex, np.float32) if outputs else None
        _check(_lib.tga_hits(self._h, iters, mode, t_lo, t_hi, _ptr(hub), _ptr(auth)))
        return hub, auth

    def degree_centrality(self, t_start: int = 0, t_end: int = 0, outputs: bool = True):
        deg = np.zeros(self.max_vertex, np.int32) if outputs else None
        avg = np.zeros(self.max_vertex, np.int64) if outputs else None
        _check(_lib.tga_degree(self._h, t_start, t_end, _ptr(deg), _ptr(avg)))
        return deg, avg

    def color(self, prio_mode: int = 0, prio: np.ndarray | None = None, java_isolated: bool = False,
              outputs: bool = True):
        col = np.zeros(self.max_vertex, np.uint32) if outputs else None
        pout = np.zeros(self.max_vertex, np.uint32) if outputs else None
        rounds = C.c_int32()
        pin = None if prio is None else np.ascontiguousarray(prio, np.uint32)
        _check(_lib.tga_color(self._h, prio_mode, _ptr(pin), GC_JAVA_ISOLATED if java_isolated else 0, _ptr(col),
                              _ptr(pout), C.byref(rounds)))
        return col, pout, rounds.value

    def bfs_batch(self, sources, t_lo, t_hi):
        src = np.ascontiguousarray(sources, np.int32)
        lo = np.ascontiguousarray(t_lo, np.int64)
        hi = np.ascontiguousarray(t_hi, np.int64)
        out = np.zeros((len(src), self.max_vertex), np.int32)
        _check(_lib.tga_bfs_batch(self._h, len(src), _ptr(src), _ptr(lo), _ptr(hi), _ptr(out)))
        return out

    def shortest(self, src: int, t_lo: int = 0, t_hi: int = T_MAX):
        """Fewest-hop temporal paths from src (tga_shortest): (hops, earliest arrival)."""
        hops = np.zeros(self.max_vertex, np.int32)
        arr = np.zeros(self.max_vertex, np.int32)
        _check(_lib.tga_shortest(self._h, src, t_lo, t_hi, _ptr(hops), _ptr(arr)))
        return hops, arr

    def fastest(self, src: int, t_lo: int = 0, t_hi: int = T_MAX):
        """Fastest temporal paths from src (tga_fastest): (duration, departure) per vertex, -1 where
        unreachable; the source has duration 0 and departure -1."""
        dur = np.zeros(self.max_vertex, np.int64)
        dep = np.zeros(self.max_vertex, np.int64)
        _check(_lib.tga_fastest(self._h, src, t_lo, t_hi, _ptr(dur), _ptr(dep)))
        return dur, dep

    def reverse(self, directory: str | os.PathLike, basename: str, pivot: int = -1) -> int:
        """Writes the time-reversed copy (edge x->y at t becomes y->x at pivot - t) to
        <directory>/<basename>.* (tga_reverse); returns the pivot (the largest timestamp when -1)."""
        out = C.c_int64()
        _check(_lib.tga_reverse(self._h, pivot, str(directory).encode(), basename.encode(), C.byref(out)))
        return out.value

    def latest_departure(self, pivot: int, target: int, t_lo: int = 0, t_hi: int = T_MAX) -> np.ndarray:
        """On a reversed copy: the latest time each vertex can leave on a path to target inside
        [t_lo, t_hi), -1 when none (tga_latest_departure)."""
        out = np.zeros(self.max_vertex, np.int64)
        _check(_lib.tga_latest_departure(self._h, pivot, target, t_lo, t_hi, _ptr(out)))
        return out

    def is_neighbor(self, node, neighbor, t_from=None, t_to=None):
        """Windowed point queries (tga_is_neighbor): True where some edge node->neighbor has a
        timestamp in [t_from, t_to] (inclusive); no bounds when t_from/t_to are None."""
        x = np.ascontiguousarray(node, np.int32)
        y = np.ascontiguousarray(neighbor, np.int32)
        lo = None if t_from is None else np.ascontiguousarray(np.broadcast_to(t_from, x.shape), np.int64)
        hi = None if t_to is None else np.ascontiguousarray(np.broadcast_to(t_to, x.shape), np.int64)
        out = np.zeros(len(x), np.uint8)
        _check(_lib.tga_is_neighbor(self._h, len(x), _ptr(x), _ptr(y), _ptr(lo), _ptr(hi), _ptr(out)))
        return out.astype(bool)

    def cc_batch(self, t_lo, t_hi, early_exit: bool = True):
        """Connected components of many windows in one launch (tga_cc_batch): labels [n, max_vertex]
        and component counts [n], each row equal to connected_components for that window."""
        lo = np.ascontiguousarray(t_lo, np.int64)
        hi = np.ascontiguousarray(t_hi, np.int64)
        lab = np.zeros((len(lo), self.max_vertex), np.int32)
        comps = np.zeros(len(lo), np.int32)
        _check(_lib.tga_cc_batch(self._h, len(lo), _ptr(lo), _ptr(hi), CC_EARLY_EXIT if early_exit else 0, _ptr(lab),
                                 _ptr(comps)))
        return lab, comps

    def pagerank_batch(self, t_lo, t_hi, iters=20, damping: float = 0.85, alpha: float = 0.1):
        """Windowed PageRanks as one strided vector; iters is one count for all or one per query."""
        lo = np.ascontiguousarray(t_lo, np.int64)
        hi = np.ascontiguousarray(t_hi, np.int64)
        out = np.zeros((len(lo), self.max_vertex), np.float32)
        if np.ndim(iters) == 0:
            _check(_lib.tga_pagerank_batch(self._h, len(lo), int(iters), damping, alpha, _ptr(lo), _ptr(hi), _ptr(out)))
        else:
            it = np.ascontiguousarray(iters, np.int32)
            _check(_lib.tga_pagerank_batch_iters(self._h, len(lo), _ptr(it), damping, alpha, _ptr(lo), _ptr(hi),
                                                 _ptr(out)))
        return out


# ---- served form -------------------------------------------------------------------------------

Q_BFS, Q_PAGERANK, Q_CC, Q_NEIGHBOR = 0, 1, 2, 3


class CcJob:
    """Resumable connected components over several windows (tga_cc_job_*): add windows, step with a
    device-time budget, take finished windows; each window's result equals connected_components."""

    def __init__(self, graph: "Graph", capacity: int = 32, early_exit: bool = True):
        self.graph = graph
        h = C.c_void_p()
        _check(_lib.tga_cc_job_create(graph.handle, capacity, CC_EARLY_EXIT if early_exit else 0, C.byref(h)))
        self._h = h

    def add(self, t_lo: int, t_hi: int) -> int:
        slot = C.c_int32()
        _check(_lib.tga_cc_job_add(self._h, t_lo, t_hi, C.byref(slot)))
        return slot.value

    def step(self, budget_ms: float = 0.0) -> list:
        """Runs batches for about budget_ms (<= 0: to the end); returns the finished slots."""
        fin = C.c_uint32()
        _check(_lib.tga_cc_job_step(self._h, budget_ms, C.byref(fin)))
        return [s for s in range(32) if fin.value >> s & 1]

    def take(self, slot: int):
        lab = np.zeros(self.graph.max_vertex, np.int32)
        k = C.c_int32()
        _check(_lib.tga_cc_job_take(self._h, slot, _ptr(lab), C.byref(k)))
        return lab, k.value

    def close(self):
        if self._h:
            _check(_lib.tga_cc_job_destroy(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Server:
    """Request loop over resident graphs (tga_server_*): submit queries, poll or drain, read the
    latency statistics.  Result arrays are owned here until the query finished."""

    def __init__(self, budget_bytes: int):
        h = C.c_void_p()
        _check(_lib.tga_server_create(int(budget_bytes), C.byref(h)))
        self._h = h
        self._graphs: list[Graph] = []
        self._keep: dict[int, np.ndarray] = {}

    def add_graph(self, g: Graph) -> int:
        gid = C.c_int32()
        _check(_lib.tga_server_add_graph(self._h, g.handle, C.byref(gid)))
        self._graphs.append(g)
        return gid.value

    def submit(self, kind: int, graph: int, src: int = 0, t_lo: int = 0, t_hi: int = T_MAX, iters: int = 0,
               dst: int = 0) -> int:
        nv = self._graphs[graph].max_vertex
        if kind == Q_NEIGHBOR:
            out = np.zeros(1, np.uint8)
        else:
            out = np.zeros(nv, np.float32 if kind == Q_PAGERANK else np.int32)
        q = _Query(kind, graph, src, iters, dst, 0, t_lo, t_hi, out.ctypes.data)
        ticket = C.c_int64()
        _check(_lib.tga_submit(self._h, C.byref(q), C.byref(ticket)))
        self._keep[ticket.value] = out
        return ticket.value

    def poll(self, ticket: int):
        """None while pending; (result array, latency ms) when done."""
        lat = C.c_double()
        rc = _lib.tga_poll(self._h, ticket, C.byref(lat))
        if rc == TGA_E_AGAIN:
            return None
        _check(rc)
        return self._keep[ticket], lat.value

    def drain(self) -> None:
        _check(_lib.tga_server_drain(self._h))

    def stats(self) -> dict:
        st = _ServerStats()
        _check(_lib.tga_server_get_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in _ServerStats._fields_}

    def close(self) -> None:
        if self._h:
            _lib.tga_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---- format layer -----------------------------------------------------------------------------

@dataclass
class GenParams:
    n: int = 10_000
    m: int = 200_000
    deg_exponent: float = 2.1
    max_degree: int = 1 << 20
    repeat_frac: float = 0.30
    local_frac: float = 0.60
    local_radius: int = 32
    pref_frac: float = 0.0
    copy_frac: float = 0.0
    ts_kind: int = 0
    ts_span: int = 1_000_000
    min_timestamp: int = 0
    seed: int = 1
    ref_safe: bool = False
    hub_count: int = 0       # this many vertices get exactly hub_degree out-edges each
    hub_degree: int = 0


# Synthetic stand-ins for the benchmark configurations (the real datasets are absent).
CONFIGS = {
    "small": GenParams(n=10_000, m=200_000, deg_exponent=2.1, repeat_frac=0.30, local_frac=0.60, local_radius=32,
                       ts_kind=0, ts_span=1_000_000, seed=1),
    "all7": GenParams(n=2_000_000, m=40_000_000, deg_exponent=2.0, max_degree=100_000, repeat_frac=0.30,
                      local_frac=0.70, local_radius=64, pref_frac=0.5, copy_frac=0.20, ts_kind=1,
                      ts_span=100_000_000, seed=2),
    "batched": GenParams(n=20_000_000, m=500_000_000, deg_exponent=1.9, max_degree=1_000_000, repeat_frac=0.30,
                         local_frac=0.70, local_radius=64, pref_frac=0.5, copy_frac=0.20, ts_kind=1,
                         ts_span=100_000_000, seed=3),
    # Served-form resident graph of 1M vertices / 20M temporal edges (same generator).
    "served1m": GenParams(n=1_000_000, m=20_000_000, deg_exponent=2.0, max_degree=50_000, repeat_frac=0.30,
                          local_frac=0.70, local_radius=64, pref_frac=0.5, copy_frac=0.20, ts_kind=1,
                          ts_span=100_000_000, seed=4),
    # Served-form resident graph of 10M vertices / 200M temporal edges.
    "served10m": GenParams(n=10_000_000, m=200_000_000, deg_exponent=2.0, max_degree=200_000, repeat_frac=0.30,
                           local_frac=0.70, local_radius=64, pref_frac=0.5, copy_frac=0.20, ts_kind=1,
                           ts_span=100_000_000, seed=4),
    # Served-form resident graph of 50M vertices / 1B temporal edges.
    "served50m": GenParams(n=50_000_000, m=1_000_000_000, deg_exponent=2.0, max_degree=1_000_000, repeat_frac=0.30,
                           local_frac=0.70, local_radius=64, pref_frac=0.5, copy_frac=0.20, ts_kind=1,
                           ts_span=100_000_000, seed=4),
    # Skew stress: Zipf 1.6 out-degrees plus 16 hubs of 5M out-edges each (block-scale lists), bursty
    # timestamps (10% of the edges in 1% of the span).
    "skew": GenParams(n=100_000_000, m=2_000_000_000, deg_exponent=1.6, max_degree=5_000_000, repeat_frac=0.30,
                      local_frac=0.70, local_radius=64, pref_frac=0.5, copy_frac=0.20, ts_kind=2,
                      ts_span=100_000_000, seed=5, hub_count=16, hub_degree=5_000_000),
}


def generate(params: GenParams, directory: str | os.PathLike, basename: str, raw_path: str | None = None) -> dict:
    p = _GenParams()
    for k, _ in _GenParams._fields_:
        setattr(p, k, int(getattr(params, k)) if k == "ref_safe" else getattr(params, k))
    s = _GenSummary()
    Path(directory).mkdir(parents=True, exist_ok=True)
    _check(_lib.tga_generate(C.byref(p), str(directory).encode(), basename.encode(),
                             raw_path.encode() if raw_path else None, C.byref(s)))
    return {k: getattr(s, k) for k, _ in _GenSummary._fields_}


def encode_raw(raw_path: str | os.PathLike, directory: str | os.PathLike, basename: str, max_label: int = -1) -> dict:
    s = _GenSummary()
    _check(_lib.tga_encode_raw(str(raw_path).encode(), str(directory).encode(), basename.encode(), max_label,
                               C.byref(s)))
    return {k: getattr(s, k) for k, _ in _GenSummary._fields_}


def write_reversed(offsets, dst, ts, pivot: int, directory: str | os.PathLike, basename: str) -> dict:
    """Writes the time-reversed graph of a CSR as a dataset (tga_write_reversed, host only)."""
    off = np.ascontiguousarray(offsets, np.int64)
    d = np.ascontiguousarray(dst, np.int32)
    t = np.ascontiguousarray(ts, np.int64)
    s = _GenSummary()
    _check(_lib.tga_write_reversed(_ptr(off), _ptr(d), _ptr(t), len(off) - 1, pivot, str(directory).encode(),
                                   basename.encode(), C.byref(s)))
    return {k: getattr(s, k) for k, _ in _GenSummary._fields_}


def reference_depths(directory: str | os.PathLike, basename: str):
    """Realised reference-chain depth of every list (tga_reference_depths, host only): returns the
    summary (nodes, referenced_nodes, truncated_nodes, maximum_depth, configured_max_ref_count,
    depth_counts) and the per-list depths."""
    r = _RefDepths()
    _check(_lib.tga_reference_depths(str(directory).encode(), basename.encode(), C.byref(r), None))
    depth = np.zeros(r.nodes, np.int32)
    _check(_lib.tga_reference_depths(str(directory).encode(), basename.encode(), C.byref(r), _ptr(depth)))
    summary = {k: getattr(r, k) for k, _ in _RefDepths._fields_ if k != "depth_counts"}
    summary["depth_counts"] = list(r.depth_counts)
    return summary, depth


def build_index(directory: str | os.PathLike, basename: str, max_label: int, device: bool = False) -> None:
    """Writes the four GPU index files of a directory that has <base>.offsets (tga_build_index;
    with device=True the walks run on the GPU, tga_build_index_device)."""
    fn = _lib.tga_build_index_device if device else _lib.tga_build_index
    _check(fn(str(directory).encode(), basename.encode(), max_label))


def barrier_selftest(limit_ms: float = 200.0) -> bool:
    """Makes a grid-barrier wait run out on the device (tga_barrier_selftest); True if it ended with
    the timeout status."""
    st = C.c_int32()
    _check(_lib.tga_barrier_selftest(limit_ms, C.byref(st)))
    return st.value == 1


def decode_table(kind: int) -> np.ndarray:
    out = np.zeros(65536, np.int32)
    _check(_lib.tga_decode_table(kind, _ptr(out)))
    return out


CODE_GAMMA, CODE_ZETA, CODE_UNARY, CODE_LONG64 = 0, 1, 2, 3


def encode_codes(kind: int, values, k: int = 0) -> tuple[bytes, int]:
    """Bit-packs values with one instantaneous code (see tga_encode_codes)."""
    v = np.ascontiguousarray(values, np.uint64)
    nbits = C.c_int64()
    _check(_lib.tga_encode_codes(kind, k, _ptr(v), len(v), None, 0, C.byref(nbits)))
    out = np.zeros((nbits.value + 7) // 8 + 1, np.uint8)
    _check(_lib.tga_encode_codes(kind, k, _ptr(v), len(v), _ptr(out), len(out), C.byref(nbits)))
    return out[: (nbits.value + 7) // 8].tobytes(), nbits.value


def ef_encode(values, l: int) -> tuple[bytes, bytes]:
    """Elias-Fano index in the GPU file layout (see tga_ef_encode)."""
    v = np.ascontiguousarray(values, np.uint64)
    lb, ub = C.c_int64(), C.c_int64()
    _check(_lib.tga_ef_encode(_ptr(v), len(v), l, None, 0, None, 0, C.byref(lb), C.byref(ub)))
    lo = np.zeros(max(lb.value, 1), np.uint8)
    up = np.zeros(max(ub.value, 1), np.uint8)
    _check(_lib.tga_ef_encode(_ptr(v), len(v), l, _ptr(lo), len(lo), _ptr(up), len(up), C.byref(lb), C.byref(ub)))
    return lo[: lb.value].tobytes(), up[: ub.value].tobytes()


def config_for(summary: dict, name: str = "synthetic", **kw) -> DatasetConfig:
    """Dataset configuration for a generated graph: MAX_LABEL = n-1, MAX_Vertex = n."""
    n = int(summary["n"])
    return DatasetConfig(name=name, max_label=n - 1, max_vertex=n, **kw)
