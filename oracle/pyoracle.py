"""ctypes wrapper of the CPU oracle (oracle.c).  TEST INFRASTRUCTURE ONLY: imported by tests/,
__graft_entry__.smoke() and the CPU-baseline leg of bench.py, never by the product package."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"


def build() -> Path:
    src = HERE / "oracle.c"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "-s"], check=True)
    return LIB


def _load() -> C.CDLL:
    build()
    lib = C.CDLL(str(LIB))
    P = C.c_void_p
    i32, i64, f64 = C.c_int32, C.c_int64, C.c_double
    sig = {
        "orc_open": (P, [C.c_char_p, C.c_char_p, i64, C.c_int]),
        "orc_close": (None, [P]),
        "orc_error": (C.c_int, [P]),
        "orc_min_ts": (i64, [P]),
        "orc_graph_offset": (i64, [P, i64]),
        "orc_ts_offset": (i64, [P, i64]),
        "orc_outdegree": (i32, [P, i64]),
        "orc_outdegrees": (None, [P, P]),
        "orc_neighbors": (i64, [P, i64, P, P, i64]),
        "orc_materialize": (i64, [P]),
        "orc_csr": (None, [P, P, P, P]),
        "orc_checksums": (None, [P, i64, i64, P, P]),
        "orc_bfs": (None, [P, i32, i32, i32, i32, i64, i64, P, P]),
        "orc_cc": (i32, [P, i32, i32, i32, i32, i64, i64, i32, P]),
        "orc_pagerank": (None, [P, i32, i32, i32, i32, f64, f64, i64, i64, P]),
        "orc_hits": (None, [P, i32, i32, i32, i32, i32, i64, i64, P, P]),
        "orc_degree": (None, [P, i32, i32, i32, i64, i64, P, P]),
        "orc_color": (i32, [P, i32, i32, i32, P, i32, P]),
        "orc_java_random256": (None, [i64, i32, P]),
        "orc_stream_pagerank": (i64, [P, i32, i32, i32, i32, f64, f64, P, i32]),
        "orc_stream_decode": (i64, [P, i64, i64, P, i32]),
        "orc_stream_bfs": (i64, [P, i32, i32, i32, i32, i64, i64, P, P]),
        "orc_stream_cc": (i64, [P, i32, i32, i32, i32, i64, i64, i32, P, P]),
        "orc_stream_hits": (i64, [P, i32, i32, i32, i32, i32, P, P, i32]),
        "orc_stream_degree": (i64, [P, i32, i32, i32, i64, i64, P, P, i32]),
        "orc_stream_color": (i64, [P, i32, i32, i32, P, i32, P, P, i32]),
        "orc_shortest": (None, [P, i32, i32, i32, i32, i64, i64, P, P]),
        "orc_max_threads": (i32, []),
        "orc_read_codes": (i64, [P, i64, i32, i32, P, i64]),
        "orc_ef_get": (C.c_uint64, [P, P, i64, i32, i64]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_lib = None
_max_threads = 1


def lib() -> C.CDLL:
    global _lib, _max_threads
    if _lib is None:
        _lib = _load()
        # Read before any call sets a thread count: OpenMP keeps the last one set.
        _max_threads = _lib.orc_max_threads()
    return _lib


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


INT64_MIN, INT64_MAX = -(1 << 63), (1 << 63) - 1


class Oracle:
    """Decoded view of one dataset from the CPU restatement (uses .offsets, not the EF files)."""

    def __init__(self, directory, basename: str, n: int, min_interval: int = 4, materialize: bool = True):
        self.L = lib()
        self.h = self.L.orc_open(str(directory).encode(), basename.encode(), n, min_interval)
        if not self.h:
            raise FileNotFoundError(f"oracle cannot open {directory}/{basename}")
        self.n = n
        self.m = self.L.orc_materialize(self.h) if materialize else None
        if self.L.orc_error(self.h):
            raise ValueError("oracle decode error")

    def close(self):
        if self.h:
            self.L.orc_close(self.h)
            self.h = None

    def __del__(self):
        self.close()

    @property
    def min_ts(self) -> int:
        return self.L.orc_min_ts(self.h)

    def outdegrees(self) -> np.ndarray:
        out = np.zeros(self.n, np.int32)
        self.L.orc_outdegrees(self.h, _p(out))
        return out

    def graph_offsets(self) -> np.ndarray:
        return np.array([self.L.orc_graph_offset(self.h, v) for v in range(self.n + 1)], np.int64)

    def ts_offsets(self) -> np.ndarray:
        return np.array([self.L.orc_ts_offset(self.h, v) for v in range(self.n + 1)], np.int64)

    def csr(self):
        off = np.zeros(self.n + 1, np.int64)
        dst = np.zeros(max(self.m, 1), np.int32)
        ts = np.zeros(max(self.m, 1), np.int64)
        self.L.orc_csr(self.h, _p(off), _p(dst), _p(ts))
        return off, dst[: self.m], ts[: self.m]

    def neighbors(self, v: int):
        d = self.L.orc_outdegree(self.h, v)
        dst = np.zeros(max(d, 1), np.int32)
        ts = np.zeros(max(d, 1), np.int64)
        k = self.L.orc_neighbors(self.h, v, _p(dst), _p(ts), d)
        return dst[:k], ts[:k]

    def checksums(self, begin: int, end: int, max_vertex: int):
        cs = np.zeros(max_vertex, np.uint64)
        small = np.zeros(max_vertex, np.uint8)
        self.L.orc_checksums(self.h, begin, end, _p(cs), _p(small))
        return small, cs

    def bfs(self, max_label, max_vertex, active, src, lo=0, hi=INT64_MAX):
        arr = np.zeros(max_vertex, np.int32)
        hops = np.zeros(max_vertex, np.int32)
        self.L.orc_bfs(self.h, max_label, max_vertex, active, src, lo, hi, _p(arr), _p(hops))
        return arr, hops

    def shortest(self, max_label, max_vertex, active, src, lo=0, hi=INT64_MAX):
        """Fewest-hop temporal paths from src: (hops, earliest arrival)."""
        arr = np.zeros(max_vertex, np.int32)
        hops = np.zeros(max_vertex, np.int32)
        self.L.orc_shortest(self.h, max_label, max_vertex, active, src, lo, hi, _p(arr), _p(hops))
        return hops, arr

    def cc(self, max_label, max_vertex, active, begin, lo=0, hi=INT64_MAX, early_exit=True):
        lab = np.zeros(max_vertex, np.int32)
        k = self.L.orc_cc(self.h, max_label, max_vertex, active, begin, lo, hi, int(early_exit), _p(lab))
        return lab, k

    def pagerank(self, max_label, max_vertex, active, iters, d=0.85, alpha=0.1, lo=0, hi=INT64_MAX):
        r = np.zeros(max_vertex, np.float64)
        self.L.orc_pagerank(self.h, max_label, max_vertex, active, iters, d, alpha, lo, hi, _p(r))
        return r

    def hits(self, max_label, max_vertex, active, iters, java=False, lo=0, hi=INT64_MAX):
        hub = np.zeros(max_vertex, np.float64)
        auth = np.zeros(max_vertex, np.float64)
        self.L.orc_hits(self.h, max_label, max_vertex, active, iters, int(java), lo, hi, _p(hub), _p(auth))
        return hub, auth

    def degree(self, max_label, max_vertex, active, s=0, e=0):
        deg = np.zeros(max_vertex, np.int32)
        avg = np.zeros(max_vertex, np.int64)
        self.L.orc_degree(self.h, max_label, max_vertex, active, s, e, _p(deg), _p(avg))
        return deg, avg

    def color(self, max_label, max_vertex, active, prio, java_isolated=False):
        col = np.zeros(max_vertex, np.uint32)
        p = np.ascontiguousarray(prio, np.uint32)
        r = self.L.orc_color(self.h, max_label, max_vertex, active, _p(p), int(java_isolated), _p(col))
        return col, r

    def stream_pagerank(self, max_label, max_vertex, active, iters, threads=0, d=0.85, alpha=0.1):
        r = np.zeros(max_vertex, np.float64)
        e = self.L.orc_stream_pagerank(self.h, max_label, max_vertex, active, iters, d, alpha, _p(r), threads)
        return r, e

    def stream_decode(self, begin, end, threads=0, max_vertex=None):
        cs = np.zeros(max_vertex or self.n, np.uint64)
        e = self.L.orc_stream_decode(self.h, begin, end, _p(cs), threads)
        return cs, e

    # Streaming forms of the remaining workloads (lists decoded at every visit); each returns its
    # result and the number of edges it decoded.

    def stream_bfs(self, max_label, max_vertex, active, src, lo=0, hi=INT64_MAX):
        arr = np.zeros(max_vertex, np.int32)
        hops = np.zeros(max_vertex, np.int32)
        e = self.L.orc_stream_bfs(self.h, max_label, max_vertex, active, src, lo, hi, _p(arr), _p(hops))
        return (arr, hops), e

    def stream_cc(self, max_label, max_vertex, active, begin, lo=0, hi=INT64_MAX, early_exit=True):
        lab = np.zeros(max_vertex, np.int32)
        k = C.c_int32()
        e = self.L.orc_stream_cc(self.h, max_label, max_vertex, active, begin, lo, hi, int(early_exit), _p(lab),
                                 C.byref(k))
        return (lab, k.value), e

    def stream_hits(self, max_label, max_vertex, active, iters, java=False, threads=0):
        hub = np.zeros(max_vertex, np.float64)
        auth = np.zeros(max_vertex, np.float64)
        e = self.L.orc_stream_hits(self.h, max_label, max_vertex, active, iters, int(java), _p(hub), _p(auth), threads)
        return (hub, auth), e

    def stream_degree(self, max_label, max_vertex, active, s=0, e=0, threads=0):
        deg = np.zeros(max_vertex, np.int32)
        avg = np.zeros(max_vertex, np.int64)
        n = self.L.orc_stream_degree(self.h, max_label, max_vertex, active, s, e, _p(deg), _p(avg), threads)
        return (deg, avg), n

    def stream_color(self, max_label, max_vertex, active, prio, java_isolated=False, threads=0):
        col = np.zeros(max_vertex, np.uint32)
        p = np.ascontiguousarray(prio, np.uint32)
        r = C.c_int32()
        e = self.L.orc_stream_color(self.h, max_label, max_vertex, active, _p(p), int(java_isolated), _p(col),
                                    C.byref(r), threads)
        return (col, r.value), e


def java_random256(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.uint32)
    lib().orc_java_random256(seed, n, _p(out))
    return out


def read_codes(data: bytes, kind: int, n: int, k: int = 0) -> tuple[np.ndarray, int]:
    buf = np.frombuffer(bytes(data) + b"\0" * 16, np.uint8)
    out = np.zeros(n, np.uint64)
    used = lib().orc_read_codes(_p(buf), len(data), kind, k, _p(out), n)
    return out, used


def ef_values(lower: bytes, upper: bytes, l: int, count: int) -> np.ndarray:
    lo = np.frombuffer(bytes(lower) + b"\0" * 16, np.uint8)
    up = np.frombuffer(bytes(upper), np.uint8)
    return np.array([lib().orc_ef_get(_p(lo), _p(up), len(upper), l, i) for i in range(count)], np.uint64)


def max_threads() -> int:
    """Threads the oracle's parallel passes use by default (OpenMP's count when the library loaded)."""
    lib()
    return _max_threads
