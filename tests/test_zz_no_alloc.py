"""tga_pagerank_noalloc through the C ABI: same result as tga_pagerank on two calls in a row, no
change of free device memory across calls once its scratch is set up, and clear rejections
beyond its fixed limits.  Named to be collected last, so it also runs after every other GPU test
in the same process (and passes alone)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

import compresstemporalgraph_b200 as tga

pytestmark = pytest.mark.gpu

MAX_VERTICES = 1 << 20
MAX_ITERS = 1024
PARAMS = tga.GenParams(n=3000, m=60000, deg_exponent=2.3, repeat_frac=0.3, local_frac=0.9, local_radius=3,
                       copy_frac=0.6, ts_kind=0, ts_span=10_000, seed=21)


@pytest.fixture(scope="module")
def data(tmp_path_factory):
    d = tmp_path_factory.mktemp("noalloc")
    s = tga.generate(PARAMS, d, "na")
    return d, s["n"]


def _open(data, **kw):
    d, n = data
    cfg = dict(name="na", max_label=n - 1, max_vertex=n)
    cfg.update(kw)
    return tga.Graph.open_dir(d, "na", tga.DatasetConfig(**cfg))


def _noalloc(g, iters, lo, hi, out_ptr) -> int:
    return tga.lib().tga_pagerank_noalloc(g.handle, iters, C.c_float(0.85), C.c_float(0.1), lo, hi, out_ptr)


def _has_cudart() -> bool:
    try:
        C.CDLL("libcudart.so.12")
        return True
    except OSError:
        return False


def _err() -> str:
    return (tga.lib().tga_last_error() or b"").decode()


@pytest.mark.parametrize("window", ["all", "windowed"])
def test_noalloc_matches_pagerank_on_two_calls(data, window):
    with _open(data) as g:
        lo, hi = (0, tga.T_MAX) if window == "all" else (2_500, 7_500)
        iters = 20
        ref = g.pagerank(iters, 0.85, 0.1, lo, hi)
        assert ref.shape[0] == g.max_vertex
        out = torch.full((g.max_vertex,), -1.0, dtype=torch.float32, device="cuda:0")
        torch.cuda.synchronize()
        for call in range(2):
            out.fill_(-1.0)
            torch.cuda.synchronize()
            assert _noalloc(g, iters, lo, hi, C.c_void_p(out.data_ptr())) == tga.TGA_OK, _err()
            r = out.cpu().numpy()
            # Same tolerance as tga_pagerank against its FP64 oracle: the two runs differ only in
            # the order of FP32 atomic additions.
            assert float(np.abs(r.astype(np.float64) - ref).sum()) <= 1e-5, call
            assert np.allclose(r, ref, rtol=1e-4, atol=1e-9), call
            t = g.timing()
            assert t["iterations"] == iters and t["total_ms"] > 0


def test_noalloc_two_handles_in_turn(data):
    """Two handles on one device share the fixed scratch: calls made one after the other (the
    documented safe use) each give their own window's tga_pagerank result."""
    windows = [(0, tga.T_MAX), (1_000, 6_000)]
    with _open(data) as g1, _open(data) as g2:
        graphs = [g1, g2]
        refs = [g.pagerank(15, 0.85, 0.1, lo, hi) for g, (lo, hi) in zip(graphs, windows)]
        outs = [torch.full((g.max_vertex,), -1.0, dtype=torch.float32, device="cuda:0") for g in graphs]
        torch.cuda.synchronize()
        for _ in range(2):
            for g, (lo, hi), out, ref in zip(graphs, windows, outs, refs):
                assert _noalloc(g, 15, lo, hi, C.c_void_p(out.data_ptr())) == tga.TGA_OK, _err()
                r = out.cpu().numpy()
                assert float(np.abs(r.astype(np.float64) - ref).sum()) <= 1e-5


def test_noalloc_leaves_free_memory_unchanged(data):
    with _open(data) as g:
        g.pagerank(2)  # the handle's own scratch exists before the measurement
        nv = g.max_vertex
        out = torch.empty(nv, dtype=torch.float32, device="cuda:0")
        # First call: scratch set-up, and the first launch of each kernel it uses.
        assert _noalloc(g, 5, 100, 9_000, C.c_void_p(out.data_ptr())) == tga.TGA_OK, _err()
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info(0)
        for _ in range(2):
            assert _noalloc(g, 5, 100, 9_000, C.c_void_p(out.data_ptr())) == tga.TGA_OK, _err()
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info(0)
        assert free1 == free0


def test_noalloc_rejects_beyond_limits(data):
    with _open(data) as g:
        nv = g.max_vertex
        out = torch.empty(nv, dtype=torch.float32, device="cuda:0")
        assert _noalloc(g, MAX_ITERS + 1, 0, tga.T_MAX, C.c_void_p(out.data_ptr())) == tga.TGA_E_ARG
        assert str(MAX_ITERS) in _err()
        host = np.zeros(nv, np.float32)
        assert _noalloc(g, 5, 0, tga.T_MAX, host.ctypes.data_as(C.c_void_p)) == tga.TGA_E_ARG
        assert "device memory" in _err()
        assert _noalloc(g, 5, 0, tga.T_MAX, None) == tga.TGA_E_ARG
        # Managed memory is refused: its device attribute does not say where the pages are.
        managed = C.c_void_p()
        cudart = C.CDLL("libcudart.so.12") if _has_cudart() else None
        if cudart is not None and cudart.cudaMallocManaged(C.byref(managed), C.c_size_t(nv * 4), 1) == 0:
            try:
                assert _noalloc(g, 5, 0, tga.T_MAX, managed) == tga.TGA_E_ARG
                assert "device memory" in _err()
            finally:
                cudart.cudaFree(managed)
    with _open(data, max_vertex=MAX_VERTICES + 1) as g:
        out = torch.empty(MAX_VERTICES + 1, dtype=torch.float32, device="cuda:0")
        assert _noalloc(g, 5, 0, tga.T_MAX, C.c_void_p(out.data_ptr())) == tga.TGA_E_ARG
        assert str(MAX_VERTICES) in _err()
