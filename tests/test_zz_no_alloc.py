"""The allocation-free query entry point against the ordinary one.

gahhg_query_device_noalloc exists for callers that cannot allocate device
memory while they query: an application whose allocator owns the whole
device, a serving loop that reserves all of its memory before taking
requests, or code that cannot afford the implicit synchronisation of
cudaMalloc/cudaFree.  It uses a fixed array in device memory instead of
scratch from the library's pool, so its labels must be exactly those of
gahhg_query_device.  Two calls in a row check that the shared array's
leftover contents from one call do not leak into the next.

This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

import gahhg_b200 as G
from gahhg_b200 import _lib, synth

pytestmark = pytest.mark.gpu


def _grid(tmp_path):
    rings = synth.c0_polygon(seed=3)
    path = str(tmp_path / "c0_noalloc.txt")
    synth.write_polygon(path, rings)
    return rings, G.Grid(G.Polygon.from_file(path), semantics=G.SEMANTICS_EXACT).classify()


@pytest.mark.parametrize("precision", [G.QUERY_FP32_FILTER, G.QUERY_FP64_FILTER])
def test_noalloc_matches_query_device_twice(tmp_path, precision):
    import torch
    rings, grid = _grid(tmp_path)
    L = _lib.lib()
    rng = np.random.default_rng(21)
    pts = np.concatenate([synth.uniform_points(700_000, rng), synth.near_edge_points(rings, 300_000, rng)])
    n = len(pts)
    assert n <= L.gahhg_query_noalloc_max_points()
    d_pts = torch.from_numpy(pts).cuda()
    want = torch.zeros(n, dtype=torch.uint8, device="cuda")
    grid.query_device(d_pts.data_ptr(), n, want.data_ptr(), precision, stream=0, sync=True)
    torch.cuda.synchronize()
    assert int((want == 0).sum()) == 0  # every label decided
    for call in range(2):
        got = torch.full((n,), 255, dtype=torch.uint8, device="cuda")
        st = L.gahhg_query_device_noalloc(grid._h, ctypes.c_void_p(d_pts.data_ptr()), n,
                                          ctypes.c_void_p(got.data_ptr()), precision, None)
        assert st == 0, L.gahhg_last_error()
        torch.cuda.synchronize()
        # integer labels: the tolerance is exact equality
        assert torch.equal(got, want), "call %d: %d labels differ" % (call, int((got != want).sum()))


def test_noalloc_rejects_oversize_and_reference_grids(tmp_path):
    import torch
    rings, grid = _grid(tmp_path)
    L = _lib.lib()
    cap = L.gahhg_query_noalloc_max_points()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    lab = torch.zeros(8, dtype=torch.uint8, device="cuda")
    # refused before any device work, so the small buffers are never touched
    st = L.gahhg_query_device_noalloc(grid._h, ctypes.c_void_p(buf.data_ptr()), cap + 1,
                                      ctypes.c_void_p(lab.data_ptr()), G.QUERY_FP32_FILTER, None)
    assert st == _lib.ERR_CAPACITY
    assert b"exceed" in L.gahhg_last_error()
    gref = G.Grid(grid.polygon, semantics=G.SEMANTICS_REFERENCE).classify()
    st = L.gahhg_query_device_noalloc(gref._h, ctypes.c_void_p(buf.data_ptr()), 8,
                                      ctypes.c_void_p(lab.data_ptr()), G.QUERY_AUTO, None)
    assert st == _lib.ERR_STATE
