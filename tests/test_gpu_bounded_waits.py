"""The bounded waits and loops of the kernels, made to run out (knobs of
gahhg_set_knob lowered), on the GPU, without a fault:

  walk step limit      every edge walk of the hierarchy stops after one cell:
                       the build completes, counts the walks (walk_limit_hits)
                       and still answers reference-precision queries; an
                       exact grid's labels do not depend on the hierarchy and
                       stay equal to the exact oracle's;
  scan look-back       every build scan's look-back gives up at once on a late
                       tile and sums that tile's inputs itself: the grids are
                       bit-identical to a normal build's (scan_fallbacks
                       counts the events);
  summary staging      every pass-1 block gives up at once on the bulk copy of
                       the coarse summary and reads it from global memory: the
                       labels are unchanged and gahhg_staging_fallbacks counts
                       the blocks (single polygons and batches);
  edge-list staging    every tier-1 block over a leaf-ordered queue (pass-2
                       order 3) gives up at once on the bulk copy of its
                       tile's leaf and edge records and reads them from global
                       memory: the labels and tier counts are unchanged and
                       the blocks are counted on top of the pass-1 ones.

Each knob is put back to its default whatever the outcome.  The reference's
walks are unbounded (source/GPISPAHHG.cu:736,872,1210); its scan and staging
have no counterpart.
"""
import contextlib

import numpy as np
import pytest

import gahhg_b200 as G
from gahhg_b200 import synth
from oracle import exact

pytestmark = pytest.mark.gpu


@contextlib.contextmanager
def knob(k, v):
    old = G.set_knob(k, v)
    try:
        yield
    finally:
        G.set_knob(k, old)


def test_walk_step_limit_runs_out(inputs, tmp_path):
    path = inputs.polygon_file("various/NA0.txt", tmp_path)
    P = G.Polygon.from_file(path)
    q = inputs.query("uniform")
    g0 = G.Grid(P, semantics=G.SEMANTICS_REFERENCE, device=0).classify()
    assert g0.stats()["walk_limit_hits"] == 0
    with knob(G.KNOB_WALK_STEP_LIMIT, 1):
        gr = G.Grid(P, semantics=G.SEMANTICS_REFERENCE, device=0).classify()
        g = G.Grid(P, semantics=G.SEMANTICS_EXACT, device=0).classify()
        assert g.depth > 0  # the exact grid's hierarchy, built now, under the same limit
    assert gr.stats()["walk_limit_hits"] > 0 and g.stats()["walk_limit_hits"] > 0
    assert set(np.unique(gr.query(q, G.QUERY_REFERENCE_FP64))) <= {0, 1, 2}
    xyz, pe = P.export()
    want = exact.ExactPolygon(xyz, pe, len(inputs.rings_deg("various/NA0.txt")[0])).query_lonlat(q)
    assert np.array_equal(g.query(q, G.QUERY_FP32_FILTER), want)


def test_scan_lookback_runs_out():
    rng = np.random.default_rng(5)
    rings = [synth.star_ring(-40.0, 10.0, 200_000, 25.0, 0.2, rng), synth.star_ring(-40.0, 10.0, 5_000, 4.0, 0.0, rng)]
    P = G.Polygon.from_rings(rings)
    normal = G.Grid(P, semantics=G.SEMANTICS_REFERENCE, device=0).classify()
    with knob(G.KNOB_SCAN_SPIN_LIMIT, 0):
        late = G.Grid(P, semantics=G.SEMANTICS_REFERENCE, device=0).classify()
        late_exact = G.Grid(P, semantics=G.SEMANTICS_EXACT, device=0).classify()
    assert late.stats()["scan_fallbacks"] + late_exact.stats()["scan_fallbacks"] > 0
    assert normal.stats()["scan_fallbacks"] == 0
    for a, b in zip(normal.export(), late.export()):
        assert np.array_equal(a, b)
    q = synth.uniform_points(200_000, rng)
    ex = G.Grid(P, semantics=G.SEMANTICS_EXACT, device=0).classify()
    assert np.array_equal(late_exact.query(q, G.QUERY_FP32_FILTER), ex.query(q, G.QUERY_FP32_FILTER))
    assert np.array_equal(late.query(q, G.QUERY_REFERENCE_FP64), normal.query(q, G.QUERY_REFERENCE_FP64))


def test_summary_staging_runs_out():
    import torch
    rng = np.random.default_rng(6)
    polys = synth.c3_polygons(16, seed=9, vmax=5000)
    P = [G.Polygon.from_rings(r) for r, _c, _r in polys]
    pts = synth.c3_points(polys, seed=10, pmax=5000)
    g = G.Grid(P[0], semantics=G.SEMANTICS_EXACT, device=0).classify()
    q = np.concatenate([pts[0], synth.uniform_points(50_000, rng)])
    want = g.query(q, G.QUERY_FP32_FILTER)
    B = G.Batch(P)
    off = np.zeros(len(pts) + 1, dtype=np.int64)
    off[1:] = np.cumsum([len(p) for p in pts])
    d_pts = torch.from_numpy(np.concatenate(pts)).cuda()
    lab = torch.zeros(len(d_pts), dtype=torch.uint8, device="cuda")
    B.query_device(d_pts.data_ptr(), off, lab.data_ptr(), G.QUERY_FP32_FILTER, sync=True)
    want_b = lab.cpu().numpy()
    before = G.staging_fallbacks(0)
    with knob(G.KNOB_STAGING_POLL_LIMIT, 0):
        got = g.query(q, G.QUERY_FP32_FILTER)
        mid = G.staging_fallbacks(0)
        lab.zero_()
        B.query_device(d_pts.data_ptr(), off, lab.data_ptr(), G.QUERY_FP32_FILTER, sync=True)
    after = G.staging_fallbacks(0)
    assert np.array_equal(got, want)
    assert np.array_equal(lab.cpu().numpy(), want_b)
    assert mid > before and after > mid


def test_edge_list_staging_runs_out():
    import torch
    # a C1-style polygon a tenth the size, so that a tile of the leaf-ordered
    # queue of 1e6 C2 points spans few enough leaves to be staged
    rings = synth.c1_polygon(n_outer=100_000, hole_n=1_000)
    g = G.Grid(G.Polygon.from_rings(rings), semantics=G.SEMANTICS_EXACT, device=0).classify()
    d = synth.device_c2_points(rings, 1_000_000, 17, "cuda:0")
    lab = torch.empty(d.shape[0], dtype=torch.uint8, device="cuda")

    def run(order):
        with knob(G.KNOB_GROUPED_PASS2, order):
            lab.fill_(9)
            before = G.staging_fallbacks(0)
            g.query_device(d.data_ptr(), d.shape[0], lab.data_ptr(), G.QUERY_FP32_FILTER, sync=True)
            return lab.cpu().numpy(), g.stats(), G.staging_fallbacks(0) - before

    want, sw, f0 = run(0)
    assert f0 == 0
    got, sg, f3 = run(3)
    assert f3 == 0 and np.array_equal(got, want)
    with knob(G.KNOB_STAGING_POLL_LIMIT, 0):
        _, _, f2 = run(2)       # pass-1 blocks only
        late, sl, f3 = run(3)   # and the staging tier-1 blocks
    assert np.array_equal(late, want)
    for k in ("boundary_points", "esc_fp64", "esc_exact", "in_count"):
        assert sl[k] == sw[k] == sg[k], k
    assert f2 > 0 and f3 > f2
