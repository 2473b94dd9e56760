"""The pass-1 queue put in leaf-window order before the tiers run
(knob GAHHG_KNOB_GROUPED_PASS2 = 1; k_part_count / k_part_scatter: a
counting sort of the queue by window of consecutive leaves, each window
about 24 MB of index records), in leaf order (= 2; k_ls_*: a counting sort
by leaf) or in leaf order with tier 1 reading each tile's leaf and edge
records from shared memory, staged there by bulk copies (= 3; k_leaf_t1s),
against the tiers over the queue in pass-1 order (= 0, the default): the same labels and the same per-tier escalation counts, for both
precisions, on near-edge points of the 1.1M-edge C1 polygon (a long queue:
ordered) and on uniform points and the shipped NA0 polygon (short queues or
one window: pass-1 order kept).  Labels are also checked against the exact
oracle where it is cheap.
Reference boundary loop: source/GPISPAHHG.cu:1481-1501.
"""
import numpy as np
import pytest

import gahhg_b200 as G
from gahhg_b200 import synth
from oracle import exact
from tests.conftest import report

pytestmark = pytest.mark.gpu


def _run(g, d_pts, prec, order):
    import torch
    old = G.set_knob(G.KNOB_GROUPED_PASS2, order)
    try:
        n = d_pts.shape[0]
        lab = torch.full((n,), 9, dtype=torch.uint8, device=d_pts.device)
        g.query_device(d_pts.data_ptr(), n, lab.data_ptr(), prec, sync=True)
        return lab.cpu().numpy(), g.stats()
    finally:
        G.set_knob(G.KNOB_GROUPED_PASS2, old)


@pytest.fixture(scope="module")
def c1_grid():
    rings = synth.c1_polygon()
    P = G.Polygon.from_rings(rings)
    return rings, P, G.Grid(P, semantics=G.SEMANTICS_EXACT, device=0).classify()


ORDERS = {1: "leaf-window", 2: "leaf", 3: "leaf (tier 1 on staged edge lists)"}


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("prec", [G.QUERY_FP32_FILTER, G.QUERY_FP64_FILTER])
def test_grouped_equals_per_point_c2(c1_grid, prec, order):
    rings, _P, g = c1_grid
    pts = synth.device_c2_points(rings, 2_000_000, 7, "cuda:0")
    fallbacks = G.staging_fallbacks(0)
    a, sa = _run(g, pts, prec, order)
    b, sb = _run(g, pts, prec, 0)
    assert np.array_equal(a, b), "%d labels differ" % int((a != b).sum())
    assert set(np.unique(a)) <= {1, 2}
    for k in ("boundary_points", "esc_fp64", "esc_exact", "in_count"):
        assert sa[k] == sb[k], (k, sa[k], sb[k])
    assert G.staging_fallbacks(0) == fallbacks
    report("tiers over the %s-ordered queue == pass-1 order on 2e6 C2 points (%s): boundary %d, FP32->FP64 %d, "
           "FP64->exact %d" % (ORDERS[order], "FP32 filter" if prec == G.QUERY_FP32_FILTER else "FP64 filter",
                               sa["boundary_points"], sa["esc_fp64"], sa["esc_exact"]))


@pytest.mark.parametrize("order", [1, 2, 3])
def test_grouped_equals_per_point_uniform(c1_grid, order):
    _rings, _P, g = c1_grid
    pts = synth.device_points(4_000_000, 11, "cuda:0")
    a, sa = _run(g, pts, G.QUERY_FP32_FILTER, order)
    b, sb = _run(g, pts, G.QUERY_FP32_FILTER, 0)
    assert np.array_equal(a, b)
    assert sa["boundary_points"] == sb["boundary_points"] > 0


def test_grouped_against_oracle_small(inputs, tmp_path):
    import torch
    path = inputs.polygon_file("various/NA0.txt", tmp_path)
    P = G.Polygon.from_file(path)
    xyz, pe = P.export()
    E = exact.ExactPolygon(xyz, pe, len(inputs.rings_deg("various/NA0.txt")[0]))
    g = G.Grid(P, semantics=G.SEMANTICS_EXACT, device=0).classify()
    rng = np.random.default_rng(3)
    rings = inputs.rings_deg("various/NA0.txt")
    q = np.concatenate([inputs.query("uniform"), synth.near_edge_points(rings, 40_000, rng)])
    d = torch.from_numpy(q).cuda()
    want = E.query_lonlat(q)
    for order in (1, 2, 3):
        for prec in (G.QUERY_FP32_FILTER, G.QUERY_FP64_FILTER):
            a, _ = _run(g, d, prec, order)
            assert np.array_equal(a, want), (order, prec)
