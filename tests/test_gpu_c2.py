"""C2: the C1 polygon (1.1M edges) queried with points placed within
10^U[-15,-3] rad of its edges, where the FP32 filter must hand tests on to
FP64 and the exact predicate.

Labels must be bit-exact against the brute-force exact oracle on a sample,
equal between the FP32-filtered and FP64-filtered paths on all points, and
the escalations must actually happen (the near-edge points are the cases the
filters exist for).
"""
import numpy as np
import pytest

import gahhg_b200 as G
from gahhg_b200 import synth
from oracle import exact

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1():
    rings = synth.c1_polygon()
    P = G.Polygon.from_rings(rings)
    g = G.Grid(P, semantics=G.SEMANTICS_EXACT).classify()
    return rings, P, g


def _c2_points(rings, n, seed):
    rng = np.random.default_rng(seed)
    return np.concatenate([synth.uniform_points(n // 2, rng), synth.near_edge_points(rings, n - n // 2, rng)])


def test_c2_sample_against_oracle(c1):
    rings, P, g = c1
    pts = _c2_points(rings, 3000, 31)
    xyz, pe = P.export()
    want = exact.ExactPolygon(xyz, pe, len(rings[0])).query_lonlat(pts)
    for prec in (G.QUERY_FP32_FILTER, G.QUERY_FP64_FILTER):
        got = g.query(pts, prec)
        bad = np.nonzero(got != want)[0]
        assert len(bad) == 0, "precision %d: %d of %d labels differ, first %s" % (prec, len(bad), len(pts), bad[:5])


def test_c2_filters_agree_and_escalate(c1):
    import torch
    rings, P, g = c1
    pts = _c2_points(rings, 2_000_000, 32)
    d = torch.from_numpy(pts).cuda()
    lab32 = torch.empty(len(pts), dtype=torch.uint8, device="cuda")
    lab64 = torch.empty_like(lab32)
    g.query_device(d.data_ptr(), len(pts), lab32.data_ptr(), G.QUERY_FP32_FILTER, sync=True)
    st32 = g.stats()
    g.query_device(d.data_ptr(), len(pts), lab64.data_ptr(), G.QUERY_FP64_FILTER, sync=True)
    assert torch.equal(lab32, lab64)
    assert set(torch.unique(lab32).tolist()) <= {1, 2}
    # near-edge points reach the crossing tests, and some of those are too
    # close for the FP32 bound
    assert st32["boundary_points"] > len(pts) // 10
    assert st32["esc_fp64"] > 0
