"""Batches: many polygons built concurrently and queried in one launch.

Every label from the batch query must equal the label the single-polygon
path gives for the same polygon and point (both are exact), including
polygons around a pole, across the antimeridian, with holes, and points far
outside the polygons' domains; CUDA-graph replays must equal direct launches,
also after the points change in place.
"""
import numpy as np
import pytest

import gahhg_b200 as G
from gahhg_b200 import synth
from oracle import exact

pytestmark = pytest.mark.gpu


def _batch_inputs(count=48, seed=5, vmax=20000):
    polys = synth.c3_polygons(count, seed=seed, vmax=vmax)
    # force a few special cases: around the north pole, across the antimeridian
    rng = np.random.default_rng(seed)
    polys[0] = ([synth.star_ring(20.0, 85.0, 300, 12.0, 0.2, rng)], (20.0, 85.0), 12.0)
    polys[1] = ([synth.star_ring(179.5, -10.0, 500, 3.0, 0.2, rng), synth.star_ring(179.5, -10.0, 40, 0.8, 0.0, rng)],
                (179.5, -10.0), 3.0)
    pts = synth.c3_points(polys, seed=seed + 1, pmax=20000)
    # some points anywhere on the sphere
    pts = [np.concatenate([p, synth.uniform_points(200, rng)]) for p in pts]
    return polys, pts


def _layout(pts):
    offsets = np.zeros(len(pts) + 1, dtype=np.int64)
    offsets[1:] = np.cumsum([len(p) for p in pts])
    return np.concatenate(pts), offsets


@pytest.fixture(scope="module")
def batch_case():
    polys, pts = _batch_inputs()
    P = [G.Polygon.from_rings(r) for r, _c, _r in polys]
    return polys, pts, P


def test_batch_equals_single(batch_case):
    import torch
    polys, pts, P = batch_case
    B = G.Batch(P)
    flat, off = _layout(pts)
    d_pts = torch.from_numpy(flat).cuda()
    lab = torch.zeros(len(flat), dtype=torch.uint8, device="cuda")
    for prec in (G.QUERY_FP32_FILTER, G.QUERY_FP64_FILTER):
        lab.zero_()
        B.query_device(d_pts.data_ptr(), off, lab.data_ptr(), prec, sync=True)
        got = lab.cpu().numpy()
        for i, poly in enumerate(P):
            g = G.Grid(poly, semantics=G.SEMANTICS_EXACT).classify()
            want = g.query(pts[i], prec)
            seg = got[off[i]:off[i + 1]]
            assert np.array_equal(seg, want), "polygon %d: %d labels differ" % (i, int((seg != want).sum()))
    st = B.stats()
    assert st["polygons"] == len(P) and st["query_points"] == len(flat)
    assert st["in_count"] == int((got == 2).sum())


def test_batch_against_oracle(batch_case):
    import torch
    polys, pts, P = batch_case
    B = G.Batch(P, chunk_points=1024)
    flat, off = _layout(pts)
    d_pts = torch.from_numpy(flat).cuda()
    lab = torch.zeros(len(flat), dtype=torch.uint8, device="cuda")
    B.query_device(d_pts.data_ptr(), off, lab.data_ptr(), G.QUERY_FP32_FILTER, sync=True)
    got = lab.cpu().numpy()
    for i in (0, 1, 2, 7, 11):
        xyz, pe = P[i].export()
        want = exact.ExactPolygon(xyz, pe, len(polys[i][0][0])).query_lonlat(pts[i])
        assert np.array_equal(got[off[i]:off[i + 1]], want), i


def test_batch_graph_replay(batch_case):
    import torch
    polys, pts, P = batch_case
    B = G.Batch(P)
    flat, off = _layout(pts)
    d_pts = torch.from_numpy(flat).cuda()
    direct = torch.zeros(len(flat), dtype=torch.uint8, device="cuda")
    B.query_device(d_pts.data_ptr(), off, direct.data_ptr(), G.QUERY_FP32_FILTER, sync=True)
    lab = torch.zeros(len(flat), dtype=torch.uint8, device="cuda")
    for _ in range(3):
        lab.fill_(7)
        B.query_device(d_pts.data_ptr(), off, lab.data_ptr(), G.QUERY_FP32_FILTER, graph=True)
        torch.cuda.synchronize()
        assert torch.equal(lab, direct)
    # new points in the same buffers: the graph reads them
    rng = np.random.default_rng(99)
    flat2 = np.concatenate([synth.uniform_points(len(p), rng) for p in pts])
    d_pts.copy_(torch.from_numpy(flat2))
    B.query_device(d_pts.data_ptr(), off, lab.data_ptr(), G.QUERY_FP32_FILTER, graph=True)
    B.query_device(d_pts.data_ptr(), off, direct.data_ptr(), G.QUERY_FP32_FILTER, sync=True)
    torch.cuda.synchronize()
    assert torch.equal(lab, direct)


def test_batch_rejects_bad_offsets(batch_case):
    polys, pts, P = batch_case
    B = G.Batch(P[:4])
    with pytest.raises(G.GahhgError):
        B.query_device(0, np.array([0, 5, 3, 6, 9]), 0)


def test_summary_staged_by_bulk_copy(batch_case):
    """The locate kernels stage each polygon's coarse summary with one bulk
    copy; in batch and single-polygon queries no block fell back to plain loads
    (a wait that runs out would count one and still give correct labels)."""
    import torch
    polys, pts, P = batch_case
    before = G.staging_fallbacks(0)
    B = G.Batch(P[:8])
    flat, off = _layout(pts[:8])
    d_pts = torch.from_numpy(flat).cuda()
    lab = torch.zeros(len(flat), dtype=torch.uint8, device="cuda")
    B.query_device(d_pts.data_ptr(), off, lab.data_ptr(), G.QUERY_FP32_FILTER, sync=True)
    G.Grid(P[2], semantics=G.SEMANTICS_EXACT, device=0).classify().query(pts[2], G.QUERY_FP32_FILTER)
    assert G.staging_fallbacks(0) == before


def test_group_boundaries_equal_single():
    """Batches are built in groups of consecutive polygons of up to 2^20 edges
    (a larger polygon is a group of its own): small polygons around the
    1.1M-edge C1 polygon (groups [small], [C1], [small]) give the labels each
    polygon's own build gives, on near-edge and uniform points; the batch
    statistics count every polygon's edges."""
    import torch
    rng = np.random.default_rng(21)
    small = synth.c3_polygons(6, seed=22, vmax=3000)
    c1 = synth.c1_polygon()
    rings = [r for r, _c, _r in small[:3]] + [c1] + [r for r, _c, _r in small[3:]]
    P = [G.Polygon.from_rings(r) for r in rings]
    pts = [np.concatenate([synth.near_edge_points(r, 3000, rng), synth.uniform_points(2000, rng)]) for r in rings]
    B = G.Batch(P)
    flat, off = _layout(pts)
    d_pts = torch.from_numpy(flat).cuda()
    lab = torch.zeros(len(flat), dtype=torch.uint8, device="cuda")
    B.query_device(d_pts.data_ptr(), off, lab.data_ptr(), G.QUERY_FP32_FILTER, sync=True)
    got = lab.cpu().numpy()
    for i, poly in enumerate(P):
        want = G.Grid(poly, semantics=G.SEMANTICS_EXACT).classify().query(pts[i], G.QUERY_FP32_FILTER)
        seg = got[off[i]:off[i + 1]]
        assert np.array_equal(seg, want), "polygon %d: %d labels differ" % (i, int((seg != want).sum()))
    assert B.stats()["edges"] == sum(p.num_edges for p in P)


def test_launch_shapes_give_the_same_labels(batch_case):
    """Every pass-1 launch shape (points per thread x blocks per SM) gives the
    default shape's labels and in-count, directly and through a graph that
    the shape change recaptures; a chunk change recaptures it too."""
    import torch
    polys, pts, P = batch_case
    shapes = G.Batch.shapes()
    assert shapes[0] == (5, 5) and len(shapes) >= 2
    B = G.Batch(P)
    flat, off = _layout(pts)
    d_pts = torch.from_numpy(flat).cuda()
    want = torch.zeros(len(flat), dtype=torch.uint8, device="cuda")
    B.query_device(d_pts.data_ptr(), off, want.data_ptr(), G.QUERY_FP32_FILTER, sync=True)
    n_in = B.stats()["in_count"]
    lab = torch.zeros(len(flat), dtype=torch.uint8, device="cuda")
    B.query_device(d_pts.data_ptr(), off, lab.data_ptr(), G.QUERY_FP32_FILTER, graph=True)
    for i in range(len(shapes)):
        B.set_shape(i)
        for chunk in (1024, 4096):
            B.set_chunk(chunk)
            lab.fill_(7)
            B.query_device(d_pts.data_ptr(), off, lab.data_ptr(), G.QUERY_FP32_FILTER, sync=True)
            assert torch.equal(lab, want), (shapes[i], chunk)
            assert B.stats()["in_count"] == n_in
            lab.fill_(7)
            B.query_device(d_pts.data_ptr(), off, lab.data_ptr(), G.QUERY_FP32_FILTER, graph=True)
            torch.cuda.synchronize()
            assert torch.equal(lab, want), (shapes[i], chunk, "graph")
    with pytest.raises(G.GahhgError):
        B.set_shape(len(shapes))
