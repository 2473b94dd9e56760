"""Exact-semantics queries on the GPU against the exact brute-force oracle.

Labels must be identical (bit-exact) for every point: uniform points, points
within 1e-15..1e-3 rad of edges, points exactly on edges (symbolic
perturbation), points equal to vertices, poles, the antimeridian, and inputs
outside the nominal lon/lat ranges.  The FP32-filtered and FP64-filtered
kernels must agree with each other and with the oracle.
"""
import ctypes

import numpy as np
import pytest

import gahhg_b200 as G
from gahhg_b200 import synth
from oracle import exact
from tests.golden.make_fixtures import POLYGONS

pytestmark = pytest.mark.gpu


def _oracle_for(path, rings):
    """Exact oracle over the polygon as the reference's loader reads it."""
    from oracle import ref
    if ref.available():
        r = ref.RefGPISP(path, maxdepth=1)
        xyz, pe = r.polygon()
        r.close()
    else:
        xyz, pe = G.Polygon.from_file(path).export()
    return exact.ExactPolygon(xyz, pe, len(rings[0]))


def _check(grid, oracle, pts, expect_escalations=False):
    want = oracle.query_lonlat(pts)
    got32 = grid.query(pts, G.QUERY_FP32_FILTER)
    st = grid.stats()
    got64 = grid.query(pts, G.QUERY_FP64_FILTER)
    bad = np.nonzero(got32 != want)[0]
    assert len(bad) == 0, "fp32-filter: %d mismatches, first %s got %d want %d" % (
        len(bad), pts[bad[0]].tolist(), got32[bad[0]], want[bad[0]])
    bad = np.nonzero(got64 != want)[0]
    assert len(bad) == 0, "fp64-filter: %d mismatches, first %s" % (len(bad), pts[bad[0]].tolist())
    if expect_escalations:
        assert st["esc_fp64"] > 0
    return st


@pytest.mark.parametrize("name", POLYGONS)
def test_shipped_polygons_exact(inputs, ref_outputs, name, tmp_path):
    path = inputs.polygon_file(name, tmp_path)
    rings = inputs.rings_deg(name)
    g = G.Grid(G.Polygon.from_file(path), semantics=G.SEMANTICS_EXACT).classify()
    qname = str(ref_outputs.get("pair", name)[0])
    q = inputs.query("uniform" if qname == "uniform" else qname)
    _check(g, _oracle_for(path, rings), q)


def test_c0_uniform_and_near_edge(tmp_path):
    rings = synth.c0_polygon()
    path = str(tmp_path / "c0.txt")
    synth.write_polygon(path, rings)
    g = G.Grid(G.Polygon.from_file(path), semantics=G.SEMANTICS_EXACT).classify()
    rng = np.random.default_rng(7)
    pts = np.concatenate([synth.uniform_points(200_000, rng),
                          synth.near_edge_points(rings, 100_000, rng),
                          synth.cap_points(10.0, 20.0, 40.0, 100_000, rng)])
    st = _check(g, _oracle_for(path, rings), pts, expect_escalations=True)
    assert st["esc_exact"] > 0
    assert st["boundary_points"] > 0


def test_exact_zero_cases(tmp_path):
    """Edges on the equator and on the prime meridian: queries there have
    exactly vanishing determinants and are decided by symbolic perturbation;
    queries equal to vertices are inside."""
    rings = [np.array([[0.0, 0.0], [40.0, 0.0], [40.0, 30.0], [0.0, 30.0]]),
             np.array([[10.0, 10.0], [20.0, 10.0], [20.0, 20.0], [10.0, 20.0]])]
    path = str(tmp_path / "sq.txt")
    synth.write_polygon(path, rings)
    g = G.Grid(G.Polygon.from_file(path), semantics=G.SEMANTICS_EXACT).classify()
    lon = np.linspace(-5, 45, 1001)
    pts = np.concatenate([
        np.stack([lon, np.zeros_like(lon)], 1),              # on the equator
        np.stack([np.zeros(301), np.linspace(-5, 35, 301)], 1),  # on the meridian
        np.concatenate(rings),                                # the vertices
        np.array([[0.0, 90.0], [0.0, -90.0], [180.0, 0.0], [-180.0, 0.0], [180.0, 89.99]]),
        np.array([[380.0, 15.0], [-340.0, 15.0], [20.0, 100.0], [20.0, 170.0], [25.0, -95.0]]),
    ])
    want = _oracle_for(path, rings).query_lonlat(pts)
    vert = np.concatenate(rings)
    got = g.query(pts, G.QUERY_FP32_FILTER)
    assert np.array_equal(got, want), np.nonzero(got != want)
    assert np.array_equal(g.query(pts, G.QUERY_FP64_FILTER), want)
    # vertices whose FakeLL latitude is exact are polygon vertices -> inside
    assert (got[1001 + 301:1001 + 301 + len(vert)] == 2).all()


def test_misaligned_lonlat_is_refused(tmp_path):
    """Exact queries read lon/lat in 16-byte units: a device buffer that is
    not 16-byte aligned is refused with GAHHG_ERR_ARG (both entry points),
    never read."""
    import torch
    from gahhg_b200 import _lib
    rings = synth.c0_polygon()
    path = str(tmp_path / "c0.txt")
    synth.write_polygon(path, rings)
    g = G.Grid(G.Polygon.from_file(path), semantics=G.SEMANTICS_EXACT).classify()
    buf = torch.zeros(2 * 1000 + 1, dtype=torch.float64, device="cuda:0")
    lab = torch.zeros(1000, dtype=torch.uint8, device="cuda:0")
    with pytest.raises(_lib.GahhgError) as e:
        g.query_device(buf.data_ptr() + 8, 1000, lab.data_ptr(), G.QUERY_FP32_FILTER)
    assert e.value.status == _lib.ERR_ARG
    st = _lib.lib().gahhg_query_device_noalloc(g._h, ctypes.c_void_p(buf.data_ptr() + 8), 1000,
                                               ctypes.c_void_p(lab.data_ptr()), G.QUERY_FP32_FILTER,
                                               ctypes.c_void_p(0))
    assert st == _lib.ERR_ARG
    g.query_device(buf.data_ptr(), 1000, lab.data_ptr(), G.QUERY_FP32_FILTER, sync=True)


def test_non_finite_inputs_are_undefined(tmp_path):
    rings = synth.c0_polygon()
    path = str(tmp_path / "c0.txt")
    synth.write_polygon(path, rings)
    g = G.Grid(G.Polygon.from_file(path), semantics=G.SEMANTICS_EXACT).classify()
    pts = np.array([[np.nan, 0.0], [0.0, np.inf], [10.0, 20.0]])
    got = g.query(pts)
    assert got[0] == 0 and got[1] == 0 and got[2] in (1, 2)


def test_lattice_params_do_not_change_labels(tmp_path):
    rings = synth.c0_polygon(seed=5)
    path = str(tmp_path / "c0.txt")
    synth.write_polygon(path, rings)
    rng = np.random.default_rng(11)
    pts = np.concatenate([synth.uniform_points(50_000, rng), synth.near_edge_points(rings, 50_000, rng)])
    P = G.Polygon.from_file(path)
    ref = None
    for top, leaf in [(0, 0), (64, 2), (512, 32), (32, 4)]:
        g = G.Grid(P, semantics=G.SEMANTICS_EXACT, lattice_top=top, lattice_leaf=leaf).classify()
        lab = g.query(pts)
        if ref is None:
            ref = lab
        assert np.array_equal(lab, ref), (top, leaf)
