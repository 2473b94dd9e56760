"""The seeded workload generators (gahhg_b200/synth.py) against the
configurations they stand in for: ring sizes, radii, holes, pole and
antimeridian coverage, point distributions and near-edge offsets.  Host only
(the device point generators run on torch's CPU device here)."""
import numpy as np
import pytest

from gahhg_b200 import synth

DEG = np.pi / 180.0


def _xyz(ll):
    return synth._xyz(np.asarray(ll, dtype=np.float64))


def _dist_deg(ll, lon0, lat0):
    c = _xyz(np.array([[lon0, lat0]]))[0]
    return np.arccos(np.clip(_xyz(ll) @ c, -1.0, 1.0)) / DEG


def _center(ring):
    m = _xyz(ring).mean(0)
    m /= np.linalg.norm(m)
    return np.arctan2(m[0], m[2]) / DEG, np.arcsin(m[1]) / DEG


def test_c0_polygon():
    outer, hole = synth.c0_polygon()
    assert outer.shape == (1000, 2) and hole.shape == (100, 2)
    d = _dist_deg(outer, 10.0, 20.0)
    assert d.min() >= 24.0 - 1e-9 and d.max() <= 36.0 + 1e-9  # 30 deg x (1 +- 0.2)
    assert np.allclose(_dist_deg(hole, 10.0, 20.0), 5.0)


def test_c1_polygon():
    rings = synth.c1_polygon()
    assert len(rings) == 11
    assert len(rings[0]) == 1_000_000 and all(len(h) == 10_000 for h in rings[1:])
    d = _dist_deg(rings[0], 170.0, 70.0)
    # 60 deg with displacements of 6 deg halving per level (at most 12 in all)
    assert 48.0 <= d.min() and d.max() <= 72.0
    assert d.min() > 20.0  # the north pole (20 deg from the center) is inside
    lon = rings[0][:, 0]
    assert (lon > 170.0).any() and (lon < -170.0).any()  # across the antimeridian
    for h in rings[1:]:
        lo, la = _center(h)
        r = _dist_deg(h, lo, la)
        assert 1.0 - 1e-6 <= r.mean() <= 4.0 + 1e-6 and np.ptp(r) < 1e-6
        assert _dist_deg(np.array([[lo, la]]), 170.0, 70.0)[0] + r.max() < d.min()  # inside the outer ring


def test_uniform_points_by_area():
    p = synth.uniform_points(400_000, np.random.default_rng(5))
    s = np.sin(p[:, 1] * DEG)
    assert abs(s.mean()) < 0.01 and abs((s * s).mean() - 1.0 / 3.0) < 0.01
    assert abs(p[:, 0].mean()) < 1.5 and p[:, 0].min() >= -180.0 and p[:, 0].max() < 180.0


def test_c2_points_near_edges():
    torch = pytest.importorskip("torch")
    rings = synth.c1_polygon(n_outer=20_000, hole_n=500)
    n = 200_000
    pts = synth.device_c2_points(rings, n, 3, "cpu").numpy()
    assert pts.shape == (n, 2) and np.isfinite(pts).all()
    # half uniform by area
    s = np.sin(pts[: n // 2, 1] * DEG)
    assert abs(s.mean()) < 0.02 and abs((s * s).mean() - 1.0 / 3.0) < 0.02
    # half within 10^[-15,-3] rad of an edge: the distance to the nearest
    # vertex is at most about an edge (under 1e-3 rad on this ring and its
    # holes) plus the 1e-3 rad offset
    ll = np.concatenate(rings)
    q = _xyz(pts[n // 2:][:2000])
    v = _xyz(ll)
    near = np.arccos(np.clip((q @ v.T).max(1), -1.0, 1.0))
    assert near.max() < 3e-3
    del torch


def test_c3_polygons_shapes():
    polys = synth.c3_polygons(600, seed=11, vmax=3_000)
    nv = np.array([len(r[0]) for r, _c, _r in polys])
    holes = np.array([len(r) - 1 for r, _c, _r in polys])
    radii = np.array([rad for _r, _c, rad in polys])
    lats = np.array([c[1] for _r, c, _rad in polys])
    assert nv.min() >= 16 and nv.max() <= 3_000
    assert holes.min() >= 0 and holes.max() <= 8
    assert radii.min() >= 0.5 and radii.max() <= 40.0
    # log-uniform radius: the median near sqrt(0.5 * 40)
    assert 2.5 < np.median(radii) < 7.5
    # about 5 % moved onto a pole (the pole lies inside those polygons)
    polar = np.abs(lats) >= 90.0 - 0.3 * radii - 1e-9
    assert 0.02 < polar.mean() < 0.09
    for rings, (lon, lat), radius in polys[:50]:
        d = _dist_deg(rings[0], lon, lat)
        assert d.max() < 1.5 * radius * 1.2  # inside the query cap
        for h in rings[1:]:
            assert _dist_deg(h, lon, lat).max() < d.min()  # holes inside the outer ring


def test_c3_points_in_caps():
    polys = synth.c3_polygons(40, seed=12, vmax=500)
    pts = synth.c3_points(polys, seed=13, pmax=20_000)
    for (rings, (lon, lat), radius), p in zip(polys, pts):
        assert 1_000 <= len(p) <= 20_000
        assert _dist_deg(p, lon, lat).max() <= 1.5 * radius * 1.2 + 1e-9
