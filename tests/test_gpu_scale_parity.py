"""Exact labels at the benchmark configurations' scale, every label checked
against the exact oracle's brute force over every edge.

The oracle here is oracle/brute_gpu.cu: the brute force of oracle/exact_pip.c
run on the GPU with its own FP64 predicates and error bounds; the points it
cannot decide there go to the CPU brute force, so every expected label is
the CPU oracle's definition.  Its agreement with the CPU oracle is pinned
first.  Then:
  C1  1e6 points of the benchmark's own uniform generator (synth.device_points)
      on the 1.1M-edge C1 polygon, FP32-filtered and FP64-filtered queries;
  C2  2e6 points of the benchmark's C2 generator (synth.device_c2_points: half
      uniform, half within 10^U[-15,-3] rad of a random edge), both precisions;
  C3  256 batch-configuration polygons chosen to include the largest rings
      (up to 200,000 vertices), 8-hole polygons, polygons around a pole and
      polygons across the antimeridian, every point of every polygon checked,
      from a direct batch launch and from a CUDA-graph replay.
The per-tier escalation counts of each run are printed in the session's
summary.  Reference path: kernel_PISP (source/GPISPAHHG.cu:1422-1504), with
the labels of the library's exact semantics.
"""
import time

import numpy as np
import pytest

import gahhg_b200 as G
from gahhg_b200 import synth
from oracle import exact
from tests.conftest import report

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1():
    rings = synth.c1_polygon()
    P = G.Polygon.from_rings(rings)
    xyz, pe = P.export()
    E = exact.ExactPolygon(xyz, pe, len(rings[0]))
    g = G.Grid(P, semantics=G.SEMANTICS_EXACT, device=0).classify()
    return rings, P, E, g


def test_gpu_brute_force_equals_cpu_oracle(c1):
    """The GPU brute force gives the CPU oracle's labels (or none) on C0
    (uniform, near-edge and vertex-adjacent points) and on C1 samples."""
    rng = np.random.default_rng(17)
    r0 = synth.c0_polygon()
    P0 = G.Polygon.from_rings(r0)
    x0, p0 = P0.export()
    E0 = exact.ExactPolygon(x0, p0, len(r0[0]))
    q0 = np.concatenate([synth.uniform_points(4000, rng), synth.near_edge_points(r0, 4000, rng),
                         np.concatenate(r0)[::7]])
    got, und = E0.query_lonlat_gpu(q0)
    assert np.array_equal(got, E0.query_lonlat(q0))
    rings, _P, E, _g = c1
    q1 = np.concatenate([synth.uniform_points(200, rng), synth.near_edge_points(rings, 200, rng)])
    got1, und1 = E.query_lonlat_gpu(q1)
    assert np.array_equal(got1, E.query_lonlat(q1))
    report("oracle pin: GPU brute force == CPU brute force on %d C0 + %d C1 points (%d + %d left to the CPU)"
           % (len(q0), len(q1), und, und1))


def _device_labels(g, d_pts, prec):
    import torch
    n = d_pts.shape[0]
    lab = torch.zeros(n, dtype=torch.uint8, device=d_pts.device)
    g.query_device(d_pts.data_ptr(), n, lab.data_ptr(), prec, sync=True)
    return lab.cpu().numpy(), g.stats()


def _check_config(name, g, E, d_pts):
    t0 = time.time()
    want, und = E.query_lonlat_gpu(d_pts.cpu().numpy())
    t_oracle = time.time() - t0
    n = len(want)
    for prec, pname in ((G.QUERY_FP32_FILTER, "FP32 filter"), (G.QUERY_FP64_FILTER, "FP64 filter")):
        got, st = _device_labels(g, d_pts, prec)
        bad = int((got != want).sum())
        report("%s: %d points, %s: %d labels differ from the oracle; boundary %d, FP32->FP64 %d, FP64->exact %d"
               % (name, n, pname, bad, st["boundary_points"], st["esc_fp64"], st["esc_exact"]))
        assert bad == 0, "%s %s: %d of %d labels differ" % (name, pname, bad, n)
    report("%s: oracle %.1f s on the GPU, %d points left to the CPU" % (name, t_oracle, und))
    return want


def test_c1_uniform_against_oracle(c1):
    _rings, _P, E, g = c1
    pts = synth.device_points(1_000_000, 1234, "cuda:0")
    want = _check_config("C1", g, E, pts)
    assert 0.05 < (want == 2).mean() < 0.95


def test_c2_near_edge_against_oracle(c1):
    rings, _P, E, g = c1
    pts = synth.device_c2_points(rings, 2_000_000, 2222, "cuda:0")
    _check_config("C2", g, E, pts)


def _c3_sample(n_pick=256, seed=3):
    """256 polygons of the batch configuration's generator: the largest
    rings, those with 8 holes, those around a pole, those across the
    antimeridian, then others in generation order."""
    polys = synth.c3_polygons(1024, seed=seed)
    nv = np.array([len(r[0]) for r, _c, _r in polys])
    holes = np.array([len(r) - 1 for r, _c, _r in polys])
    polar = np.array([abs(c[1]) + 1.2 * rad >= 90.0 for _r, c, rad in polys])
    anti = np.array([np.ptp(r[0][:, 0]) > 180.0 and not pl for (r, _c, _r), pl in zip(polys, polar)])
    pick = []
    for group in (np.argsort(-nv)[:24], np.nonzero(holes == 8)[0][:24], np.nonzero(polar)[0][:24],
                  np.nonzero(anti)[0][:24], np.arange(len(polys))):
        for i in group:
            if len(pick) < n_pick and i not in pick:
                pick.append(int(i))
    sel = [polys[i] for i in pick]
    return sel, nv[pick], holes[pick], polar[pick], anti[pick]


def test_c3_batch_against_oracle():
    import torch
    polys, nv, holes, polar, anti = _c3_sample()
    assert nv.max() >= 190_000 and (holes == 8).any() and polar.any() and anti.any()
    pts = synth.c3_points(polys, seed=4, pmax=20_000)
    P = [G.Polygon.from_rings(r) for r, _c, _r in polys]
    B = G.Batch(P)
    off = np.zeros(len(pts) + 1, dtype=np.int64)
    off[1:] = np.cumsum([len(p) for p in pts])
    flat = np.concatenate(pts)
    d_pts = torch.from_numpy(flat).cuda()
    direct = torch.zeros(len(flat), dtype=torch.uint8, device="cuda")
    B.query_device(d_pts.data_ptr(), off, direct.data_ptr(), G.QUERY_FP32_FILTER, sync=True)
    st = B.stats()
    replay = torch.zeros(len(flat), dtype=torch.uint8, device="cuda")
    B.query_device(d_pts.data_ptr(), off, replay.data_ptr(), G.QUERY_FP32_FILTER, graph=True)
    torch.cuda.synchronize()
    got, got_replay = direct.cpu().numpy(), replay.cpu().numpy()
    assert np.array_equal(got, got_replay)
    bad_polys, undecided = [], 0
    t0 = time.time()
    for i, (rings, _c, _r) in enumerate(polys):
        xyz, pe = P[i].export()
        want, und = exact.ExactPolygon(xyz, pe, len(rings[0])).query_lonlat_gpu(pts[i])
        undecided += und
        if not np.array_equal(got[off[i]:off[i + 1]], want):
            bad_polys.append((i, int((got[off[i]:off[i + 1]] != want).sum())))
    report("C3: %d polygons (max %d vertices, %d with 8 holes, %d polar, %d across the antimeridian), %d points: "
           "%d polygons differ from the oracle; boundary %d, FP32->FP64 %d, FP64->exact %d; oracle %.1f s, "
           "%d points left to the CPU" % (len(polys), nv.max(), (holes == 8).sum(), polar.sum(), anti.sum(),
                                          len(flat), len(bad_polys), st["boundary_points"], st["esc_fp64"],
                                          st["esc_exact"], time.time() - t0, undecided))
    assert not bad_polys, bad_polys[:10]
