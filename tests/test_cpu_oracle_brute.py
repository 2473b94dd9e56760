"""The GPU brute force of the exact oracle (oracle/brute_gpu.cu) runs its
per-point steps on the host as well; there they must give the CPU oracle's
labels (oracle/exact_pip.c) wherever they decide, on uniform, near-edge and
vertex-adjacent points of C0 and on near-edge points of the 1.1M-edge C1
polygon, and leave undecided only points the FP64 bounds cannot separate.
Host code only: this checks the brute force's logic without a GPU.
"""
import numpy as np

import gahhg_b200 as G
from gahhg_b200 import synth
from oracle import exact
from tests.conftest import report


def _oracle(rings):
    P = G.Polygon.from_rings(rings)
    xyz, pe = P.export()
    return exact.ExactPolygon(xyz, pe, len(rings[0]))


def test_brute_steps_equal_cpu_oracle_c0():
    rng = np.random.default_rng(23)
    rings = synth.c0_polygon()
    E = _oracle(rings)
    q = np.concatenate([synth.uniform_points(3000, rng), synth.near_edge_points(rings, 3000, rng),
                        np.concatenate(rings)[::3]])
    got, und = E.query_lonlat_brute_host(q)
    want = E.query_lonlat(q)
    dec = got != 0
    assert np.array_equal(got[dec], want[dec])
    assert und == int((~dec).sum()) and und < 0.05 * len(q)
    # points 1e-15 rad from an edge are decided: the bound follows the edge's length
    assert dec[3000:6000].mean() > 0.99
    report("brute force steps on the host == CPU oracle on %d C0 points (%d undecided)" % (len(q), und))


def test_brute_steps_equal_cpu_oracle_c1_near_edge():
    rng = np.random.default_rng(29)
    rings = synth.c1_polygon()
    E = _oracle(rings)
    q = synth.near_edge_points(rings, 60, rng, umin=-15.0, umax=-12.0)
    got, und = E.query_lonlat_brute_host(q)
    want = E.query_lonlat(q)
    dec = got != 0
    assert np.array_equal(got[dec], want[dec]) and und <= 3
