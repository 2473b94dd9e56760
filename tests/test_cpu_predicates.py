"""Soundness of the FP64 orientation filters against the exact oracle.

A filter may answer "undecided" (0) as often as it likes, but every sign it
does return must be the exact sign of det[a; b; c].  The triples mimic the
query's crossing tests: an edge (a, b) a few micro-radians long with a point
c placed 10^U[-20,-3] rad off its great circle, and a leaf center with a
point and an edge end near it.  The filters are compiled for the host from
the same headers the kernels use.  The FP32 local-frame tier is checked the
same way on cells of 1e-7..1e-1 rad with points near an edge's great circle
or near the arc from the cell center to an edge end.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from oracle import exact

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("pred") / "libpred_probe.so")
    subprocess.check_call(["g++", "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-I",
                           os.path.join(os.path.dirname(HERE), "include"), "-o", out,
                           os.path.join(HERE, "native", "pred_probe.cpp")])
    lib = ctypes.CDLL(out)
    lib.filter_signs.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_void_p]
    lib.filter_signs.restype = None
    lib.local_signs.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p]
    lib.local_signs.restype = None

    def signs(tri, near):
        tri = np.ascontiguousarray(tri, dtype=np.float64)
        res = np.zeros(len(tri), dtype=np.int32)
        lib.filter_signs(tri.ctypes.data, len(tri), 1 if near else 0, res.ctypes.data)
        return res

    def local(cfg):
        cfg = np.ascontiguousarray(cfg, dtype=np.float64)
        res = np.zeros((len(cfg), 4), dtype=np.int32)
        lib.local_signs(cfg.ctypes.data, len(cfg), res.ctypes.data)
        return res

    signs.local = local
    return signs


def _unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def _triples(n, seed):
    rng = np.random.default_rng(seed)
    a = _unit(rng.normal(size=(n, 3)))
    t = _unit(np.cross(a, rng.normal(size=(n, 3))))
    length = 10.0 ** rng.uniform(-7, -3, n)[:, None]
    b = _unit(a + length * t)
    nrm = _unit(np.cross(a, b))
    off = 10.0 ** rng.uniform(-20, -3, n)[:, None] * np.where(rng.random((n, 1)) < 0.5, -1.0, 1.0)
    s = rng.uniform(-0.5, 1.5, (n, 1))
    c = _unit((1 - s) * a + s * b + off * nrm)
    edge = np.stack([a, b, c], 1)          # orient(A, B, q)
    center = np.stack([c, a, b], 1)        # orient(R, q, A) with R near q and A
    return np.concatenate([edge, center]).reshape(-1, 9)


def test_fp64_filters_are_sound(probe):
    tri = _triples(20000, 5)
    want = np.array([exact.orient(t[0:3], t[3:6], t[6:9], sos=False) for t in tri])
    for near in (False, True):
        got = probe(tri, near)
        decided = got != 0
        assert np.array_equal(got[decided], want[decided]), "filter %s returned a wrong sign" % near
    near_decided = (probe(tri, True) != 0).mean()
    plain_decided = (probe(tri, False) != 0).mean()
    # the translated rows resolve points far closer to short edges
    assert near_decided > 0.9 and near_decided > plain_decided + 0.2, (near_decided, plain_decided)


def _lonlat(v):
    v = _unit(v)
    return np.stack([np.degrees(np.arctan2(v[:, 0], v[:, 2])), np.degrees(np.arcsin(np.clip(v[:, 1], -1, 1)))], 1)


def _xyz(ll):
    lo, la = np.radians(ll[:, 0]), np.radians(ll[:, 1])
    return np.stack([np.cos(la) * np.sin(lo), np.sin(la), np.cos(la) * np.cos(lo)], 1)


def _local_cases(n, seed, polar=0.1):
    """Cells of 1e-7..1e-1 rad anywhere (a fraction `polar` of them within 5
    degrees of a pole; antimeridian wraps); the point on the edge's great
    circle or on the arc from the center to an edge end, pushed off it by
    10^U[-19,-2] times the cell size; longitudes wrapped by +-360 degrees on
    either side."""
    rng = np.random.default_rng(seed)
    Rll = np.stack([rng.uniform(-180, 180, n), np.degrees(np.arcsin(rng.uniform(-1, 1, n)))], 1)
    pole = rng.random(n) < polar
    Rll[pole, 1] = np.sign(rng.uniform(-1, 1, pole.sum())) * rng.uniform(85, 90, pole.sum())
    R = _xyz(Rll)
    r = 10.0 ** rng.uniform(-7, -1, n)[:, None]
    def near(scale):
        return _unit(R + scale * r * rng.normal(size=(n, 3)))
    A, B = near(1.0), near(1.0)
    kind = rng.integers(0, 3, n)[:, None]  # 0: near edge AB, 1: near arc R-A, 2: near arc R-B
    P0 = np.where(kind == 0, A, R)
    P1 = np.where(kind == 2, B, np.where(kind == 0, B, A))
    t = rng.uniform(-0.3, 1.3, (n, 1))
    q = _unit((1 - t) * P0 + t * P1)
    nrm = _unit(np.cross(P0, P1))
    off = 10.0 ** rng.uniform(-19, -2, (n, 1)) * r * np.where(rng.random((n, 1)) < 0.5, -1.0, 1.0)
    q = _unit(q + off * nrm)
    qll, All, Bll = _lonlat(q), _lonlat(A), _lonlat(B)
    qll[:, 0] += 360.0 * rng.integers(-1, 2, n) * (rng.random(n) < 0.2)
    Rll[:, 0] += 360.0 * (rng.random(n) < 0.1)
    return np.concatenate([qll, Rll, All, Bll], 1)


@pytest.mark.parametrize("seed,polar", [(11, 0.1), (23, 0.6)])
def test_fp32_local_frame_is_sound(probe, seed, polar):
    cfg = _local_cases(30000, seed, polar)
    got = probe.local(cfg)
    ok = got[:, 0] != 9
    # near a pole cells span wide longitude differences, and more offsets are
    # refused (those points defer to the FP64 tier)
    assert ok.mean() > (0.99 if polar < 0.5 else 0.95)
    want = np.zeros((len(cfg), 3), dtype=np.int32)
    cross = np.full(len(cfg), -1, dtype=np.int32)  # exact crossing of the stored record, -1: degenerate
    for i in np.nonzero(ok)[0]:
        c = cfg[i]
        q = exact.query_xyz(c[0:2].reshape(1, 2))[0]
        R, A, B = exact.vertex_xyz(c[2:8].reshape(3, 2))
        want[i] = (exact.orient(A, B, q, sos=False), exact.orient(R, q, A, sos=False), exact.orient(R, q, B, sos=False))
        # the record is stored in the order that makes orient(A, B, R) = +1
        s2, s3, s4 = want[i]
        if exact.orient(A, B, R, sos=False) < 0:
            s2, s3, s4 = -s2, s4, s3
        if s2 == 1 or s3 == 1 or s4 == -1:
            cross[i] = 0
        elif s2 == -1 and s3 == -1 and s4 == 1:
            cross[i] = 1
    g, w = got[ok, :3], want[ok]
    decided = g != 0
    assert np.array_equal(g[decided], w[decided]), "the local-frame FP32 tier returned a wrong sign"
    # points 1e-5 of the cell size or more from the arc are decided in FP32
    assert decided.mean() > 0.6, decided.mean()
    # the tier's combined test: decided answers are the exact crossing, and a
    # degenerate case (an exact zero and no sign that rules the crossing out)
    # is never decided
    gx, wx = got[ok, 3], cross[ok]
    dx = gx >= 0
    assert np.array_equal(gx[dx], wx[dx]), "the local-frame FP32 crossing test returned a wrong answer"
    assert dx.mean() > 0.7, dx.mean()
