"""Soundness of the FP64 orientation filters against the exact oracle.

A filter may answer "undecided" (0) as often as it likes, but every sign it
does return must be the exact sign of det[a; b; c].  The triples mimic the
query's crossing tests: an edge (a, b) a few micro-radians long with a point
c placed 10^U[-20,-3] rad off its great circle, and a leaf center with a
point and an edge end near it.  The filters are compiled for the host from
the same header the kernels use.
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
    subprocess.check_call(["g++", "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-o", out,
                           os.path.join(HERE, "native", "pred_probe.cpp")])
    lib = ctypes.CDLL(out)
    lib.filter_signs.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_void_p]
    lib.filter_signs.restype = None

    def signs(tri, near):
        tri = np.ascontiguousarray(tri, dtype=np.float64)
        res = np.zeros(len(tri), dtype=np.int32)
        lib.filter_signs(tri.ctypes.data, len(tri), 1 if near else 0, res.ctypes.data)
        return res

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
