"""GPU grid, classification and FP64 query against the reference's own code.

The reference (source/GPISPAHHG.cu) is built for the CPU by oracle/build_ref.py
and run serially; its outputs on the shipped polygons are committed in
tests/golden/reference_outputs.npz and, where the prebuilt oracle library is
present, also recomputed live so a mismatch can be located array by array.
Everything here is bit-exact: grid vertices, borders, cells, edge lists, cell
types, labels.
"""
import hashlib

import numpy as np
import pytest

import gahhg_b200 as G
from tests.golden.make_fixtures import POLYGONS

pytestmark = pytest.mark.gpu


def _digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def _first_diff(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if a.shape != b.shape:
        return "shape %s vs %s" % (a.shape, b.shape)
    if a.dtype.names:
        for f in a.dtype.names:
            d = _first_diff(a[f], b[f])
            if d:
                return "field %s: %s" % (f, d)
        return None
    bad = np.argwhere(a != b)
    if len(bad) == 0:
        return None
    i = tuple(bad[0])
    return "first at %s: %r vs %r (%d differ)" % (i, a[i], b[i], len(bad))


def _build(inputs, name, tmp_path):
    path = inputs.polygon_file(name, tmp_path)
    P = G.Polygon.from_file(path)
    g = G.Grid(P, semantics=G.SEMANTICS_REFERENCE)
    g.classify()
    return path, P, g


@pytest.mark.parametrize("name", POLYGONS)
def test_grid_bitwise(inputs, ref_outputs, name, tmp_path, request):
    path, P, g = _build(inputs, name, tmp_path)
    lv, V, B, C, R = g.export()
    st = ref_outputs.get("stats", name)
    assert [len(lv), lv[-1]["vstart"] + lv[-1]["vnum"], lv[-1]["bstart"] + lv[-1]["bnum"],
            lv[-1]["cstart"] + lv[-1]["cnum"], lv[-1]["rnum"]] == list(st[:5])
    want = str(ref_outputs.get("digest_grid", name)[0])
    if _digest(lv, V, B, C, R) != want:
        from oracle import ref
        msg = "grid digest differs"
        if ref.available():
            r = ref.RefGPISP(path, threads=1)
            rl, rV, rB, rC, rR = r.export()
            for nm, a, b in (("levels", lv, rl), ("V", V, rV), ("B", B, rB), ("C", C, rC), ("refs", R, rR)):
                d = _first_diff(a, b)
                if d:
                    msg += "; %s: %s" % (nm, d)
        pytest.fail(msg)


@pytest.mark.parametrize("name", POLYGONS)
def test_labels_fp64_match_reference(inputs, ref_outputs, name, tmp_path):
    path, P, g = _build(inputs, name, tmp_path)
    qname = str(ref_outputs.get("pair", name)[0])
    q = inputs.query("uniform" if qname == "uniform" else qname)
    lab = g.query(q, G.QUERY_REFERENCE_FP64)
    want = ref_outputs.get("labels", name)
    d = _first_diff(lab, want)
    assert d is None, d
    st = g.stats()
    ref_st = ref_outputs.get("stats", name)
    assert st["depth"] == ref_st[0]
    assert st["cpu_space"] == ref_st[5]
    assert st["gpu_min_space"] == ref_st[6]
