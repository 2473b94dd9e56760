"""The drop-in acceptance set: every test/explist.bat invocation whose query
file is shipped, 3,125 in all: every Mars polygon and the shipped `various`
ones (tests/golden/explist.npz, which also holds 16 Tennessee polygons) and
all 2,498 Tennessee polygons (tests/golden/explist_tennessee.npz; both from
tests/golden/make_explist_fixtures.py).

Per invocation, through the same C ABI the `gahhg` CLI uses: the polygon file
loaded by our loader; the reference-semantics grid must equal the reference's
(level statistics, report space figures and a digest of every grid array) and
give its labels bit for bit; the exact-semantics labels must equal the exact
oracle's.  The reference's labels include its misclassifications (five Mars
polygons 0.01 degrees across where it puts thousands of the query points
inside); the exact labels do not.
"""
import os

import numpy as np
import pytest

import gahhg_b200 as G
from tests.golden.fixtures import Inputs, fmt6
from tests.golden.make_fixtures import digest
from tests.conftest import report

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURE = os.path.join(GOLDEN, "explist.npz")
FIXTURE_TN = os.path.join(GOLDEN, "explist_tennessee.npz")


class Explist:
    def __init__(self, path=FIXTURE):
        z = np.load(path)
        self.z = z
        self.names = list(z["names"])
        n = z["npoints"]
        self.n = n
        self.boff = np.concatenate([[0], np.cumsum((n + 7) // 8)])
        self.zoff = np.concatenate([[0], np.cumsum(z["ref_zero_count"])])
        self.text = None
        if "text_xz" in z.files:
            import lzma
            self.text = lzma.decompress(z["text_xz"].tobytes())
            self.toff = z["text_off"]

    def polygon_text(self, i):
        z = self.z
        if self.text is not None:
            return self.text[self.toff[i]:self.toff[i + 1]].decode()
        r0, r1 = z["poly_ring"][i], z["poly_ring"][i + 1]
        lines = ["POLYGON 1 %d" % (r1 - r0 - 1)]
        for r in range(r0, r1):
            a, b = z["ring_heads"][r]
            lines.append("%d %d" % (a, b))
            c = z["coords"][z["ring_start"][r]:z["ring_start"][r + 1]]
            lines.extend("%s %s" % (fmt6(x), fmt6(y)) for x, y in c)
        return "\n".join(lines) + "\n"

    def labels(self, kind, i):
        bits = np.unpackbits(self.z[kind + "_in"][self.boff[i]:self.boff[i + 1]], count=self.n[i])
        lab = bits.astype(np.uint8) + 1
        if kind == "ref":
            lab[self.z["ref_zero"][self.zoff[i]:self.zoff[i + 1]]] = 0
        return lab


@pytest.fixture(scope="module")
def explist():
    return Explist()


def _check(explist, i, q, path):
    """The invocation's mismatches (empty when it passes)."""
    name = explist.names[i]
    with open(path, "w") as f:
        f.write(explist.polygon_text(i))
    P = G.Polygon.from_file(path)
    g = G.Grid(P, semantics=G.SEMANTICS_REFERENCE, max_depth=15).classify()
    st = g.stats()
    got = np.array([st["depth"], st["vnum"], st["bnum"], st["cnum"], st["rnum"], st["cpu_space"],
                    st["gpu_min_space"]], dtype=np.int64)
    if not np.array_equal(got, explist.z["stats"][i]):
        return [(name, "stats", got, explist.z["stats"][i])]
    if digest(*g.export()) != str(explist.z["grid_digest"][i]):
        return [(name, "grid arrays")]
    bad = []
    lab = g.query(q, G.QUERY_REFERENCE_FP64)
    want = explist.labels("ref", i)
    if not np.array_equal(lab, want):
        bad.append((name, "reference labels", int((lab != want).sum())))
    ge = G.Grid(P, semantics=G.SEMANTICS_EXACT).classify()
    lab = ge.query(q, G.QUERY_FP32_FILTER)
    want = explist.labels("exact", i)
    if not np.array_equal(lab, want):
        bad.append((name, "exact labels", int((lab != want).sum())))
    return bad


def test_explist_invocations(explist, tmp_path):
    store = Inputs()
    queries = {}
    bad = []
    for i, name in enumerate(explist.names):
        qname = str(explist.z["queries"][i])
        if qname not in queries:
            queries[qname] = store.query(qname)
        bad += _check(explist, i, queries[qname], str(tmp_path / "p.txt"))
    assert not bad, bad[:10]
    assert len(explist.names) >= 640


def test_explist_tennessee_invocations(explist, tmp_path):
    """All 2,498 Tennessee invocations (the same boundary at 5 to 25,003
    vertices; test/explist.bat:645-3142)."""
    tn = Explist(FIXTURE_TN)
    q = Inputs().query("Tennessee_query")
    bad = []
    for i in range(len(tn.names)):
        bad += _check(tn, i, q, str(tmp_path / "p.txt"))
    assert not bad, bad[:10]
    assert len(tn.names) == 2498
    # the 16 Tennessee polygons of the main fixture are the same invocations
    shared = [n for n in explist.names if n.startswith("Tennessee/")]
    assert shared and set(shared) <= set(tn.names)
    others = sum(1 for n in explist.names if not n.startswith("Tennessee/"))
    report("explist: %d invocations (%d Mars/various + %d Tennessee): grids, reference labels and exact labels "
           "all equal" % (others + len(tn.names), others, len(tn.names)))
