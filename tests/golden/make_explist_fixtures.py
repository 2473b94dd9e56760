"""Generate tests/golden/explist.npz: the drop-in acceptance set.

test/explist.bat runs the reference's GPISP.exe 3,135 times; 3,125 of those
invocations have their query files shipped (Mars, Tennessee, various).  The
Tennessee polygons are 601 MB of text, so the fixture keeps every Mars
invocation (624), the shipped `various` ones, and 16 Tennessee polygons
spread over the set by index.  For each invocation it stores the polygon (as
integer micro-degrees, with the ring headers, so the text is re-created byte
for byte), the query file's name, and what the reference code (built for the
CPU, run serially) produces at its default depth: labels, the grid
statistics of the report and a SHA-256 digest of the grid arrays; plus the
exact oracle's labels.

    python tests/golden/make_explist_fixtures.py [/path/to/reference]
    python tests/golden/make_explist_fixtures.py --tennessee [/path/to/reference]

The second form writes explist_tennessee.npz, every Tennessee invocation
(main_tennessee below).

Needs the reference checkout and the CPU builds (python oracle/build_ref.py,
python oracle/build_oracle.py) and libgahhg.so (host code only).
"""
import multiprocessing as mp
import os
import re
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from tests.golden.make_fixtures import digest, read_polygon_text  # noqa: E402

TENNESSEE_SAMPLE = 16


def invocations(refroot):
    pat = re.compile(r"/polyfile\s+\.\\polygon\\(\S+)\s+/tpfile\s+\.\\query\\(\S+)")
    out = []
    with open(os.path.join(refroot, "test/explist.bat")) as f:
        for ln in f:
            m = pat.search(ln)
            if m:
                out.append((m.group(1).replace("\\", "/"), m.group(2)))
    shipped = set(os.listdir(os.path.join(refroot, "test/query")))
    return [(p, q) for p, q in out if q in shipped]


def select(invs):
    mars = [i for i in invs if i[0].startswith("Mars/")]
    various = [i for i in invs if i[0].startswith("various/")]
    tn = sorted(i for i in invs if i[0].startswith("Tennessee/"))
    pick = np.unique(np.linspace(0, len(tn) - 1, TENNESSEE_SAMPLE).round().astype(int))
    return mars + various + [tn[k] for k in pick]


def _run_one(args):
    """Reference (CPU build, serial) and exact oracle on one invocation."""
    text, qmicro = args
    from oracle import exact, ref
    import gahhg_b200 as G
    from tests.golden.fixtures import fmt6
    d = tempfile.mkdtemp()
    path = os.path.join(d, "p.txt")
    with open(path, "w") as f:
        f.write(text)
    q = np.array([[float(fmt6(a)), float(fmt6(b))] for a, b in qmicro])
    R = ref.RefGPISP(path, threads=1)
    st = R.stats()
    lv, V, B, C, refs = R.export()
    stats = np.array([st["gnum"], st["vnum"], st["bnum"], st["cnum"], st["rnum"], st["cpu_space"],
                      st["gpu_min_space"]], dtype=np.int64)
    dig = digest(lv, V, B, C, refs)
    lab = R.query(q).astype(np.uint8)
    R.close()
    P = G.Polygon.from_file(path)
    xyz, pe = P.export()
    n_outer = int(text.split("\n")[1].split()[1]) - 1
    ex = exact.ExactPolygon(xyz, pe, n_outer).query_lonlat(q, threads=1)
    os.unlink(path)
    os.rmdir(d)
    return stats, dig, lab, ex


def main(refroot=None):
    refroot = refroot or os.environ.get("GAHHG_REFERENCE", "/root/reference")
    from tests.golden.fixtures import Inputs, fmt6
    store = Inputs()
    invs = select(invocations(refroot))
    qkey = {"Mars_query.csv": "Mars_query", "Tennessee_query.csv": "Tennessee_query",
            "Radiometer_query.csv": "Radiometer_query", "Square_72_query.csv": "Square_72_query"}
    coords, ring_heads, ring_start, poly_ring = [], [], [0], [0]
    texts = []
    for p, _q in invs:
        heads, rings = read_polygon_text(os.path.join(refroot, "test/polygon", p))
        for h, r in zip(heads, rings):
            ring_heads.append(h)
            coords.append(r.astype(np.int32))
            ring_start.append(ring_start[-1] + len(r))
        poly_ring.append(poly_ring[-1] + len(heads))
        lines = ["POLYGON 1 %d" % (len(rings) - 1)]
        for (a, b), r in zip(heads, rings):
            lines.append("%d %d" % (a, b))
            lines.extend("%s %s" % (fmt6(x), fmt6(y)) for x, y in r)
        text = "\n".join(lines) + "\n"
        with open(os.path.join(refroot, "test/polygon", p), "rb") as f:
            shipped = f.read().decode().replace("\r\n", "\n")
        assert shipped.rstrip("\n") == text.rstrip("\n"), p  # re-created byte for byte
        texts.append(text)
    jobs = [(t, store.z["query_" + qkey[q]]) for t, (_p, q) in zip(texts, invs)]
    with mp.get_context("spawn").Pool(os.cpu_count()) as pool:
        res = pool.map(_run_one, jobs, chunksize=4)
    out = {
        "names": np.array([p for p, _q in invs]),
        "queries": np.array([qkey[q] for _p, q in invs]),
        "coords": np.concatenate(coords),
        "ring_heads": np.array(ring_heads, dtype=np.int32),
        "ring_start": np.array(ring_start, dtype=np.int64),
        "poly_ring": np.array(poly_ring, dtype=np.int64),
        "stats": np.stack([r[0] for r in res]),
        "grid_digest": np.array([r[1] for r in res]),
        "ref_in": np.concatenate([np.packbits(r[2] == 2) for r in res]),
        "ref_zero": np.concatenate([np.nonzero(r[2] == 0)[0] for r in res] + [np.zeros(0, np.int64)]),
        "ref_zero_count": np.array([int((r[2] == 0).sum()) for r in res]),
        "exact_in": np.concatenate([np.packbits(r[3] == 2) for r in res]),
        "npoints": np.array([len(r[2]) for r in res]),
    }
    np.savez_compressed(os.path.join(HERE, "explist.npz"), **out)
    print("wrote", len(invs), "invocations;", sum(int((r[2] != r[3]).sum()) for r in res),
          "points where the reference and the exact oracle differ")


def main_tennessee(refroot=None):
    """tests/golden/explist_tennessee.npz: every Tennessee invocation of
    test/explist.bat (2,498 polygons of the same boundary at 5 to 25,003
    vertices, 601 MB of text).  The polygon texts are stored as one
    LZMA-compressed blob (the polygons share most of their lines, so it
    compresses to a few MB) with each polygon's byte range; the outputs as in
    explist.npz."""
    import lzma
    refroot = refroot or os.environ.get("GAHHG_REFERENCE", "/root/reference")
    from tests.golden.fixtures import Inputs
    store = Inputs()
    invs = sorted(i for i in invocations(refroot) if i[0].startswith("Tennessee/"))
    assert all(q == "Tennessee_query.csv" for _p, q in invs)
    texts = []
    for p, _q in invs:
        with open(os.path.join(refroot, "test/polygon", p), "rb") as f:
            texts.append(f.read().decode().replace("\r\n", "\n"))
    blob = "".join(texts).encode()
    offs = np.concatenate([[0], np.cumsum([len(t.encode()) for t in texts])]).astype(np.int64)
    q = store.z["query_Tennessee_query"]
    with mp.get_context("spawn").Pool(os.cpu_count()) as pool:
        res = pool.map(_run_one, [(t, q) for t in texts], chunksize=1)
    out = {
        "names": np.array([p for p, _q in invs]),
        "queries": np.array(["Tennessee_query"] * len(invs)),
        "text_xz": np.frombuffer(lzma.compress(blob, preset=9), dtype=np.uint8),
        "text_off": offs,
        "stats": np.stack([r[0] for r in res]),
        "grid_digest": np.array([r[1] for r in res]),
        "ref_in": np.concatenate([np.packbits(r[2] == 2) for r in res]),
        "ref_zero": np.concatenate([np.nonzero(r[2] == 0)[0] for r in res] + [np.zeros(0, np.int64)]),
        "ref_zero_count": np.array([int((r[2] == 0).sum()) for r in res]),
        "exact_in": np.concatenate([np.packbits(r[3] == 2) for r in res]),
        "npoints": np.array([len(r[2]) for r in res]),
    }
    np.savez_compressed(os.path.join(HERE, "explist_tennessee.npz"), **out)
    print("wrote", len(invs), "Tennessee invocations;", sum(int((r[2] != r[3]).sum()) for r in res),
          "points where the reference and the exact oracle differ")


if __name__ == "__main__":
    if sys.argv[1:2] == ["--tennessee"]:
        main_tennessee(*sys.argv[2:])
    else:
        main(*sys.argv[1:])
