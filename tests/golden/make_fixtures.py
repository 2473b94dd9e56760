"""Generate tests/golden/*.npz from the reference's shipped test data.

Run in a container that has the reference checkout (default /root/reference)
and the CPU build of the reference (python oracle/build_ref.py):

    python tests/golden/make_fixtures.py [/path/to/reference]

Writes
  shipped_inputs.npz   a subset of test/polygon/** and test/query/*.csv,
                       coordinates as integer micro-degrees (every shipped
                       coordinate has exactly six decimals, checked here), so
                       tests/golden/fixtures.py re-creates the files byte for
                       byte on a machine without the reference;
  reference_outputs.npz  what the reference code (built for the CPU, run
                       serially) produces on those inputs: labels per
                       (polygon, query) pair, grid statistics, and SHA-256
                       digests of the grid arrays.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

POLYGONS = [
    "various/Square_72.txt", "various/Radiometer.txt", "various/NA0.txt", "various/NA2.txt",
    "various/Antarctic.txt", "various/Tennessee.txt",
    "Mars/001.txt", "Mars/017.txt", "Mars/100.txt", "Mars/250.txt", "Mars/400.txt", "Mars/624.txt",
    "Tennessee/Tennessee_00005.txt", "Tennessee/Tennessee_03990.txt", "Tennessee/Tennessee_11990.txt",
    "Tennessee/Tennessee_20000.txt",
]
QUERIES = ["Square_72_query.csv", "Radiometer_query.csv", "Mars_query.csv", "Tennessee_query.csv"]
# polygon -> query file, as test/explist.bat pairs them; NA0/NA2/Antarctic use a
# seeded uniform sample (their query files are not shipped)
PAIRS = {
    "various/Square_72.txt": "Square_72_query.csv",
    "various/Radiometer.txt": "Radiometer_query.csv",
    "various/Tennessee.txt": "Tennessee_query.csv",
}


def _key(name):
    return name.replace("/", "__").replace(".txt", "").replace(".csv", "")


def _micro(tok):
    """'-83.918080' -> -83918080, insisting on exactly six decimals."""
    neg = tok.startswith("-")
    t = tok[1:] if neg else tok
    whole, frac = t.split(".")
    assert len(frac) == 6, tok
    v = int(whole) * 1000000 + int(frac)
    return -v if neg else v


def read_polygon_text(path):
    with open(path, "rb") as f:
        lines = f.read().decode().splitlines()
    header = lines[0].split()
    nholes = int(header[2])
    pos = 1
    rings, heads = [], []
    for r in range(nholes + 1):
        a, b = lines[pos].split()
        heads.append((int(a), int(b)))
        pos += 1
        pts = []
        for _ in range(int(b)):
            lo, la = lines[pos].split()
            pts.append((_micro(lo), _micro(la)))
            pos += 1
        rings.append(np.array(pts, dtype=np.int64))
    return heads, rings


def read_query_text(path):
    with open(path, "rb") as f:
        rows = [ln.split(",") for ln in f.read().decode().splitlines() if ln.strip()]
    return np.array([(_micro(a), _micro(b)) for a, b in rows], dtype=np.int64)


def uniform_points(n, seed):
    rng = np.random.default_rng(seed)
    lon = rng.uniform(-180.0, 180.0, n)
    lat = np.degrees(np.arcsin(rng.uniform(-1.0, 1.0, n)))
    return np.round(np.stack([lon, lat], 1) * 1e6).astype(np.int64)


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main(refroot=None):
    refroot = refroot or os.environ.get("GAHHG_REFERENCE", "/root/reference")
    from tests.golden import fixtures
    from oracle import ref

    inputs = {}
    for p in POLYGONS:
        heads, rings = read_polygon_text(os.path.join(refroot, "test/polygon", p))
        k = _key(p)
        inputs["poly_" + k + "_heads"] = np.array(heads, dtype=np.int64)
        for i, r in enumerate(rings):
            inputs["poly_%s_ring%d" % (k, i)] = r
    for q in QUERIES:
        inputs["query_" + _key(q)] = read_query_text(os.path.join(refroot, "test/query", q))
    inputs["query_uniform"] = uniform_points(20000, 1234)
    np.savez_compressed(os.path.join(HERE, "shipped_inputs.npz"), **inputs)

    # the regenerated text must equal the shipped files byte for byte
    import tempfile
    tmp = tempfile.mkdtemp()
    store = fixtures.Inputs(os.path.join(HERE, "shipped_inputs.npz"))
    for p in POLYGONS:
        path = store.polygon_file(p, tmp)
        with open(path, "rb") as a, open(os.path.join(refroot, "test/polygon", p), "rb") as b:
            ta, tb = a.read(), b.read()
            assert ta.replace(b"\r\n", b"\n").rstrip() == tb.replace(b"\r\n", b"\n").rstrip(), p

    outputs = {}
    for p in POLYGONS:
        path = store.polygon_file(p, tmp)
        R = ref.RefGPISP(path, threads=1)
        st = R.stats()
        lv, V, B, C, refs = R.export()
        k = _key(p)
        outputs["stats_" + k] = np.array([st["gnum"], st["vnum"], st["bnum"], st["cnum"], st["rnum"],
                                          st["cpu_space"], st["gpu_min_space"]], dtype=np.int64)
        outputs["gamma_" + k] = np.array([st["gamma"]], dtype=np.float32)
        outputs["digest_grid_" + k] = np.array([digest(lv, V, B, C, refs)])
        qname = PAIRS.get(p)
        if qname is None:
            qname = "Mars_query.csv" if p.startswith("Mars/") else (
                "Tennessee_query.csv" if p.startswith("Tennessee/") else "uniform")
        q = store.query("uniform" if qname == "uniform" else qname)
        outputs["labels_" + k] = R.query(q).astype(np.uint8)
        outputs["pair_" + k] = np.array([qname])
        R.close()
    np.savez_compressed(os.path.join(HERE, "reference_outputs.npz"), **outputs)
    print("wrote", len(inputs), "input arrays and", len(outputs), "output arrays")


if __name__ == "__main__":
    main(*sys.argv[1:])
