"""CPU checks: the oracle against what the reference ships, and product host
logic against the oracle (no GPU)."""
import ctypes
import re

import numpy as np
import pytest

from tests.golden.make_fixtures import POLYGONS


def test_grid0_product_equals_oracle(oracle_ref):
    import gahhg_b200 as G
    V, B, C = G.grid0()
    rV, rB, rC = oracle_ref.grid0()
    assert V.tobytes() == rV.tobytes()
    assert B.tobytes() == rB.tobytes()
    assert C.tobytes() == rC.tobytes()


def test_grid0_contract():
    """42 cells (12 pentagons, 30 hexagons), 80 vertices, 240 twin half-edges,
    inward normals (source/GPISPAHHG.cu:208-224 inside test)."""
    import gahhg_b200 as G
    V, B, C = G.grid0()
    assert len(C) == 42 and sorted(np.bincount(C["bnum"])[5:7]) == [12, 30]
    assert np.allclose(np.linalg.norm(V, axis=1), 1.0)
    assert (B["partner"] >= 0).all()
    assert (B["partner"][B["partner"]] == np.arange(240)).all()
    for k, c in enumerate(C):
        ring = B[c["bstart"]:c["bstart"] + c["bnum"]]
        center = V[ring["v"][:, 0]].mean(0)
        center /= np.linalg.norm(center)
        assert (np.einsum("ij,j->i", ring["n"], center) > 0).all()
        assert (ring["parent"] == k).all()
    # the cells cover the sphere: every random point is inside some cell
    rng = np.random.default_rng(0)
    p = rng.normal(size=(20000, 3))
    p /= np.linalg.norm(p, axis=1)[:, None]
    inside = np.zeros(len(p), bool)
    for c in C:
        ring = B[c["bstart"]:c["bstart"] + c["bnum"]]
        inside |= (p @ ring["n"].T >= -1e-8).all(1)
    assert inside.all()


def test_reference_cpu_space_pin(oracle_ref, inputs, tmp_path):
    """source/work/report.txt:8,10 pins depth 5 and 932 bytes for NA0."""
    r = oracle_ref.RefGPISP(inputs.polygon_file("various/NA0.txt", tmp_path))
    st = r.stats()
    assert st["gnum"] == 5
    assert st["cpu_space"] == 932
    assert oracle_ref.lib().ref_sizeof(3) + 28 * 5 == 932


def test_square72_reference_labels_closed_form(oracle_ref, inputs, tmp_path):
    """Square_72: the region left of four great circles through lat-18 vertices
    (test/polygon/various/Square_72.txt).  Away from the 1e-8 tolerance band
    the reference's labels must equal the closed form."""
    from tests.include_canon import query_xyz, vertex_xyz
    r = oracle_ref.RefGPISP(inputs.polygon_file("various/Square_72.txt", tmp_path))
    q = inputs.query("Square_72_query.csv")
    lab = r.query(q)
    verts = np.array([vertex_xyz(lo, 18.0) for lo in (-135.0, -45.0, 45.0, 135.0)])
    P = np.array([query_xyz(lo, la) for lo, la in q])
    # counter-clockwise seen from outside around the north pole
    s = np.stack([np.einsum("ij,j->i", P, np.cross(verts[i], verts[(i + 1) % 4])) for i in range(4)], 1)
    inside = (s > 0).all(1)
    margin = np.abs(s).min(1) > 1e-7
    assert margin.sum() > 9000
    assert np.array_equal(lab[margin] == 2, inside[margin])


def test_loader_matches_reference(oracle_ref, inputs, tmp_path):
    import gahhg_b200 as G
    for name in POLYGONS:
        path = inputs.polygon_file(name, tmp_path)
        P = G.Polygon.from_file(path)
        xyz, pe = P.export()
        r = oracle_ref.RefGPISP(path, maxdepth=1)
        rx, rp = r.polygon()
        assert np.array_equal(xyz, rx), name
        assert np.array_equal(pe, rp), name


@pytest.mark.parametrize("text,line,msg", [
    ("POLYGON 2 0\n0 5\n", 1, "Wrong format."),
    ("POLYGON 1 0\n0 3\n0 0\n1 0\n0 0\n", 2, "Number of edges should be greater than 3. "),
    ("POLYGON 1 0\n0 5\n0 0\n1 0\nx y\n0 1\n0 0\n", 5, "Wrong format."),
    ("POLYGON 1 1\n0 5\n0 0\n10 0\n10 10\n0 10\n0 0\n1 2\n", 8, "Number of edges should be greater than 3. "),
    ("POLYGON 1 1\n0 5\n0 0\n10 0\n10 10\n0 10\n0 0\n", 8, "Wrong format."),
])
def test_loader_errors_match_reference(text, line, msg, tmp_path, capfd, oracle_ref):
    import gahhg_b200 as G
    path = tmp_path / "bad.txt"
    path.write_text(text)
    with pytest.raises(G.GahhgError) as ei:
        G.Polygon.from_file(path)
    assert ei.value.status == -2
    out = capfd.readouterr().out
    want = "Error. Line %d of %s. %s\n" % (line, path, msg)
    assert want in out
    with pytest.raises(ValueError):
        oracle_ref.RefGPISP(path)
    assert want in capfd.readouterr().out


def test_points_loader_errors(tmp_path, capfd):
    import gahhg_b200 as G
    p = tmp_path / "q.csv"
    p.write_text("1.0,2.0\n3.0;4.0\n")
    with pytest.raises(G.GahhgError):
        G.load_points(p)
    assert "Error. Line 2 of %s. Wrong format.\n" % p in capfd.readouterr().out
    p.write_text("1.5,2.5\n-3.25, 4\n")
    q = G.load_points(p)
    assert q.tolist() == [[1.5, 2.5], [-3.25, 4.0]]
    with pytest.raises(G.GahhgError) as ei:
        G.load_points(tmp_path / "missing.csv")
    assert ei.value.status == -1


def test_c_abi_exports_every_declared_symbol():
    """libgahhg.so loads without a GPU and exports every function of include/gahhg.h."""
    import os
    from gahhg_b200 import _lib
    L = _lib.lib()
    hdr = open(os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "gahhg.h")).read()
    names = re.findall(r"\b(gahhg_[a-z0-9_]+)\s*\(", hdr)
    assert len(names) > 20
    for n in set(names):
        assert hasattr(L, n), n
    assert L.gahhg_abi_version() == 1


def test_batch_launch_shapes_listed_without_a_gpu():
    """The batch query's pass-1 launch shapes are a host table: the default
    first, each within the SM's resident-thread and shared-memory limits
    (256 threads and 32 KB per block), and an index past the end is refused."""
    import ctypes
    import gahhg_b200 as G
    from gahhg_b200 import _lib
    shapes = G.Batch.shapes()
    assert shapes[0] == (5, 5) and len(set(shapes)) == len(shapes) >= 4
    for u, blocks in shapes:
        assert 1 <= u <= 16 and blocks * 256 <= 2048 and blocks * 33 <= 227
    a, b = ctypes.c_int(), ctypes.c_int()
    assert _lib.lib().gahhg_batch_shape_info(len(shapes), ctypes.byref(a), ctypes.byref(b)) == _lib.ERR_ARG
    assert _lib.lib().gahhg_batch_shape_info(-1, ctypes.byref(a), ctypes.byref(b)) == _lib.ERR_ARG


def test_exact_oracle_agrees_with_reference_on_shipped_queries(oracle_ref, inputs, ref_outputs, tmp_path):
    """Away from the reference's tolerance band the two oracles must agree.
    Known exception: one Mars/001 query 5e-4 rad from the boundary that the
    reference's cell classification labels inside."""
    from oracle import exact
    known = {"Mars/001.txt": 1}
    for name in POLYGONS:
        qname = str(ref_outputs.get("pair", name)[0])
        q = inputs.query("uniform" if qname == "uniform" else qname)
        path = inputs.polygon_file(name, tmp_path)
        r = oracle_ref.RefGPISP(path, maxdepth=1)
        xyz, pe = r.polygon()
        r.close()
        e = exact.ExactPolygon(xyz, pe, len(inputs.rings_deg(name)[0]))
        lab = e.query_lonlat(q)
        want = ref_outputs.get("labels", name)
        assert int(((lab == 2) != (want == 2)).sum()) == known.get(name, 0), name


def test_knobs_host_side():
    """gahhg_set_knob: defaults, accepted ranges, refusals (host only)."""
    import gahhg_b200 as G
    assert G.get_knob(G.KNOB_GROUPED_PASS2) == 0
    assert G.get_knob(G.KNOB_WALK_STEP_LIMIT) == 1 << 16
    assert G.get_knob(G.KNOB_SCAN_SPIN_LIMIT) == 1 << 22
    assert G.get_knob(G.KNOB_STAGING_POLL_LIMIT) == 1 << 20
    for k, bad in [(G.KNOB_GROUPED_PASS2, 4), (G.KNOB_GROUPED_PASS2, -1), (G.KNOB_WALK_STEP_LIMIT, -1),
                   (G.KNOB_SCAN_SPIN_LIMIT, 1 << 23), (0, 1), (99, 1)]:
        with pytest.raises(G.GahhgError):
            G.set_knob(k, bad)
    for mode in (3, 2, 1, 0):
        G.set_knob(G.KNOB_GROUPED_PASS2, mode)
        assert G.get_knob(G.KNOB_GROUPED_PASS2) == mode
    old = G.set_knob(G.KNOB_WALK_STEP_LIMIT, 1)
    assert G.get_knob(G.KNOB_WALK_STEP_LIMIT) == 1
    G.set_knob(G.KNOB_WALK_STEP_LIMIT, old)
    assert G.get_knob(G.KNOB_WALK_STEP_LIMIT) == 1 << 16
