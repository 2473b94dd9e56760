"""Serving: resident indexes, builds admitted by HBM footprint, queries
batched continuously.

The central property: a request's labels are the same when it runs alone and
when it is batched with other requests (split across slots, mixed with other
polygons' points, overlapping builds), and they equal the single-polygon exact
path and the exact oracle.
"""
import threading

import numpy as np
import pytest

import gahhg_b200 as G
from gahhg_b200 import _lib, synth
from oracle import exact

pytestmark = pytest.mark.gpu


def _polygons(count=20, seed=21, vmax=20000):
    polys = synth.c3_polygons(count, seed=seed, vmax=vmax)
    rng = np.random.default_rng(seed)
    polys[0] = ([synth.star_ring(-60.0, -88.0, 400, 9.0, 0.2, rng)], (-60.0, -88.0), 9.0)  # south pole
    polys[1] = ([synth.star_ring(-179.8, 35.0, 700, 4.0, 0.2, rng), synth.star_ring(-179.8, 35.0, 60, 1.0, 0.0, rng)],
                (-179.8, 35.0), 4.0)  # antimeridian, one hole
    return polys


def _requests(polys, seed=22, sizes=(1, 3, 100, 4097, 30000, 200000)):
    """(polygon index, (n, 2) lon/lat) with points in the polygon's cap and
    some anywhere on the sphere."""
    rng = np.random.default_rng(seed)
    reqs = []
    for i, (rings, (lon, lat), radius) in enumerate(polys):
        for n in sizes:
            if n > 50000 and i % 4:
                continue
            k = max(1, n // 10)
            pts = np.concatenate([synth.cap_points(lon, lat, 1.8 * radius, n - k, rng) if n > k
                                  else np.zeros((0, 2)), synth.uniform_points(k, rng)])
            reqs.append((i, np.ascontiguousarray(pts[:n])))
    order = rng.permutation(len(reqs))
    return [reqs[j] for j in order]


@pytest.fixture(scope="module")
def serve_case():
    polys = _polygons()
    P = [G.Polygon.from_rings(r) for r, _c, _r in polys]
    reqs = _requests(polys)
    return polys, P, reqs


def _build_all(srv, P, pinned=True):
    built = [srv.build(p, pinned=pinned) for p in P]
    for _pid, tk in built:
        srv.wait(tk)
    return [pid for pid, _tk in built]


def test_alone_equals_mix(serve_case):
    import torch
    polys, P, reqs = serve_case
    # small slots force splitting and many batches; a low threshold sends the
    # page-locked requests around the staging copy
    srv = G.Server(slots=3, slot_points=1 << 16, max_pieces=64, chunk_points=1024, direct_min_points=2048)
    ids = _build_all(srv, P)
    # alone: one request at a time
    alone = []
    for i, pts in reqs:
        tk, lab = srv.query(ids[i], pts)
        srv.wait(tk)
        alone.append(lab.copy())
    assert srv.stats()["queries_done"] == len(reqs)
    # mixed: four client threads submit everything at once (some from
    # page-locked memory), while more polygons are being built
    pinned = {}
    for j, (i, pts) in enumerate(reqs):
        if j % 3 == 0 and len(pts) >= 2048:
            pinned[j] = (torch.from_numpy(pts).pin_memory(), torch.empty(len(pts), dtype=torch.uint8).pin_memory())
    mixed = [None] * len(reqs)
    errors = []

    def client(c):
        try:
            mine = []
            for j in range(c, len(reqs), 4):
                i, pts = reqs[j]
                if j in pinned:
                    t, lab_t = pinned[j]
                    lab_t.fill_(9)
                    tk = srv.query_raw(ids[i], t.data_ptr(), len(pts), lab_t.data_ptr(), detached=False)
                    mine.append((j, tk, lab_t.numpy()))
                else:
                    tk, lab = srv.query(ids[i], pts, labels=np.full(len(pts), 9, np.uint8))
                    mine.append((j, tk, lab))
            for j, tk, lab in mine:
                srv.wait(tk)
                mixed[j] = lab.copy()
        except Exception as e:  # surfaced below
            errors.append(e)

    extra = [G.Polygon.from_rings(r) for r, _c, _r in synth.c3_polygons(6, seed=23, vmax=30000)]
    th = [threading.Thread(target=client, args=(c,)) for c in range(4)]
    for t in th:
        t.start()
    extra_t = [srv.build(p)[1] for p in extra]
    for t in th:
        t.join()
    for tk in extra_t:
        srv.wait(tk)
    assert not errors, errors
    for j in range(len(reqs)):
        assert np.array_equal(alone[j], mixed[j]), "request %d differs alone vs mixed" % j
    st = srv.stats()
    assert st["batches"] > 0 and st["mean_batch_pieces"] > 1.0  # requests were batched together
    # the single-polygon exact path gives the same labels
    seen = set()
    for j, (i, pts) in enumerate(reqs):
        if i in seen or i > 6:
            continue
        seen.add(i)
        g = G.Grid(P[i], semantics=G.SEMANTICS_EXACT).classify()
        assert np.array_equal(g.query(pts, G.QUERY_FP32_FILTER), alone[j]), j
    # and the exact oracle, on the special polygons
    for j, (i, pts) in enumerate(reqs):
        if i in (0, 1) and len(pts) <= 30000:
            xyz, pe = P[i].export()
            want = exact.ExactPolygon(xyz, pe, len(polys[i][0][0])).query_lonlat(pts)
            assert np.array_equal(alone[j], want), j
    srv.close()


def test_queries_held_until_built(serve_case):
    polys, P, reqs = serve_case
    srv = G.Server(slots=2, slot_points=1 << 18)
    pid, btk = srv.build(P[3])
    _i, pts = next((i, p) for i, p in reqs if len(p) >= 4097)
    tk, lab = srv.query(pid, pts)  # submitted while the polygon is queued or building
    srv.wait(tk)
    srv.wait(btk)
    assert srv.state(pid)[0] == _lib.POLY_READY
    g = G.Grid(P[3], semantics=G.SEMANTICS_EXACT).classify()
    assert np.array_equal(lab, g.query(pts, G.QUERY_FP32_FILTER))
    srv.close()


def test_admission_and_eviction(serve_case):
    polys, P, reqs = serve_case
    poly = max(P, key=lambda p: p.num_edges)
    E = poly.num_edges
    # the measured footprint of one index of this polygon
    probe = G.Server(slots=1, slot_points=1 << 16)
    pid, tk = probe.build(poly)
    probe.wait(tk)
    b = probe.state(pid)[1]
    probe.close()
    assert b > 0
    first_estimate = 1.5 * 1024 * E + 32 * E  # before any build has been measured
    # room for about three indexes: every build is admitted, the least
    # recently used unpinned indexes make room
    budget = int(max(3 * b, 1.2 * first_estimate))
    srv = G.Server(slots=2, slot_points=1 << 18, hbm_budget=budget, evict_lru=True, build_workers=2)
    ids = []
    for _ in range(6):
        pid, tk = srv.build(poly)
        srv.wait(tk)
        ids.append(pid)
        st = srv.stats()
        assert st["resident_bytes"] <= st["hbm_budget"]
    st = srv.stats()
    assert st["evictions"] >= 1 and st["builds_done"] == 6
    assert srv.state(ids[-1])[0] == _lib.POLY_READY
    g = G.Grid(poly, semantics=G.SEMANTICS_EXACT).classify()
    pts = reqs[0][1]
    tk, lab = srv.query(ids[-1], pts)
    srv.wait(tk)
    assert np.array_equal(lab, g.query(pts, G.QUERY_FP32_FILTER))
    srv.close()
    # without eviction, a build that cannot fit while nothing can be freed
    # is refused on its ticket
    srv = G.Server(slots=1, slot_points=1 << 16, hbm_budget=int(1.2 * first_estimate), evict_lru=False,
                   build_workers=1)
    a, tka = srv.build(poly, pinned=True)
    srv.wait(tka)
    c, tkc = srv.build(poly)
    with pytest.raises(G.GahhgError) as e:
        srv.wait(tkc)
    assert e.value.status == _lib.ERR_CAPACITY
    assert srv.state(c)[0] == _lib.POLY_FAILED
    with pytest.raises(G.GahhgError):  # a query of a failed polygon is refused at submission
        srv.query(c, pts)
    srv.evict(a)  # an explicit eviction frees the memory and the id
    assert srv.stats()["resident_bytes"] == 0
    with pytest.raises(G.GahhgError):
        srv.query(a, pts)
    srv.close()


def test_eviction_waits_for_submitted_queries(serve_case):
    polys, P, reqs = serve_case
    srv = G.Server(slots=2, slot_points=1 << 16)
    pid, tk = srv.build(P[2])
    srv.wait(tk)
    g = G.Grid(P[2], semantics=G.SEMANTICS_EXACT).classify()
    big = [p for _i, p in reqs if len(p) >= 30000][:3]
    tks = [srv.query(pid, p) for p in big]
    srv.evict(pid)  # queries submitted before still complete with correct labels
    for (tk, lab), p in zip(tks, big):
        srv.wait(tk)
        assert np.array_equal(lab, g.query(p, G.QUERY_FP32_FILTER))
    assert srv.state(pid)[0] == _lib.POLY_FREE
    srv.close()


def test_stats_latencies_trace(serve_case):
    polys, P, reqs = serve_case
    srv = G.Server(slots=4, precision=G.QUERY_FP64_FILTER)
    ids = _build_all(srv, P[:5])
    srv.reset_stats()
    tks = [srv.query(ids[i % 5], pts) for i, pts in reqs[:40]]
    for tk, _lab in tks:
        srv.wait(tk)
    st = srv.stats()
    lat = srv.latencies(0)
    assert st["queries_done"] == 40 and len(lat) == 40
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    assert st["query_points"] == sum(len(p) for _i, p in reqs[:40])
    assert st["inflight_batches"] == 0 and st["pending_queries"] == 0
    tr = srv.trace()
    assert len(tr) == st["batches"] and tr[:, 4].sum() == st["query_points"]
    assert (tr[:, 2] > 0).all() and (tr[:, 3] >= tr[:, 1]).all()
    srv.close()
