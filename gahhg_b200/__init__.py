"""gahhg_b200 - point-in-spherical-polygon tests on one NVIDIA B200.

Host-side mirror of the reference's objects (source/GPISPPolygon.cuh,
source/GPISPTP.cuh, source/GPISPAHHG.cuh) over the C ABI of libgahhg.so:

    poly = GPISPPolygon(); poly.loadPolyFromTXT("NA0.txt")
    tp = GPISPTP(); tp.loadTPFromCSV("query.csv")
    g = GPISP(poly, tp, semantics="reference")
    g.createAHHGInit(); g.createAHHG(15); g.classifyAHHG(); g.test()
    g.getStat(); g.exportStat2TXT("report.txt", 1); tp.exportResult2CSV("result.csv")

and a numpy-level API (Polygon, Grid) used by the tests and the benchmark.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import (BORDER_DTYPE, CELL_DTYPE, LEVEL_DTYPE, QUERY_AUTO, QUERY_FP32_FILTER,
                   QUERY_FP64_FILTER, QUERY_REFERENCE_FP64, SEMANTICS_EXACT, SEMANTICS_REFERENCE,
                   GahhgError, check)

CELL_UNDEFINED, CELL_OUT, CELL_IN = 0, 1, 2


class Polygon:
    """A loaded spherical polygon (rings re-oriented as the reference does)."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def from_file(cls, path):
        h = ctypes.c_void_p()
        check(_lib.lib().gahhg_polygon_load(str(path).encode(), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_rings(cls, rings):
        """rings: list of (k, 2) lon/lat arrays without closing vertex; ring 0 is outer."""
        ll = np.ascontiguousarray(np.concatenate([np.asarray(r, dtype=np.float64).reshape(-1, 2) for r in rings]))
        offs = np.zeros(len(rings) + 1, dtype=np.int64)
        offs[1:] = np.cumsum([len(r) for r in rings])
        h = ctypes.c_void_p()
        check(_lib.lib().gahhg_polygon_from_rings(_lib.ptr(ll), _lib.ptr(offs), len(rings), ctypes.byref(h)))
        return cls(h)

    @property
    def num_edges(self):
        return _lib.lib().gahhg_polygon_num_edges(self._h)

    def export(self):
        n = self.num_edges
        xyz = np.zeros((n, 3), dtype=np.float64)
        pe = np.zeros((n, 2), dtype=np.int32)
        check(_lib.lib().gahhg_polygon_export(self._h, _lib.ptr(xyz), _lib.ptr(pe)))
        return xyz, pe

    def __del__(self):
        # at interpreter exit the module's globals may already be gone; the
        # process is ending and frees the handle itself
        if getattr(self, "_h", None) and _lib is not None:
            _lib.lib().gahhg_polygon_free(self._h)
            self._h = None


def load_points(path, sidecar=False):
    """GPISPTP::loadTPFromCSV -> (n, 2) float64 lon/lat.  sidecar=True reads
    `<path>.f64` when it matches the CSV and writes it otherwise."""
    h = ctypes.c_void_p()
    L = _lib.lib()
    if sidecar:
        check(L.gahhg_points_load_ex(str(path).encode(), _lib.POINTS_USE_SIDECAR | _lib.POINTS_WRITE_SIDECAR,
                                     ctypes.byref(h)))
    else:
        check(L.gahhg_points_load(str(path).encode(), ctypes.byref(h)))
    n = L.gahhg_points_count(h)
    out = np.empty((n, 2), dtype=np.float64)
    if n:
        ctypes.memmove(out.ctypes.data, L.gahhg_points_lonlat(h), n * 16)
    L.gahhg_points_free(h)
    return out


class Grid:
    """The hexagon hierarchy (+ the exact-label lattice for exact semantics)."""

    def __init__(self, polygon, semantics=SEMANTICS_EXACT, max_depth=15, auto_depth=True, device=0,
                 verbose=False, lattice_top=0, lattice_leaf=0):
        L = _lib.lib()
        o = _lib.BuildOpts()
        L.gahhg_build_opts_init(ctypes.byref(o))
        o.max_depth = max_depth
        o.auto_depth = 1 if auto_depth else 0
        o.semantics = semantics
        o.device = device
        o.verbose = 1 if verbose else 0
        o.lattice_top = lattice_top
        o.lattice_leaf = lattice_leaf
        self.polygon = polygon  # the native grid keeps a pointer to it
        self.semantics = semantics
        h = ctypes.c_void_p()
        check(L.gahhg_build(polygon._h, ctypes.byref(o), ctypes.byref(h)))
        self._h = h

    def classify(self):
        check(_lib.lib().gahhg_classify(self._h))
        return self

    def query(self, lonlat, precision=QUERY_AUTO):
        ll = np.ascontiguousarray(np.asarray(lonlat, dtype=np.float64).reshape(-1, 2))
        out = np.zeros(len(ll), dtype=np.uint8)
        check(_lib.lib().gahhg_query(self._h, _lib.ptr(ll), len(ll), _lib.ptr(out), precision))
        return out

    def query_device(self, d_lonlat, n, d_labels, precision=QUERY_AUTO, stream=0, sync=False):
        """Device pointers (ints), e.g. from torch tensors' data_ptr()."""
        check(_lib.lib().gahhg_query_device(self._h, ctypes.c_void_p(d_lonlat), n, ctypes.c_void_p(d_labels),
                                            precision, ctypes.c_void_p(stream), 1 if sync else 0))

    def stats(self):
        s = _lib.Stats()
        check(_lib.lib().gahhg_stats_get(self._h, ctypes.byref(s)))
        return s.as_dict()

    @property
    def depth(self):
        return _lib.lib().gahhg_grid_depth(self._h)

    def export(self):
        """(levels, V, B, C, refs) as numpy arrays."""
        L = _lib.lib()
        d = self.depth
        lv = np.zeros(d, dtype=LEVEL_DTYPE)
        L.gahhg_grid_export(self._h, _lib.ptr(lv), None, None, None, None)
        last = lv[-1]
        nv = int(last["vstart"] + last["vnum"])
        nb = int(last["bstart"] + last["bnum"])
        nc = int(last["cstart"] + last["cnum"])
        nr = int(last["rnum"])
        V = np.zeros((nv, 3), dtype=np.float64)
        B = np.zeros(nb, dtype=BORDER_DTYPE)
        C = np.zeros(nc, dtype=CELL_DTYPE)
        R = np.zeros(max(nr, 1), dtype=np.int32)
        check(L.gahhg_grid_export(self._h, _lib.ptr(lv), _lib.ptr(V), _lib.ptr(B), _lib.ptr(C), _lib.ptr(R)))
        return lv, V, B, C, R[:nr]

    def report_append(self, polyfile, tpfile, npoints, path, to_stdout=False):
        check(_lib.lib().gahhg_report_append(self._h, str(polyfile).encode(), str(tpfile).encode(), npoints,
                                             str(path).encode(), 1 if to_stdout else 0))

    def __del__(self):
        # at interpreter exit the module's globals may already be gone; the
        # process is ending and frees the handle itself
        if getattr(self, "_h", None) and _lib is not None:
            _lib.lib().gahhg_grid_free(self._h)
            self._h = None


class Batch:
    """Exact indexes of many polygons, queried together (see gahhg_batch_* in
    include/gahhg.h)."""

    def __init__(self, polygons, device=0, top_cells=None, leaf_edges=None, workers=0, chunk_points=None):
        L = _lib.lib()
        o = _lib.BuildOpts()
        L.gahhg_build_opts_init(ctypes.byref(o))
        o.device = device
        self.polygons = list(polygons)
        arr = (ctypes.c_void_p * len(self.polygons))(*[p._h.value for p in self.polygons])
        tc = np.ascontiguousarray(top_cells, dtype=np.int32) if top_cells is not None else None
        le = np.ascontiguousarray(leaf_edges, dtype=np.int32) if leaf_edges is not None else None
        h = ctypes.c_void_p()
        check(L.gahhg_batch_build(arr, len(self.polygons), ctypes.byref(o), _lib.ptr(tc), _lib.ptr(le), workers,
                                  ctypes.byref(h)))
        self._h = h
        if chunk_points:
            check(L.gahhg_batch_set_chunk(h, chunk_points))

    @staticmethod
    def shapes():
        """The query's pass-1 launch shapes, by index: (points per thread,
        blocks per SM)."""
        L = _lib.lib()
        out = []
        a, b = ctypes.c_int(), ctypes.c_int()
        while L.gahhg_batch_shape_info(len(out), ctypes.byref(a), ctypes.byref(b)) == 0:
            out.append((a.value, b.value))
        return out

    def set_chunk(self, chunk_points):
        check(_lib.lib().gahhg_batch_set_chunk(self._h, chunk_points))

    def set_shape(self, shape):
        check(_lib.lib().gahhg_batch_set_shape(self._h, shape))

    def query_device(self, d_lonlat, offsets, d_labels, precision=QUERY_AUTO, stream=0, sync=False, graph=False):
        """d_lonlat / d_labels: device pointers; offsets: host int64 array (count+1)."""
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        assert len(off) == len(self.polygons) + 1
        self._off = off  # keep alive for the call
        L = _lib.lib()
        if graph:
            check(L.gahhg_batch_query_graph(self._h, ctypes.c_void_p(d_lonlat), _lib.ptr(off),
                                            ctypes.c_void_p(d_labels), precision, ctypes.c_void_p(stream)))
        else:
            check(L.gahhg_batch_query_device(self._h, ctypes.c_void_p(d_lonlat), _lib.ptr(off),
                                             ctypes.c_void_p(d_labels), precision, ctypes.c_void_p(stream),
                                             1 if sync else 0))

    def stats(self):
        s = _lib.BatchStats()
        check(_lib.lib().gahhg_batch_stats_get(self._h, ctypes.byref(s)))
        return s.as_dict()

    def __del__(self):
        # at interpreter exit the module's globals may already be gone; the
        # process is ending and frees the handle itself
        if getattr(self, "_h", None) and _lib is not None:
            _lib.lib().gahhg_batch_free(self._h)
            self._h = None


class Server:
    """A request loop over resident exact indexes (gahhg_server_* in
    include/gahhg.h): builds admitted by HBM footprint, queries batched
    continuously into in-flight slots, latency percentiles.

    Query buffers must stay alive and unmoved until the request completes;
    `query` keeps references to the numpy arrays it was given until then.
    """

    def __init__(self, device=0, slots=4, slot_points=1 << 22, max_pieces=4096, chunk_points=4096,
                 build_workers=4, max_polygons=65536, hbm_budget=0, evict_lru=False,
                 precision=QUERY_FP32_FILTER, direct_min_points=65536):
        L = _lib.lib()
        o = _lib.ServerOpts()
        L.gahhg_server_opts_init(ctypes.byref(o))
        o.device, o.slots, o.slot_points, o.max_pieces = device, slots, slot_points, max_pieces
        o.chunk_points, o.build_workers, o.max_polygons = chunk_points, build_workers, max_polygons
        o.hbm_budget, o.evict_lru, o.precision = int(hbm_budget), 1 if evict_lru else 0, precision
        o.direct_min_points = direct_min_points
        h = ctypes.c_void_p()
        check(L.gahhg_server_create(ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self._keep = {}

    def build(self, polygon, top_cells=0, leaf_edges=0, pinned=False, detached=False):
        """Queues a build; returns (polygon id, ticket)."""
        pid, tk = ctypes.c_int(), ctypes.c_int64()
        flags = (_lib.SERVE_PINNED if pinned else 0) | (_lib.SERVE_DETACHED if detached else 0)
        check(_lib.lib().gahhg_server_submit_build(self._h, polygon._h, int(top_cells), int(leaf_edges), flags,
                                                   ctypes.byref(pid), ctypes.byref(tk)))
        return pid.value, tk.value

    def query(self, pid, lonlat, labels=None, detached=False):
        """Queues a query of (n, 2) float64 lon/lat; returns (ticket, labels array)."""
        ll = np.asarray(lonlat)
        assert ll.dtype == np.float64 and ll.flags.c_contiguous and ll.ndim == 2 and ll.shape[1] == 2
        if labels is None:
            labels = np.empty(len(ll), dtype=np.uint8)
        assert labels.dtype == np.uint8 and labels.flags.c_contiguous and len(labels) >= len(ll)
        tk = ctypes.c_int64()
        check(_lib.lib().gahhg_server_submit_query(self._h, int(pid), ctypes.c_void_p(ll.ctypes.data), len(ll),
                                                   ctypes.c_void_p(labels.ctypes.data),
                                                   _lib.SERVE_DETACHED if detached else 0, ctypes.byref(tk)))
        if not detached:
            self._keep[tk.value] = (ll, labels)
        return tk.value, labels

    def query_raw(self, pid, ll_ptr, n, labels_ptr, detached=True):
        """Pointer form (the caller keeps the buffers alive); returns the ticket."""
        tk = ctypes.c_int64()
        check(_lib.lib().gahhg_server_submit_query(self._h, int(pid), ctypes.c_void_p(ll_ptr), int(n),
                                                   ctypes.c_void_p(labels_ptr),
                                                   _lib.SERVE_DETACHED if detached else 0, ctypes.byref(tk)))
        return tk.value

    def wait(self, ticket, timeout_s=60.0):
        st = _lib.lib().gahhg_server_wait(self._h, int(ticket), float(timeout_s))
        if st != _lib.ERR_STATE:
            self._keep.pop(ticket, None)
        check(st)

    def drain(self, timeout_s=120.0):
        check(_lib.lib().gahhg_server_drain(self._h, float(timeout_s)))

    def evict(self, pid):
        check(_lib.lib().gahhg_server_evict(self._h, int(pid)))

    def state(self, pid):
        st, b = ctypes.c_int(), ctypes.c_longlong()
        check(_lib.lib().gahhg_server_polygon_state(self._h, int(pid), ctypes.byref(st), ctypes.byref(b)))
        return st.value, b.value

    def stats(self):
        s = _lib.ServerStats()
        check(_lib.lib().gahhg_server_stats_get(self._h, ctypes.byref(s)))
        return s.as_dict()

    def reset_stats(self):
        check(_lib.lib().gahhg_server_stats_reset(self._h))

    def latencies(self, kind=0):
        L = _lib.lib()
        n = L.gahhg_server_latencies(self._h, kind, None, 0)
        out = np.zeros(n, dtype=np.float64)
        if n:
            L.gahhg_server_latencies(self._h, kind, _lib.ptr(out), n)
        return out

    def trace(self):
        """Per query batch: formed (s), host enqueue ms, device ms, completion
        ms after forming, points, pieces."""
        L = _lib.lib()
        n = L.gahhg_server_trace(self._h, None, 0)
        out = np.zeros((n, 6), dtype=np.float64)
        if n:
            L.gahhg_server_trace(self._h, _lib.ptr(out), n)
        return out

    def stalls(self):
        """Host-side stalls of 2 ms or more: start (s), kind, ms (kinds in include/gahhg.h)."""
        L = _lib.lib()
        n = L.gahhg_server_stalls(self._h, None, 0)
        out = np.zeros((n, 3), dtype=np.float64)
        if n:
            L.gahhg_server_stalls(self._h, _lib.ptr(out), n)
        return out

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().gahhg_server_free(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        self.close()


def write_result(path, labels):
    labels = np.ascontiguousarray(labels, dtype=np.uint8)
    check(_lib.lib().gahhg_result_write(str(path).encode(), _lib.ptr(labels), len(labels)))


def staging_fallbacks(device=0):
    """Blocks on `device` whose bulk copy into shared memory (the locate
    pass's coarse summary, or a staged tier-1 tile's edge lists) ran out of
    time and fell back to plain loads (0 in normal operation)."""
    v = ctypes.c_ulonglong(0)
    check(_lib.lib().gahhg_staging_fallbacks(int(device), ctypes.byref(v)))
    return int(v.value)


KNOB_GROUPED_PASS2 = 1
KNOB_WALK_STEP_LIMIT = 2
KNOB_SCAN_SPIN_LIMIT = 3
KNOB_STAGING_POLL_LIMIT = 4


def set_knob(knob, value):
    """Process-wide tuning/test knob (gahhg_set_knob); returns the old value."""
    old = get_knob(knob)
    check(_lib.lib().gahhg_set_knob(int(knob), int(value)))
    return old


def get_knob(knob):
    return int(_lib.lib().gahhg_get_knob(int(knob)))


def grid0():
    V = np.zeros((80, 3), dtype=np.float64)
    B = np.zeros(240, dtype=BORDER_DTYPE)
    C = np.zeros(42, dtype=CELL_DTYPE)
    check(_lib.lib().gahhg_grid0_export(_lib.ptr(V), _lib.ptr(B), _lib.ptr(C)))
    return V, B, C


# ---------------------------------------------------------------------------
# Mirror of the reference's host objects (names and call order of
# source/GPISP.cu:15-70 and source/GPISPAHHG.cuh:59-75).

class GPISPPolygon:
    def __init__(self):
        self.poly = None

    def loadPolyFromTXT(self, filename):
        """0 on success, -1 on failure (message printed), as the reference."""
        try:
            self.poly = Polygon.from_file(filename)
        except GahhgError:
            return -1
        self.filename = str(filename)
        return 0

    @property
    def pv_num(self):
        return self.poly.num_edges


class GPISPTP:
    def __init__(self):
        self.tp = None
        self.result = None

    def loadTPFromCSV(self, filename):
        try:
            self.tp = load_points(filename)
        except GahhgError:
            return -1
        self.filename = str(filename)
        return 0

    @property
    def tpNum(self):
        return 0 if self.tp is None else len(self.tp)

    def exportResult2CSV(self, filename):
        write_result(filename, self.result)


class GPISP:
    def __init__(self, polygon, tp, semantics=SEMANTICS_REFERENCE, precision=QUERY_AUTO):
        self.pPolygon = polygon
        self.pTP = tp
        self.semantics = semantics
        self.precision = precision
        self.grid = None
        self.maxDepth = 15

    def createAHHGInit(self):
        pass  # capacities and the level-0 grid are set up inside createAHHG

    def createAHHG(self, maxdepth=15):
        self.grid = Grid(self.pPolygon.poly, semantics=self.semantics, max_depth=maxdepth)

    def classifyAHHG(self):
        self.grid.classify()

    def test(self):
        self.pTP.result = self.grid.query(self.pTP.tp, self.precision)

    def getStat(self):
        self.stat = self.grid.stats()
        return self.stat

    def exportStat2TXT(self, filename, desttype=1):
        self.grid.report_append(self.pPolygon.filename, self.pTP.filename, self.pTP.tpNum, filename,
                                to_stdout=(desttype == 0))
