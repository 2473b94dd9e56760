"""ctypes wrapper of oracle/_ref/libgahhg_ref.so (TEST INFRASTRUCTURE).

The reference's own GAHHG code built for the CPU by oracle/build_ref.py.
Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libgahhg_ref.so")
REF_EXE = os.path.join(HERE, "_ref", "gpisp_ref")

BORDER_DTYPE = np.dtype([("parent", "<i4"), ("partner", "<i4"), ("v", "<i4", 2), ("subcell", "<i4"),
                         ("id", "<i4"), ("n", "<f8", 3)])
CELL_DTYPE = np.dtype([("bstart", "<i4"), ("bnum", "<i4"), ("rstart", "<i4"), ("rnum", "<i4"),
                       ("upcell", "<i4"), ("subcell", "<i4"), ("type", "<i4")])
LEVEL_DTYPE = np.dtype([("vstart", "<i4"), ("vnum", "<i4"), ("bstart", "<i4"), ("bnum", "<i4"),
                        ("cstart", "<i4"), ("cnum", "<i4"), ("rnum", "<i4")])


class RefStats(ctypes.Structure):
    _fields_ = [("gnum", ctypes.c_int), ("pv_num", ctypes.c_int), ("vnum", ctypes.c_int),
                ("bnum", ctypes.c_int), ("cnum", ctypes.c_int), ("rnum", ctypes.c_int),
                ("cpu_space", ctypes.c_int), ("gpu_min_space", ctypes.c_int), ("gamma", ctypes.c_float),
                ("create_s", ctypes.c_double), ("classify_s", ctypes.c_double), ("query_s", ctypes.c_double),
                ("in_count", ctypes.c_int)]


_lib = None


def available():
    return os.path.exists(REF_LIB)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError("oracle/_ref/libgahhg_ref.so not built (python oracle/build_ref.py)")
        L = ctypes.CDLL(REF_LIB)
        P = ctypes.c_void_p
        L.ref_set_threads.argtypes = [ctypes.c_int, ctypes.c_int]
        L.ref_open.restype = P
        L.ref_open.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
        L.ref_query.argtypes = [P, P, ctypes.c_int, P]
        L.ref_stats_get.argtypes = [P, ctypes.POINTER(RefStats)]
        L.ref_grid_export.argtypes = [P, P, P, P, P, P]
        L.ref_polygon_export.argtypes = [P, P, P]
        L.ref_close.argtypes = [P]
        L.ref_grid0_export.argtypes = [P, P, P]
        L.ref_sizeof.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


class RefGPISP:
    """One polygon built and classified by the reference code on the CPU."""

    def __init__(self, polyfile, maxdepth=15, autodepth=True, threads=1, reverse=False):
        L = lib()
        L.ref_set_threads(threads, 1 if reverse else 0)
        h = L.ref_open(str(polyfile).encode(), maxdepth, 1 if autodepth else 0)
        if not h:
            raise ValueError("reference loader rejected %s" % polyfile)
        self._h = h
        self.threads = threads
        self.reverse = reverse

    def query(self, lonlat):
        L = lib()
        L.ref_set_threads(self.threads, 1 if self.reverse else 0)
        ll = np.ascontiguousarray(np.asarray(lonlat, dtype=np.float64).reshape(-1, 2))
        out = np.zeros(len(ll), dtype=np.int32)
        L.ref_query(self._h, _p(ll), len(ll), _p(out))
        return out

    def stats(self):
        s = RefStats()
        lib().ref_stats_get(self._h, ctypes.byref(s))
        return {k: getattr(s, k) for k, _ in s._fields_}

    def export(self):
        st = self.stats()
        g = st["gnum"]
        lv = np.zeros(g, dtype=LEVEL_DTYPE)
        V = np.zeros((st["vnum"], 3), dtype=np.float64)
        B = np.zeros(st["bnum"], dtype=BORDER_DTYPE)
        C = np.zeros(st["cnum"], dtype=CELL_DTYPE)
        R = np.zeros(max(st["rnum"], 1), dtype=np.int32)
        lib().ref_grid_export(self._h, _p(lv), _p(V), _p(B), _p(C), _p(R))
        return lv, V, B, C, R[:st["rnum"]]

    def polygon(self):
        n = self.stats()["pv_num"]
        xyz = np.zeros((n, 3), dtype=np.float64)
        pe = np.zeros((n, 2), dtype=np.int32)
        lib().ref_polygon_export(self._h, _p(xyz), _p(pe))
        return xyz, pe

    def close(self):
        if self._h:
            lib().ref_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def grid0():
    V = np.zeros((80, 3), dtype=np.float64)
    B = np.zeros(240, dtype=BORDER_DTYPE)
    C = np.zeros(42, dtype=CELL_DTYPE)
    lib().ref_grid0_export(_p(V), _p(B), _p(C))
    return V, B, C
