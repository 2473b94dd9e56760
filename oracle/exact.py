"""ctypes wrapper of the exact oracle (TEST INFRASTRUCTURE).

See oracle/exact_pip.c for the definitions of the exact labels.
"""
import ctypes
import os

import numpy as np

from . import build_oracle

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = build_oracle.OUT
        if not os.path.exists(path):
            path = build_oracle.build()
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        L.exact_poly_new.restype = P
        L.exact_poly_new.argtypes = [P, P, ctypes.c_int, ctypes.c_int]
        L.exact_poly_free.argtypes = [P]
        L.exact_poly_info.argtypes = [P, P, P, P, P]
        L.exact_poly_query_xyz.argtypes = [P, P, ctypes.c_long, P, ctypes.c_int]
        L.exact_poly_query_lonlat.argtypes = [P, P, ctypes.c_long, P, ctypes.c_int]
        L.exact_poly_arc_parity.argtypes = [P, P, P]
        L.oracle_orient.argtypes = [P, P, P]
        L.oracle_orient_nosos.argtypes = [P, P, P]
        L.oracle_crossing.argtypes = [P, P, P, P]
        L.oracle_canon_query_xyz.argtypes = [P, ctypes.c_long, P]
        L.oracle_canon_vertex_xyz.argtypes = [P, ctypes.c_long, P]
        _lib = L
    return _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def orient(a, b, c, sos=True):
    a, b, c = (np.ascontiguousarray(x, dtype=np.float64) for x in (a, b, c))
    f = lib().oracle_orient if sos else lib().oracle_orient_nosos
    return f(_p(a), _p(b), _p(c))


def query_xyz(lonlat):
    ll = np.ascontiguousarray(np.asarray(lonlat, dtype=np.float64).reshape(-1, 2))
    out = np.zeros((len(ll), 3))
    lib().oracle_canon_query_xyz(_p(ll), len(ll), _p(out))
    return out


def vertex_xyz(lonlat):
    ll = np.ascontiguousarray(np.asarray(lonlat, dtype=np.float64).reshape(-1, 2))
    out = np.zeros((len(ll), 3))
    lib().oracle_canon_vertex_xyz(_p(ll), len(ll), _p(out))
    return out


class ExactPolygon:
    """Exact labels for a polygon given as canonical XYZ vertices + oriented edges
    (e.g. gahhg_b200.Polygon.export()); n_outer = number of outer-ring edges."""

    def __init__(self, xyz, pe, n_outer=None):
        self.xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        self.pe = np.ascontiguousarray(pe, dtype=np.int32)
        n = len(self.pe)
        self._h = lib().exact_poly_new(_p(self.xyz), _p(self.pe), n, n if n_outer is None else n_outer)
        if not self._h:
            raise ValueError("no usable reference edge on the outer ring")

    def info(self):
        x = np.zeros(3)
        hubs = np.zeros((6, 3))
        hl = np.zeros(6, dtype=np.int32)
        e = ctypes.c_int()
        lib().exact_poly_info(self._h, _p(x), _p(hubs), _p(hl), ctypes.byref(e))
        return x, hubs, hl, e.value

    def query_lonlat(self, lonlat, threads=os.cpu_count()):
        ll = np.ascontiguousarray(np.asarray(lonlat, dtype=np.float64).reshape(-1, 2))
        out = np.zeros(len(ll), dtype=np.uint8)
        lib().exact_poly_query_lonlat(self._h, _p(ll), len(ll), _p(out), threads)
        return out

    def query_xyz(self, xyz, threads=os.cpu_count()):
        q = np.ascontiguousarray(np.asarray(xyz, dtype=np.float64).reshape(-1, 3))
        out = np.zeros(len(q), dtype=np.uint8)
        lib().exact_poly_query_xyz(self._h, _p(q), len(q), _p(out), threads)
        return out

    def arc_parity(self, p, q):
        p = np.ascontiguousarray(p, dtype=np.float64)
        q = np.ascontiguousarray(q, dtype=np.float64)
        return lib().exact_poly_arc_parity(self._h, _p(p), _p(q))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().exact_poly_free(self._h)
            self._h = None
