"""ctypes wrapper of the exact oracle (TEST INFRASTRUCTURE).

See oracle/exact_pip.c for the definitions of the exact labels, and
oracle/brute_gpu.cu for the same brute force run on a GPU (for point sets of
the benchmark configurations' size; points it cannot decide in FP64 go to
the CPU brute force).
"""
import ctypes
import os

import numpy as np

from . import build_oracle

_lib = None
_brute = None


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
        L.exact_poly_hub_sides.argtypes = [P, P, ctypes.c_int]
        _lib = L
    return _lib


def brute_lib():
    global _brute
    if _brute is None:
        path = build_oracle.BRUTE
        if not os.path.exists(path):
            path = build_oracle.build_brute()
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        L.brute_gpu_label.restype = ctypes.c_longlong
        L.brute_gpu_label.argtypes = [P, P, ctypes.c_int, P, P, P, P, ctypes.c_longlong, P, ctypes.c_int]
        L.brute_host_label.restype = ctypes.c_longlong
        L.brute_host_label.argtypes = [P, P, ctypes.c_int, P, P, P, P, ctypes.c_longlong, P]
        _brute = L
    return _brute


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

    def hub_sides(self, threads=os.cpu_count()):
        """orient(a_e, b_e, hub_k) for every edge e and hub k, (n, 6) int8."""
        if getattr(self, "_sides", None) is None:
            side = np.zeros((len(self.pe), 6), dtype=np.int8)
            lib().exact_poly_hub_sides(self._h, _p(side), threads)
            self._sides = side
        return self._sides

    def query_lonlat_gpu(self, lonlat, device=0, threads=os.cpu_count()):
        """The same labels as query_lonlat, by the GPU brute force
        (oracle/brute_gpu.cu); the points it leaves undecided are labelled by
        the CPU brute force.  Returns (labels, number of undecided points)."""
        ll = np.ascontiguousarray(np.asarray(lonlat, dtype=np.float64).reshape(-1, 2))
        out = np.zeros(len(ll), dtype=np.uint8)
        _x, hubs, hl, _e = self.info()
        side = self.hub_sides(threads)
        und = brute_lib().brute_gpu_label(_p(self.xyz), _p(self.pe), len(self.pe), _p(side),
                                          _p(np.ascontiguousarray(hubs)), _p(hl), _p(ll), len(ll), _p(out),
                                          device)
        if und < 0:
            raise RuntimeError("GPU brute force failed (CUDA error)")
        if und:
            idx = np.nonzero(out == 0)[0]
            out[idx] = self.query_lonlat(ll[idx], threads=threads)
        return out, int(und)

    def query_lonlat_brute_host(self, lonlat, threads=os.cpu_count()):
        """The GPU brute force's per-point steps run on the host (one thread):
        its labels, 0 where it is undecided (a check of its logic without a
        GPU).  Returns (labels, number of undecided points)."""
        ll = np.ascontiguousarray(np.asarray(lonlat, dtype=np.float64).reshape(-1, 2))
        out = np.zeros(len(ll), dtype=np.uint8)
        _x, hubs, hl, _e = self.info()
        side = self.hub_sides(threads)
        und = brute_lib().brute_host_label(_p(self.xyz), _p(self.pe), len(self.pe), _p(side),
                                           _p(np.ascontiguousarray(hubs)), _p(hl), _p(ll), len(ll), _p(out))
        return out, int(und)

    def arc_parity(self, p, q):
        p = np.ascontiguousarray(p, dtype=np.float64)
        q = np.ascontiguousarray(q, dtype=np.float64)
        return lib().exact_poly_arc_parity(self._h, _p(p), _p(q))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().exact_poly_free(self._h)
            self._h = None
