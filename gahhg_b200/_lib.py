"""ctypes binding of libgahhg.so (include/gahhg.h).

The native library is the product; this module only declares its C ABI.  It
raises at import time when the library has not been built, so nothing can
silently run without the CUDA path.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgahhg.so")

OK = 0
ERR_IO = -1
ERR_FORMAT = -2
ERR_ARG = -3
ERR_CUDA = -4
ERR_DEVICE = -5
ERR_NOMEM = -6
ERR_STATE = -7
ERR_CAPACITY = -8

SEMANTICS_EXACT = 0
SEMANTICS_REFERENCE = 1

QUERY_AUTO = 0
QUERY_FP32_FILTER = 1
QUERY_FP64_FILTER = 2
QUERY_REFERENCE_FP64 = 3

# grid records (geom.cuh; layout of the reference's AHHGBorder / AHHGCell)
BORDER_DTYPE = np.dtype([("parent", "<i4"), ("partner", "<i4"), ("v", "<i4", 2), ("subcell", "<i4"),
                         ("id", "<i4"), ("n", "<f8", 3)])
CELL_DTYPE = np.dtype([("bstart", "<i4"), ("bnum", "<i4"), ("rstart", "<i4"), ("rnum", "<i4"),
                       ("upcell", "<i4"), ("subcell", "<i4"), ("type", "<i4")])
LEVEL_DTYPE = np.dtype([("vstart", "<i4"), ("vnum", "<i4"), ("bstart", "<i4"), ("bnum", "<i4"),
                        ("cstart", "<i4"), ("cnum", "<i4"), ("rnum", "<i4")])
assert BORDER_DTYPE.itemsize == 48 and CELL_DTYPE.itemsize == 28


class BuildOpts(ctypes.Structure):
    _fields_ = [("max_depth", ctypes.c_int), ("auto_depth", ctypes.c_int), ("semantics", ctypes.c_int),
                ("lattice_top", ctypes.c_int), ("lattice_leaf", ctypes.c_int), ("device", ctypes.c_int),
                ("verbose", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("depth", ctypes.c_int), ("pv_num", ctypes.c_int), ("vnum", ctypes.c_int),
                ("bnum", ctypes.c_int), ("cnum", ctypes.c_int), ("rnum", ctypes.c_int),
                ("cpu_space", ctypes.c_int), ("gpu_min_space", ctypes.c_int), ("gamma", ctypes.c_float),
                ("create_s", ctypes.c_double), ("classify_s", ctypes.c_double), ("pre_s", ctypes.c_double),
                ("lattice_s", ctypes.c_double), ("lattice_bytes", ctypes.c_longlong),
                ("query_s", ctypes.c_double), ("query_points", ctypes.c_longlong),
                ("in_count", ctypes.c_longlong), ("esc_fp64", ctypes.c_longlong),
                ("esc_exact", ctypes.c_longlong), ("boundary_points", ctypes.c_longlong),
                ("walk_limit_hits", ctypes.c_longlong), ("scan_fallbacks", ctypes.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchStats(ctypes.Structure):
    _fields_ = [("polygons", ctypes.c_int), ("workers", ctypes.c_int), ("edges", ctypes.c_longlong),
                ("lattice_bytes", ctypes.c_longlong), ("build_s", ctypes.c_double), ("query_s", ctypes.c_double),
                ("query_points", ctypes.c_longlong), ("boundary_points", ctypes.c_longlong),
                ("esc_fp64", ctypes.c_longlong), ("esc_exact", ctypes.c_longlong), ("in_count", ctypes.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerOpts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("slots", ctypes.c_int), ("slot_points", ctypes.c_longlong),
                ("max_pieces", ctypes.c_int), ("chunk_points", ctypes.c_int), ("build_workers", ctypes.c_int),
                ("max_polygons", ctypes.c_int), ("hbm_budget", ctypes.c_longlong), ("evict_lru", ctypes.c_int),
                ("precision", ctypes.c_int), ("direct_min_points", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    _fields_ = [("queries_done", ctypes.c_longlong), ("query_points", ctypes.c_longlong),
                ("builds_done", ctypes.c_longlong), ("builds_failed", ctypes.c_longlong),
                ("evictions", ctypes.c_longlong), ("batches", ctypes.c_longlong), ("pieces", ctypes.c_longlong),
                ("resident_polygons", ctypes.c_int), ("pending_queries", ctypes.c_int),
                ("pending_builds", ctypes.c_int), ("inflight_batches", ctypes.c_int),
                ("resident_bytes", ctypes.c_longlong), ("hbm_budget", ctypes.c_longlong),
                ("window_s", ctypes.c_double), ("points_per_s", ctypes.c_double),
                ("p50_ms", ctypes.c_double), ("p90_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("max_ms", ctypes.c_double), ("build_p50_ms", ctypes.c_double), ("build_p99_ms", ctypes.c_double),
                ("mean_batch_points", ctypes.c_double), ("mean_batch_pieces", ctypes.c_double),
                ("boundary_points", ctypes.c_longlong), ("esc_fp64", ctypes.c_longlong),
                ("esc_exact", ctypes.c_longlong), ("in_count", ctypes.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


POINTS_USE_SIDECAR = 1
POINTS_WRITE_SIDECAR = 2

SERVE_PINNED = 1
SERVE_DETACHED = 2
POLY_FREE, POLY_QUEUED, POLY_BUILDING, POLY_READY, POLY_FAILED, POLY_EVICTING = range(6)

# name: (restype, argtypes)
_P = ctypes.c_void_p
_SIGS = {
    "gahhg_build_opts_init": (None, [ctypes.POINTER(BuildOpts)]),
    "gahhg_last_error": (ctypes.c_char_p, []),
    "gahhg_abi_version": (ctypes.c_int, []),
    "gahhg_staging_fallbacks": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong)]),
    "gahhg_set_knob": (ctypes.c_int, [ctypes.c_int, ctypes.c_longlong]),
    "gahhg_get_knob": (ctypes.c_longlong, [ctypes.c_int]),
    "gahhg_polygon_load": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_P)]),
    "gahhg_polygon_from_rings": (ctypes.c_int, [_P, _P, ctypes.c_int, ctypes.POINTER(_P)]),
    "gahhg_polygon_num_edges": (ctypes.c_int, [_P]),
    "gahhg_polygon_export": (ctypes.c_int, [_P, _P, _P]),
    "gahhg_polygon_free": (None, [_P]),
    "gahhg_points_load": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_P)]),
    "gahhg_points_load_ex": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(_P)]),
    "gahhg_points_count": (ctypes.c_size_t, [_P]),
    "gahhg_points_lonlat": (_P, [_P]),
    "gahhg_points_free": (None, [_P]),
    "gahhg_build": (ctypes.c_int, [_P, ctypes.POINTER(BuildOpts), ctypes.POINTER(_P)]),
    "gahhg_classify": (ctypes.c_int, [_P]),
    "gahhg_grid_free": (None, [_P]),
    "gahhg_query_device": (ctypes.c_int, [_P, _P, ctypes.c_size_t, _P, ctypes.c_int, _P, ctypes.c_int]),
    "gahhg_query": (ctypes.c_int, [_P, _P, ctypes.c_size_t, _P, ctypes.c_int]),
    "gahhg_query_device_noalloc": (ctypes.c_int, [_P, _P, ctypes.c_size_t, _P, ctypes.c_int, _P]),
    "gahhg_query_noalloc_max_points": (ctypes.c_longlong, []),
    "gahhg_stats_get": (ctypes.c_int, [_P, ctypes.POINTER(Stats)]),
    "gahhg_grid_depth": (ctypes.c_int, [_P]),
    "gahhg_grid_export": (ctypes.c_int, [_P, _P, _P, _P, _P, _P]),
    "gahhg_report_append": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_longlong,
                                           ctypes.c_char_p, ctypes.c_int]),
    "gahhg_result_write": (ctypes.c_int, [ctypes.c_char_p, _P, ctypes.c_size_t]),
    "gahhg_grid0_export": (ctypes.c_int, [_P, _P, _P]),
    "gahhg_batch_build": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(BuildOpts), _P, _P, ctypes.c_int,
                                         ctypes.POINTER(_P)]),
    "gahhg_batch_size": (ctypes.c_int, [_P]),
    "gahhg_batch_set_chunk": (ctypes.c_int, [_P, ctypes.c_int]),
    "gahhg_batch_shape_info": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(ctypes.c_int)]),
    "gahhg_batch_set_shape": (ctypes.c_int, [_P, ctypes.c_int]),
    "gahhg_batch_query_device": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_int, _P, ctypes.c_int]),
    "gahhg_batch_query_graph": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_int, _P]),
    "gahhg_batch_stats_get": (ctypes.c_int, [_P, ctypes.POINTER(BatchStats)]),
    "gahhg_batch_free": (None, [_P]),
    "gahhg_server_opts_init": (None, [ctypes.POINTER(ServerOpts)]),
    "gahhg_server_create": (ctypes.c_int, [ctypes.POINTER(ServerOpts), ctypes.POINTER(_P)]),
    "gahhg_server_submit_build": (ctypes.c_int, [_P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                 ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int64)]),
    "gahhg_server_submit_query": (ctypes.c_int, [_P, ctypes.c_int, _P, ctypes.c_int64, _P, ctypes.c_int,
                                                 ctypes.POINTER(ctypes.c_int64)]),
    "gahhg_server_wait": (ctypes.c_int, [_P, ctypes.c_int64, ctypes.c_double]),
    "gahhg_server_drain": (ctypes.c_int, [_P, ctypes.c_double]),
    "gahhg_server_evict": (ctypes.c_int, [_P, ctypes.c_int]),
    "gahhg_server_polygon_state": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                                  ctypes.POINTER(ctypes.c_longlong)]),
    "gahhg_server_stats_get": (ctypes.c_int, [_P, ctypes.POINTER(ServerStats)]),
    "gahhg_server_stats_reset": (ctypes.c_int, [_P]),
    "gahhg_server_latencies": (ctypes.c_longlong, [_P, ctypes.c_int, _P, ctypes.c_longlong]),
    "gahhg_server_trace": (ctypes.c_longlong, [_P, _P, ctypes.c_longlong]),
    "gahhg_server_stalls": (ctypes.c_longlong, [_P, _P, ctypes.c_longlong]),
    "gahhg_server_free": (None, [_P]),
}

_lib = None


def lib():
    """Load libgahhg.so once; raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libgahhg.so is not built: run `python gahhg_b200/build.py` "
                              "(or __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def declared_symbols():
    return list(_SIGS)


class GahhgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("gahhg status %d: %s" % (status, msg))
        self.status = status


def check(status):
    if status != OK:
        raise GahhgError(status, lib().gahhg_last_error().decode(errors="replace"))
    return status


def ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None
