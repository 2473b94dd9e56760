"""numpy restatement of include/gahhg_canon.h for CPU-side checks (uses libm
sin/cos, so agreement with the canonical functions is to ~1 ulp)."""
import math

PI_T = 3.14159265


def vertex_xyz(lon, lat):
    a = lat * PI_T / 180.0
    o = lon * PI_T / 180.0
    return (math.cos(a) * math.sin(o), math.sin(a), math.cos(a) * math.cos(o))


def query_xyz(lon, lat):
    f = lat + 90.0
    lat2 = 270.0 - f if f > 180.0 else f - 90.0
    return vertex_xyz(lon, lat2)
