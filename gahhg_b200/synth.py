"""Seeded synthetic polygons and query points with the shapes of the
benchmark configurations (the reference's own query sets are not shipped and
no public dataset is involved).

C0  star polygon, 1,000 vertices at bearings 2 pi k / 1000 around (10E, 20N),
    radius 30 deg x (1 + U[-0.2, 0.2]); one 100-vertex hole of radius 5 deg at
    the center; 1e6 points uniform by area.
C1  1,000,000-vertex outer ring by midpoint displacement of a 64-gon of
    radius 60 deg around (170E, 70N) (amplitude halving per level, last level
    refined partially), so it crosses the antimeridian and contains the north
    pole; ten 10,000-vertex holes of radius U[1, 4] deg; 1e8 points uniform.
C2  the C1 polygon; half the points uniform, half on random edges offset
    along the edge normal by +-10^u rad, u ~ U[-15, -3].
C3  batch of polygons: vertex count log-uniform in [16, 200000] (fractal
    outer rings by midpoint displacement of a 16-gon with amplitude 10 % of
    the radius, star rings below 64 vertices), 0-8 holes (about 1/20 of the
    outer vertex count each, radius 5-15 % of the outer radius), radius
    log-uniform in [0.5, 40] deg, centers uniform on the sphere with about 5 %
    moved onto a pole; per polygon a log-uniform 1e3-1e6 points inside the
    1.5x bounding cap.

Rings are star-shaped around their center with monotonic bearings and radius
below 85 deg, so in the gnomonic projection at the center they are simple
polygons; holes lie inside the outer ring's minimum radius and do not overlap.
"""
import numpy as np

DEG = np.pi / 180.0


def destination(lon0, lat0, bearing, dist):
    """Points at angular distance `dist` (rad) along `bearing` (rad, clockwise
    from north) from (lon0, lat0) degrees -> (lon, lat) degrees."""
    la1, lo1 = lat0 * DEG, lon0 * DEG
    sl = np.sin(la1) * np.cos(dist) + np.cos(la1) * np.sin(dist) * np.cos(bearing)
    la2 = np.arcsin(np.clip(sl, -1.0, 1.0))
    lo2 = lo1 + np.arctan2(np.sin(bearing) * np.sin(dist) * np.cos(la1), np.cos(dist) - np.sin(la1) * sl)
    lon = (lo2 / DEG + 180.0) % 360.0 - 180.0
    return np.stack([lon, la2 / DEG], 1)


def star_ring(lon0, lat0, n, radius_deg, jitter, rng):
    theta = 2.0 * np.pi * np.arange(n) / n
    r = radius_deg * (1.0 + rng.uniform(-jitter, jitter, n)) if jitter else np.full(n, radius_deg)
    return destination(lon0, lat0, theta, r * DEG)


def uniform_points(n, rng):
    lon = rng.uniform(-180.0, 180.0, n)
    lat = np.arcsin(rng.uniform(-1.0, 1.0, n)) / DEG
    return np.stack([lon, lat], 1)


def cap_points(lon0, lat0, radius_deg, n, rng):
    """Uniform by area inside the cap of angular radius `radius_deg`."""
    c = rng.uniform(np.cos(min(radius_deg, 180.0) * DEG), 1.0, n)
    return destination(lon0, lat0, rng.uniform(0, 2 * np.pi, n), np.arccos(c))


def c0_polygon(seed=0):
    rng = np.random.default_rng(seed)
    outer = star_ring(10.0, 20.0, 1000, 30.0, 0.2, rng)
    hole = star_ring(10.0, 20.0, 100, 5.0, 0.0, rng)
    return [outer, hole]


def displaced_ring(lon0, lat0, n_target, r0_deg, base=64, amp_deg=6.0, rng=None):
    """Midpoint displacement in (bearing, radius) from a regular `base`-gon."""
    theta = 2.0 * np.pi * np.arange(base) / base
    r = np.full(base, r0_deg)
    amp = amp_deg
    while len(r) < n_target:
        m = len(r)
        k = min(m, n_target - m)  # the last level is refined partially
        tn = np.concatenate([theta[1:], [2 * np.pi]])
        rn = np.concatenate([r[1:], r[:1]])
        mid_t = 0.5 * (theta[:k] + tn[:k])
        mid_r = 0.5 * (r[:k] + rn[:k]) + rng.uniform(-amp, amp, k)
        nt = np.empty(m + k)
        nr = np.empty(m + k)
        idx = np.arange(k)
        nt[2 * idx] = theta[:k]
        nt[2 * idx + 1] = mid_t
        nr[2 * idx] = r[:k]
        nr[2 * idx + 1] = mid_r
        nt[2 * k:] = theta[k:]
        nr[2 * k:] = r[k:]
        theta, r = nt, nr
        amp *= 0.5
    return destination(lon0, lat0, theta, r * DEG), r


def c1_polygon(seed=1, n_outer=1_000_000, n_holes=10, hole_n=10_000):
    rng = np.random.default_rng(seed)
    outer, r = displaced_ring(170.0, 70.0, n_outer, 60.0, rng=rng)
    rmin = r.min()
    holes, centers = [], []
    while len(holes) < n_holes:
        hr = rng.uniform(1.0, 4.0)
        d = rng.uniform(0.0, rmin - hr - 2.0)
        c = destination(170.0, 70.0, np.array([rng.uniform(0, 2 * np.pi)]), np.array([d * DEG]))[0]
        ok = True
        for (cc, rr) in centers:
            if _angdist(c, cc) < hr + rr + 1.0:
                ok = False
                break
        if ok:
            centers.append((c, hr))
            holes.append(star_ring(c[0], c[1], hole_n, hr, 0.0, rng))
    return [outer] + holes


def _angdist(a, b):
    la1, lo1, la2, lo2 = a[1] * DEG, a[0] * DEG, b[1] * DEG, b[0] * DEG
    c = np.sin(la1) * np.sin(la2) + np.cos(la1) * np.cos(la2) * np.cos(lo1 - lo2)
    return np.arccos(np.clip(c, -1, 1)) / DEG


def near_edge_points(rings, n, rng, umin=-15.0, umax=-3.0):
    """Points on random edges offset along the edge normal by +-10^u rad."""
    ll = np.concatenate(rings)
    starts = np.cumsum([0] + [len(r) for r in rings])
    nxt = np.arange(len(ll)) + 1
    for a, b in zip(starts[:-1], starts[1:]):
        nxt[b - 1] = a
    xyz = _xyz(ll)
    e = rng.integers(0, len(ll), n)
    A, B = xyz[e], xyz[nxt[e]]
    t = rng.uniform(0.0, 1.0, n)[:, None]
    P = (1 - t) * A + t * B
    P /= np.linalg.norm(P, axis=1)[:, None]
    N = np.cross(A, B)
    N /= np.maximum(np.linalg.norm(N, axis=1), 1e-300)[:, None]
    off = 10.0 ** rng.uniform(umin, umax, n) * np.where(rng.random(n) < 0.5, -1.0, 1.0)
    Q = P + off[:, None] * N
    Q /= np.linalg.norm(Q, axis=1)[:, None]
    lat = np.arcsin(np.clip(Q[:, 1], -1, 1)) / DEG
    lon = np.arctan2(Q[:, 0], Q[:, 2]) / DEG
    return np.stack([lon, lat], 1)


def _xyz(ll):
    lo, la = ll[:, 0] * DEG, ll[:, 1] * DEG
    return np.stack([np.cos(la) * np.sin(lo), np.sin(la), np.cos(la) * np.cos(lo)], 1)


def c3_polygons(count=4096, seed=3, vmin=16, vmax=200_000):
    """List of (rings, center, radius_deg) for the batch configuration."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        nv = int(round(np.exp(rng.uniform(np.log(vmin), np.log(vmax)))))
        radius = float(np.exp(rng.uniform(np.log(0.5), np.log(40.0))))
        if rng.random() < 0.05:
            lat = (90.0 - 0.3 * radius) * (1 if rng.random() < 0.5 else -1)
            lon = rng.uniform(-180, 180)
        else:
            lon, lat = uniform_points(1, rng)[0]
        if nv < 64:
            outer = star_ring(lon, lat, nv, radius, 0.2, rng)
        else:
            # a fractal boundary like C1's: midpoint displacement of a 16-gon,
            # amplitude 10 % of the radius halving per level
            outer, _r = displaced_ring(lon, lat, nv, radius, base=16, amp_deg=0.1 * radius, rng=rng)
        rings = [outer]
        nh = int(rng.integers(0, 9))
        placed = []
        for _h in range(nh):
            hr = radius * rng.uniform(0.05, 0.15)
            d = rng.uniform(0, 0.75 * radius - hr)
            c = destination(lon, lat, np.array([rng.uniform(0, 2 * np.pi)]), np.array([d * DEG]))[0]
            if any(_angdist(c, pc) < hr + pr + 0.01 * radius for pc, pr in placed):
                continue
            placed.append((c, hr))
            rings.append(star_ring(c[0], c[1], max(4, nv // 20), hr, 0.0, rng))
        out.append((rings, (lon, lat), radius))
    return out


def c3_points(polys, seed=4, pmin=1_000, pmax=1_000_000, scale=1.0):
    rng = np.random.default_rng(seed)
    pts = []
    for rings, (lon, lat), radius in polys:
        n = int(round(np.exp(rng.uniform(np.log(pmin), np.log(pmax))) * scale))
        pts.append(cap_points(lon, lat, 1.5 * radius * 1.2, max(n, 1), rng))
    return pts


def write_polygon(path, rings):
    """POLYGON text file (README.md format): closing vertex repeated."""
    with open(path, "w") as f:
        f.write("POLYGON 1 %d\n" % (len(rings) - 1))
        for i, r in enumerate(rings):
            f.write("%d %d\n" % (0 if i == 0 else i, len(r) + 1))
            for lo, la in np.concatenate([r, r[:1]]):
                f.write("%.17g %.17g\n" % (lo, la))


def write_points(path, pts):
    with open(path, "w") as f:
        for lo, la in pts:
            f.write("%.17g,%.17g\n" % (lo, la))


# ---- the benchmark's point sets, generated on the device (torch) --------

def device_points(n, seed, device):
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    u = torch.rand((n, 2), generator=g, device=device, dtype=torch.float64)
    pts = torch.empty((n, 2), device=device, dtype=torch.float64)
    pts[:, 0] = u[:, 0] * 360.0 - 180.0
    pts[:, 1] = torch.rad2deg(torch.asin(u[:, 1] * 2.0 - 1.0))
    return pts


def device_c2_points(rings, n, seed, device):
    """C2 points on the device: half uniform by area, half on a uniform random
    edge at a uniform arc parameter, offset along the edge-plane normal by
    +-10^u rad with u ~ U[-15, -3] (the construction of synth.near_edge_points)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    ll = torch.as_tensor(np.concatenate(rings), dtype=torch.float64, device=device)
    starts = np.cumsum([0] + [len(r) for r in rings])
    nxt = np.arange(len(ll)) + 1
    for a, b in zip(starts[:-1], starts[1:]):
        nxt[b - 1] = a
    nxt = torch.as_tensor(nxt, device=device)
    lo, la = torch.deg2rad(ll[:, 0]), torch.deg2rad(ll[:, 1])
    xyz = torch.stack([torch.cos(la) * torch.sin(lo), torch.sin(la), torch.cos(la) * torch.cos(lo)], 1)
    pts = device_points(n, seed + 1, device)
    m = n // 2
    e = torch.randint(0, len(ll), (m,), generator=g, device=device)
    A, B = xyz[e], xyz[nxt[e]]
    t = torch.rand((m, 1), generator=g, device=device, dtype=torch.float64)
    P = (1 - t) * A + t * B
    P = P / torch.linalg.norm(P, dim=1, keepdim=True)
    N = torch.linalg.cross(A, B)
    N = N / torch.clamp(torch.linalg.norm(N, dim=1, keepdim=True), min=1e-300)
    u = torch.rand(m, generator=g, device=device, dtype=torch.float64) * 12.0 - 15.0
    sign = torch.where(torch.rand(m, generator=g, device=device) < 0.5, -1.0, 1.0).to(torch.float64)
    Q = P + (torch.pow(10.0, u) * sign)[:, None] * N
    Q = Q / torch.linalg.norm(Q, dim=1, keepdim=True)
    pts[m:, 1] = torch.rad2deg(torch.asin(torch.clamp(Q[:, 1], -1.0, 1.0)))
    pts[m:, 0] = torch.rad2deg(torch.atan2(Q[:, 0], Q[:, 2]))
    return pts


def device_cap_points(lons, lats, radii_deg, counts, seed, device):
    """Points uniform by area inside each polygon's cap (1.5 x the bounding
    radius 1.2 r of a star polygon of radius r), generated on the device."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    counts = np.asarray(counts, dtype=np.int64)
    n = int(counts.sum())
    pts = torch.empty((n, 2), dtype=torch.float64, device=device)
    lon_all = torch.as_tensor(lons, dtype=torch.float64, device=device) * (np.pi / 180)
    lat_all = torch.as_tensor(lats, dtype=torch.float64, device=device) * (np.pi / 180)
    R_all = torch.clamp(torch.as_tensor(radii_deg, dtype=torch.float64, device=device) * (1.5 * 1.2 * np.pi / 180),
                        max=np.pi)
    starts = np.concatenate([[0], np.cumsum(counts)])
    p0 = 0
    while p0 < len(counts):  # polygon ranges of about 32M points keep the temporaries small
        p1 = p0
        while p1 < len(counts) and (p1 == p0 or starts[p1 + 1] - starts[p0] <= (1 << 25)):
            p1 += 1
        cnt = torch.as_tensor(counts[p0:p1], dtype=torch.int64, device=device)
        idx = torch.repeat_interleave(torch.arange(p0, p1, device=device), cnt)
        m = int(starts[p1] - starts[p0])
        lon0, lat0, R = lon_all[idx], lat_all[idx], R_all[idx]
        u = torch.rand((m, 2), generator=g, device=device, dtype=torch.float64)
        c = torch.cos(R) + (1.0 - torch.cos(R)) * u[:, 0]
        d = torch.arccos(torch.clamp(c, -1.0, 1.0))
        b = u[:, 1] * 2 * np.pi
        sl = torch.sin(lat0) * torch.cos(d) + torch.cos(lat0) * torch.sin(d) * torch.cos(b)
        la2 = torch.asin(torch.clamp(sl, -1.0, 1.0))
        lo2 = lon0 + torch.atan2(torch.sin(b) * torch.sin(d) * torch.cos(lat0), torch.cos(d) - torch.sin(lat0) * sl)
        out = pts[starts[p0]:starts[p1]]
        out[:, 0] = torch.remainder(lo2 * (180 / np.pi) + 180.0, 360.0) - 180.0
        out[:, 1] = la2 * (180 / np.pi)
        del idx, lon0, lat0, R, u, c, d, b, sl, la2, lo2
        p0 = p1
    return pts
