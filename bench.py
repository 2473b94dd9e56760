"""Benchmark: exact-label point-in-spherical-polygon queries on one B200.

Workload (C1): one polygon with a 1,000,000-vertex outer ring (midpoint
displacement of a 64-gon of radius 60 deg around 170E 70N, crossing the
antimeridian and containing the north pole) and ten 10,000-vertex holes;
1e8 FP64 lon/lat query points uniform by area, generated on the device
(seeded).  A step = one query pass over all points.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is the FP32-filtered exact query rate with inputs resident in HBM
(1.6 GB, larger than L2), timed with CUDA events on the launching stream;
`e2e` is the same metric through the public C ABI (gahhg_query) with pinned
host buffers, host->device and device->host copies inside the timed region.
With N > 1 (torchrun) each rank queries its own replica (the path shards by
points, with no exchange); the slowest rank's time is used.

At N = 1 the same line carries the other configurations as keys (skipped
with --no-legs): "c2" (the C1 polygon's index on 2e7 points, half within
10^U[-15,-3] rad of an edge: FP32-filtered and FP64-filtered rates and
escalation fractions), "c3" (a batch of 1,024 batch-configuration polygons,
autotuned, CUDA-graph replay) and "c4" (10 s of serving at 2,000 requests/s
over those 1,024 polygons: p50/p99 latency and sustained points/s).
--config c2|c3|c4 runs one configuration alone at full size.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "query Mpts/s (FP32-filter vs FP64, exact labels), grid build ms, serve p99"
BYTES_PER_POINT = 17  # 16 B lon/lat in + 1 B label out
REF_DEPTH_C1 = 11     # deepest level at which the reference's edge walks terminate on C1


def _traffic_per_point():
    """DRAM bytes per point of the query kernel from the committed ncu summary."""
    try:
        with open(os.path.join(REPO, "profiles", "locate_traffic.json")) as f:
            return float(json.load(f)["bytes_per_point"])
    except Exception:
        return None


def _peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def gpu_uuid(local):
    """nvidia-smi id of the GPU this process uses: its UUID (nvidia-smi's own
    indices ignore CUDA_VISIBLE_DEVICES, so a local ordinal may name another
    job's GPU)."""
    try:
        import torch
        u = str(torch.cuda.get_device_properties(local).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return str(local)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs
    (read-only queries of the GPU given by its UUID)."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local):
        self.index = gpu_uuid(local)
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "gpu": self.index}


class quiet_stdout:
    """Route C-level stdout to stderr (the reference code prints progress
    lines) so that stdout carries only the JSON result line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        try:
            import ctypes as _c
            _c.CDLL(None).fflush(None)
        except Exception:
            pass
        os.dup2(self.saved, 1)
        os.close(self.saved)
        return False


def c1_polygon_cached():
    """The C1 polygon (generated in under a second; kept for the process)."""
    global _C1_RINGS
    if _C1_RINGS is None:
        from gahhg_b200 import synth
        _C1_RINGS = synth.c1_polygon()
    return _C1_RINGS


_C1_RINGS = None


def timed_loop(fn, steps, stream):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) * 1e-3


def cpu_reference_rate(rings, sample_points, threads, budget_s=12.0):
    """The reference's own GAHHG code built for the CPU (oracle/_ref), all host
    threads, on a bounded sample of the workload; returns (Mpts/s, info)."""
    from oracle import ref
    from gahhg_b200 import synth
    if not ref.available():
        return None, "oracle/_ref not built"
    tmp = os.path.join("/tmp", "gahhg_bench_c1_%d.txt" % os.getpid())
    synth.write_polygon(tmp, rings)
    with quiet_stdout():
        t0 = time.time()
        r = ref.RefGPISP(tmp, maxdepth=REF_DEPTH_C1, threads=threads)
        build_s = time.time() - t0
        done, t1 = 0, time.time()
        while time.time() - t1 < budget_s:
            r.query(sample_points)
            done += len(sample_points)
        dt = time.time() - t1
        r.close()
    os.unlink(tmp)
    return done / dt / 1e6, {"build_s": round(build_s, 3), "points": done, "seconds": round(dt, 3)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from gahhg_b200 import synth
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (reference built for the CPU) missing"}))
        return 0
    threads = os.cpu_count()
    rings = c1_polygon_cached()
    tmp = os.path.join("/tmp", "gahhg_bench_ref_%d.txt" % os.getpid())
    synth.write_polygon(tmp, rings)
    with quiet_stdout():
        t0 = time.time()
        r = ref.RefGPISP(tmp, maxdepth=REF_DEPTH_C1, threads=threads)
        build_s = time.time() - t0
        sample = synth.uniform_points(args.ref_sample, np.random.default_rng(0))
        for _ in range(args.warmup):
            r.query(sample)
        t1 = time.time()
        for _ in range(args.steps):
            r.query(sample)
        dt = time.time() - t1
        r.close()
    os.unlink(tmp)
    rate = args.steps * len(sample) / dt / 1e6
    desc = ("reference GAHHG kernels built for the CPU (oracle/_ref), OpenMP over %d threads, maxDepth %d; "
            "each step queries %d of the 1e8 C1 points" % (threads, REF_DEPTH_C1, len(sample)))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(rate, 3), "unit": "Mpts/s", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "C1: 1.1M-edge polygon, uniform FP64 lon/lat points (sampled)",
                   "points_per_step": len(sample), "max_depth": REF_DEPTH_C1},
        "cpu_baseline": {"value": round(rate, 3), "unit": "Mpts/s", "cores": threads, "kind": "reference",
                         "sample": desc},
        "build_ms": round(build_s * 1e3, 1),
        "e2e": {"value": round(rate, 3), "unit": "Mpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


def run_c3(args, count=None, tune_budget=None, steps=None, polys=None):
    """Batch configuration: 4,096 star polygons (16-200,000 vertices, 0-8
    holes, radius 0.5-40 deg, ~5 % around a pole), each with 1e3-1e6 points
    inside its 1.5x bounding cap; autotuned lattices; one CUDA-graph query
    over all points per step.  `count` polygons of that generator (default
    --c3-polygons); returns the result line as a dict (and the polygons)."""
    import torch
    import gahhg_b200 as G
    from gahhg_b200 import autotune, synth
    dev = "cuda:0"
    t0 = time.time()
    if polys is None:
        polys = synth.c3_polygons(count or args.c3_polygons, seed=3)
    P = [G.Polygon.from_rings(r) for r, _c, _r in polys]
    gen_s = time.time() - t0
    rng = np.random.default_rng(4)
    counts = np.maximum(1, np.round(np.exp(rng.uniform(np.log(1e3), np.log(1e6), len(polys))) *
                                    args.c3_scale)).astype(np.int64)
    offsets = np.zeros(len(polys) + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(counts)
    lons = [c[0] for _r, c, _ in polys]
    lats = [c[1] for _r, c, _ in polys]
    radii = [r for _p, _c, r in polys]
    t0 = time.time()

    def sample(i):
        return synth.cap_points(lons[i], lats[i], 1.5 * 1.2 * radii[i], 20000, np.random.default_rng(100 + i))

    tuning = autotune.tune(P, sample, per_class=2, reps=3,
                           budget_s=args.tune_budget if tune_budget is None else tune_budget)
    tune_s = time.time() - t0
    tc, le = tuning.for_polygons(P)
    torch.cuda.synchronize()
    t0 = time.time()
    B = G.Batch(P, top_cells=tc, leaf_edges=le)
    build_wall = time.time() - t0
    bst = B.stats()
    d_pts = synth.device_cap_points(lons, lats, radii, counts, 5, dev)
    n = int(offsets[-1])
    d_lab = torch.empty(n, dtype=torch.uint8, device=dev)
    chunk, shape = autotune.tune_launch(B, d_pts, offsets, d_lab, reps=2)
    stream = torch.cuda.current_stream()
    B.query_device(d_pts.data_ptr(), offsets, d_lab.data_ptr(), G.QUERY_FP32_FILTER, stream.cuda_stream, sync=True)
    esc = B.stats()

    def step():
        B.query_device(d_pts.data_ptr(), offsets, d_lab.data_ptr(), G.QUERY_FP32_FILTER, stream.cuda_stream,
                       graph=True)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    time.sleep(0.3)
    steps = steps or max(3, args.steps // 20)
    t = timed_loop(step, steps, stream)
    clk = clocks.stop()
    per = t / steps
    peak, peak_kind = _peaks()
    achieved = BYTES_PER_POINT * n / per / 1e9
    del d_pts, d_lab, B
    torch.cuda.empty_cache()
    return ({
        "metric": METRIC, "value": round(n / per / 1e6, 1), "unit": "Mpts/s", "n_gpus": 1, "steps": steps,
        "warmup": args.warmup, "ms_per_step": round(per * 1e3, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "C3: %d star polygons (16-200,000 vertices, 0-8 holes, radius 0.5-40 deg), "
                               "%d FP64 points inside the polygons' 1.5x bounding caps; exact labels; one CUDA-graph "
                               "query launch per step" % (len(P), n),
                   "polygons": len(P), "edges": bst["edges"], "points_per_step": n},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None, "bytes_per_point": BYTES_PER_POINT,
                     "peak_source": peak_kind},
        "gpu_launches": 4 * steps, "clocks": clk,
        "build_ms": {"batch_build_wall": round(build_wall * 1e3, 1), "workers": bst["workers"],
                     "generate_s": round(gen_s, 1), "autotune_s": round(tune_s, 1)},
        "lattice_bytes": bst["lattice_bytes"], "tuning": tuning.as_dict(), "chunk_points": chunk,
        "launch_shape": dict(zip(("points_per_thread", "blocks_per_sm"), G.Batch.shapes()[shape])),
        "escalation": {"boundary_points": esc["boundary_points"], "fp64_tests": esc["esc_fp64"],
                       "exact_tests": esc["esc_exact"], "boundary_fraction": round(esc["boundary_points"] / n, 6)},
    }, polys)


def run_c4(args, polys=None, seconds=None, pool_n=None, tune_budget=None):
    """Serving configuration: 1,024 resident C3-style polygons (built through
    the server, pinned); open-loop Poisson arrivals at `--c4-rate` requests/s
    for `--c4-seconds`: 95 % queries (polygon uniform over the residents,
    log-uniform 1-1e6 points inside its 1.5x bounding cap, from pageable host
    memory), 5 % builds of new C3-style polygons admitted by HBM footprint
    (the budget leaves `--c4-headroom` GB above the residents; the least
    recently used unpinned indexes are evicted).  Latency is submission to
    labels in host memory.  `polys` (generator output) replaces the resident
    set's generation; returns the result line as a dict."""
    import torch
    import gahhg_b200 as G
    from gahhg_b200 import autotune, synth
    dev = "cuda:0"
    t0 = time.time()
    if polys is None:
        polys = synth.c3_polygons(args.c4_polygons, seed=41)
    fresh = synth.c3_polygons(args.c4_new, seed=42)
    P = [G.Polygon.from_rings(r) for r, _c, _r in polys]
    NP = [G.Polygon.from_rings(r) for r, _c, _r in fresh]
    gen_s = time.time() - t0
    lons = [c[0] for _r, c, _ in polys]
    lats = [c[1] for _r, c, _ in polys]
    radii = [r for _p, _c, r in polys]

    def sample(i):
        return synth.cap_points(lons[i], lats[i], 1.5 * 1.2 * radii[i], 20000, np.random.default_rng(200 + i))

    t0 = time.time()
    tuning = autotune.tune(P, sample, per_class=1, reps=2,
                           budget_s=args.tune_budget if tune_budget is None else tune_budget)
    tune_s = time.time() - t0
    tc, le = tuning.for_polygons(P)
    ntc, nle = tuning.for_polygons(NP)

    def serve(budget):
        srv = G.Server(slots=args.c4_slots, slot_points=args.c4_slot_points, build_workers=args.c4_workers,
                       evict_lru=True, hbm_budget=int(budget))
        t0 = time.time()
        built = [srv.build(p, tc[i], le[i], pinned=True) for i, p in enumerate(P)]
        for _pid, tk in built:
            srv.wait(tk, 600.0)
        return srv, [pid for pid, _tk in built], time.time() - t0

    # the resident set's footprint, then the served configuration with a
    # budget of the residents plus the headroom
    srv, ids, resident_build_s = serve(150e9)
    resident = srv.stats()["resident_bytes"]
    srv.close()
    srv, ids, _ = serve(resident * 1.02 + args.c4_headroom * 1e9)
    # point pools: pool_n points per polygon inside its cap, pageable host memory
    pool_n = pool_n or args.c4_pool
    seconds = seconds or args.c4_seconds
    d_pool = synth.device_cap_points(lons, lats, radii, [pool_n] * len(P), 43, dev)
    pool = d_pool.cpu().numpy()
    del d_pool
    torch.cuda.empty_cache()
    lab_pool = np.zeros(len(pool), dtype=np.uint8)
    total = len(pool)
    # the arrival schedule
    rng = np.random.default_rng(44)
    nev = int(args.c4_rate * seconds * 1.1) + 16
    times = np.cumsum(rng.exponential(1.0 / args.c4_rate, nev))
    times = times[times < seconds]
    nev = len(times)
    is_build = rng.random(nev) < args.c4_build_frac
    qpoly = rng.integers(0, len(P), nev)
    qn = np.maximum(1, np.round(np.exp(rng.uniform(0.0, np.log(1e6), nev)))).astype(np.int64)
    qoff = np.empty(nev, dtype=np.int64)
    for k in range(nev):
        n = qn[k]
        if n <= pool_n:
            qoff[k] = qpoly[k] * pool_n + rng.integers(0, pool_n - n + 1)
        else:  # a request longer than one pool continues into the next polygons' pools
            qoff[k] = min(qpoly[k] * pool_n, total - n)
    q_idx = np.nonzero(~is_build)[0]
    b_idx = np.nonzero(is_build)[0]
    offered_pts = int(qn[q_idx].sum())
    pool_ptr, lab_ptr = pool.ctypes.data, lab_pool.ctypes.data
    lags = np.zeros(len(q_idx))
    build_lag = []

    def builds(t_start):
        for j, k in enumerate(b_idx):
            target = t_start + times[k]
            d = target - time.perf_counter()
            if d > 0:
                time.sleep(d)
            build_lag.append(time.perf_counter() - target)
            m = j % len(NP)
            srv.build(NP[m], ntc[m], nle[m], detached=True)

    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    time.sleep(0.3)
    srv.reset_stats()
    t_start = time.perf_counter() + 0.02
    bt = threading.Thread(target=builds, args=(t_start,))
    bt.start()
    for j, k in enumerate(q_idx):
        target = t_start + times[k]
        while True:
            now = time.perf_counter()
            d = target - now
            if d <= 0:
                break
            if d > 0.0006:
                time.sleep(d - 0.0005)
        lags[j] = now - target
        off = int(qoff[k])
        srv.query_raw(ids[qpoly[k]], pool_ptr + 16 * off, int(qn[k]), lab_ptr + off, detached=True)
    t_submit_end = time.perf_counter()
    bt.join()
    srv.drain(300.0)
    t_end = time.perf_counter()
    st = srv.stats()
    clk = clocks.stop()
    lat = srv.latencies(0)
    tr = srv.trace()
    stalls = srv.stalls()
    if args.c4_trace:
        np.savez(args.c4_trace, trace=tr, latencies=lat, builds=srv.latencies(1), stalls=stalls)
    window = t_end - t_start
    srv.close()
    sustained = st["query_points"] / window

    def pct(a, q):
        return round(float(np.percentile(a, q)), 4) if len(a) else None

    del pool, lab_pool
    return {
        "metric": METRIC, "value": round(st["p99_ms"], 3), "unit": "ms (query p99)", "n_gpus": 1,
        "steps": int(st["queries_done"]), "warmup": 0,
        "ms_per_step": round(float(lat.mean()), 4) if len(lat) else None,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "C4: %d resident C3-style polygons; Poisson arrivals at %g req/s for %g s: %d %% "
                               "queries (uniform polygon, log-uniform 1-1e6 points from pageable host memory), %d %% "
                               "builds of new C3-style polygons admitted by HBM footprint with LRU eviction"
                               % (len(P), args.c4_rate, seconds, round(100 * (1 - args.c4_build_frac)),
                                  round(100 * args.c4_build_frac)),
                   "polygons": len(P), "slots": args.c4_slots, "slot_points": args.c4_slot_points,
                   "build_workers": args.c4_workers, "pool_points_per_polygon": pool_n,
                   "hbm_budget_gb": round(st["hbm_budget"] / 1e9, 2)},
        "latency_ms": {"p50": round(st["p50_ms"], 3), "p90": round(st["p90_ms"], 3), "p99": round(st["p99_ms"], 3),
                       "max": round(st["max_ms"], 3), "build_p50": round(st["build_p50_ms"], 2),
                       "build_p99": round(st["build_p99_ms"], 2)},
        "throughput": {"sustained_mpts_s": round(sustained / 1e6, 3),
                       "offered_mpts_s": round(offered_pts / seconds / 1e6, 3),
                       "queries": int(st["queries_done"]), "builds_done": int(st["builds_done"]),
                       "builds_failed": int(st["builds_failed"]), "evictions": int(st["evictions"]),
                       "batches": int(st["batches"]), "mean_batch_pieces": round(st["mean_batch_pieces"], 2),
                       "mean_batch_points": round(st["mean_batch_points"], 1),
                       "drain_s": round(t_end - t_submit_end, 4)},
        "host_stalls": {int(k): [int((stalls[:, 1] == k).sum()), round(float(stalls[stalls[:, 1] == k, 2].max()), 2)]
                        for k in np.unique(stalls[:, 1])} if len(stalls) else {},
        "batch_trace_ms": {"enqueue_p99": pct(tr[:, 1], 99), "device_p50": pct(tr[:, 2], 50),
                           "device_p99": pct(tr[:, 2], 99), "device_max": pct(tr[:, 2], 100),
                           "complete_p99": pct(tr[:, 3], 99)},
        "e2e": {"value": round(sustained / 1e6, 3), "unit": "Mpts/s",
                "h2d_bytes_per_step": int(16 * st["query_points"] / max(st["queries_done"], 1)),
                "d2h_bytes_per_step": int(st["query_points"] / max(st["queries_done"], 1))},
        "arrival_lag_ms": {"p50": round(float(np.median(lags)) * 1e3, 4),
                           "p99": round(float(np.percentile(lags, 99)) * 1e3, 4),
                           "build_p99": round(float(np.percentile(build_lag, 99)) * 1e3, 4) if build_lag else None},
        "escalation": {"boundary_points": st["boundary_points"], "fp64_tests": st["esc_fp64"],
                       "exact_tests": st["esc_exact"]},
        "gpu_launches": 4 * int(st["batches"]), "clocks": clk,
        "build_ms": {"resident_set_wall": round(resident_build_s * 1e3, 1), "resident_bytes": resident,
                     "generate_s": round(gen_s, 1), "autotune_s": round(tune_s, 1)},
        "tuning": tuning.as_dict(),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--points", type=int, default=100_000_000)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--ref-sample", type=int, default=2_000_000)
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--traffic", type=float, default=None,
                    help="DRAM bytes per launch of the query kernel from an ncu capture (profiles/)")
    ap.add_argument("--config", default="c1", choices=["c1", "c2", "c3", "c4"])
    ap.add_argument("--c2-points", type=int, default=20_000_000)
    ap.add_argument("--c3-polygons", type=int, default=4096)
    ap.add_argument("--c3-scale", type=float, default=1.0, help="scale the C3 point counts")
    ap.add_argument("--tune-budget", type=float, default=60.0)
    ap.add_argument("--c4-polygons", type=int, default=1024)
    ap.add_argument("--c4-new", type=int, default=256, help="distinct new polygons the build requests cycle over")
    ap.add_argument("--c4-rate", type=float, default=2000.0, help="requests per second (Poisson)")
    ap.add_argument("--c4-seconds", type=float, default=20.0)
    ap.add_argument("--c4-build-frac", type=float, default=0.05)
    ap.add_argument("--c4-slots", type=int, default=4)
    ap.add_argument("--c4-slot-points", type=int, default=1 << 22)
    ap.add_argument("--c4-workers", type=int, default=4)
    ap.add_argument("--c4-pool", type=int, default=1 << 19, help="host points per resident polygon")
    ap.add_argument("--c4-headroom", type=float, default=8.0, help="GB of budget above the resident set")
    ap.add_argument("--c4-trace", default=None, help="save the per-batch trace and latencies (.npz)")
    ap.add_argument("--no-legs", action="store_true", help="C1 only (no C2/C3/C4 keys in the default run)")
    ap.add_argument("--legs", default="c2,c3,c4", help="configurations added as keys of the C1 line")
    ap.add_argument("--leg-c3-polygons", type=int, default=1024)
    ap.add_argument("--leg-tune-budget", type=float, default=15.0)
    ap.add_argument("--leg-c4-seconds", type=float, default=10.0)
    ap.add_argument("--leg-c4-pool", type=int, default=1 << 17)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.config == "c3":
        print(json.dumps(run_c3(args)[0]))
        return 0
    if args.config == "c4":
        print(json.dumps(run_c4(args)))
        return 0

    import torch
    import torch.distributed as dist
    from gahhg_b200 import replicas
    rank, world, local = replicas.world()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    import gahhg_b200 as G

    rings = c1_polygon_cached()
    P = G.Polygon.from_rings(rings)
    # one-time process costs (CUDA context, lazy module loading) land in a
    # build of the small C0 polygon, not in the timed C1 builds
    from gahhg_b200 import synth
    t0 = time.time()
    G.Grid(G.Polygon.from_rings(synth.c0_polygon()), semantics=G.SEMANTICS_EXACT, device=local).classify()
    G.Grid(G.Polygon.from_rings(synth.c0_polygon()), semantics=G.SEMANTICS_REFERENCE, device=local).classify()
    cold_s = time.time() - t0
    # the first C1 build of the process also grows the device memory pool
    # (first use of the memory it maps): timed apart as the cold build; the
    # second, timed build is the warm one the queries use
    t0 = time.time()
    g = G.Grid(P, semantics=G.SEMANTICS_EXACT, device=local).classify()
    cold_build_wall = time.time() - t0
    st_cold = g.stats()
    del g
    t0 = time.time()
    g = G.Grid(P, semantics=G.SEMANTICS_EXACT, device=local).classify()
    build_wall = time.time() - t0
    st_build = g.stats()
    t0 = time.time()
    gref = G.Grid(P, semantics=G.SEMANTICS_REFERENCE, max_depth=REF_DEPTH_C1, device=local).classify()
    ref_build_wall = time.time() - t0
    st_ref = gref.stats()

    c2 = args.config == "c2"
    n = args.c2_points if c2 else args.points
    if c2:
        pts = synth.device_c2_points(rings, n, 2222 + rank, "cuda:%d" % local)
    else:
        pts = synth.device_points(n, 1234 + rank, "cuda:%d" % local)
    labels = torch.empty(n, dtype=torch.uint8, device="cuda:%d" % local)
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    lp, pp = labels.data_ptr(), pts.data_ptr()

    def q32():
        g.query_device(pp, n, lp, G.QUERY_FP32_FILTER, sh)

    def q64():
        g.query_device(pp, n, lp, G.QUERY_FP64_FILTER, sh)

    def qref():
        gref.query_device(pp, n, lp, G.QUERY_REFERENCE_FP64, sh)

    # escalation statistics from one counted pass
    g.query_device(pp, n, lp, G.QUERY_FP32_FILTER, sh, sync=True)
    esc = g.stats()
    inside = int((labels == 2).sum().item())

    for _ in range(args.warmup):
        q32()
    torch.cuda.synchronize()
    replicas.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    replicas.barrier()
    t = timed_loop(q32, args.steps, stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    t = replicas.max_over_ranks(t, "cuda:%d" % local)
    rate = world * n * args.steps / t / 1e6
    per_launch = t / args.steps

    # comparison paths (same points, same stream)
    for _ in range(2):
        q64()
    t64 = timed_loop(q64, max(10, args.steps // 4), stream) / max(10, args.steps // 4)
    for _ in range(2):
        qref()
    kref = max(3, args.steps // 40)
    tref = timed_loop(qref, kref, stream) / kref

    # end to end through the C ABI with pinned host buffers
    e2e_n = n
    host_ll = torch.empty((e2e_n, 2), dtype=torch.float64, pin_memory=True)
    host_ll.copy_(pts[:e2e_n])
    host_lab = torch.empty(e2e_n, dtype=torch.uint8, pin_memory=True)
    L = G._lib.lib()
    hp, hl = ctypes.c_void_p(host_ll.data_ptr()), ctypes.c_void_p(host_lab.data_ptr())
    G.check(L.gahhg_query(g._h, hp, e2e_n, hl, G.QUERY_FP32_FILTER))
    torch.cuda.synchronize()
    te = time.perf_counter()
    for _ in range(args.e2e_steps):
        G.check(L.gahhg_query(g._h, hp, e2e_n, hl, G.QUERY_FP32_FILTER))
    te = (time.perf_counter() - te) / args.e2e_steps
    te = replicas.max_over_ranks(te, "cuda:%d" % local)
    e2e_rate = world * e2e_n / te / 1e6

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from gahhg_b200 import synth
        rs = np.random.default_rng(0)
        if c2:
            sample = np.concatenate([synth.uniform_points(args.ref_sample // 2, rs),
                                     synth.near_edge_points(rings, args.ref_sample - args.ref_sample // 2, rs)])
        else:
            sample = synth.uniform_points(args.ref_sample, rs)
        threads = os.cpu_count()
        v, info = cpu_reference_rate(rings, sample, threads, args.cpu_budget)
        if v is not None:
            cpu = {"value": round(v, 3), "unit": "Mpts/s", "cores": threads, "kind": "reference",
                   "sample": "reference GAHHG kernels built for the CPU, maxDepth %d, OpenMP %d threads; "
                             "%d %s points per pass for %.0f s (%s)" % (
                                 REF_DEPTH_C1, threads, len(sample), "C2 (half near-edge)" if c2 else "uniform C1",
                                 args.cpu_budget, json.dumps(info))}
        else:
            cpu = {"value": None, "unit": "Mpts/s", "cores": 0, "kind": "reference", "sample": info}

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    peak, peak_kind = _peaks()
    achieved = BYTES_PER_POINT * n / per_launch / 1e9
    out = {
        "metric": METRIC, "value": round(rate, 1), "unit": "Mpts/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(per_launch * 1e3, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": ("C2: the C1 polygon (1.1M edges); %d FP64 points per GPU, half uniform by area, "
                                "half within 10^U[-15,-3] rad of a random edge; exact labels, FP32 certified filter"
                                % n) if c2 else
                               "C1: 1,000,000-vertex outer ring + 10 x 10,000-vertex holes (1.1M edges), "
                               "1e8 uniform FP64 lon/lat points per GPU; exact labels, FP32 certified filter",
                   "points_per_step": n, "edges": int(P.num_edges),
                   "inputs": "%.2f GB per GPU, larger than L2" % (16 * n / 1e9),
                   "parallelism": "replicas" if world > 1 else "single"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4),
                     "traffic": args.traffic if args.traffic is not None else (
                         round(_traffic_per_point() * n) if _traffic_per_point() else None),
                     "traffic_source": "given on the command line" if args.traffic is not None else
                                       "scaled ncu capture (profiles/locate_traffic.json: DRAM bytes per point "
                                       "of one k_locate launch on 1e7 C1 points, times the points per step)",
                     "bytes_per_point": BYTES_PER_POINT, "peak_source": peak_kind},
        "cpu_baseline": cpu,
        "e2e": {"value": round(e2e_rate, 1), "unit": "Mpts/s", "h2d_bytes_per_step": 16 * e2e_n,
                "d2h_bytes_per_step": e2e_n},
        # per chunk of 2^27 points: k_locate and the three pass-2 tiers
        "gpu_launches": 4 * args.steps * ((n + (1 << 27) - 1) // (1 << 27)),
        "clocks": clk,
        "comparison": {
            "fp64_filter_exact_mpts": round(world * n / t64 / 1e6, 1),
            "reference_fp64_descent_mpts": round(world * n / tref / 1e6, 1),
            "speedup_vs_reference_fp64": round(tref / per_launch, 2),
            "reference_fp64_max_depth": REF_DEPTH_C1,
        },
        "build_ms": {"exact_total_wall": round(build_wall * 1e3, 1),
                     "exact_total_wall_first_in_process": round(cold_build_wall * 1e3, 1),
                     "lattice_first_in_process": round(st_cold["lattice_s"] * 1e3, 2),
                     "lattice": round(st_build["lattice_s"] * 1e3, 2),
                     "exact_grid": "exact index only; the hexagon hierarchy is built when a report, an "
                                   "export or a reference-precision query needs it",
                     "reference_semantics_total_wall": round(ref_build_wall * 1e3, 1),
                     "reference_semantics_create": round(st_ref["create_s"] * 1e3, 2),
                     "process_warmup_c0": round(cold_s * 1e3, 1)},
        "escalation": {"boundary_points": esc["boundary_points"], "fp64_tests": esc["esc_fp64"],
                       "exact_tests": esc["esc_exact"],
                       "boundary_fraction": round(esc["boundary_points"] / n, 6),
                       "fp32_to_fp64_per_point": esc["esc_fp64"] / n,
                       "fp32_to_fp64_per_boundary_point": esc["esc_fp64"] / max(esc["boundary_points"], 1),
                       "fp64_to_exact_per_point": esc["esc_exact"] / n},
        "inside_fraction": round(inside / n, 6),
        "lattice_bytes": st_build["lattice_bytes"],
    }
    if args.config == "c1" and world == 1 and not args.no_legs:
        # the other configurations as keys of the same line: C2 on the same
        # polygon and index, then a reduced C3 batch and a shortened C4
        # serving run on the same 1,024 batch-configuration polygons
        del pts, labels, host_ll, host_lab
        torch.cuda.empty_cache()
        legs = set(args.legs.split(","))
        if "c2" in legs:
            out["c2"] = leg_c2(args, g, gref, rings, stream)
        del g, gref
        torch.cuda.empty_cache()
        polys = None
        if "c3" in legs:
            out["c3"], polys = run_c3(args, count=args.leg_c3_polygons, tune_budget=args.leg_tune_budget,
                                      steps=max(3, args.steps // 4))
            torch.cuda.empty_cache()
        if "c4" in legs:
            out["c4"] = run_c4(args, polys=polys, seconds=args.leg_c4_seconds, pool_n=args.leg_c4_pool,
                               tune_budget=args.leg_tune_budget)
    print(json.dumps(out))
    return 0


def leg_c2(args, g, gref, rings, stream):
    """C2 on the C1 polygon's index: FP32-filtered and FP64-filtered exact
    query rates and escalation fractions, and the reference algorithm's FP64
    descent, on `--c2-points` points (half uniform, half within
    10^U[-15,-3] rad of a random edge) resident in HBM."""
    import torch
    import gahhg_b200 as G
    from gahhg_b200 import synth
    n = args.c2_points
    pts = synth.device_c2_points(rings, n, 2222, "cuda:0")
    labels = torch.empty(n, dtype=torch.uint8, device="cuda:0")
    sh = stream.cuda_stream
    lp, pp = labels.data_ptr(), pts.data_ptr()
    rates, esc = {}, {}
    steps = max(10, args.steps)
    for name, prec in (("fp32_filter", G.QUERY_FP32_FILTER), ("fp64_filter", G.QUERY_FP64_FILTER)):
        g.query_device(pp, n, lp, prec, sh, sync=True)
        esc[name] = g.stats()
        for _ in range(max(3, args.warmup)):
            g.query_device(pp, n, lp, prec, sh)
        t = timed_loop(lambda: g.query_device(pp, n, lp, prec, sh), steps, stream)
        rates[name] = n * steps / t / 1e6
    # pass 2 over the queue in leaf-window order and in leaf order (the
    # default keeps pass-1 order), both precisions, for comparison
    old = G.set_knob(G.KNOB_GROUPED_PASS2, 0)
    for order, oname in ((1, "window_ordered"), (2, "leaf_sorted"), (3, "leaf_sorted_staged")):
        G.set_knob(G.KNOB_GROUPED_PASS2, order)
        for name, prec in (("fp32_filter", G.QUERY_FP32_FILTER), ("fp64_filter", G.QUERY_FP64_FILTER)):
            for _ in range(max(3, args.warmup)):
                g.query_device(pp, n, lp, prec, sh)
            t = timed_loop(lambda: g.query_device(pp, n, lp, prec, sh), steps, stream)
            rates["%s_%s_pass2" % (name, oname)] = n * steps / t / 1e6
    G.set_knob(G.KNOB_GROUPED_PASS2, old)
    for _ in range(2):
        gref.query_device(pp, n, lp, G.QUERY_REFERENCE_FP64, sh)
    kref = 3
    tref = timed_loop(lambda: gref.query_device(pp, n, lp, G.QUERY_REFERENCE_FP64, sh), kref, stream) / kref
    peak, peak_kind = _peaks()
    e32 = esc["fp32_filter"]
    per32 = n / (rates["fp32_filter"] * 1e6)
    del pts, labels
    return {
        "workload": "C2: the C1 polygon (1.1M edges); %d FP64 points, half uniform by area, half within "
                    "10^U[-15,-3] rad of a random edge; exact labels" % n,
        "points_per_step": n, "steps": steps,
        "value": round(rates["fp32_filter"], 1), "unit": "Mpts/s",
        "fp32_filter_mpts": round(rates["fp32_filter"], 1),
        "fp64_filter_mpts": round(rates["fp64_filter"], 1),
        "fp32_over_fp64_filter": round(rates["fp32_filter"] / rates["fp64_filter"], 3),
        "pass2_orders_mpts": {k[:-len("_pass2")]: round(v, 1) for k, v in rates.items() if k.endswith("_pass2")},
        "reference_fp64_descent_mpts": round(n / tref / 1e6, 1),
        "reference_fp64_max_depth": REF_DEPTH_C1,
        "roofline": {"bound": "hbm", "achieved": round(BYTES_PER_POINT * n / per32 / 1e9, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(BYTES_PER_POINT * n / per32 / 1e9 / peak, 4),
                     "peak_source": peak_kind},
        "escalation": {"boundary_points": e32["boundary_points"],
                       "fp32_to_fp64_points": e32["esc_fp64"], "fp64_to_exact_points": e32["esc_exact"],
                       "fp32_to_fp64_per_point": round(e32["esc_fp64"] / n, 6),
                       "fp32_to_fp64_per_boundary_point": round(e32["esc_fp64"] / max(e32["boundary_points"], 1), 4),
                       "fp64_to_exact_per_point": e32["esc_exact"] / n,
                       "fp64_filter_mode_exact_points": esc["fp64_filter"]["esc_exact"]},
    }


if __name__ == "__main__":
    sys.exit(main())
