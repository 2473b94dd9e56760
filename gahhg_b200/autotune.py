"""Autotuner for the exact index of many polygons.

Chooses, per size class of polygon (edge count rounded to a power of two),
the lattice parameters that give the fastest queries on a sample of the
class:

  cells_per_edge  top-level cells per edge (lattice_top = cells_per_edge x
                  edges, clamped to [1024, 8M]); more cells mean more points
                  answered from a cell without edges, at more build time and
                  memory;
  leaf_edges      edges per leaf before a cell is split (lattice_leaf);
                  fewer mean shorter crossing loops and deeper lattices;

and then, per batch, the point-chunk size of the persistent batch query
(the load balancing grain) and the launch shape of its first pass (points
per thread in flight x resident blocks per SM; threads per block stay 256).  Candidates are measured, not modelled: each candidate
builds the sampled polygons as a batch and times queries of their own points
with CUDA events.  The result is a plain table that `Batch` takes as its
per-polygon `top_cells` / `leaf_edges`.
"""
import math
import time

import numpy as np

from . import Batch, QUERY_FP32_FILTER

CELLS_PER_EDGE = (2, 8, 32)
LEAF_EDGES = (4, 8, 16)
CHUNKS = (2048, 8192, 32768)


def size_class(edges):
    return max(0, int(math.log2(max(edges, 1))))


def top_cells(edges, cells_per_edge):
    return int(min(max(cells_per_edge * edges, 1024), 8 << 20))


def _time_batch(batch, d_pts, offsets, d_lab, reps):
    import torch
    stream = torch.cuda.current_stream()
    batch.query_device(d_pts.data_ptr(), offsets, d_lab.data_ptr(), QUERY_FP32_FILTER, stream.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        batch.query_device(d_pts.data_ptr(), offsets, d_lab.data_ptr(), QUERY_FP32_FILTER, stream.cuda_stream)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) * 1e-3 / reps


def tune(polygons, points, per_class=3, reps=5, seed=0, budget_s=60.0, mem_ratio=2.0, log=None):
    """polygons: list of gahhg_b200.Polygon; points: list of (n_i, 2) float64
    lon/lat arrays (the polygon's own query sample), or a function of the
    polygon index returning one.  Returns a Tuning."""
    import torch
    rng = np.random.default_rng(seed)
    classes = {}
    for i, p in enumerate(polygons):
        classes.setdefault(size_class(p.num_edges), []).append(i)
    table = {}
    t_start = time.time()
    for c in sorted(classes):
        idx = classes[c]
        pick = list(rng.choice(idx, size=min(per_class, len(idx)), replace=False))
        polys = [polygons[i] for i in pick]
        pts = [points(i) if callable(points) else points[i] for i in pick]
        offsets = np.zeros(len(pts) + 1, dtype=np.int64)
        offsets[1:] = np.cumsum([len(q) for q in pts])
        d_pts = torch.from_numpy(np.concatenate(pts)).cuda()
        d_lab = torch.empty(len(d_pts), dtype=torch.uint8, device="cuda")
        results = []
        for f in CELLS_PER_EDGE:
            for k in LEAF_EDGES:
                if time.time() - t_start > budget_s and results:
                    break
                tc = [top_cells(p.num_edges, f) for p in polys]
                t0 = time.time()
                b = Batch(polys, top_cells=tc, leaf_edges=[k] * len(polys))
                tb = time.time() - t0
                tq = _time_batch(b, d_pts, offsets, d_lab, reps)
                mem = b.stats()["lattice_bytes"]
                del b
                results.append((tq, tb, mem, f, k))
                if log:
                    log("class 2^%d f=%d K=%d query %.3f ms build %.1f ms %.1f MB" % (
                        c, f, k, tq * 1e3, tb * 1e3, mem / 1e6))
        # fastest queries among candidates within `mem_ratio` of the smallest
        # index (memory decides how many polygons stay resident); build time
        # breaks near-ties
        mmin = min(r[2] for r in results)
        ok = [r for r in results if r[2] <= mem_ratio * mmin] or results
        tq, tb, mem, f, k = min(ok, key=lambda r: r[0] * (1.0 + 0.02 * r[1] / max(r[0] * 1000.0, 1e-9)))
        table[c] = (f, k)
    return Tuning(table)


def tune_chunk(batch, d_pts, offsets, d_lab, reps=5):
    """Sets and returns the fastest chunk size of `batch` on these points."""
    best = None
    for ch in CHUNKS:
        batch.set_chunk(ch)
        t = _time_batch(batch, d_pts, offsets, d_lab, reps)
        if best is None or t < best[0]:
            best = (t, ch)
    batch.set_chunk(best[1])
    return best[1]


def tune_shape(batch, d_pts, offsets, d_lab, reps=5, log=None):
    """Sets and returns the index of the fastest pass-1 launch shape (points
    per thread x blocks per SM, `Batch.shapes()`) of `batch` on these points:
    the descent is latency-bound, and how many points a thread keeps in
    flight against how many warps an SM holds depends on the mix of polygon
    sizes and points."""
    best = None
    for i, (u, blocks) in enumerate(Batch.shapes()):
        batch.set_shape(i)
        t = _time_batch(batch, d_pts, offsets, d_lab, reps)
        if log:
            log("shape %d (%d points x %d blocks) query %.3f ms" % (i, u, blocks, t * 1e3))
        if best is None or t < best[0]:
            best = (t, i)
    batch.set_shape(best[1])
    return best[1]


def tune_launch(batch, d_pts, offsets, d_lab, reps=5, log=None):
    """Chunk size, then launch shape, of `batch`'s query; returns both."""
    ch = tune_chunk(batch, d_pts, offsets, d_lab, reps)
    return ch, tune_shape(batch, d_pts, offsets, d_lab, reps, log)


class Tuning:
    def __init__(self, table):
        self.table = dict(table)

    def params(self, edges):
        c = size_class(edges)
        if c in self.table:
            f, k = self.table[c]
        elif self.table:
            near = min(self.table, key=lambda x: abs(x - c))
            f, k = self.table[near]
        else:
            f, k = 8, 8
        return top_cells(edges, f), k

    def for_polygons(self, polygons):
        tc, le = zip(*[self.params(p.num_edges) for p in polygons]) if polygons else ((), ())
        return list(tc), list(le)

    def as_dict(self):
        return {"2^%d" % c: {"cells_per_edge": f, "leaf_edges": k} for c, (f, k) in sorted(self.table.items())}
