"""Replicas on CPU: two gloo ranks, as torchrun would start them.

Each rank labels its own shard of a common point array (the exact oracle
stands in for its GPU), and the ranks agree on the slowest rank's time.  The
shards must cover the array without overlap, and their labels must equal one
process's labels: the path shards by points with no exchange.
"""
import os
import socket

import numpy as np
import pytest

from gahhg_b200 import replicas, synth


def test_shard_partitions():
    for n in (0, 1, 7, 1000, 1001):
        for size in (1, 2, 3, 8):
            spans = [replicas.shard(n, r, size) for r in range(size)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            lens = [e - s for s, e in spans]
            assert max(lens) - min(lens) <= 1


def _oracle(rings):
    """Exact oracle over the polygon as the library loads it (rings re-oriented
    as the reference does; host code only)."""
    import gahhg_b200 as G
    from oracle import exact
    xyz, pe = G.Polygon.from_rings(rings).export()
    return exact.ExactPolygon(xyz, pe, len(rings[0]))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, size, port, outdir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(size),
                      LOCAL_RANK=str(rank))
    from datetime import timedelta
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    r, w, _ = replicas.world()
    rings = synth.c0_polygon(seed=2)
    rng = np.random.default_rng(3)
    pts = np.concatenate([synth.uniform_points(3000, rng), synth.near_edge_points(rings, 3000, rng)])
    a, b = replicas.shard(len(pts), r, w)
    E = _oracle(rings)
    lab = E.query_lonlat(pts[a:b], threads=1)
    replicas.barrier()
    slowest = replicas.max_over_ranks(10.0 + r)
    np.save(os.path.join(outdir, "lab%d.npy" % r), lab)
    np.save(os.path.join(outdir, "t%d.npy" % r), np.array([slowest]))
    dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    labs = [np.load(tmp_path / ("lab%d.npy" % r)) for r in range(2)]
    for r in range(2):
        assert float(np.load(tmp_path / ("t%d.npy" % r))[0]) == 11.0
    # one process over the whole array
    rings = synth.c0_polygon(seed=2)
    rng = np.random.default_rng(3)
    pts = np.concatenate([synth.uniform_points(3000, rng), synth.near_edge_points(rings, 3000, rng)])
    whole = _oracle(rings).query_lonlat(pts, threads=1)
    assert np.array_equal(np.concatenate(labs), whole)
    assert set(np.unique(whole)) <= {1, 2}
