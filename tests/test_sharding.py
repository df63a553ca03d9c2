"""Orientation sharding: shard ranges, and the cross-rank argmin with the
reference's first-strict-minimum rule, over two gloo ranks on the CPU."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from tomo_shell2026_b200 import sharding


def test_shard_ranges_cover_exactly():
    for n in (0, 1, 7, 684, 21960):
        for world in (1, 2, 3, 8):
            spans = [sharding.shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))


CASES = [
    np.array([3.0, 1.0, 2.0, 1.0, 5.0], np.float32),                  # tie: first index wins
    np.array([2e5, 3e5, 1e5, 4e5], np.float32),                       # nothing below 1e5 -> 0
    np.array([0.5, -1.0, -1.0, 7.0, -3.0, -3.0, 2.0], np.float32),   # negatives, tie across shards
    np.array([9.0], np.float32),                                      # single orientation -> 0
]


def test_first_optimal_rule():
    assert sharding.first_optimal(CASES[0]) == 1
    assert sharding.first_optimal(CASES[1]) == 0
    assert sharding.first_optimal(CASES[2]) == 4
    assert sharding.first_optimal(CASES[3]) == 0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, results):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out = []
        for mss in CASES:
            b, e = sharding.shard_range(len(mss), rank, world)
            out.append(sharding.global_first_optimal(mss[b:e], b, len(mss)))
        results[rank] = out
    finally:
        dist.destroy_process_group()


def test_global_argmin_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    results = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, results)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    want = [sharding.first_optimal(m) for m in CASES]
    assert results[0] == want and results[1] == want


def _oracle_engine(mesh, ypr, opts):
    from oracle.oracle import Oracle
    return Oracle().sweep(mesh, ypr, opts, threads=2)


def _sweep_worker(rank, world, port, results, n_keep):
    import torch.distributed as dist
    from tomo_shell2026_b200 import meshgen
    from tomo_shell2026_b200.options import PrintOptions
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mesh = meshgen.small_solid(0)
        ypr = meshgen.ypr_grid(np.arange(0, 360, 10), np.arange(0, 190, 10))[:n_keep]
        r = sharding.sweep_shard(mesh, ypr, PrintOptions(explicit_ss=True), engine=_oracle_engine, gather=True)
        results[rank] = (r.optID, r.begin, r.end, r.Mss.view(np.int32).tolist(), r.Vss64.tolist(), r.Vo64.tolist())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_keep,world", [(684, 2), (1, 2), (7, 3)])
def test_sharded_sweep_equals_undivided_sweep(n_keep, world):
    """Each gloo rank sweeps its contiguous shard of the 684-orientation
    grid of the small solid (the oracle stands in for the device, which
    makes no difference to the host-side split and combine); the combined
    optID and the gathered Mss bits, Vss and Vo equal one undivided sweep."""
    from oracle.oracle import Oracle
    from tomo_shell2026_b200 import meshgen
    from tomo_shell2026_b200.options import PrintOptions
    mesh = meshgen.small_solid(0)
    ypr = meshgen.ypr_grid(np.arange(0, 360, 10), np.arange(0, 190, 10))[:n_keep]
    want = Oracle().sweep(mesh, ypr, PrintOptions(explicit_ss=True), threads=4)
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    results = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_sweep_worker, args=(r, world, port, results, n_keep)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    spans = [sharding.shard_range(n_keep, r, world) for r in range(world)]
    for r in range(world):
        opt, b, e, mss_bits, vss, vo = results[r]
        assert (b, e) == spans[r]
        assert opt == want["optID"]
        assert mss_bits == want["Mss"].view(np.int32).tolist()
        assert vss == want["Vss64"].tolist() and vo == want["Vo64"].tolist()
