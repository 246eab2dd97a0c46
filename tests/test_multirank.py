"""Multi-rank host logic on CPU (gloo, world size 2): the timing reduction the benchmark uses and
the cross-replica result check (the reference's burn-in comparison), with a planted mismatch."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import PKG, REPO


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, plant, q):
    import sys
    import datetime

    for p in (REPO, PKG):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import numpy as np
    import torch.distributed as dist

    from oracle import oracle as O
    from tconvolve import replicas
    from tconvolve.workload import PROBLEMS, normal_vis

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # each replica times its "step"; the benchmark reports the slowest rank
        mx = replicas.max_over_ranks([1.0 + rank, 5.0 - rank])
        # each replica runs the same problem (the oracle stands in for the device here)
        prob = PROBLEMS["g1"]
        vis = normal_vis(prob.n_data(), 99)
        r = O.run_plain(O.Config(prob.n_samples, prob.w_size, prob.n_chan, prob.g_size, prob.cell_size), vis=vis)
        grid = r["grid"].copy()
        if plant and rank == 1:
            grid[1234] += np.complex64(1e-3)  # a planted disagreement on one replica
        same = replicas.cross_check(replicas.checksum(grid))
        # each rank's own autotuner choice; every rank ends with rank 0's
        mine = {"r32": ((16, 64, 0, 64 * (rank + 1)), 1.0 + rank), "c64": ((8, 32, 128 * rank, 0, rank), None)}
        agreed = replicas.rank0_tunings(mine)
        q.put((rank, mx, same, agreed))
    finally:
        dist.destroy_process_group()


def _run(plant: bool):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, plant, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(out)


def test_replicas_agree_and_time_is_max():
    out = _run(plant=False)
    for rank, mx, same, agreed in out:
        assert mx == [2.0, 5.0]
        assert same
        # rank 0's tunings everywhere (its own "extra" value kept)
        assert agreed["r32"][0] == (16, 64, 0, 64) and agreed["c64"][0] == (8, 32, 0, 0)
        assert agreed["r32"][1] == 1.0 + rank


def test_cross_check_detects_planted_mismatch():
    out = _run(plant=True)
    assert all(not same for _, _, same, _ in out)


def test_single_process_defaults():
    import sys

    sys.path.insert(0, PKG)
    from tconvolve import replicas

    assert replicas.world() == (0, 1)
    assert replicas.max_over_ranks([3.0]) == [3.0]
    assert replicas.cross_check(123)
    assert replicas.rank0_tunings({"r32": ((16, 64, 0, 64), 2.0)}) == {"r32": ((16, 64, 0, 64), 2.0)}
