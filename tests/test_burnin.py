"""Burn-in soak test (attic/tConvolveBurnIn): the exchange partners, the element-wise comparison
with the reference's FLT_EPSILON test, error accumulation and time statistics, on CPU with gloo at
world sizes 2 and 3 (with a planted disagreement), and one GPU run of the whole loop."""
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
    import datetime
    import sys

    for p in (REPO, PKG):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch
    import torch.distributed as dist

    from tconvolve import burnin

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        g = torch.Generator().manual_seed(5)
        data = torch.randn(50_000, dtype=torch.complex64, generator=g)  # the same on every rank
        if plant is not None and rank == plant:
            data[777] = data[777] + 1e-3
        ok, count, first, src = burnin.share_and_compare(data)
        errors = burnin.accumulate_errors(ok)
        tmin, tavg, tmax = burnin.gather_times(0.5 + rank)
        q.put((rank, ok, count, first, src, errors, (tmin, tavg, tmax)))
    finally:
        dist.destroy_process_group()


def _run(world, plant):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, plant, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(out)


def test_partners():
    import sys

    sys.path.insert(0, PKG)
    from tconvolve.burnin import partners

    assert partners(0, 1) == (0, 0)
    assert [partners(r, 2) for r in range(2)] == [(1, 1), (0, 0)]
    assert [partners(r, 3) for r in range(3)] == [(1, 2), (2, 0), (0, 1)]
    for n in range(1, 9):  # every rank receives from exactly the rank that sends to it
        assert sorted(partners(r, n)[0] for r in range(n)) == list(range(n))
        assert all(partners(partners(r, n)[1], n)[0] == r for r in range(n))


@pytest.mark.parametrize("world", [2, 3])
def test_replicas_agree(world):
    out = _run(world, None)
    for rank, ok, count, first, src, errors, times in out:
        assert ok and count == 0 and first == -1 and errors == 0
        assert times == (0.5, 0.5 + (world - 1) / 2, 0.5 + world - 1)


@pytest.mark.parametrize("world", [2, 3])
def test_planted_disagreement_is_found(world):
    out = _run(world, 1)
    from tconvolve.burnin import partners

    for rank, ok, count, first, src, errors, _ in out:
        involved = rank == 1 or src == 1  # rank 1 differs from what it receives; its receiver too
        assert ok == (not involved)
        if involved:
            assert count == 1 and first == 777
        assert errors == sum(1 for r in range(world) if r == 1 or partners(r, world)[1] == 1)


@pytest.mark.gpu
def test_burnin_on_gpu(tcv, cuda_ok):
    """Two cycles of the loop on one GPU (a small problem): no errors, and the grid accumulates
    (the second pass doubles it, exactly: unit data on the same grid points)."""
    import torch

    from tconvolve import burnin

    lines = []
    r = burnin.run(2, printer=lines.append, n_samples=4000, w_size=9, g_size=1024, cell_size=40.286094970136006)
    assert r["grid_errors"] == 0 and r["degrid_errors"] == 0 and r["ranks"] == 1
    assert any("Gridding error count:           0" in s for s in lines)
    b = burnin.BurnIn(n_samples=4000, w_size=9, g_size=1024, cell_size=40.286094970136006)
    b.run_grid()
    g1 = b.grid.clone()
    b.run_grid()
    assert torch.equal(b.grid, 2 * g1)
