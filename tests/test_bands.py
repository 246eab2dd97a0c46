"""Row-band split of one job over several ranks (tconvolve.bands, csrc/tcv_bands.cu).

CPU: the bounds (host arithmetic of the library), the exchange plan, and the whole split as gloo
ranks with the oracle standing in for the device (world sizes 2 and 3, and a planted dropped
halo that the check must catch).  GPU: the device steps bit for bit against numpy, and the whole
split with its ranks as threads on one GPU (each on its own stream; no kernel waits on another
rank's), checked against the oracle and against the one-GPU plan.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import PKG, REL_L2_FP32, REPO, VIS_SEED, oracle_config
from tconvolve.workload import PROBLEMS, normal_vis


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _setup(orc, prob):
    cfg = oracle_config(orc, prob)
    u, v, w = orc.init_uvw(cfg)
    c, _, support, os_, wcs, _ = orc.init_c(cfg, want_f64=False)
    iu, iv, co = orc.init_offsets(cfg, u, v, w, wcs, support, os_)
    return c, support, iu, iv, co


def _shares(n: int, size: int):
    return [(r * n // size, (r + 1) * n // size) for r in range(size)]


# ----------------------------------------------------------------------------------------------
# CPU
# ----------------------------------------------------------------------------------------------
def test_bounds_balance_and_heights(tcv):
    from tconvolve.bands import band_bounds

    rng = np.random.default_rng(5)
    g = 512
    for support, nb in [(0, 1), (14, 2), (14, 3), (22, 8), (64, 8), (1, 64)]:
        for hist in (np.full(g, 7, np.int64),
                     np.bincount(np.clip(rng.normal(g / 2, g / 12, 20000).astype(int), 0, g - 1), minlength=g),
                     np.zeros(g, np.int64)):
            rows = band_bounds(hist, g, support, nb)
            assert rows[0] == 0 and rows[-1] == g and len(rows) == nb + 1
            h = np.diff(rows)
            assert np.all(h >= max(support, 1))
            # where no height bound moved them, the bounds cut the samples into equal shares
            # (to within one row's samples)
            total = int(hist.sum())
            cum = np.concatenate([[0], np.cumsum(hist)])
            free = all(rows[b] - rows[b - 1] > max(support, 1) and rows[b + 1] - rows[b] > max(support, 1)
                       for b in range(1, nb))
            if free and total:
                for b in range(1, nb):
                    target = -(-total * b // nb)
                    assert cum[rows[b]] >= target
                    assert cum[rows[b] - 1] < target
            assert rows == band_bounds(hist, g, support, nb)  # deterministic


def test_bounds_reject_bad_arguments(tcv):
    from tconvolve.bands import band_bounds

    hist = np.ones(256, np.int64)
    with pytest.raises(tcv.TcvError):
        band_bounds(hist, 256, 64, 5)  # 5 bands of 64 rows do not fit 256 rows
    with pytest.raises(tcv.TcvError):
        band_bounds(hist, 256, 1, 0)
    with pytest.raises(tcv.TcvError):
        band_bounds(hist, 256, 1, 65)
    bad = hist.copy()
    bad[3] = -1
    with pytest.raises(tcv.TcvError):
        band_bounds(bad, 256, 1, 2)


def test_halo_plan_pairs_up():
    from tconvolve.bands import halo_plan

    rows, s = [0, 100, 140, 300, 512], 40
    plans = [halo_plan(rows, b, s) for b in range(4)]
    for b in range(4):
        for kind, other in (("grid_send", "grid_recv"), ("fetch_send", "fetch_recv")):
            for peer, a, e in plans[b][kind]:
                assert e - a == s
                assert (b, a, e) in plans[peer][other]  # the peer expects exactly these rows
    assert plans[0]["grid_send"] == [(1, 100, 140)] and plans[0]["fetch_recv"] == [(1, 100, 140)]
    assert plans[3]["grid_send"] == [(2, 260, 300)] and plans[3]["fetch_recv"] == [(2, 260, 300)]
    assert halo_plan(rows, 1, 0) == {"grid_send": [], "grid_recv": [], "fetch_send": [], "fetch_recv": []}


def _gloo_worker(rank, world, port, prob_name, drop_halo, q):
    import datetime
    import sys

    for p in (REPO, PKG, os.path.join(REPO, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch
    import torch.distributed as dist

    from band_helpers import NumpyBandOps
    from oracle import oracle as O
    from tconvolve.bands import BandJob, DistComm
    from tconvolve.workload import PROBLEMS, normal_vis

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        prob = PROBLEMS[prob_name]
        c, support, iu, iv, co = _setup(O, prob)
        vis = normal_vis(iu.size, VIS_SEED)
        a, e = _shares(iu.size, world)[rank]
        comm = DistComm()
        if drop_halo:
            real_exchange = comm.exchange

            def exchange(sends, recvs):  # a planted fault: the halos arrive as zeros
                real_exchange(sends, recvs)
                for _, t in recvs:
                    t.zero_()

            comm.exchange = exchange
        t = torch.from_numpy
        job = BandJob(t(vis[a:e].copy()), t(iu[a:e].copy()), t(iv[a:e].copy()), t(co[a:e].copy()), support,
                      prob.g_size, c.size, comm=comm, ops=NumpyBandOps(O, c))
        grid = torch.zeros(prob.g_size ** 2, dtype=torch.complex64)
        job.grid(grid, None, 0)
        r0, r1 = job.band
        band_rows = grid[r0 * prob.g_size:r1 * prob.g_size].numpy().copy()
        out = torch.empty(e - a, dtype=torch.complex64)
        job.degrid(grid, None, 0, out)
        q.put((rank, job.rows, band_rows, out.numpy().copy(), job.n_band))
    finally:
        dist.destroy_process_group()


def _run_gloo(world: int, prob_name: str, drop_halo: bool = False):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_worker, args=(r, world, port, prob_name, drop_halo, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=180) for _ in procs], key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


def _assemble(out, g):
    grid = np.zeros(g * g, np.complex64)
    rows = out[0][1]
    for rank, r, band_rows, _, _ in out:
        assert r == rows  # every rank computed the same bounds
        grid[rows[rank] * g:rows[rank + 1] * g] = band_rows
    return grid, np.concatenate([o[3] for o in out])


@pytest.mark.parametrize("world", [2, 3])
def test_band_split_gloo_matches_oracle(orc, world):
    prob = PROBLEMS["g2"]
    c, support, iu, iv, co = _setup(orc, prob)
    vis = normal_vis(iu.size, VIS_SEED)
    ref = np.zeros(prob.g_size ** 2, np.complex64)
    orc.grid_f32(vis, support, c, co, iu, iv, ref, prob.g_size)
    out = _run_gloo(world, "g2")
    assert sum(o[4] for o in out) == iu.size  # every sample gridded by exactly one rank
    assert min(o[4] for o in out) > 0
    grid, deg = _assemble(out, prob.g_size)
    assert orc.rel_l2(grid, ref) <= REL_L2_FP32
    # degridding reads the same rows as the whole grid holds: the reference's per-sample sums
    assert np.array_equal(deg, orc.degrid_f32(grid, prob.g_size, support, c, co, iu, iv))
    assert orc.rel_l2(deg, orc.degrid_f32(ref, prob.g_size, support, c, co, iu, iv)) <= REL_L2_FP32


def test_band_split_gloo_dropped_halo_is_caught(orc):
    prob = PROBLEMS["g2"]
    c, support, iu, iv, co = _setup(orc, prob)
    vis = normal_vis(iu.size, VIS_SEED)
    ref = np.zeros(prob.g_size ** 2, np.complex64)
    orc.grid_f32(vis, support, c, co, iu, iv, ref, prob.g_size)
    grid, _ = _assemble(_run_gloo(2, "g2", drop_halo=True), prob.g_size)
    assert orc.rel_l2(grid, ref) > 1e-3


# ----------------------------------------------------------------------------------------------
# GPU
# ----------------------------------------------------------------------------------------------
def _random_samples(n: int, g: int, support: int, seed: int):
    rng = np.random.default_rng(seed)
    iv = rng.integers(-3 * support, g + support, n).astype(np.int32)  # some outside the grid
    iu = rng.integers(0, g, n).astype(np.int32)
    co = rng.integers(0, 1 << 20, n).astype(np.int32)
    return normal_vis(n, seed), iu, iv, co


@pytest.mark.gpu
@pytest.mark.parametrize("n", [0, 1, 4095, 4096, 4097, 100003])
@pytest.mark.parametrize("nb", [1, 2, 5, 64])
def test_histogram_and_bucket_match_numpy(tcv, cuda_ok, n, nb):
    import sys

    import torch

    sys.path.insert(0, os.path.join(REPO, "tests"))
    from band_helpers import bucket_numpy, centre_rows
    from tconvolve.bands import CudaBandOps, band_bounds

    g, support = 4096, 64 if nb < 64 else 8
    vis, iu, iv, co = _random_samples(n, g, support, 11 + n + nb)
    d = [torch.from_numpy(a).cuda() for a in (vis, iu, iv, co)]
    ops = CudaBandOps()
    hist = ops.histogram(d[2], support, g).cpu().numpy()
    assert np.array_equal(hist, np.bincount(centre_rows(iv, support, g), minlength=g))
    rows = band_bounds(hist, g, support, nb)
    rec, perm, counts = ops.bucket(*d, support, g, rows)
    ref_rec, ref_perm, ref_counts = bucket_numpy(vis, iu, iv, co, support, g, rows)
    assert counts == [int(x) for x in ref_counts]
    assert np.array_equal(rec.cpu().numpy(), ref_rec)
    assert np.array_equal(perm.cpu().numpy(), ref_perm)
    # unpack, scatter and the halo add undo / redo the partition exactly
    data, iu2, iv2, co2 = ops.unpack(rec)
    assert np.array_equal(data.cpu().numpy()[np.argsort(ref_perm)], vis)
    assert np.array_equal(iv2.cpu().numpy(), iv[ref_perm]) and np.array_equal(co2.cpu().numpy(), co[ref_perm])
    back = torch.empty_like(d[0])
    ops.scatter(data, perm, back)
    assert np.array_equal(back.cpu().numpy(), vis)
    if n:
        acc = d[0].clone()
        ops.rows_add(acc, d[0])
        assert np.array_equal(acc.cpu().numpy(), vis + vis)
        odd = d[0][1:].clone()  # an unaligned, odd-length add
        ops.rows_add(odd, d[0][:-1])
        assert np.array_equal(odd.cpu().numpy(), vis[1:] + vis[:-1])


def _band_split_on_threads(prob, size, c, support, iu, iv, co, vis, tuning):
    import sys

    import torch

    sys.path.insert(0, os.path.join(REPO, "tests"))
    from band_helpers import run_threads
    from tconvolve.bands import BandJob, CudaBandOps

    g = prob.g_size
    dc = torch.from_numpy(c).cuda()
    shares = _shares(iu.size, size)

    def rank_fn(rank, comm):
        a, e = shares[rank]
        d = [torch.from_numpy(np.ascontiguousarray(x[a:e])).cuda() for x in (vis, iu, iv, co)]
        job = BandJob(*d, support, g, c.size, comm=comm, ops=CudaBandOps(), tuning=tuning)
        grid = torch.zeros(g * g, dtype=torch.complex64, device="cuda")
        job.grid(grid, dc, tcv_c64())
        r0, r1 = job.band
        band_rows = grid[r0 * g:r1 * g].cpu().numpy()
        out = torch.empty(e - a, dtype=torch.complex64, device="cuda")
        job.degrid(grid, dc, tcv_c64(), out)
        return job.rows, band_rows, out.cpu().numpy(), job.rejected()

    res = run_threads(size, rank_fn)
    rows = res[0][0]
    grid = np.zeros(g * g, np.complex64)
    for rank, (r, band_rows, _, rej) in enumerate(res):
        assert r == rows and rej == 0
        grid[rows[rank] * g:rows[rank + 1] * g] = band_rows
    return rows, grid, np.concatenate([x[2] for x in res])


def tcv_c64():
    import tconvolve

    return tconvolve.C64


@pytest.mark.gpu
@pytest.mark.parametrize("size", [1, 2, 3, 4])
def test_band_split_threads_match_oracle_and_one_gpu(tcv, orc, cuda_ok, size):
    import torch

    from tconvolve import raw

    prob = PROBLEMS["c1"]
    c, support, iu, iv, co = _setup(orc, prob)
    vis = normal_vis(iu.size, VIS_SEED)
    tuning = (16, 32, 0, 0)
    rows, grid, deg = _band_split_on_threads(prob, size, c, support, iu, iv, co, vis, tuning)
    assert len(rows) == size + 1
    ref = np.zeros(prob.g_size ** 2, np.complex64)
    orc.grid_f32(vis, support, c, co, iu, iv, ref, prob.g_size)
    assert orc.rel_l2(grid, ref) <= REL_L2_FP32
    assert orc.rel_l2(deg, orc.degrid_f32(ref, prob.g_size, support, c, co, iu, iv)) <= REL_L2_FP32
    # degridding the assembled grid on one GPU with the same tile shape gives the same bits
    d = [torch.from_numpy(a).cuda() for a in (iu, iv, co)]
    plan = raw.Plan(*d, support, prob.g_size, c.size, tuning=tuning)
    one = torch.empty(iu.size, dtype=torch.complex64, device="cuda")
    plan.degrid(torch.from_numpy(grid).cuda(), torch.from_numpy(c).cuda(), tcv.C64, one)
    assert np.array_equal(deg, one.cpu().numpy())


@pytest.mark.gpu
def test_band_split_threads_full_size(tcv, cuda_ok):
    """The 4096^2 problem of 160000 samples split over 4 bands against one GPU's plan (grid within
    the path's bar; degridding of the same grid bit for bit)."""
    import torch

    import tconvolve
    from tconvolve import raw

    prob = PROBLEMS["c2"]
    with tconvolve.Benchmark(**prob.kwargs(), device=0) as b:
        b.init()
        support = b.getSupport()
        iu, iv, co = b.offsets()
        c = b.C()
    vis = normal_vis(iu.size, VIS_SEED)
    tuning = (16, 64, 0, 64)
    rows, grid, deg = _band_split_on_threads(prob, 4, c, support, iu, iv, co, vis, tuning)
    d = [torch.from_numpy(a).cuda() for a in (vis, iu, iv, co)]
    dc = torch.from_numpy(c).cuda()
    plan = raw.Plan(*d[1:], support, prob.g_size, c.size, tuning=tuning)
    one = torch.zeros(prob.g_size ** 2, dtype=torch.complex64, device="cuda")
    plan.grid(d[0], dc, tcv.C64, one)
    one_h = one.cpu().numpy()
    num = np.linalg.norm((grid - one_h).astype(np.complex128))
    assert num / np.linalg.norm(one_h.astype(np.complex128)) <= REL_L2_FP32
    out = torch.empty(iu.size, dtype=torch.complex64, device="cuda")
    plan.degrid(torch.from_numpy(grid).cuda(), dc, tcv.C64, out)
    assert np.array_equal(deg, out.cpu().numpy())
    # the bands balance the samples: no band holds more than 1.5x its share
    counts = np.bincount(np.searchsorted(np.asarray(rows[1:-1]), np.clip(iv + support, 0, prob.g_size - 1),
                                         side="right"), minlength=4)
    assert counts.max() <= 1.5 * iu.size / 4


def _narrow_samples(orc, prob):
    """The problem's samples moved into a narrow band of rows (so that the bounds leave some band
    without samples), plus a few whose footprint leaves the grid."""
    c, support, iu, iv, co = _setup(orc, prob)
    g = prob.g_size
    rng = np.random.default_rng(3)
    iv = (g // 3 + rng.integers(0, 8, iv.size)).astype(np.int32)  # centre rows in [g/3 + s, g/3 + s + 8)
    bad = np.array([5, 17, iu.size - 1])
    iv[bad[:2]] = -1  # footprint starts above the first row
    iu = iu.copy()
    iu[bad[2]] = support - 1  # one column past the left edge
    return c, support, iu, iv, co, bad


def _band_worker_narrow(rank, world, port, q):
    import datetime
    import sys

    for p in (REPO, PKG, os.path.join(REPO, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch
    import torch.distributed as dist

    from band_helpers import NumpyBandOps
    from oracle import oracle as O
    from tconvolve.bands import BandJob, DistComm
    from tconvolve.workload import PROBLEMS, normal_vis

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        prob = PROBLEMS["g2"]
        c, support, iu, iv, co, bad = _narrow_samples(O, prob)
        keep = np.ones(iu.size, bool)
        keep[bad] = False
        vis = normal_vis(iu.size, VIS_SEED)
        a, e = _shares(iu.size, world)[rank]
        t = torch.from_numpy
        # the oracle plans grid every sample they are given: hand them the in-bounds ones, as the
        # device plans do after counting the others out
        sl = slice(a, e)
        m = keep[sl]
        job = BandJob(t(vis[sl][m].copy()), t(iu[sl][m].copy()), t(iv[sl][m].copy()), t(co[sl][m].copy()), support,
                      prob.g_size, c.size, comm=DistComm(), ops=NumpyBandOps(O, c))
        grid = torch.zeros(prob.g_size ** 2, dtype=torch.complex64)
        job.grid(grid, None, 0)
        r0, r1 = job.band
        q.put((rank, job.rows, grid[r0 * prob.g_size:r1 * prob.g_size].numpy().copy(), np.zeros(0, np.complex64),
               job.n_band))
    finally:
        dist.destroy_process_group()


def test_band_split_gloo_empty_band(orc):
    """Samples in a narrow range of rows: the bounds keep every band at least `support` rows high,
    so one band holds no sample and its rank only takes part in the exchanges."""
    prob = PROBLEMS["g2"]
    c, support, iu, iv, co, bad = _narrow_samples(orc, prob)
    keep = np.ones(iu.size, bool)
    keep[bad] = False
    vis = normal_vis(iu.size, VIS_SEED)
    ref = np.zeros(prob.g_size ** 2, np.complex64)
    orc.grid_f32(vis[keep], support, c, co[keep], iu[keep], iv[keep], ref, prob.g_size)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_band_worker_narrow, args=(r, 3, port, q)) for r in range(3)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=180) for _ in procs], key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert min(o[4] for o in out) == 0  # a band without samples
    assert sum(o[4] for o in out) == int(keep.sum())
    grid, _ = _assemble(out, prob.g_size)
    assert orc.rel_l2(grid, ref) <= REL_L2_FP32


@pytest.mark.gpu
def test_band_split_threads_empty_band_and_rejected(tcv, orc, cuda_ok):
    """On one GPU (ranks as threads): a band without samples, and samples outside the grid counted
    out by whichever rank receives them, as one GPU's plan counts them."""
    import sys

    import torch

    sys.path.insert(0, os.path.join(REPO, "tests"))
    from band_helpers import run_threads
    from tconvolve import raw
    from tconvolve.bands import BandJob, CudaBandOps

    prob = PROBLEMS["g2"]
    c, support, iu, iv, co, bad = _narrow_samples(orc, prob)
    g = prob.g_size
    vis = normal_vis(iu.size, VIS_SEED)
    dc = torch.from_numpy(c).cuda()
    shares = _shares(iu.size, 3)

    def rank_fn(rank, comm):
        a, e = shares[rank]
        d = [torch.from_numpy(np.ascontiguousarray(x[a:e])).cuda() for x in (vis, iu, iv, co)]
        job = BandJob(*d, support, g, c.size, comm=comm, ops=CudaBandOps(), tuning=(16, 32, 0, 0))
        grid = torch.zeros(g * g, dtype=torch.complex64, device="cuda")
        job.grid(grid, dc, tcv.C64)
        r0, r1 = job.band
        out = torch.full((e - a,), 7 + 7j, dtype=torch.complex64, device="cuda")
        job.degrid(grid, dc, tcv.C64, out)
        return job.rows, grid[r0 * g:r1 * g].cpu().numpy(), out.cpu().numpy(), job.rejected(), job.n_band

    res = run_threads(3, rank_fn)
    rows = res[0][0]
    assert min(x[4] for x in res) == 0  # a band without samples
    assert res[0][4] > 0  # band 0: the samples above the first row (counted out) beside valid ones
    assert sum(x[3] for x in res) == bad.size
    grid = np.zeros(g * g, np.complex64)
    for rank, (_, band_rows, _, _, _) in enumerate(res):
        grid[rows[rank] * g:rows[rank + 1] * g] = band_rows
    keep = np.ones(iu.size, bool)
    keep[bad] = False
    ref = np.zeros(g * g, np.complex64)
    orc.grid_f32(vis[keep], support, c, co[keep], iu[keep], iv[keep], ref, g)
    assert orc.rel_l2(grid, ref) <= REL_L2_FP32
    deg = np.concatenate([x[2] for x in res])
    assert np.all(deg[bad] == 0)  # counted out: nothing degridded into them
    plan = raw.Plan(*[torch.from_numpy(x).cuda() for x in (iu, iv, co)], support, g, c.size, tuning=(16, 32, 0, 0))
    one = torch.empty(iu.size, dtype=torch.complex64, device="cuda")
    plan.degrid(torch.from_numpy(grid).cuda(), dc, tcv.C64, one)
    assert plan.rejected() == bad.size
    assert np.array_equal(deg, one.cpu().numpy())


@pytest.mark.gpu
def test_bands_program_one_rank(tcv, cuda_ok):
    """`python -m tconvolve.bands` on one process (one band): the reference's report lines."""
    import subprocess
    import sys

    out = subprocess.run([sys.executable, "-m", "tconvolve.bands", "2"], cwd=PKG, capture_output=True, text=True,
                         timeout=600, check=True).stdout
    for line in ("+++++ Forward processing (row bands) +++++", "    Number of processes: 1",
                 "+++++ Reverse processing (row bands) +++++", "Done"):
        assert line in out.splitlines(), line
    rates = [float(ln.split()[2]) for ln in out.splitlines() if ln.strip().startswith(("Gridding rate",
                                                                                     "Degridding rate"))]
    assert len(rates) == 2 and min(rates) > 1e5  # million grid points per second


def test_bands_program_usage():
    import subprocess
    import sys

    r = subprocess.run([sys.executable, "-m", "tconvolve.bands", "x"], cwd=PKG, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 1 and "usage" in r.stderr


def test_band_split_one_rank_without_a_process_group(orc):
    """One band (SoloComm): the split reduces to the plain passes; the oracle stands in for the
    device."""
    import sys

    import torch

    sys.path.insert(0, os.path.join(REPO, "tests"))
    from band_helpers import NumpyBandOps
    from tconvolve.bands import BandJob, SoloComm

    prob = PROBLEMS["g1"]
    c, support, iu, iv, co = _setup(orc, prob)
    vis = normal_vis(iu.size, VIS_SEED)
    t = torch.from_numpy
    job = BandJob(t(vis.copy()), t(iu.copy()), t(iv.copy()), t(co.copy()), support, prob.g_size, c.size,
                  comm=SoloComm(), ops=NumpyBandOps(orc, c))
    assert job.rows == [0, prob.g_size] and job.n_band == iu.size
    assert job.halo == {"grid_send": [], "grid_recv": [], "fetch_send": [], "fetch_recv": []}
    grid = torch.zeros(prob.g_size ** 2, dtype=torch.complex64)
    job.grid(grid, None, 0)
    ref = np.zeros(prob.g_size ** 2, np.complex64)
    orc.grid_f32(vis, support, c, co, iu, iv, ref, prob.g_size)
    assert np.array_equal(grid.numpy(), ref)  # one rank, samples in input order: the reference's sums
    out = torch.empty(iu.size, dtype=torch.complex64)
    job.degrid(grid, None, 0, out)
    assert np.array_equal(out.numpy(), orc.degrid_f32(ref, prob.g_size, support, c, co, iu, iv))
