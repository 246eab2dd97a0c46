"""Batched plans (many jobs sharing one table), CUDA-graph replay and the autotuner.

Bars (written here, used below):
  * a job's grid and degridded samples from a batch are bit-identical to the same job run alone
    with the same tuning: the order of the sums at a grid point or a sample does not depend on
    the other jobs;
  * every job, and every tuning, is within the FP32 bar (rel-L2 <= 1e-5, REL_L2_FP32) of the
    oracle run on that job's in-bounds samples;
  * gridding with the same plane groups is bit-identical for every tile shape (a grid point's
    samples are summed in index order within each group whatever the tile);
  * a captured graph gives bit-identical results to the direct calls.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import REL_L2_FP32, VIS_SEED
from tconvolve.workload import ARCSEC_CELL_1024, batch_sizes

pytestmark = pytest.mark.gpu

# uneven jobs on the 9-plane, 45^2-footprint table; the 256 grid is too small for some of its
# footprints (those samples are rejected), one job is empty
SIZES = [(3000, 512), (0, 384), (5000, 1024), (1500, 256), (4000, 384), (700, 2048)]
W_SIZE = 9


@pytest.fixture(scope="module")
def prob(tcv, cuda_ok):
    from tconvolve.batch import make_problem

    return make_problem(SIZES, w_size=W_SIZE, cell_size=ARCSEC_CELL_1024, vis_seed=VIS_SEED)


def _zeros(sizes):
    import torch

    return [torch.zeros(g * g, dtype=torch.complex64, device="cuda") for _, g in sizes]


def _keep(iu, iv, co, support, g, c_len):
    s = 2 * support + 1
    fx = iu.astype(np.int64) - support
    return (fx >= 0) & (fx + s <= g) & (iv >= 0) & (iv.astype(np.int64) + s <= g) & (co >= 0) & \
        (co.astype(np.int64) + s * s <= c_len)


def _host(prob):
    return {k: prob[k].cpu().numpy() for k in ("iu", "iv", "coff", "data", "c64")}


def _oracle_job(orc, h, at, n, g, support, c_len):
    sl = slice(at, at + n)
    iu, iv, co, vis = h["iu"][sl], h["iv"][sl], h["coff"][sl], h["data"][sl]
    keep = _keep(iu, iv, co, support, g, c_len)
    ref = np.zeros(g * g, np.complex64)
    orc.grid_f32(vis[keep], support, h["c64"], co[keep], iu[keep], iv[keep], ref, g, threads=8)
    ref_o = orc.degrid_f32(ref, g, support, h["c64"], co[keep], iu[keep], iv[keep], threads=8)
    return ref, ref_o, keep


def _run_batch(tcv, prob, sizes, tuning=None, c=None, c_type=None, c_scale=1.0):
    import torch

    from tconvolve.batch import Batch

    c = prob["c64"] if c is None else c
    c_type = tcv.C64 if c_type is None else c_type
    grids = _zeros(sizes)
    b = Batch(sizes, grids, prob["iu"], prob["iv"], prob["coff"], prob["support"], prob["c_len"], tuning=tuning)
    b.grid(prob["data"], c, c_type, c_scale)
    out = torch.full((prob["total"],), 7 + 7j, dtype=torch.complex64, device="cuda")
    b.degrid(c, c_type, out, c_scale)
    torch.cuda.synchronize()
    return b, grids, out


def test_batch_matches_single_jobs_and_oracle(tcv, orc, prob):
    import torch

    from tconvolve import raw

    b, grids, out = _run_batch(tcv, prob, SIZES)
    h = _host(prob)
    support, c_len = prob["support"], prob["c_len"]
    at, rejected = 0, 0
    for j, (n, g) in enumerate(SIZES):
        sl = slice(at, at + n)
        alone = torch.zeros(g * g, dtype=torch.complex64, device="cuda")
        plan = raw.Plan(prob["iu"][sl].contiguous(), prob["iv"][sl].contiguous(), prob["coff"][sl].contiguous(),
                        support, g, c_len)
        plan.grid(prob["data"][sl].contiguous(), prob["c64"], tcv.C64, alone)
        alone_out = torch.empty(n, dtype=torch.complex64, device="cuda")
        plan.degrid(alone, prob["c64"], tcv.C64, alone_out)
        torch.cuda.synchronize()
        assert torch.equal(grids[j], alone), f"job {j} grid differs from the job alone"
        assert torch.equal(out[sl], alone_out), f"job {j} samples differ from the job alone"
        ref, ref_o, keep = _oracle_job(orc, h, at, n, g, support, c_len)
        o = out[sl].cpu().numpy()
        assert np.all(o[~keep] == 0)
        if n:
            assert orc.rel_l2(grids[j].cpu().numpy(), ref) <= REL_L2_FP32
            assert orc.rel_l2(o[keep], ref_o) <= REL_L2_FP32
        rejected += int((~keep).sum())
        at += n
    assert rejected > 0  # the 256 grid is too small for some footprints
    assert b.rejected() == rejected


@pytest.mark.parametrize("rows", [8, 16, 32])
@pytest.mark.parametrize("mib", [32, 8, -1])
@pytest.mark.parametrize("split,dsplit", [(0, 0), (64, 64), (0, 128)])
def test_tunings_agree(tcv, orc, prob, rows, mib, split, dsplit):
    """Every tile shape, plane-group size and work-unit size gives the oracle's answer; with cells
    whole, gridding is bit-identical across tile shapes with the same plane groups."""
    b, grids, out = _run_batch(tcv, prob, SIZES, tuning=(rows, mib, split, dsplit))
    assert b.tuning() == (rows, mib, split, dsplit)
    _, base_grids, _ = _run_batch(tcv, prob, SIZES, tuning=(16, mib, 0, 0))
    h = _host(prob)
    at = 0
    for j, (n, g) in enumerate(SIZES):
        if split == 0:
            assert np.array_equal(grids[j].cpu().numpy(), base_grids[j].cpu().numpy())
        if n:
            ref, ref_o, keep = _oracle_job(orc, h, at, n, g, prob["support"], prob["c_len"])
            assert orc.rel_l2(grids[j].cpu().numpy(), ref) <= REL_L2_FP32
            assert orc.rel_l2(out[at:at + n].cpu().numpy()[keep], ref_o) <= REL_L2_FP32
        at += n


def test_graph_replay_matches_direct_calls(tcv, prob):
    import torch

    from tconvolve._lib import PASS_BIN, PASS_DEGRID, PASS_GRID
    from tconvolve.batch import Batch

    _, direct, direct_out = _run_batch(tcv, prob, SIZES, tuning=(8, 32, 64, 256))
    grids = _zeros(SIZES)
    b = Batch(SIZES, grids, prob["iu"], prob["iv"], prob["coff"], prob["support"], prob["c_len"],
              tuning=(8, 32, 64, 256))
    out = torch.empty(prob["total"], dtype=torch.complex64, device="cuda")
    graph = b.capture(PASS_BIN | PASS_GRID | PASS_DEGRID, prob["data"], prob["c64"], tcv.C64, vis=out)
    for gr in grids:
        gr.zero_()
    graph.launch()
    torch.cuda.synchronize()
    for j in range(len(SIZES)):
        assert torch.equal(grids[j], direct[j])
    assert torch.equal(out, direct_out)
    graph.launch()  # gridding accumulates: two replays add the pass twice
    torch.cuda.synchronize()
    for j in range(len(SIZES)):
        assert torch.allclose(grids[j], 2 * direct[j], rtol=1e-6, atol=1e-6)
    graph.close()


def test_autotuner(tcv, prob):
    from tconvolve.batch import Batch, autotune

    best, ms, report = autotune(SIZES, prob["iu"], prob["iv"], prob["coff"], prob["data"], prob["c64"], tcv.C64,
                                prob["support"], reps=2)
    assert ms > 0 and len(report) >= 3
    assert best in [t for t, _ in report]
    assert ms == min(m for _, m in report)
    assert {t[0] for t, _ in report} == {8, 16, 32}
    assert {t[2] for t, _ in report} == {0, 512, 256, 128, 64}
    assert {t[3] for t, _ in report} == {0, 512, 256, 128, 64}
    again, ms2, _ = autotune(SIZES, prob["iu"], prob["iv"], prob["coff"], prob["data"], prob["c64"], tcv.C64,
                             prob["support"], reps=2)
    assert again == best and ms2 == ms  # cached
    b = Batch(SIZES, _zeros(SIZES), prob["iu"], prob["iv"], prob["coff"], prob["support"], prob["c_len"],
              tuning=best)
    assert b.tuning() == best


@pytest.mark.parametrize("form", ["r32", "rbf16"])
def test_batch_table_forms(tcv, orc, prob, form):
    """The batched path takes every table form: r32 is bit-identical to c64, bf16 within its bound."""
    from tconvolve import raw

    c, scale, _ = raw.convert_c(prob["c64"], tcv.CTYPE_BY_NAME[form])
    _, grids, out = _run_batch(tcv, prob, SIZES, c=c, c_type=tcv.CTYPE_BY_NAME[form], c_scale=scale)
    _, g64, o64 = _run_batch(tcv, prob, SIZES)
    for j in range(len(SIZES)):
        if form == "r32":
            assert np.array_equal(grids[j].cpu().numpy(), g64[j].cpu().numpy())
        else:
            assert orc.rel_l2(grids[j].cpu().numpy(), g64[j].cpu().numpy()) <= 6e-3
    if form == "r32":
        assert np.array_equal(out.cpu().numpy(), o64.cpu().numpy())


def test_full_size_batch(tcv):
    """The 64-job batch (6.7 M samples, 2048^2 and 4096^2 grids, 129^2 footprints): the rejected
    samples are exactly those whose footprint leaves their grid (the reference's footprint spans
    rows iv .. iv + 2*support, so on a 2048 grid samples with v above about 958 m would write past
    the last row), and the first and the largest job are bit-identical to the job alone."""
    import torch

    from tconvolve import raw
    from tconvolve.batch import make_problem

    sizes = batch_sizes(64, seed=0)
    p = make_problem(sizes, vis_seed=VIS_SEED)
    b, grids, out = _run_batch(tcv, p, sizes)
    first = np.cumsum([0] + [n for n, _ in sizes])
    iu, iv, co = (p[k].cpu().numpy() for k in ("iu", "iv", "coff"))
    outside = 0
    for j, (n, g) in enumerate(sizes):
        sl = slice(int(first[j]), int(first[j]) + n)
        keep = _keep(iu[sl], iv[sl], co[sl], p["support"], g, p["c_len"])
        outside += int((~keep).sum())
        if g == 4096:
            assert keep.all()
    assert 0 < outside < p["total"] // 50
    assert b.rejected() == outside
    for j in (0, int(np.argmax([n for n, _ in sizes]))):
        n, g = sizes[j]
        sl = slice(int(first[j]), int(first[j]) + n)
        alone = torch.zeros(g * g, dtype=torch.complex64, device="cuda")
        plan = raw.Plan(p["iu"][sl].contiguous(), p["iv"][sl].contiguous(), p["coff"][sl].contiguous(),
                        p["support"], g, p["c_len"])
        plan.grid(p["data"][sl].contiguous(), p["c64"], tcv.C64, alone)
        o = torch.empty(n, dtype=torch.complex64, device="cuda")
        plan.degrid(alone, p["c64"], tcv.C64, o)
        torch.cuda.synchronize()
        assert torch.equal(grids[j], alone)
        assert torch.equal(out[sl], o)


@pytest.mark.parametrize("tuning", [(8, 32, 0, 128, 2), (8, 32, 128, 128, 3), (8, -1, 64, 64, 3)])
def test_sample_parallel_passes(tcv, orc, prob, tuning):
    """The sample-parallel kernels on a fixed-width batch (45^2 footprints): every job within the
    FP32 bar of the oracle, each job bit-identical to the same job alone with the same tuning, and
    the batch bit-identical when rerun."""
    import torch

    from tconvolve import raw

    b, grids, out = _run_batch(tcv, prob, SIZES, tuning=tuning)
    assert b.tuning() == tuning
    _, grids2, out2 = _run_batch(tcv, prob, SIZES, tuning=tuning)
    assert torch.equal(out, out2)
    h = _host(prob)
    support, c_len = prob["support"], prob["c_len"]
    at = 0
    for j, (n, g) in enumerate(SIZES):
        assert torch.equal(grids[j], grids2[j])
        if n:
            sl = slice(at, at + n)
            alone = torch.zeros(g * g, dtype=torch.complex64, device="cuda")
            plan = raw.Plan(prob["iu"][sl].contiguous(), prob["iv"][sl].contiguous(), prob["coff"][sl].contiguous(),
                            support, g, c_len, tuning=tuning)
            plan.grid(prob["data"][sl].contiguous(), prob["c64"], tcv.C64, alone)
            alone_out = torch.empty(n, dtype=torch.complex64, device="cuda")
            plan.degrid(alone, prob["c64"], tcv.C64, alone_out)
            torch.cuda.synchronize()
            assert torch.equal(grids[j], alone), f"job {j} grid differs from the job alone"
            assert torch.equal(out[sl], alone_out), f"job {j} samples differ from the job alone"
            ref, ref_o, keep = _oracle_job(orc, h, at, n, g, support, c_len)
            assert orc.rel_l2(grids[j].cpu().numpy(), ref) <= REL_L2_FP32
            assert orc.rel_l2(out[sl].cpu().numpy()[keep], ref_o) <= REL_L2_FP32
            assert np.all(out[sl].cpu().numpy()[~keep] == 0)
        at += n
