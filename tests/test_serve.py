"""Serving: the request loop with continuous batching (tcv_server_*).

Bars (written here, used below):
  * each request's result is the same alone and in a mix: bit-identical (tolerance 0), since a
    job's sums do not depend on the other jobs of its batch;
  * requests on one grid apply in submission order (the mix equals the sequential solo runs);
  * the results are the reference's: rel-L2 <= 1e-5 (REL_L2_FP32) against the oracle;
  * grids beyond the device-memory budget and requests beyond the batch size are refused.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import REL_L2_FP32
from tconvolve.workload import ARCSEC_CELL_1024

pytestmark = pytest.mark.gpu

N = 6000  # samples per request (the served geometry is the 1024^2, 9-plane, 5 arcsec problem)


def _server(tcv, **kw):
    from tconvolve.serve import Server

    args = dict(streams=2, max_batch=8, batch_samples=4 * N)
    args.update(kw)
    return Server(**args)


def _random_grid(seed, g=1024):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(g * g, dtype=np.float32) + 1j * rng.standard_normal(g * g, dtype=np.float32)).astype(
        np.complex64)


def _oracle_offsets(orc, u, v, w):
    from tconvolve.workload import Problem

    prob = Problem("served", u.size, 9, 1, 1024, ARCSEC_CELL_1024)
    cfg = orc.Config(prob.n_samples, prob.w_size, 1, prob.g_size, prob.cell_size, prob.baseline, 0)
    c, _, support, os_, wcs, _ = orc.init_c(cfg)
    iu, iv, co = orc.init_offsets(cfg, u, v, w, wcs, support, os_)
    return c, support, iu, iv, co


def test_same_result_alone_and_in_mix(tcv, orc, cuda_ok):
    from tconvolve._lib import REQ_DEGRID, REQ_GRID
    from tconvolve.serve import request_pool

    pool = request_pool(12, N, seed=3)
    srv = _server(tcv)
    images = [_random_grid(10 + k) for k in range(3)]
    gd = []
    for img in images:
        g = srv.grid_alloc()
        srv.grid_write(g, img)
        gd.append(g)
    # the mix: 6 gridding requests on their own grids and 6 degridding requests on 3 grids, all
    # submitted at once so that they share batches and slots
    ga = [srv.grid_alloc() for _ in range(6)]
    mix = []
    for i in range(6):
        u, v, w, vis = pool[i]
        mix.append(srv.submit(REQ_GRID, ga[i], u, v, w, vis))
        u, v, w, _ = pool[6 + i]
        mix.append(srv.submit(REQ_DEGRID, gd[i % 3], u, v, w))
    infos = [r.wait() for r in mix]
    assert all(i.status == 0 for i in infos)
    assert max(i.batch_requests for i in infos) > 1, "the mix never shared a batch"
    mix_grids = [srv.grid_read(g) for g in ga]
    mix_out = [mix[2 * i + 1].vis_out.copy() for i in range(6)]
    # alone: each request by itself, waited before the next
    ga2 = [srv.grid_alloc() for _ in range(6)]
    for i in range(6):
        u, v, w, vis = pool[i]
        r = srv.submit(REQ_GRID, ga2[i], u, v, w, vis)
        assert r.wait().batch_requests == 1
        assert np.array_equal(srv.grid_read(ga2[i]), mix_grids[i]), f"gridding request {i} differs"
        u, v, w, _ = pool[6 + i]
        r = srv.submit(REQ_DEGRID, gd[i % 3], u, v, w)
        assert r.wait().batch_requests == 1
        assert np.array_equal(r.vis_out, mix_out[i]), f"degridding request {i} differs"
    # the reference's answers (oracle) for one request of each kind
    u, v, w, vis = pool[0]
    c, support, iu, iv, co = _oracle_offsets(orc, u, v, w)
    ref = np.zeros(1024 * 1024, np.complex64)
    orc.grid_f32(vis, support, c, co, iu, iv, ref, 1024, threads=8)
    assert orc.rel_l2(mix_grids[0], ref) <= REL_L2_FP32
    u, v, w, _ = pool[6]
    c, support, iu, iv, co = _oracle_offsets(orc, u, v, w)
    ref_o = orc.degrid_f32(images[0], 1024, support, c, co, iu, iv, threads=8)
    assert orc.rel_l2(mix_out[0], ref_o) <= REL_L2_FP32
    srv.close()


def test_requests_on_one_grid_apply_in_order(tcv, cuda_ok):
    from tconvolve._lib import REQ_DEGRID, REQ_GRID
    from tconvolve.serve import request_pool

    pool = request_pool(3, N, seed=5)
    srv = _server(tcv)
    g = srv.grid_alloc()
    a = srv.submit(REQ_GRID, g, *pool[0])
    b = srv.submit(REQ_GRID, g, *pool[1])
    d = srv.submit(REQ_DEGRID, g, *pool[2][:3])
    for r in (a, b, d):
        assert r.wait().status == 0
    mixed_grid, mixed_out = srv.grid_read(g), d.vis_out.copy()
    g2 = srv.grid_alloc()
    for i in range(2):
        srv.submit(REQ_GRID, g2, *pool[i]).wait()
    d2 = srv.submit(REQ_DEGRID, g2, *pool[2][:3])
    d2.wait()
    assert np.array_equal(srv.grid_read(g2), mixed_grid)
    assert np.array_equal(d2.vis_out, mixed_out)
    assert np.count_nonzero(mixed_out) > 0
    srv.close()


def test_admission_limits(tcv, cuda_ok):
    from tconvolve._lib import REQ_GRID, TcvError
    from tconvolve.serve import request_pool

    srv = _server(tcv)
    held = srv.stats()["bytes_held"]
    srv.close()
    grid_bytes = 1024 * 1024 * 8
    srv = _server(tcv, hbm_budget=held + 2.5 * grid_bytes)
    g0, g1 = srv.grid_alloc(), srv.grid_alloc()
    with pytest.raises(TcvError) as e:
        srv.grid_alloc()
    assert e.value.status == 3  # TCV_ERR_OOM: over the budget
    srv.grid_free(g1)
    srv.grid_alloc()  # the freed grid's memory is admitted again
    big = request_pool(1, 4 * N + 1, seed=1)[0]
    with pytest.raises(TcvError) as e:
        srv.submit(REQ_GRID, g0, *big)
    assert e.value.status == 8  # larger than a batch
    srv.close()
    with pytest.raises(TcvError) as e:
        _server(tcv, hbm_budget=held // 2)
    assert e.value.status == 3


def test_poisson_load(tcv, cuda_ok):
    from tconvolve.serve import poisson_run, request_pool

    srv = _server(tcv, batch_samples=32 * 16000, max_batch=32)
    grids = [srv.grid_alloc() for _ in range(16)]
    pool = request_pool(8, 16000, seed=2)
    r = poisson_run(srv, rate=300, duration=0.5, pool=pool, grids=grids)
    assert r["requests"] > 50 and r["errors"] == 0
    assert 0 < r["p50_ms"] <= r["p99_ms"]
    assert srv.stats()["completed"] == r["requests"]
    srv.close()


@pytest.mark.parametrize("tuning", [(8, 32, 32, 128, 2), (16, 32, 32, 32)], ids=["default", "tile-kernels"])
def test_graph_replay_matches_direct_launches(tcv, cuda_ok, tuning):
    """Batches replayed as CUDA graphs (the default, for batches of up to 4 requests) and launched
    call by call give the same bits; the same batch shapes repeat, so the graph path updates its
    executable graphs in place."""
    from tconvolve._lib import REQ_DEGRID, REQ_GRID
    from tconvolve.serve import request_pool

    pool = request_pool(8, N, seed=11)
    image = _random_grid(21)
    results = []
    for graphs in (True, False):
        srv = _server(tcv, graphs=graphs, tuning=tuning)
        gd = srv.grid_alloc()
        srv.grid_write(gd, image)
        grids, outs = [], []
        for rnd in range(3):  # three rounds of the same shapes
            ga = [srv.grid_alloc() for _ in range(2)]
            reqs = [srv.submit(REQ_GRID, ga[i], *pool[i]) for i in range(2)]
            degs = [srv.submit(REQ_DEGRID, gd, *pool[4 + i][:3]) for i in range(2)]
            assert all(r.wait().status == 0 for r in reqs + degs)
            assert max(r.info.batch_requests for r in reqs + degs) <= 4
            grids.append([srv.grid_read(g) for g in ga])
            outs.append([d.vis_out.copy() for d in degs])
        results.append((grids, outs))
        srv.close()
    (g1, o1), (g2, o2) = results
    for rnd in range(3):
        for i in range(2):
            assert np.array_equal(g1[rnd][i], g2[rnd][i])
            assert np.array_equal(o1[rnd][i], o2[rnd][i])
            assert np.array_equal(g1[rnd][i], g1[0][i]) and np.array_equal(o1[rnd][i], o1[0][i])
    assert np.count_nonzero(o1[0][0]) > 0
