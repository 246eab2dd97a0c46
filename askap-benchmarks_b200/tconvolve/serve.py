"""Serving: gridding and degridding requests through the library's request loop (tcv_server_*,
include/tconvolve.h) with continuous batching, resident grids and table, and device-memory
admission; plus a Poisson load generator that reports p50/p99 latency and throughput.

A request is one channel of samples at the reference's first frequency (Benchmark.cc:89): u, v, w
in metres and, for gridding, the visibilities, all host arrays.  Latency is measured by the
server from submission to result-ready (the degridded samples in the caller's buffer, or the
gridding pass complete on the device).
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _lib
from ._lib import TcvRequest, TcvRequestInfo, TcvServerConfig, check, lib


class Request:
    """A submitted request; keeps its host arrays alive until it completes."""

    def __init__(self, server, ticket, keep, vis_out):
        self.server, self.ticket, self._keep, self.vis_out = server, ticket, keep, vis_out
        self.info = None

    def wait(self, timeout: float = -1.0):
        if self.info is None:
            info = TcvRequestInfo()
            st = lib().tcv_server_wait(self.server._h, self.ticket, float(timeout), ctypes.byref(info))
            check(st, "tcv_server_wait")
            self.info = info
            self._keep = None
        return self.info

    @property
    def latency_s(self) -> float:
        i = self.wait()
        return i.t_done - i.t_submit


class Server:
    def __init__(self, g_size: int = 1024, w_size: int = 9, cell_size: float | None = None, baseline: int = 2000,
                 c_type: int | str = "r32", streams: int = 2, max_batch: int = 32, batch_samples: int = 262144,
                 hbm_budget: float = 150e9, tuning=(8, 32, 32, 128, 2), device: int = 0, graphs: bool = True):
        cfg = TcvServerConfig()
        lib().tcv_server_config_default(ctypes.byref(cfg))
        cfg.g_size, cfg.w_size, cfg.baseline = g_size, w_size, baseline
        if cell_size is not None:
            cfg.cell_size = cell_size
        cfg.c_type = _lib.CTYPE_BY_NAME[c_type] if isinstance(c_type, str) else int(c_type)
        cfg.streams, cfg.max_batch, cfg.batch_samples = streams, max_batch, batch_samples
        cfg.hbm_budget = int(hbm_budget)
        (cfg.tuning.tile_rows, cfg.tuning.group_mib, cfg.tuning.split, cfg.tuning.degrid_split,
         cfg.tuning.kernel) = (tuple(tuning) + (0, 0, 0))[:5]
        cfg.device = device
        cfg.graphs = 1 if graphs else 0
        self.cfg = cfg
        self._h = ctypes.c_void_p()
        check(lib().tcv_server_create(ctypes.byref(cfg), ctypes.byref(self._h)), "tcv_server_create")

    def grid_alloc(self) -> int:
        g = ctypes.c_int32()
        check(lib().tcv_server_grid_alloc(self._h, ctypes.byref(g)), "tcv_server_grid_alloc")
        return g.value

    def grid_free(self, g: int):
        check(lib().tcv_server_grid_free(self._h, g), "tcv_server_grid_free")

    def grid_read(self, g: int) -> np.ndarray:
        out = np.empty(self.cfg.g_size * self.cfg.g_size, np.complex64)
        check(lib().tcv_server_grid_read(self._h, g, out.ctypes.data_as(ctypes.c_void_p)), "tcv_server_grid_read")
        return out

    def grid_write(self, g: int, values: np.ndarray):
        values = np.ascontiguousarray(values, np.complex64)
        check(lib().tcv_server_grid_write(self._h, g, values.ctypes.data_as(ctypes.c_void_p)), "tcv_server_grid_write")

    def submit(self, kind: int, grid: int, u, v, w, vis=None) -> Request:
        u, v, w = (np.ascontiguousarray(a, np.float64) for a in (u, v, w))
        n = u.size
        r = TcvRequest()
        r.kind, r.grid, r.n = kind, grid, n
        r.u, r.v, r.w = (a.ctypes.data_as(ctypes.c_void_p) for a in (u, v, w))
        keep = [u, v, w]
        out = None
        if kind == _lib.REQ_GRID:
            vis = np.ascontiguousarray(vis, np.complex64)
            r.vis = vis.ctypes.data_as(ctypes.c_void_p)
            keep.append(vis)
        else:
            out = np.empty(n, np.complex64)
            r.vis_out = out.ctypes.data_as(ctypes.c_void_p)
        t = ctypes.c_uint64()
        check(lib().tcv_server_submit(self._h, ctypes.byref(r), ctypes.byref(t)), "tcv_server_submit")
        return Request(self, t.value, keep, out)

    def stats(self) -> dict:
        held, done, batches, pending = ctypes.c_size_t(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        check(lib().tcv_server_stats(self._h, ctypes.byref(held), ctypes.byref(done), ctypes.byref(batches),
                                     ctypes.byref(pending)), "tcv_server_stats")
        return {"bytes_held": held.value, "completed": done.value, "batches": batches.value,
                "pending": pending.value}

    def close(self):
        if self._h:
            lib().tcv_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def request_pool(n_requests: int, n_samples: int = 16000, baseline: int = 2000, seed: int = 0):
    """Inputs for requests: u, v, w uniform in [-baseline/2, baseline/2] m (the reference's
    distribution, Benchmark.cc:71-75) and N(0,1) complex64 visibilities, from PCG64(seed)."""
    rng = np.random.default_rng(seed)
    pool = []
    for _ in range(n_requests):
        u, v, w = (rng.uniform(-baseline / 2, baseline / 2, n_samples) for _ in range(3))
        vis = (rng.standard_normal(n_samples, dtype=np.float32) +
               1j * rng.standard_normal(n_samples, dtype=np.float32)).astype(np.complex64)
        pool.append((u, v, w, vis))
    return pool


def poisson_run(server: Server, rate: float, duration: float, pool, grids, degrid_fraction: float = 0.5,
                seed: int = 1) -> dict:
    """Submit requests at Poisson arrival times (rate per second) for `duration` seconds: each a
    gridding or (with probability degrid_fraction) a degridding request on a random resident grid
    with inputs from the pool; wait for all and summarise the server-measured latencies."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, int(rate * duration * 2) + 16)
    t_arr = np.cumsum(gaps)
    t_arr = t_arr[t_arr < duration]
    kinds = rng.random(t_arr.size) < degrid_fraction
    picks = rng.integers(0, len(pool), t_arr.size)
    gsel = rng.integers(0, len(grids), t_arr.size)
    reqs = []
    start = time.perf_counter()
    for i, t in enumerate(t_arr):
        while time.perf_counter() - start < t:
            pass
        u, v, w, vis = pool[picks[i]]
        kind = _lib.REQ_DEGRID if kinds[i] else _lib.REQ_GRID
        reqs.append(server.submit(kind, grids[gsel[i]], u, v, w, vis if kind == _lib.REQ_GRID else None))
    submit_end = time.perf_counter() - start
    infos = [r.wait() for r in reqs]
    lat = np.array([i.t_done - i.t_submit for i in infos]) * 1e3
    queue = np.array([i.t_start - i.t_submit for i in infos]) * 1e3
    span = max(i.t_done for i in infos) - min(i.t_submit for i in infos) if infos else 0.0
    n_samples = sum(pool[p][0].size for p in picks)
    return {
        "rate_req_s": rate, "requests": len(infos), "duration_s": duration, "submit_span_s": submit_end,
        "p50_ms": float(np.percentile(lat, 50)) if lat.size else None,
        "p99_ms": float(np.percentile(lat, 99)) if lat.size else None,
        "mean_ms": float(lat.mean()) if lat.size else None,
        "queue_p50_ms": float(np.percentile(queue, 50)) if queue.size else None,
        "throughput_req_s": len(infos) / span if span > 0 else None,
        "samples": int(n_samples),
        "mean_batch": float(np.mean([i.batch_requests for i in infos])) if infos else None,
        "errors": int(sum(1 for i in infos if i.status != 0)),
    }
