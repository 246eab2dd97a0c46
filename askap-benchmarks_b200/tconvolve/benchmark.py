"""Python mirror of the reference's Benchmark class (attic/tConvolveMPI/Benchmark.h:55-99).

Same method names, argument meaning and call order as the reference:

    b = Benchmark()          # reference defaults, or Benchmark(n_samples=..., ...)
    b.init()                 # u, v, w, C, offsets (+ the device binning plan)
    b.runGrid()              # grid += gridding of the samples
    b.runDegrid()            # outdata = degridding of the grid
    b.getSupport()

All buffers live on the GPU inside a libtconvolve context; results are copied to numpy only on
request (grid(), outdata(), C(), samples()).  Errors raise TcvError, as the reference's helpers
throw std::runtime_error (attic/tConvolveMPI/Stopwatch.cc:47-61).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import TcvConfig, TcvDeviceBuffers, check, lib


def _p(a: np.ndarray):
    assert a.flags.c_contiguous
    return ctypes.c_void_p(a.ctypes.data)


class Benchmark:
    """The tConvolve benchmark object with every buffer resident on one GPU."""

    def __init__(self, n_samples: int = 160000, w_size: int = 33, n_chan: int = 1,
                 g_size: int = 4096, cell_size: float = 5.0, baseline: int = 2000, seed: int = 0,
                 c_type: int | str = _lib.C64, device: int = 0):
        if isinstance(c_type, str):
            c_type = _lib.CTYPE_BY_NAME[c_type]
        self.cfg = TcvConfig(n_samples=n_samples, w_size=w_size, n_chan=n_chan, g_size=g_size,
                             baseline=baseline, cell_size=float(cell_size), seed=seed,
                             c_type=int(c_type), device=device)
        self._ctx = ctypes.c_void_p()
        check(lib().tcv_create(ctypes.byref(self.cfg), ctypes.byref(self._ctx)), "tcv_create")
        self._next = seed + 1  # host copy of the reference generator state (randomInt)

    # ---- lifetime ----
    def close(self):
        if self._ctx:
            lib().tcv_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def ctx(self):
        return self._ctx

    # ---- reference interface ----
    def randomInt(self) -> int:
        """attic/tConvolveMPI/Benchmark.cc:53-58 (host copy of the generator)."""
        self._next = (self._next * 1103515245 + 12345) & 0xFFFFFFFFFFFFFFFF
        return int(((self._next // 65536) & 0xFFFFFFFF) % 2147483647)

    def init(self):
        check(lib().tcv_init(self._ctx), "tcv_init", self._ctx)

    def runGrid(self):
        check(lib().tcv_run_grid(self._ctx), "tcv_run_grid", self._ctx)

    def runDegrid(self):
        check(lib().tcv_run_degrid(self._ctx), "tcv_run_degrid", self._ctx)

    def getSupport(self) -> int:
        return lib().tcv_support(self._ctx)

    # ---- extras ----
    def sync(self):
        check(lib().tcv_sync(self._ctx), "tcv_sync", self._ctx)

    def set_stream(self, stream_handle: int | None):
        check(lib().tcv_set_stream(self._ctx, ctypes.c_void_p(stream_handle or 0)),
              "tcv_set_stream", self._ctx)

    def set_ctype(self, c_type: int | str):
        if isinstance(c_type, str):
            c_type = _lib.CTYPE_BY_NAME[c_type]
        check(lib().tcv_set_ctype(self._ctx, int(c_type)), "tcv_set_ctype", self._ctx)

    def set_path(self, path: int | str):
        """Kernel family: "direct" (default: tile kernels on the reference-layout table), "paired"
        (two columns per lane on the paired table) or "tma" (TMA pipeline on the padded table)."""
        if isinstance(path, str):
            path = {"tma": _lib.PATH_TMA, "direct": _lib.PATH_DIRECT, "paired": _lib.PATH_PAIRED}[path]
        check(lib().tcv_set_path(self._ctx, int(path)), "tcv_set_path", self._ctx)

    def set_degrid_variant(self, variant: int | str):
        """Degridding kernel on the direct path: "tiles" (default) or "anchor"."""
        if isinstance(variant, str):
            variant = {"tiles": _lib.DEGRID_TILES, "anchor": _lib.DEGRID_ANCHOR}[variant]
        plan = ctypes.c_void_p(self.device_buffers().plan)
        check(lib().tcv_plan_set_degrid_variant(plan, int(variant)), "tcv_plan_set_degrid_variant")

    def set_tuning(self, tile_rows: int = 16, group_mib: int = 32, split: int = 0, degrid_split: int = 0,
                   kernel: int = 0):
        """Tile shape (grid rows per warp: 8, 16 or 32), plane-group slice (MiB of complex64
        table; -1 = the whole table in one group), work-unit sizes of busy cells for gridding
        and degridding (samples; 0 = cells whole) and the passes that use the sample-parallel
        kernels (bit mask: 1 gridding, 2 degridding; 8-row tiles) of the plan.  Rebuilds the plan
        (the degridding variant returns to "tiles")."""
        t = _lib.TcvTuning(int(tile_rows), int(group_mib), int(split), int(degrid_split), int(kernel))
        check(lib().tcv_set_tuning(self._ctx, ctypes.byref(t)), "tcv_set_tuning", self._ctx)

    def tuning(self) -> tuple:
        t = _lib.TcvTuning()
        check(lib().tcv_get_tuning(self._ctx, ctypes.byref(t)), "tcv_get_tuning", self._ctx)
        return t.as_tuple()

    def tune(self, reps: int = 3):
        """Autotune the plan on this problem, table form and grid (tcv_tune): the fastest
        (tile_rows, group_mib, split, degrid_split) and its median ms per bin + grid + degrid pass."""
        t = _lib.TcvTuning()
        ms = ctypes.c_float()
        check(lib().tcv_tune(self._ctx, int(reps), ctypes.byref(t), ctypes.byref(ms)), "tcv_tune", self._ctx)
        return t.as_tuple(), float(ms.value)

    @property
    def path(self) -> int:
        return lib().tcv_get_path(self._ctx)

    @property
    def overSample(self) -> int:
        return lib().tcv_over_sample(self._ctx)

    @property
    def wCellSize(self) -> float:
        return lib().tcv_w_cell_size(self._ctx)

    @property
    def sumC(self) -> float:
        return lib().tcv_sum_c(self._ctx)

    @property
    def n_data(self) -> int:
        return int(lib().tcv_n_data(self._ctx))

    @property
    def c_len(self) -> int:
        return int(lib().tcv_c_len(self._ctx))

    def updates_per_pass(self) -> float:
        return lib().tcv_updates_per_pass(self._ctx)

    def set_data(self, vis: np.ndarray):
        vis = np.ascontiguousarray(vis, np.complex64)
        check(lib().tcv_set_data(self._ctx, _p(vis), vis.size), "tcv_set_data", self._ctx)

    def data(self) -> np.ndarray:
        out = np.empty(self.n_data, np.complex64)
        check(lib().tcv_get_data(self._ctx, _p(out), out.size), "tcv_get_data", self._ctx)
        return out

    def outdata(self) -> np.ndarray:
        out = np.empty(self.n_data, np.complex64)
        check(lib().tcv_get_outdata(self._ctx, _p(out), out.size), "tcv_get_outdata", self._ctx)
        return out

    def grid(self) -> np.ndarray:
        g = np.empty(self.cfg.g_size * self.cfg.g_size, np.complex64)
        check(lib().tcv_get_grid(self._ctx, _p(g)), "tcv_get_grid", self._ctx)
        return g

    def set_grid(self, grid: np.ndarray):
        grid = np.ascontiguousarray(grid, np.complex64)
        assert grid.size == self.cfg.g_size * self.cfg.g_size
        check(lib().tcv_set_grid(self._ctx, _p(grid)), "tcv_set_grid", self._ctx)

    def zero_grid(self):
        check(lib().tcv_zero_grid(self._ctx), "tcv_zero_grid", self._ctx)

    def C(self) -> np.ndarray:
        c = np.empty(self.c_len, np.complex64)
        check(lib().tcv_get_c(self._ctx, _p(c), c.size), "tcv_get_c", self._ctx)
        return c

    def offsets(self):
        n = self.n_data
        iu, iv, co = (np.empty(n, np.int32) for _ in range(3))
        check(lib().tcv_get_offsets(self._ctx, _p(iu), _p(iv), _p(co)), "tcv_get_offsets", self._ctx)
        return iu, iv, co

    def uvw(self):
        n = self.cfg.n_samples
        u, v, w = (np.empty(n, np.float64) for _ in range(3))
        check(lib().tcv_get_uvw(self._ctx, _p(u), _p(v), _p(w)), "tcv_get_uvw", self._ctx)
        return u, v, w

    def set_uvw(self, u, v, w):
        u, v, w = (np.ascontiguousarray(a, np.float64) for a in (u, v, w))
        check(lib().tcv_set_uvw(self._ctx, _p(u), _p(v), _p(w)), "tcv_set_uvw", self._ctx)

    def plan_info(self) -> dict:
        """Tile geometry the binning plan chose (tcv_plan_info)."""
        plan = ctypes.c_void_p(self.device_buffers().plan)
        vals = [ctypes.c_int() for _ in range(5)]
        check(lib().tcv_plan_info(plan, *[ctypes.byref(v) for v in vals]), "tcv_plan_info")
        return dict(zip(["tile_w", "tile_h", "anchor", "degrid_mode", "n_tiles"],
                        [v.value for v in vals]))

    def device_buffers(self) -> TcvDeviceBuffers:
        b = TcvDeviceBuffers()
        check(lib().tcv_get_device_buffers(self._ctx, ctypes.byref(b)), "tcv_get_device_buffers",
              self._ctx)
        return b
