"""Raw device-pointer entry points on torch CUDA tensors.

torch provides device memory and the stream; every computation is a libtconvolve call
(include/tconvolve.h).  These mirror cuda_gridKernel / cuda_degridKernel
(attic/tConvolveCuda/CudaGridKernel.h:33-42): the caller owns the data, table, offsets and grid.
"""
from __future__ import annotations

import ctypes

from . import _lib
from ._lib import check, lib


def _ptr(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream=None) -> ctypes.c_void_p:
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def c_geometry(freq0: float, cell_size: float, baseline: int, w_size: int):
    sup, os_, wcs, clen = ctypes.c_int(), ctypes.c_int(), ctypes.c_double(), ctypes.c_int64()
    check(lib().tcv_c_geometry(freq0, cell_size, baseline, w_size, ctypes.byref(sup),
                               ctypes.byref(os_), ctypes.byref(wcs), ctypes.byref(clen)),
          "tcv_c_geometry")
    return sup.value, os_.value, wcs.value, clen.value


def init_c(freq0: float, cell_size: float, baseline: int, w_size: int, device="cuda"):
    """The normalised complex64 table (as a complex64 tensor) and sumC."""
    import torch

    _, _, _, clen = c_geometry(freq0, cell_size, baseline, w_size)
    c = torch.empty(clen, dtype=torch.complex64, device=device)
    scratch = torch.empty(lib().tcv_init_c_scratch_bytes(), dtype=torch.uint8, device=device)
    s = ctypes.c_float()
    check(lib().tcv_init_c_raw(freq0, cell_size, baseline, w_size, _ptr(c), _ptr(scratch),
                               ctypes.byref(s), _stream()), "tcv_init_c_raw")
    return c, s.value


def convert_c(c64, c_type: int):
    """Table in another storage form: (tensor of raw bytes, c_scale, imaginary-nonzero count)."""
    import torch

    nb = lib().tcv_ctype_bytes(c_type)
    out = torch.empty(c64.numel() * nb, dtype=torch.uint8, device=c64.device)
    scale = ctypes.c_float()
    nz = ctypes.c_int64()
    check(lib().tcv_convert_c(_ptr(c64), c64.numel(), c_type, _ptr(out), ctypes.byref(scale),
                              ctypes.byref(nz), _stream()), "tcv_convert_c")
    return out, scale.value, nz.value


def init_uvw(n: int, baseline: int = 2000, state0: int = 1, device="cuda"):
    import torch

    u, v, w = (torch.empty(n, dtype=torch.float64, device=device) for _ in range(3))
    check(lib().tcv_init_uvw_raw(n, baseline, state0, _ptr(u), _ptr(v), _ptr(w), _stream()),
          "tcv_init_uvw_raw")
    return u, v, w


def init_offsets(u, v, w, freq, cell_size, w_cell_size, w_size, g_size, support, over_sample):
    import torch

    n_samples = u.numel()
    n_chan = freq.numel()
    n = n_samples * n_chan
    iu, iv, co = (torch.empty(n, dtype=torch.int32, device=u.device) for _ in range(3))
    check(lib().tcv_init_offsets_raw(_ptr(u), _ptr(v), _ptr(w), n_samples, _ptr(freq), n_chan,
                                     float(cell_size), float(w_cell_size), w_size, g_size, support,
                                     over_sample, _ptr(iu), _ptr(iv), _ptr(co), _stream()),
          "tcv_init_offsets_raw")
    return iu, iv, co


class Plan:
    """A binning plan (tcv_plan) in a torch-allocated workspace."""

    def __init__(self, iu, iv, coff, support: int, g_size: int, c_len: int, stream=None, tuning=None):
        """tuning: (tile_rows, group_mib, split, degrid_split) for tcv_plan_build_tuned; None for
        the default plan (tcv_plan_build)."""
        import torch

        from ._lib import TcvTuning

        self.n = iu.numel()
        self.support, self.g_size, self.c_len = support, g_size, c_len
        self._keep = (iu, iv, coff)
        self.handle = ctypes.c_void_p()
        if tuning is None:
            nbytes = lib().tcv_plan_workspace_bytes(self.n, support, g_size, c_len)
            self.work = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=iu.device)
            check(lib().tcv_plan_build(ctypes.byref(self.handle), _ptr(iu), _ptr(iv), _ptr(coff),
                                       self.n, support, g_size, c_len, _ptr(self.work), nbytes,
                                       _stream(stream)), "tcv_plan_build")
        else:
            t = TcvTuning(*(tuple(tuning) + (0, 0, 0, 0, 0))[:5])
            nbytes = lib().tcv_plan_workspace_bytes_tuned(self.n, support, g_size, c_len, ctypes.byref(t))
            if nbytes == 0:
                raise _lib.TcvError(1, "tcv_plan_workspace_bytes_tuned")
            self.work = torch.empty(nbytes, dtype=torch.uint8, device=iu.device)
            check(lib().tcv_plan_build_tuned(ctypes.byref(self.handle), _ptr(iu), _ptr(iv), _ptr(coff),
                                             self.n, support, g_size, c_len, ctypes.byref(t),
                                             _ptr(self.work), nbytes, _stream(stream)), "tcv_plan_build_tuned")

    def grid(self, data, c, c_type: int, grid, c_scale: float = 1.0, stream=None):
        check(lib().tcv_plan_grid(self.handle, _ptr(data), _ptr(c), c_type, c_scale, _ptr(grid),
                                  _stream(stream)), "tcv_plan_grid")

    def degrid(self, grid, c, c_type: int, out, c_scale: float = 1.0, stream=None):
        check(lib().tcv_plan_degrid(self.handle, _ptr(grid), _ptr(c), c_type, c_scale, _ptr(out),
                                    _stream(stream)), "tcv_plan_degrid")

    def capture(self, passes: int, data, c, c_type: int, grid, vis=None, c_scale: float = 1.0):
        """CUDA graph of this plan's passes (tcv_graph_capture: bin, grid into `grid`, degrid into
        `vis`, as the _lib.PASS_* bits say), replayed with Graph.launch()."""
        from .batch import Graph

        iu, iv, coff = self._keep
        h = ctypes.c_void_p()
        check(lib().tcv_graph_capture(ctypes.byref(h), self.handle, passes, _ptr(iu), _ptr(iv), _ptr(coff),
                                      _ptr(data), _ptr(c), c_type, c_scale, _ptr(grid),
                                      _ptr(vis) if vis is not None else None), "tcv_graph_capture")
        return Graph(h, (data, c, grid, vis, self))

    def set_degrid_variant(self, variant: int):
        check(lib().tcv_plan_set_degrid_variant(self.handle, variant), "tcv_plan_set_degrid_variant")

    def rejected(self, stream=None) -> int:
        r = ctypes.c_int64()
        check(lib().tcv_plan_rejected(self.handle, ctypes.byref(r), _stream(stream)),
              "tcv_plan_rejected")
        return r.value

    def status(self, stream=None) -> int:
        return lib().tcv_plan_status(self.handle, _stream(stream))

    def info(self):
        vals = [ctypes.c_int() for _ in range(5)]
        check(lib().tcv_plan_info(self.handle, *[ctypes.byref(v) for v in vals]), "tcv_plan_info")
        return dict(zip(["tile_w", "tile_h", "anchor", "degrid_mode", "n_tiles"],
                        [v.value for v in vals]))

    def close(self):
        if self.handle:
            lib().tcv_plan_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class VarPlan(Plan):
    """A variable-width plan (tcv_plan_build_var): every sample grids with the footprint width of
    its w-plane, s_size[wplane[k]] (current/tConvolveMPI/Benchmark.cc:373-452); s_size and c_off0
    are per-plane host arrays."""

    def __init__(self, iu, iv, coff, wplane, s_size, c_off0, g_size: int, c_len: int, tuning=None, stream=None):
        import numpy as np
        import torch

        from ._lib import TcvTuning

        self.n = iu.numel()
        self.g_size, self.c_len = g_size, c_len
        s_size = np.ascontiguousarray(s_size, np.int32)
        c_off0 = np.ascontiguousarray(c_off0, np.int32)
        # (tile_rows, group_mib, split, degrid_split[, kernel bits]); missing entries are 0 (defaults)
        t = TcvTuning(*(tuple(tuning) + (0, 0, 0, 0, 0))[:5]) if tuning is not None else None
        tp = ctypes.byref(t) if t is not None else None
        sp, op = ctypes.c_void_p(s_size.ctypes.data), ctypes.c_void_p(c_off0.ctypes.data)
        nbytes = lib().tcv_plan_workspace_bytes_var(self.n, sp, op, s_size.size, g_size, c_len, tp)
        if nbytes == 0:
            raise _lib.TcvError(1, "tcv_plan_workspace_bytes_var")
        self.work = torch.empty(nbytes, dtype=torch.uint8, device=iu.device)
        self._keep = (iu, iv, coff, wplane, s_size, c_off0)
        self.handle = ctypes.c_void_p()
        check(lib().tcv_plan_build_var(ctypes.byref(self.handle), _ptr(iu), _ptr(iv), _ptr(coff), _ptr(wplane), self.n,
                                       sp, op, s_size.size, g_size, c_len, tp, _ptr(self.work), nbytes,
                                       _stream(stream)), "tcv_plan_build_var")


def grid_raw(data, support, c, c_type, c_scale, coff, iu, iv, grid, g_size, stream=None):
    """One call: plan + gridding (tcv_grid_raw), workspace allocated by torch."""
    import torch

    n = data.numel()
    c_len = c.numel() if c_type == _lib.C64 else c.numel() // lib().tcv_ctype_bytes(c_type)
    nbytes = lib().tcv_plan_workspace_bytes(n, support, g_size, c_len)
    work = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=data.device)
    check(lib().tcv_grid_raw(_ptr(data), n, support, _ptr(c), c_type, c_scale, c_len, _ptr(coff),
                             _ptr(iu), _ptr(iv), _ptr(grid), g_size, _ptr(work), nbytes,
                             _stream(stream)), "tcv_grid_raw")
    return work


def degrid_raw(grid, g_size, support, c, c_type, c_scale, coff, iu, iv, out, stream=None):
    import torch

    n = out.numel()
    c_len = c.numel() if c_type == _lib.C64 else c.numel() // lib().tcv_ctype_bytes(c_type)
    nbytes = lib().tcv_plan_workspace_bytes(n, support, g_size, c_len)
    work = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=grid.device)
    check(lib().tcv_degrid_raw(_ptr(grid), g_size, support, _ptr(c), c_type, c_scale, c_len,
                               _ptr(coff), _ptr(iu), _ptr(iv), _ptr(out), n, _ptr(work), nbytes,
                               _stream(stream)), "tcv_degrid_raw")
    return work
