"""Batched gridding and degridding: many jobs (channels, Taylor terms) of uneven sample counts and
grid sizes that share one table, binned by one plan and run as one sequence of persistent
launches (tcv_batch_plan_create), optionally captured into one CUDA graph (tcv_graph_capture)
with the tile shape and sort granularity chosen by the autotuner (tcv_autotune).

The reference runs one job per process or thread (attic/tConvolveMPI/tConvolveMPI.cc:78-119,
attic/tConvolveMT/tConvolveMT.cc:65-77); each job's result here is that job's Benchmark result.
"""
from __future__ import annotations

import ctypes

from . import _lib
from ._lib import TcvJob, TcvTuning, autotune_report, check, lib
from .raw import _ptr, _stream


def _jobs_array(sizes, grids):
    arr = (TcvJob * len(sizes))()
    for j, (n, g) in enumerate(sizes):
        arr[j].n = int(n)
        arr[j].g_size = int(g)
        arr[j].d_grid = ctypes.c_void_p(grids[j].data_ptr()) if grids is not None else None
    return arr


def _tuning(t):
    if t is None:
        return None
    if isinstance(t, TcvTuning):
        return t
    rows, mib, split, dsplit, kernel = (tuple(t) + (0, 0, 0))[:5]
    return TcvTuning(int(rows), int(mib), int(split), int(dsplit), int(kernel))


def table_len(c, c_type: int) -> int:
    return c.numel() if c_type == _lib.C64 else c.numel() // lib().tcv_ctype_bytes(c_type)


class Graph:
    """A captured sequence of a plan's passes, replayed with one launch."""

    def __init__(self, handle, keep):
        self.handle = handle
        self._keep = keep

    def launch(self, stream=None):
        check(lib().tcv_graph_launch(self.handle, _stream(stream)), "tcv_graph_launch")

    def close(self):
        if self.handle:
            lib().tcv_graph_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """A batched plan over jobs [(n_j, g_size_j)] whose samples are consecutive in iu/iv/coff
    (job 0 first) and whose grids are the complex64 tensors `grids` (g_size_j x g_size_j)."""

    def __init__(self, sizes, grids, iu, iv, coff, support: int, c_len: int, tuning=None, stream=None):
        import torch

        self.sizes = [(int(n), int(g)) for n, g in sizes]
        self.grids = list(grids)
        assert len(self.grids) == len(self.sizes)
        self.n = sum(n for n, _ in self.sizes)
        assert iu.numel() == self.n and iv.numel() == self.n and coff.numel() == self.n
        self.support, self.c_len = support, c_len
        self._jobs = _jobs_array(self.sizes, self.grids)
        t = _tuning(tuning)
        tp = ctypes.byref(t) if t is not None else None
        nbytes = lib().tcv_batch_workspace_bytes(self._jobs, len(self.sizes), support, c_len, tp)
        if nbytes == 0:
            raise _lib.TcvError(1, "tcv_batch_workspace_bytes")
        self.work = torch.empty(nbytes, dtype=torch.uint8, device=iu.device)
        self.handle = ctypes.c_void_p()
        check(lib().tcv_batch_plan_create(ctypes.byref(self.handle), self._jobs, len(self.sizes), support,
                                          c_len, tp, _ptr(self.work), nbytes, _stream(stream)),
              "tcv_batch_plan_create")
        self._keep = (iu, iv, coff)
        self.bin(iu, iv, coff, stream)

    def bin(self, iu, iv, coff, stream=None):
        self._keep = (iu, iv, coff)
        check(lib().tcv_plan_bin(self.handle, _ptr(iu), _ptr(iv), _ptr(coff), _stream(stream)), "tcv_plan_bin")

    def grid(self, data, c, c_type: int, c_scale: float = 1.0, stream=None):
        """Every job's grid += gridding of its samples (Benchmark.cc:125-155)."""
        check(lib().tcv_plan_grid(self.handle, _ptr(data), _ptr(c), c_type, c_scale, None, _stream(stream)),
              "tcv_plan_grid")

    def degrid(self, c, c_type: int, out, c_scale: float = 1.0, stream=None):
        """out[k] = degridding of sample k from its job's grid (Benchmark.cc:158-195)."""
        check(lib().tcv_plan_degrid(self.handle, None, _ptr(c), c_type, c_scale, _ptr(out), _stream(stream)),
              "tcv_plan_degrid")

    def capture(self, passes: int, data, c, c_type: int, vis=None, c_scale: float = 1.0) -> Graph:
        iu, iv, coff = self._keep
        h = ctypes.c_void_p()
        check(lib().tcv_graph_capture(ctypes.byref(h), self.handle, passes, _ptr(iu), _ptr(iv), _ptr(coff),
                                      _ptr(data), _ptr(c), c_type, c_scale, None,
                                      _ptr(vis) if vis is not None else None), "tcv_graph_capture")
        return Graph(h, (data, c, vis, self))

    def tuning(self):
        t = TcvTuning()
        check(lib().tcv_plan_tuning(self.handle, ctypes.byref(t)), "tcv_plan_tuning")
        return t.as_tuple()

    def rejected(self, stream=None) -> int:
        r = ctypes.c_int64()
        check(lib().tcv_plan_rejected(self.handle, ctypes.byref(r), _stream(stream)), "tcv_plan_rejected")
        return r.value

    def close(self):
        if self.handle:
            lib().tcv_plan_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(sizes, iu, iv, coff, data, c, c_type: int, support: int, c_scale: float = 1.0, reps: int = 3,
             stream=None):
    """Fastest tuning (tile_rows, group_mib, split, degrid_split) for this batch, its median ms per bin+grid+degrid
    pass, and the candidates of the last timing run [((rows, mib, split, dsplit), ms)] (a cached result times
    nothing and leaves that report as it was)."""
    jobs = _jobs_array(sizes, None)  # the tuner grids into scratch grids of its own
    best = TcvTuning()
    ms = ctypes.c_float()
    check(lib().tcv_autotune(jobs, len(sizes), _ptr(iu), _ptr(iv), _ptr(coff), _ptr(data), _ptr(c), c_type,
                             c_scale, table_len(c, c_type), support, reps, ctypes.byref(best), ctypes.byref(ms),
                             _stream(stream)), "tcv_autotune")
    return best.as_tuple(), float(ms.value), autotune_report()


def make_problem(sizes, w_size: int = 33, cell_size: float = 5.0, baseline: int = 2000, vis_seed: int = 0,
                 device="cuda"):
    """Device inputs of a batch: one table (Benchmark::initC for w_size, cell_size, baseline), u, v, w
    from the reference generator for all samples in job order (state 1, as one long run of
    Benchmark::init), each job's offsets for its own grid size, and N(0,1) visibilities
    (workload.normal_vis(total, vis_seed)).  Returns a dict of tensors and scalars."""
    import torch

    from . import raw
    from .workload import normal_vis

    freq0 = 1.4e9 / 2.998e8
    support, over_sample, w_cell, c_len = raw.c_geometry(freq0, cell_size, baseline, w_size)
    c64, sum_c = raw.init_c(freq0, cell_size, baseline, w_size, device=device)
    total = sum(int(n) for n, _ in sizes)
    u, v, w = raw.init_uvw(total, baseline, 1, device=device)
    freq = torch.tensor([freq0], dtype=torch.float64, device=device)
    iu = torch.empty(total, dtype=torch.int32, device=device)
    iv = torch.empty_like(iu)
    coff = torch.empty_like(iu)
    at = 0
    for n, g in sizes:
        n = int(n)
        if n:
            a, b, c = raw.init_offsets(u[at:at + n], v[at:at + n], w[at:at + n], freq, cell_size, w_cell, w_size,
                                       int(g), support, over_sample)
            iu[at:at + n], iv[at:at + n], coff[at:at + n] = a, b, c
        at += n
    data = torch.from_numpy(normal_vis(total, vis_seed)).to(device)
    return dict(c64=c64, sum_c=sum_c, support=support, c_len=c_len, w_cell=w_cell, iu=iu, iv=iv, coff=coff,
                data=data, u=u, v=v, w=w, total=total)
