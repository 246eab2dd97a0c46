"""Python mirror of the Benchmark class of current/tConvolveMPI (current/tConvolveMPI/Benchmark.h:38-111):
the variable-support W-projection benchmark (per-plane kernel widths, complex kernels, samples of a
12 h track of the 36-antenna array), with every buffer on one GPU (libtconvolve tcv_cur_*).

Same method names and call order as the reference's driver (current/tConvolveMPI/tConvolveMPI.cc:61-186):

    b = Benchmark()
    b.setSort(0)
    for run in (0, 1):          # continuum, then spectral line
        b.setRunType(run)
        b.init()                # the generator continues across init() calls, as in the reference
        b.runGrid()
        b.runDegrid()
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import TcvCurGeometry, TcvTuning, check, lib

RUN_TYPES = {0: "continuum", 1: "spectral", 2: "nearest-neighbour", 3: "7x7", 4: "87x87"}


def _p(a: np.ndarray):
    assert a.flags.c_contiguous
    return ctypes.c_void_p(a.ctypes.data)


def geometry(run_type: int) -> TcvCurGeometry:
    g = TcvCurGeometry()
    check(lib().tcv_cur_geometry_of(run_type, ctypes.byref(g)), "tcv_cur_geometry_of")
    return g


def required_rate():
    """Benchmark::requiredRate (current/tConvolveMPI/Benchmark.cc:697-739): [continuum, spectral]."""
    r = (ctypes.c_float * 2)()
    lib().tcv_cur_required_rate(r)
    return [float(r[0]), float(r[1])]


class Benchmark:
    def __init__(self, device: int = 0):
        self._ctx = ctypes.c_void_p()
        self._tuning = (16, 32, 0, 0)
        check(lib().tcv_cur_create(device, ctypes.byref(self._ctx)), "tcv_cur_create")

    def close(self):
        if self._ctx:
            lib().tcv_cur_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- reference interface ----
    def setMPIrank(self, rank: int):
        """Printing is rank 0's in the reference; nothing is printed here."""
        self.rank = rank

    def setSort(self, sort: int):
        check(lib().tcv_cur_set_sort(self._ctx, int(sort)), "tcv_cur_set_sort")

    def setRunType(self, run_type: int):
        check(lib().tcv_cur_set_run_type(self._ctx, int(run_type)), "tcv_cur_set_run_type")

    def getRunType(self) -> int:
        return lib().tcv_cur_get_run_type(self._ctx)

    def init(self):
        st = lib().tcv_cur_init(self._ctx)
        if st:
            raise _lib.TcvError(st, "tcv_cur_init (" + lib().tcv_cur_last_error(self._ctx).decode() + ")")

    def runGrid(self):
        check(lib().tcv_cur_run_grid(self._ctx), "tcv_cur_run_grid")

    def runDegrid(self):
        check(lib().tcv_cur_run_degrid(self._ctx), "tcv_cur_run_degrid")

    def getSupport(self) -> int:
        return lib().tcv_cur_support(self._ctx)

    def nVisibilitiesGridded(self) -> int:
        return int(lib().tcv_cur_n_visibilities(self._ctx))

    def nPixelsGridded(self) -> int:
        return int(lib().tcv_cur_n_pixels(self._ctx))

    def requiredRate(self):
        return required_rate()

    # ---- extras ----
    def sync(self):
        check(lib().tcv_cur_sync(self._ctx), "tcv_cur_sync")

    @property
    def stream(self) -> int:
        return lib().tcv_cur_get_stream(self._ctx) or 0

    def set_ctype(self, c_type: int | str):
        if isinstance(c_type, str):
            c_type = _lib.CTYPE_BY_NAME[c_type]
        check(lib().tcv_cur_set_ctype(self._ctx, int(c_type)), "tcv_cur_set_ctype")

    def set_tuning(self, group_mib: int = 32, split: int = 0, degrid_split: int = 0, tile_rows: int = 16,
                   kernel: int = 0):
        """Plane-group slice, work-unit sizes, tile height (rows per warp, 8 or 16) and the passes
        that use the sample-parallel kernels (bit mask: 1 gridding, 2 degridding; needs tile_rows
        8) of the plan."""
        t = TcvTuning(int(tile_rows), int(group_mib), int(split), int(degrid_split), int(kernel))
        check(lib().tcv_cur_set_tuning(self._ctx, ctypes.byref(t)), "tcv_cur_set_tuning")
        self._tuning = t.as_tuple()

    def tuning(self):
        """The plan's (tile_rows, group_mib, split, degrid_split)."""
        return self._tuning

    def tune(self, reps: int = 3):
        """Autotune the plan on the initialised problem (tcv_cur_tune): keeps the fastest tuning
        and returns it with its median ms per gridding + degridding pass, and the candidates
        timed as [((rows, group_mib, split, degrid_split), ms), ...]."""
        t = TcvTuning()
        ms = ctypes.c_float()
        st = lib().tcv_cur_tune(self._ctx, int(reps), ctypes.byref(t), ctypes.byref(ms))
        if st != _lib.TCV_OK:
            raise _lib.TcvError(st, "tcv_cur_tune (" + lib().tcv_cur_last_error(self._ctx).decode() + ")")
        self._tuning = t.as_tuple()
        return t.as_tuple(), float(ms.value), _lib.autotune_report()

    def geometry(self) -> TcvCurGeometry:
        g = TcvCurGeometry()
        check(lib().tcv_cur_info(self._ctx, ctypes.byref(g)), "tcv_cur_info")
        return g

    @property
    def generator_state(self) -> int:
        return int(lib().tcv_cur_generator_state(self._ctx))

    def set_data(self, vis: np.ndarray):
        vis = np.ascontiguousarray(vis, np.complex64)
        check(lib().tcv_cur_set_data(self._ctx, _p(vis), vis.size), "tcv_cur_set_data")

    def zero_grid(self):
        check(lib().tcv_cur_zero_grid(self._ctx), "tcv_cur_zero_grid")

    def grid(self) -> np.ndarray:
        g = self.geometry()
        out = np.empty(g.g_size * g.g_size, np.complex64)
        check(lib().tcv_cur_get_grid(self._ctx, _p(out)), "tcv_cur_get_grid")
        return out

    def outdata(self) -> np.ndarray:
        out = np.empty(self.nVisibilitiesGridded(), np.complex64)
        check(lib().tcv_cur_get_outdata(self._ctx, _p(out), out.size), "tcv_cur_get_outdata")
        return out

    def C(self) -> np.ndarray:
        out = np.empty(self.geometry().c_len, np.complex64)
        check(lib().tcv_cur_get_c(self._ctx, _p(out), out.size), "tcv_cur_get_c")
        return out

    def uvw(self):
        n = self.nVisibilitiesGridded()
        u, v, w = (np.empty(n, np.float64) for _ in range(3))
        check(lib().tcv_cur_get_uvw(self._ctx, _p(u), _p(v), _p(w)), "tcv_cur_get_uvw")
        return u, v, w

    def offsets(self):
        n = self.nVisibilitiesGridded()
        iu, iv, wp, co = (np.empty(n, np.int32) for _ in range(4))
        check(lib().tcv_cur_get_offsets(self._ctx, _p(iu), _p(iv), _p(wp), _p(co)), "tcv_cur_get_offsets")
        return iu, iv, wp, co

    def planes(self):
        g = self.geometry()
        s, o = np.empty(g.w_size, np.int32), np.empty(g.w_size, np.int32)
        check(lib().tcv_cur_get_planes(self._ctx, _p(s), _p(o)), "tcv_cur_get_planes")
        return s, o


def main(argv=None) -> int:
    """current/tConvolveMPI's driver (current/tConvolveMPI/tConvolveMPI.cc:61-186) on one GPU:
    the continuum then the spectral run on one object, runGrid and runDegrid each timed, and the
    reference's report lines.  --tune picks the plan with tcv_cur_tune first (untimed);
    --runs selects run types; --repeat times each pass that many times (the last is reported)."""
    import argparse
    import time

    ap = argparse.ArgumentParser(prog="python -m tconvolve.current")
    ap.add_argument("--runs", default="0,1", help="run types in order (0 continuum, 1 spectral, 2-4 tests)")
    ap.add_argument("--sort", type=int, default=0)
    ap.add_argument("--tune", action="store_true")
    ap.add_argument("--tuning", default=None,
                    help="fixed plan: tile rows,group MiB,split,degrid split[,kernel bits (1 gridding, "
                         "2 degridding: sample-parallel)]")
    ap.add_argument("--repeat", type=int, default=1)
    a = ap.parse_args(argv)
    b = Benchmark()
    b.setSort(a.sort)
    for run in (int(r) for r in a.runs.split(",")):
        b.setRunType(run)
        print(f"+++++ Test {b.getRunType()} +++++")
        if a.tuning:
            v = [int(x) for x in a.tuning.split(",")]
            b.set_tuning(v[1], v[2], v[3], v[0], v[4] if len(v) > 4 else 0)
        b.init()
        if a.tune:
            best, ms, _ = b.tune()
            print(f"    Tuned plan (rows, group MiB, split, degrid split) = {best}, {ms:.3f} ms per grid+degrid")
        ngridvis = float(b.nVisibilitiesGridded())
        ngridpix = float(b.nPixelsGridded())
        label = {0: "Continuum", 1: "Spectral"}.get(run)
        for kind in ("grid", "degrid"):
            for _ in range(a.repeat):
                b.sync()
                t0 = time.perf_counter()
                b.runGrid() if kind == "grid" else b.runDegrid()
                b.sync()
                t = time.perf_counter() - t0
            if kind == "grid":
                print("  Forward processing")
                print("    Number of processes: 1")
                print(f"    Time {t} (s) ")
                print(f"    Time per visibility spectral sample {1e6 * t / ngridvis} (us) ")
                print(f"    Time per gridding   {1e9 * t / ngridpix} (ns) ")
                print(f"    Gridding rate (per process)   {(ngridvis / 1e6) / t} (Mvis/sec)")
                print(f"    Gridding rate (per process)   {(ngridpix / 1e6) / t} (Mpix/sec)")
                print(f"    Gridding rate (total)      {(ngridpix / 1e6) / t} (Mpix/sec)")
                if label:
                    print(f"    {label} gridding performance (per process):   {(ngridpix / 1e6) / t} (Mpix/sec)")
            else:
                print("  Reverse processing")
                print("    Number of processes: 1")
                print(f"    Time {t} (s) ")
                print(f"    Time per visibility spectral sample {1e6 * t / ngridvis} (us) ")
                print(f"    Time per degridding {1e9 * t / ngridpix} (ns) ")
                print(f"    Degridding rate (per node) {(ngridvis / 1e6) / t} (Mvis/sec)")
                print(f"    Degridding rate (per node) {(ngridpix / 1e6) / t} (Mpix/sec)")
                print(f"    Degridding rate (total)    {(ngridpix / 1e6) / t} (Mpix/sec)")
                if label:
                    print(f"    {label} degridding performance (per process):   {(ngridpix / 1e6) / t} (Mpix/sec)")
        print("Done")
    b.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
