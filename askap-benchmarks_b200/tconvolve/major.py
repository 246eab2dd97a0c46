"""The imaging major cycle of current/tMajorACC on the GPU (libtconvolve tcv_major_*), with the FFT
steps either side of gridding (tcv_fft_exec, tcv_image_from_grid, tcv_grid_from_image).

tMajorACC is one program (current/tMajorACC/tMajorACC.cc:889-1635); its driver loop becomes

    m = MajorCycle()                  # the program's constants: 160000 samples, 33 planes, 4096^2 ...
    m.init()                          # samples, delta table, offsets, the 100-source sky, its visibilities
    for it in range(m.config.n_major):
        m.run_cycle()                 # PSF (first cycle), grid, inverse FFT, Hogbom, FFT, degrid, subtract
    m.stage_ms()                      # device time per stage, as the reference's timers

Images come back as float32 (the reference's complex images have zero imaginary parts after fftFix).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import MAJOR_STAGES, TcvMajorConfig, TcvTuning, check, lib
from .raw import _ptr, _stream


def default_config(**kw) -> TcvMajorConfig:
    cfg = TcvMajorConfig()
    lib().tcv_major_config_default(ctypes.byref(cfg))
    for k, v in kw.items():
        if k == "tuning":
            cfg.tuning = TcvTuning(*v)
        else:
            setattr(cfg, k, v)
    return cfg


class MajorCycle:
    def __init__(self, config: TcvMajorConfig | None = None, **kw):
        self.config = config if config is not None else default_config(**kw)
        self._ctx = ctypes.c_void_p()
        check(lib().tcv_major_create(ctypes.byref(self.config), ctypes.byref(self._ctx)), "tcv_major_create")

    def close(self):
        if self._ctx:
            lib().tcv_major_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st != _lib.TCV_OK:
            raise _lib.TcvError(st, f"{what} ({lib().tcv_major_last_error(self._ctx).decode()})")

    def init(self):
        self._check(lib().tcv_major_init(self._ctx), "tcv_major_init")

    def run_cycle(self):
        self._check(lib().tcv_major_run_cycle(self._ctx), "tcv_major_run_cycle")

    def sync(self):
        self._check(lib().tcv_major_sync(self._ctx), "tcv_major_sync")

    @property
    def stream(self) -> int:
        return lib().tcv_major_get_stream(self._ctx) or 0

    def stage_ms(self):
        """{stage: device ms summed over the cycles run}, and the number of cycles."""
        ms = (ctypes.c_double * len(MAJOR_STAGES))()
        n = ctypes.c_int()
        self._check(lib().tcv_major_stage_ms(self._ctx, ms, ctypes.byref(n)), "tcv_major_stage_ms")
        return dict(zip(MAJOR_STAGES, list(ms))), n.value

    def info(self):
        sup, nv, cl, sc = ctypes.c_int(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_float()
        self._check(lib().tcv_major_info(self._ctx, ctypes.byref(sup), ctypes.byref(nv), ctypes.byref(cl),
                                         ctypes.byref(sc)), "tcv_major_info")
        return {"support": sup.value, "n_vis": nv.value, "c_len": cl.value, "scale": sc.value}

    def image(self, which: int) -> np.ndarray:
        g = self.config.g_size
        out = np.empty(g * g, np.float32)
        self._check(lib().tcv_major_get_image(self._ctx, int(which), ctypes.c_void_p(out.ctypes.data)),
                    "tcv_major_get_image")
        return out

    def grid(self, which: int = 2) -> np.ndarray:
        g = self.config.g_size
        out = np.empty(g * g, np.complex64)
        self._check(lib().tcv_major_get_grid(self._ctx, int(which), ctypes.c_void_p(out.ctypes.data)),
                    "tcv_major_get_grid")
        return out

    def vis(self, which: int = 0) -> np.ndarray:
        out = np.empty(self.info()["n_vis"], np.complex64)
        self._check(lib().tcv_major_get_vis(self._ctx, int(which), ctypes.c_void_p(out.ctypes.data)),
                    "tcv_major_get_vis")
        return out

    def offsets(self):
        n = self.info()["n_vis"]
        iu, iv, co = (np.empty(n, np.int32) for _ in range(3))
        self._check(lib().tcv_major_get_offsets(self._ctx, *(ctypes.c_void_p(a.ctypes.data) for a in (iu, iv, co))),
                    "tcv_major_get_offsets")
        return iu, iv, co


# ---- the FFT steps on torch tensors ----
def fft_exec(grid, g_size: int, forward: bool, stream=None):
    """fftExec in place on a complex64 CUDA tensor of g_size^2."""
    check(lib().tcv_fft_exec(_ptr(grid), int(g_size), 1 if forward else 0, _stream(stream)), "tcv_fft_exec")


def fft_fix(grid, scale: float, stream=None):
    check(lib().tcv_fft_fix(_ptr(grid), int(grid.numel()), ctypes.c_float(scale), _stream(stream)), "tcv_fft_fix")


def image_from_grid(grid, g_size: int, scale: float, image, stream=None):
    """image (float32) = Re(fftExec(grid, backward)) * scale; grid is overwritten."""
    check(lib().tcv_image_from_grid(_ptr(grid), int(g_size), ctypes.c_float(scale), _ptr(image), _stream(stream)),
          "tcv_image_from_grid")


def grid_from_image(image, g_size: int, grid, stream=None):
    """grid (complex64) = fftExec(complex(image), forward)."""
    check(lib().tcv_grid_from_image(_ptr(image), int(g_size), _ptr(grid), _stream(stream)), "tcv_grid_from_image")


def main(argv=None) -> int:
    """tMajorACC's driver (current/tMajorACC/tMajorACC.cc:889-1635) on the GPU with its options
    (-n samples, -w planes, -c channels, -f cell-size factor) and its timing report."""
    import argparse

    ap = argparse.ArgumentParser(prog="python -m tconvolve.major")
    ap.add_argument("-n", type=int, default=160000)
    ap.add_argument("-w", type=int, default=33)
    ap.add_argument("-c", type=int, default=1)
    ap.add_argument("-f", type=float, default=1.0)
    ap.add_argument("--g-size", type=int, default=4096)
    ap.add_argument("--major", type=int, default=5)
    ap.add_argument("--minor", type=int, default=100)
    a = ap.parse_args(argv)
    print(f"nSamples = {a.n}\nnChan = {a.c}\nwSize = {a.w}\ncellSize = {5.0 * a.f}")
    m = MajorCycle(n_samples=a.n, w_size=a.w, n_chan=a.c, cell_size=5.0 * a.f, g_size=a.g_size, n_major=a.major,
                   n_minor=a.minor)
    m.init()
    for it in range(a.major):
        print(f"cycle {it}")
        m.run_cycle()
    m.sync()
    ms, n = m.stage_ms()
    info = m.info()
    s = 2 * info["support"] + 1
    nv = info["n_vis"]
    griddings = nv * s * s
    print("\n+++++ B200 times +++++\n")

    def rates(title, t):
        print(title)
        print(f"    Time per major cycle {t} (s) ")
        print(f"    Time per visibility sample {1e6 * t / nv} (us) ")
        print(f"    Time per gridding   {1e9 * t / griddings} (ns) ")
        print(f"    Gridding rate   {griddings / 1e6 / t} (million grid points per second)")

    rates("Gridding PSF", ms["psf_grid"] * 1e-3)
    rates("Gridding data", ms["grid"] * 1e-3 / n)
    print(f"Inverse FFTs\n    Time per major cycle {ms['ifft'] * 1e-3 / n} (s) ")
    t = ms["hogbom"] * 1e-3 / n
    print(f"Hogbom clean\n    Time per major cycle {t} (s) \n    Time per minor cycle {t / a.minor * 1000} (ms)")
    print(f"    Cleaning rate  {a.minor / t} (iterations per second)")
    print(f"Forward FFT\n    Time per major cycle {ms['fft'] * 1e-3 / n} (s) ")
    t = ms["degrid"] * 1e-3 / n
    print("Degridding data")
    print(f"    Time per major cycle {t} (s) ")
    print(f"    Time per visibility sample {1e6 * t / nv} (us) ")
    print(f"    Time per degridding   {1e9 * t / griddings} (ns) ")
    print(f"    Degridding rate   {griddings / 1e6 / t} (million grid points per second)")
    m.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
