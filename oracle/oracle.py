"""numpy front end for the C restatement in tconvolve_oracle.c.

TEST INFRASTRUCTURE ONLY: the parity checker.  tests/, the smoke check and the cpu_baseline leg
of bench.py may import this module; the product package never does.

Each function names the reference lines it restates (paths relative to the reference project
root).  Parity status: pinned against the reference's own attic/tConvolveMPI/Benchmark.cc
(tests/golden/, tests/test_oracle.py).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle_tcv.so")
_lib = None

_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_I32 = ctypes.c_int
_F64 = ctypes.c_double


def build() -> str:
    """Compile the restatement (make restatement) and return the library path."""
    subprocess.run(["make", "-s", "-C", _HERE, "restatement"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_init_uvw.argtypes = [_I64, _I32, ctypes.c_uint64, _P, _P, _P]
        L.orc_init_freq.argtypes = [_I32, _P]
        L.orc_c_geometry.argtypes = [_F64, _F64, _I32, _I32, _P, _P, _P]
        L.orc_init_c.argtypes = [_F64, _F64, _I32, _I32, _P, _P, _P, _P, _P]
        L.orc_init_c.restype = ctypes.c_float
        L.orc_init_offsets.argtypes = [_I64, _I32, _P, _P, _P, _P, _F64, _F64, _I32, _I32, _I32,
                                       _I32, _P, _P, _P]
        L.orc_grid_f32.argtypes = [_P, _I64, _I32, _P, _P, _P, _P, _P, _I32, _I32]
        L.orc_degrid_f32.argtypes = [_P, _I32, _I32, _P, _P, _P, _P, _P, _I64, _I32]
        L.orc_grid_f64.argtypes = [_P, _I64, _I32, _P, _P, _P, _P, _P, _I32, _I32]
        L.orc_degrid_f64.argtypes = [_P, _I32, _I32, _P, _P, _P, _P, _P, _I64, _I32]
        L.orc_cur_geometry.argtypes = [_I32, _P]
        L.orc_cur_init_uvw.argtypes = [_I32, _P, _P, _P, _P]
        L.orc_cur_init_c.argtypes = [_I32, _P, _P, _P]
        L.orc_cur_init_offsets.argtypes = [_I32, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P]
        L.orc_cur_sort_by_plane.argtypes = [_I64, _I32, _P, _P, _P, _P]
        L.orc_cur_grid_f32.argtypes = [_P, _I64, _P, _P, _P, _P, _P, _P, _P, _I32, _I32]
        L.orc_cur_degrid_f32.argtypes = [_P, _I32, _I64, _P, _P, _P, _P, _P, _P, _P, _I32]
        L.orc_cur_degrid_f64.argtypes = [_P, _I32, _I64, _P, _P, _P, _P, _P, _P, _P, _I32]
        L.orc_cur_grid_f64.argtypes = [_P, _I64, _P, _P, _P, _P, _P, _P, _P, _I32, _I32]
        L.orc_find_peak.argtypes = [_P, _I64, _P, _P]
        L.orc_subtract_psf.argtypes = [_P, _I32, _P, _I32, _I64, _I64, ctypes.c_float, ctypes.c_float]
        L.orc_subtract_psf.restype = _I64
        L.orc_hogbom.argtypes = [_P, _I32, _P, _I32, _P, _P, _I32, ctypes.c_float, ctypes.c_float, _P, _P, _P,
                                 _P, _P]
        L.orc_hogbom.restype = _I32
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.flags.c_contiguous
    return ctypes.c_void_p(a.ctypes.data)


@dataclass
class Config:
    """One tConvolve problem (the constants of attic/tConvolveMPI/Benchmark.h:39-46)."""
    n_samples: int
    w_size: int
    n_chan: int
    g_size: int
    cell_size: float
    baseline: int = 2000
    seed: int = 0  # LCG start state = seed + 1; seed 0 is the reference's next = 1


ARCSEC_CELL_1024 = 1.0 / (1024 * 5.0 * math.pi / 648000.0)  # 5 arcsec cell on a 1024 grid, in wavelengths

CONFIGS = {
    "g1": Config(200, 5, 1, 128, 200.0),
    "g2": Config(1000, 9, 4, 256, 100.0),
    "c1": Config(16000, 9, 1, 1024, ARCSEC_CELL_1024),
    "c2": Config(160000, 33, 1, 4096, 5.0),
}


def init_uvw(cfg: Config):
    """u, v, w from the reference LCG (attic/tConvolveMPI/Benchmark.cc:46-80)."""
    n = cfg.n_samples
    u = np.empty(n, np.float64)
    v = np.empty(n, np.float64)
    w = np.empty(n, np.float64)
    lib().orc_init_uvw(n, cfg.baseline, cfg.seed + 1, _p(u), _p(v), _p(w))
    return u, v, w


def init_freq(cfg: Config) -> np.ndarray:
    """Inverse wavelengths per channel (attic/tConvolveMPI/Benchmark.cc:86-90)."""
    f = np.empty(cfg.n_chan, np.float64)
    lib().orc_init_freq(cfg.n_chan, _p(f))
    return f


def c_geometry(cfg: Config):
    """(support, overSample, wCellSize) as attic/tConvolveMPI/Benchmark.cc:212-217 computes them."""
    s = ctypes.c_int()
    o = ctypes.c_int()
    wc = ctypes.c_double()
    freq = init_freq(cfg)
    lib().orc_c_geometry(float(freq[0]), float(cfg.cell_size), cfg.baseline, cfg.w_size,
                         ctypes.byref(s), ctypes.byref(o), ctypes.byref(wc))
    return s.value, o.value, wc.value


def init_c(cfg: Config, want_f64: bool = False):
    """Normalised table C (attic/tConvolveMPI/Benchmark.cc:206-270).

    Returns (C complex64 flat, C64 float64 flat or None, support, overSample, wCellSize, sumC).
    """
    support, os_, _ = c_geometry(cfg)
    s = 2 * support + 1
    n = s * s * os_ * os_ * cfg.w_size
    c = np.empty(n, np.complex64)
    c64 = np.empty(n, np.float64) if want_f64 else None
    sup = ctypes.c_int()
    o = ctypes.c_int()
    wc = ctypes.c_double()
    freq = init_freq(cfg)
    sum_c = lib().orc_init_c(float(freq[0]), float(cfg.cell_size), cfg.baseline, cfg.w_size, _p(c),
                             _p(c64) if want_f64 else None, ctypes.byref(sup), ctypes.byref(o),
                             ctypes.byref(wc))
    return c, c64, sup.value, o.value, wc.value, float(sum_c)


def init_offsets(cfg: Config, u, v, w, w_cell_size: float, support: int, over_sample: int):
    """iu, iv, cOffset per sample (attic/tConvolveMPI/Benchmark.cc:281-324)."""
    n = cfg.n_samples * cfg.n_chan
    iu = np.empty(n, np.int32)
    iv = np.empty(n, np.int32)
    co = np.empty(n, np.int32)
    freq = init_freq(cfg)
    lib().orc_init_offsets(cfg.n_samples, cfg.n_chan, _p(np.ascontiguousarray(u)),
                           _p(np.ascontiguousarray(v)), _p(np.ascontiguousarray(w)), _p(freq),
                           float(cfg.cell_size), float(w_cell_size), cfg.w_size, cfg.g_size,
                           support, over_sample, _p(iu), _p(iv), _p(co))
    return iu, iv, co


def grid_f32(data, support, c, coff, iu, iv, grid, g_size, threads: int = 1):
    """grid += gridding of data, reference arithmetic and order (Benchmark.cc:125-155). In place."""
    data = np.ascontiguousarray(data, np.complex64)
    assert grid.dtype == np.complex64 and grid.size == g_size * g_size
    lib().orc_grid_f32(_p(data), data.size, support, _p(c), _p(coff), _p(iu), _p(iv), _p(grid),
                       g_size, threads)
    return grid


def degrid_f32(grid, g_size, support, c, coff, iu, iv, threads: int = 1):
    """Degridded samples, reference arithmetic and order (Benchmark.cc:158-195)."""
    n = iu.size
    out = np.empty(n, np.complex64)
    lib().orc_degrid_f32(_p(grid), g_size, support, _p(c), _p(coff), _p(iu), _p(iv), _p(out), n,
                         threads)
    return out


def grid_f64(data, support, c64, coff, iu, iv, grid64, g_size, threads: int = 1):
    """FP64 gridding (complex128 data and grid, real float64 table). In place; the same result
    for any thread count (each thread owns a band of rows and walks the samples in order)."""
    data = np.ascontiguousarray(data, np.complex128)
    assert grid64.dtype == np.complex128
    lib().orc_grid_f64(_p(data), data.size, support, _p(c64), _p(coff), _p(iu), _p(iv),
                       _p(grid64), g_size, threads)
    return grid64


def degrid_f64(grid64, g_size, support, c64, coff, iu, iv, threads: int = 1):
    n = iu.size
    out = np.empty(n, np.complex128)
    lib().orc_degrid_f64(_p(grid64), g_size, support, _p(c64), _p(coff), _p(iu), _p(iv), _p(out), n,
                         threads)
    return out


def run_plain(cfg: Config, vis: np.ndarray | None = None, threads: int = 1, want_f64: bool = False):
    """The whole reference pipeline: init, one gridding pass into a zero grid, one degridding pass.

    vis None means the reference's data = 1+0i (Benchmark.cc:76-79).
    """
    u, v, w = init_uvw(cfg)
    c, c64, support, os_, wcs, sum_c = init_c(cfg, want_f64)
    iu, iv, co = init_offsets(cfg, u, v, w, wcs, support, os_)
    n = cfg.n_samples * cfg.n_chan
    data = np.ones(n, np.complex64) if vis is None else np.ascontiguousarray(vis, np.complex64)
    grid = np.zeros(cfg.g_size * cfg.g_size, np.complex64)
    grid_f32(data, support, c, co, iu, iv, grid, cfg.g_size, threads)
    out = degrid_f32(grid, cfg.g_size, support, c, co, iu, iv, threads)
    res = dict(u=u, v=v, w=w, C=c, support=support, over_sample=os_, w_cell_size=wcs,
               sum_c=sum_c, iu=iu, iv=iv, coff=co, data=data, grid=grid, outdata=out)
    if want_f64:
        g64 = np.zeros(cfg.g_size * cfg.g_size, np.complex128)
        grid_f64(data.astype(np.complex128), support, c64, co, iu, iv, g64, cfg.g_size, threads)
        res["C64"] = c64
        res["grid64"] = g64
        res["outdata64"] = degrid_f64(g64, cfg.g_size, support, c64, co, iu, iv, threads)
    return res


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """||a - b|| / ||b|| in float64."""
    a = np.asarray(a).astype(np.complex128).ravel()
    b = np.asarray(b).astype(np.complex128).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


# -------------------------------------------------------------------------------------------------
# The variable-support path of current/tConvolveMPI (tconvolve_oracle_current.c)
# -------------------------------------------------------------------------------------------------
@dataclass(frozen=True)
class CurGeometry:
    run_type: int
    w_size: int
    over_sample: int
    support: int
    g_size: int
    n_baselines: int
    n_samples: int
    w_cell_size: float
    uv_cell_size: float
    c_len: int
    s_max: int


def cur_geometry(run_type: int) -> CurGeometry:
    """current/tConvolveMPI/Benchmark.cc:64-158 (run types 0 continuum, 1 spectral, 2 nearest
    neighbour, 3 7x7 kernels, 4 87x87 kernels)."""
    out = np.zeros(10, np.float64)
    if lib().orc_cur_geometry(run_type, _p(out)) != 0:
        raise ValueError(f"unknown run type {run_type}")
    return CurGeometry(run_type, int(out[0]), int(out[1]), int(out[2]), int(out[3]), int(out[4]),
                       int(out[5]), float(out[6]), float(out[7]), int(out[8]), int(out[9]))


def cur_init_uvw(run_type: int, state: int = 1):
    """current/tConvolveMPI/Benchmark.cc:246-262; returns u, v, w and the generator state after."""
    g = cur_geometry(run_type)
    u, v, w = (np.empty(g.n_samples, np.float64) for _ in range(3))
    st = np.array([state], np.uint64)
    lib().orc_cur_init_uvw(run_type, _p(st), _p(u), _p(v), _p(w))
    return u, v, w, int(st[0])


def cur_init_c(run_type: int):
    """current/tConvolveMPI/Benchmark.cc:487-583: (C complex64, sSize per plane, cOffset0)."""
    g = cur_geometry(run_type)
    s_size = np.empty(g.w_size, np.int32)
    off0 = np.empty(g.w_size, np.int32)
    c = np.empty(g.c_len, np.complex64)
    lib().orc_cur_init_c(run_type, _p(s_size), _p(off0), _p(c))
    return c, s_size, off0


def cur_init_offsets(run_type: int, u, v, w, s_size, off0):
    """current/tConvolveMPI/Benchmark.cc:599-650: iu, iv, wPlane, cOffset."""
    n = u.size
    iu, iv, wp, co = (np.empty(n, np.int32) for _ in range(4))
    lib().orc_cur_init_offsets(run_type, n, _p(u), _p(v), _p(w), _p(s_size), _p(off0), _p(iu), _p(iv),
                               _p(wp), _p(co))
    return iu, iv, wp, co


def cur_sort_by_plane(w_size: int, iu, iv, wp, co):
    """setSort(1), current/tConvolveMPI/Benchmark.cc:287-306: offsets stably ordered by w-plane."""
    iu, iv, wp, co = (np.ascontiguousarray(a, np.int32).copy() for a in (iu, iv, wp, co))
    lib().orc_cur_sort_by_plane(iu.size, w_size, _p(iu), _p(iv), _p(wp), _p(co))
    return iu, iv, wp, co


def cur_grid_f32(data, iu, iv, wp, co, s_size, c, grid, g_size: int, threads: int = 1):
    """current/tConvolveMPI/Benchmark.cc:373-411, reference order; grid accumulated in place."""
    data = np.ascontiguousarray(data, np.complex64)
    lib().orc_cur_grid_f32(_p(data), data.size, _p(iu), _p(iv), _p(wp), _p(co), _p(s_size), _p(c), _p(grid),
                           g_size, threads)
    return grid


def cur_degrid_f32(grid, g_size: int, iu, iv, wp, co, s_size, c, threads: int = 1):
    """current/tConvolveMPI/Benchmark.cc:414-452."""
    out = np.empty(iu.size, np.complex64)
    lib().orc_cur_degrid_f32(_p(grid), g_size, iu.size, _p(iu), _p(iv), _p(wp), _p(co), _p(s_size), _p(c),
                             _p(out), threads)
    return out


def cur_degrid_f64(grid, g_size: int, iu, iv, wp, co, s_size, c, threads: int = 1):
    """Degridding of the same float grid and table with double accumulation: the value the FP32
    sums of current/tConvolveMPI/Benchmark.cc:414-452 approximate (complex128)."""
    grid = np.ascontiguousarray(grid, np.complex64)
    out = np.empty(iu.size, np.complex128)
    lib().orc_cur_degrid_f64(_p(grid), g_size, iu.size, _p(iu), _p(iv), _p(wp), _p(co), _p(s_size), _p(c),
                             _p(out), threads)
    return out


def cur_grid_f64(data, iu, iv, wp, co, s_size, c, g_size: int, threads: int = 1):
    """Gridding of the float data and table with double accumulation (complex128 grid)."""
    data = np.ascontiguousarray(data, np.complex64)
    grid = np.zeros(g_size * g_size, np.complex128)
    lib().orc_cur_grid_f64(_p(data), data.size, _p(iu), _p(iv), _p(wp), _p(co), _p(s_size), _p(c), _p(grid),
                           g_size, threads)
    return grid


# ---- Hogbom CLEAN (tconvolve_oracle_hogbom.c; current/tHogbomCleanOMP/HogbomGolden.cc:47-141) ----
def find_peak(image: np.ndarray):
    """findPeak (HogbomGolden.cc:127-139): (value, first index) of the largest |value|."""
    img = np.ascontiguousarray(image, dtype=np.float32).ravel()
    v = ctypes.c_float()
    p = ctypes.c_int64()
    lib().orc_find_peak(_p(img), img.size, ctypes.byref(v), ctypes.byref(p))
    return float(v.value), int(p.value)


def hogbom(dirty: np.ndarray, psf: np.ndarray, niters: int, gain: float = 0.1, threshold: float = 0.0,
           model: np.ndarray | None = None):
    """HogbomGolden::deconvolve (HogbomGolden.cc:62-97) on square float images.  Returns a dict
    with model, residual, iterations done, stop iteration (-1), per-iteration peaks and the PSF
    rows skipped (reference out-of-bounds reads)."""
    d = np.ascontiguousarray(dirty, dtype=np.float32)
    p = np.ascontiguousarray(psf, dtype=np.float32)
    w, pw = int(round(np.sqrt(d.size))), int(round(np.sqrt(p.size)))
    assert w * w == d.size and pw * pw == p.size
    m = np.zeros(d.size, np.float32) if model is None else np.ascontiguousarray(model, dtype=np.float32).ravel().copy()
    r = np.empty(d.size, np.float32)
    hv = np.zeros(max(niters, 1), np.float32)
    hp = np.zeros(max(niters, 1), np.int64)
    stopped = ctypes.c_int()
    skipped = ctypes.c_int64()
    ppos = ctypes.c_int64()
    done = lib().orc_hogbom(_p(d), w, _p(p), pw, _p(m), _p(r), int(niters), ctypes.c_float(gain),
                            ctypes.c_float(threshold), _p(hv), _p(hp), ctypes.byref(stopped), ctypes.byref(skipped),
                            ctypes.byref(ppos))
    return {"model": m, "residual": r, "done": int(done), "stopped_at": int(stopped.value),
            "hist_val": hv[:done], "hist_pos": hp[:done], "skipped_rows": int(skipped.value),
            "psf_peak_pos": int(ppos.value)}


# ---- the imaging major cycle (current/tMajorACC/tMajorACC.cc:487-640, 889-1635) ----
# Restated with the gridding, degridding and Hogbom functions above (C, float) and numpy's
# double-precision FFT for fftExec (the reference calls single-precision FFTW or cuFFT there; its
# own check of one against the other is |difference| * psfScale <= 1e-5 per pixel, :1460-1580).
# tMajorACC needs FFTW, OpenACC and the PGI compiler, none of which is here: it is not built, so
# this restatement is checked piecewise (gridding, degridding and Hogbom are the pinned functions
# above; the set-up draws are the attic generator's) and its FFT against the definition.

def lcg_after(draws: int, state: int = 1) -> int:
    """The K&R generator's state after `draws` steps (attic/tConvolveMPI/Benchmark.cc:53-58)."""
    a, c, m = 1103515245, 12345, 1 << 64
    A, C = 1, 0
    while draws:
        if draws & 1:
            A, C = (a * A) % m, (a * C + c) % m
        a, c = (a * a) % m, (a * c + c) % m
        draws >>= 1
    return (A * state + C) % m


def fft_exec(grid: np.ndarray, g_size: int, forward: bool) -> np.ndarray:
    """fftExec (tMajorACC.cc:487-545): half-size rotation, unnormalised 2-D transform (forward
    exp(-i..), backward exp(+i..)), rotation back; in double, returned as complex64."""
    x = np.fft.fftshift(np.asarray(grid, np.complex128).reshape(g_size, g_size))
    y = np.fft.fft2(x) if forward else np.fft.ifft2(x, norm="forward")
    return np.fft.fftshift(y).astype(np.complex64).ravel()


def fft_fix(grid: np.ndarray, scale: float) -> np.ndarray:
    """fftFix (tMajorACC.cc:620-626): Re * scale in float; returned as the float real image."""
    return (np.real(grid).astype(np.float32) * np.float32(scale)).astype(np.float32)


def major_setup(n_samples: int = 160000, w_size: int = 33, n_chan: int = 1, cell_size: float = 5.0,
                g_size: int = 4096, baseline: int = 2000, n_sources: int = 100, threads: int = 16):
    """tMajorACC's set-up (:930-1035): samples, the delta table of its initC (:349-434), offsets,
    the true sky of n_sources points and its degridded visibilities."""
    cfg = Config(n_samples, w_size, n_chan, g_size, cell_size, baseline, 0)
    u, v, w = init_uvw(cfg)
    support, os_, wcs = c_geometry(cfg)
    s = 2 * support + 1
    c = np.zeros(s * s * os_ * os_ * w_size, np.complex64)
    c[::s * s] = 1.0  # C[cind] = 1 at i == 0 && j == 0; the float normalisation factor is exactly 1
    iu, iv, co = init_offsets(cfg, u, v, w, wcs, support, os_)
    state = lcg_after(3 * n_samples)
    maxint = 2147483647

    def draw():
        nonlocal state
        state = (state * 1103515245 + 12345) % (1 << 64)
        return ((state // 65536) & 0xFFFFFFFF) % maxint

    true = np.zeros(g_size * g_size, np.complex64)
    for _ in range(n_sources):
        l = int(g_size * float(draw()) / float(maxint))
        m = int(g_size * float(draw()) / float(maxint))
        true[m * g_size + l] += np.float32(draw()) / np.float32(2147483648.0)
    true_uv = fft_exec(true, g_size, True)
    vis = degrid_f32(true_uv, g_size, support, c, co, iu, iv, threads)
    n = n_samples * n_chan
    scale = float(np.float32(1.0 / float(np.float32(n))))
    return {"cfg": cfg, "support": support, "C": c, "iu": iu, "iv": iv, "coff": co, "vis": vis, "scale": scale,
            "true": true}


def major_cycle(st: dict, data: np.ndarray, psf_image: np.ndarray | None, n_minor: int = 100, gain: float = 0.1,
                threads: int = 16) -> dict:
    """One major cycle of tMajorACC's CPU path (:1096-1236): grid (the PSF too when psf_image is
    None), inverse FFT + fix, Hogbom (no threshold), forward FFT of the model, degrid, subtract.
    Returns every stage's output and the updated data."""
    g = st["cfg"].g_size
    sup, c, iu, iv, co, scale = st["support"], st["C"], st["iu"], st["iv"], st["coff"], st["scale"]
    out = {}
    if psf_image is None:
        uv_psf = np.zeros(g * g, np.complex64)
        grid_f32(np.ones(iu.size, np.complex64), sup, c, co, iu, iv, uv_psf, g, threads)
        out["uv_psf"] = uv_psf
        psf_image = fft_fix(fft_exec(uv_psf, g, False), scale)
    out["psf"] = psf_image
    uv = np.zeros(g * g, np.complex64)
    grid_f32(data, sup, c, co, iu, iv, uv, g, threads)
    out["uv_data"] = uv
    dirty = fft_fix(fft_exec(uv, g, False), scale)
    out["dirty"] = dirty
    h = hogbom(dirty, psf_image, n_minor, gain, 0.0)
    out["residual"], out["model"] = h["residual"], h["model"]
    out["model_grid"] = fft_exec(h["model"].astype(np.complex64), g, True)
    out["model_vis"] = degrid_f32(out["model_grid"], g, sup, c, co, iu, iv, threads)
    out["data"] = (data - out["model_vis"]).astype(np.complex64)
    return out
