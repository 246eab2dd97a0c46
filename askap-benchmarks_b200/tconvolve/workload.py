"""Problem definitions of the tConvolve benchmark and the synthetic visibility generator.

Named problems (the constants of attic/tConvolveMPI/Benchmark.h:39-46):

    c2  the reference default: 160000 samples, 33 w-planes, 4096^2 grid, 5 wavelength cells,
        2000 m baseline (support 64, 129^2 footprint, 2.66e9 updates per pass)
    c1  the CPU-sized case: 16000 samples, 9 w-planes, 1024^2 grid, 5 arcsec cells
        (1/(1024 * 5 arcsec) = 40.286 wavelengths; support 22, 45^2 footprint)
    g1, g2  small test problems (support 10 and 14; g2 has 4 channels)

Visibilities: the reference sets every sample to 1+0i (Benchmark.cc:76-79).  The N(0,1) form
draws real then imaginary parts as float32 standard normals from numpy's PCG64 generator seeded
with `seed` (normal_vis), so every consumer sees the same bytes.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, replace

import numpy as np

ARCSEC_CELL_1024 = 1.0 / (1024 * 5.0 * math.pi / 648000.0)


@dataclass(frozen=True)
class Problem:
    name: str
    n_samples: int
    w_size: int
    n_chan: int
    g_size: int
    cell_size: float
    baseline: int = 2000
    seed: int = 0

    @property
    def freq0(self) -> float:
        return 1.4e9 / 2.998e8

    def support(self) -> int:
        return int(1.5 * math.sqrt(abs(self.baseline) * self.cell_size * self.freq0) / self.cell_size)

    def s_size(self) -> int:
        return 2 * self.support() + 1

    def n_data(self) -> int:
        return self.n_samples * self.n_chan

    def updates_per_pass(self) -> float:
        return float(self.n_data()) * self.s_size() ** 2

    def kwargs(self) -> dict:
        return dict(n_samples=self.n_samples, w_size=self.w_size, n_chan=self.n_chan,
                    g_size=self.g_size, cell_size=self.cell_size, baseline=self.baseline,
                    seed=self.seed)

    def with_(self, **kw) -> "Problem":
        return replace(self, **kw)


PROBLEMS = {
    "g1": Problem("g1", 200, 5, 1, 128, 200.0),
    "g2": Problem("g2", 1000, 9, 4, 256, 100.0),
    "c1": Problem("c1", 16000, 9, 1, 1024, ARCSEC_CELL_1024),
    "c2": Problem("c2", 160000, 33, 1, 4096, 5.0),
}


def normal_vis(n: int, seed: int) -> np.ndarray:
    """n complex64 visibilities with N(0,1) real and imaginary parts (PCG64(seed))."""
    rng = np.random.default_rng(seed)
    re = rng.standard_normal(n, dtype=np.float32)
    im = rng.standard_normal(n, dtype=np.float32)
    out = np.empty(n, np.complex64)
    out.real = re
    out.imag = im
    return out


def batch_sizes(n_jobs: int = 64, seed: int = 0, n_min: float = 1e4, n_max: float = 4e5,
                g_sizes=(2048, 4096)) -> list:
    """Jobs of the batched workload: [(n_samples, g_size)] with n log-uniform in [n_min, n_max] and
    g_size drawn uniformly from g_sizes (PCG64(seed)).  With the default 5 wavelength cells and
    2000 m baseline every footprint reaches at most 999 cells from the centre, inside both sizes."""
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(math.log(n_min), math.log(n_max), n_jobs)).astype(np.int64)
    g = rng.choice(np.asarray(g_sizes, dtype=np.int64), n_jobs)
    return [(int(a), int(b)) for a, b in zip(n, g)]


def _splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser on uint64 counters (exact integer arithmetic, same bits everywhere)."""
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def synthetic_psf(width: int, scale: float | None = None) -> np.ndarray:
    """A point-spread function of width x width float32 pixels with its peak, 1.0, at
    (width/2, width/2) and a negative sidelobe ring decaying as 1/r^2: psf(r) = (1 - r^2 / 2s^2) /
    (1 + r^2 / s^2)^2 with s = width / 64 (at least 2).  Rational arithmetic in float64 only (no
    transcendental functions), so the same bits on every host.  It stands in for the reference's
    psf_<width>.img inputs of current/tHogbomCleanOMP, which are not in its tree."""
    s = float(scale) if scale else max(2.0, width / 64.0)
    c = width // 2
    d = np.arange(width, dtype=np.float64) - c
    r2 = d[:, None] ** 2 + d[None, :] ** 2
    s2 = s * s
    q = 1.0 + r2 / s2
    return ((1.0 - r2 / (2.0 * s2)) / (q * q)).astype(np.float32)


def synthetic_dirty(width: int, n_sources: int = 20, noise: float = 1e-3, seed: int = 0,
                    psf_scale: float | None = None) -> np.ndarray:
    """A dirty image of width x width float32 pixels: n_sources point sources, each the
    synthetic_psf shape centred on its pixel with amplitude in [0.1, 1), plus uniform noise in
    [-noise/2, noise/2).  Positions and amplitudes come from the reference's K&R generator
    (state seed + 1, three draws per source: x, y, amplitude), positions in the inner 80% of the
    image; the noise from SplitMix64 of the pixel index and seed.  Float64 rational arithmetic,
    rounded to float32 once."""
    s = float(psf_scale) if psf_scale else max(2.0, width / 64.0)
    s2 = s * s
    state = seed + 1
    maxint = 2147483647

    def draw():
        nonlocal state
        state = (state * 1103515245 + 12345) & 0xFFFFFFFFFFFFFFFF
        return ((state // 65536) & 0xFFFFFFFF) % maxint

    img = np.zeros((width, width), np.float64)
    d = np.arange(width, dtype=np.float64)
    lo, span = int(0.1 * width), max(1, int(0.8 * width))
    for _ in range(n_sources):
        x = lo + int(span * (draw() / maxint))
        y = lo + int(span * (draw() / maxint))
        a = 0.1 + 0.9 * (draw() / maxint)
        r2 = (d[:, None] - y) ** 2 + (d[None, :] - x) ** 2
        q = 1.0 + r2 / s2
        img += a * (1.0 - r2 / (2.0 * s2)) / (q * q)
    if noise:
        idx = np.arange(width * width, dtype=np.uint64) + np.uint64(seed) * np.uint64(0x100000000)
        u = (_splitmix64(idx) >> np.uint64(11)).astype(np.float64) / float(1 << 53)
        img += (noise * (u - 0.5)).reshape(width, width)
    return img.astype(np.float32)
