"""GPU major cycle (tcv_major_*) and FFT steps (tcv_fft_*) against the oracle.

Bars (written here, used below) are the reference's own check between its CPU and GPU pipelines
(current/tMajorACC/tMajorACC.cc:1460-1580), applied per stage and per cycle:
  * uv grids: |difference of real parts| / |largest grid value| <= 1e-5;
  * images (PSF, dirty, residual, model), the model grid and the model visibilities:
    |difference| * psfScale <= 1e-5, psfScale = 1 / PSF peak (here on real and imaginary parts);
  * the fused image step equals fftFix(fftExec(backward)) bit for bit (same transform);
  * FFT steps against numpy's double-precision transform: max |difference| <= 2e-6 x max |value|.
The oracle's FFT is double precision; the reference's is single-precision FFTW or cuFFT.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
THRESH = 1e-5


def _fft_case(n, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(n * n) + 1j * rng.standard_normal(n * n)).astype(np.complex64)


@pytest.mark.parametrize("n", [128, 256, 512, 1034, 2048, 4096, 8192])
def test_fft_steps(tcv, orc, cuda_ok, n):
    """Power-of-two sizes 128 .. 8192 run the library's own two-pass transform (an odd power of
    two takes one radix-2 stage), 1034 runs cuFFT; both against numpy's double transform."""
    import torch

    from tconvolve import major

    x = _fft_case(n, 1)
    for forward in (True, False):
        g = torch.from_numpy(x.copy()).cuda()
        major.fft_exec(g, n, forward)
        ref = orc.fft_exec(x, n, forward)
        got = g.cpu().numpy()
        assert np.abs(got - ref).max() <= 2e-6 * np.abs(ref).max(), forward
    # the fused dirty-image step is fftFix(fftExec(backward)) bit for bit
    g1 = torch.from_numpy(x.copy()).cuda()
    major.fft_exec(g1, n, False)
    major.fft_fix(g1, 1.0 / 3.0)
    g2 = torch.from_numpy(x.copy()).cuda()
    img = torch.empty(n * n, dtype=torch.float32, device="cuda")
    major.image_from_grid(g2, n, 1.0 / 3.0, img)
    assert np.array_equal(img.cpu().numpy(), np.real(g1.cpu().numpy()).astype(np.float32))
    # the fused model step against the definition
    m = np.zeros(n * n, np.float32)
    rng = np.random.default_rng(2)
    m[rng.integers(0, n * n, 100)] = rng.random(100, dtype=np.float32)
    out = torch.empty(n * n, dtype=torch.complex64, device="cuda")
    major.grid_from_image(torch.from_numpy(m).cuda(), n, out)
    ref = orc.fft_exec(m.astype(np.complex64), n, True)
    assert np.abs(out.cpu().numpy() - ref).max() <= 2e-6 * np.abs(ref).max()


def test_fft_odd_size_refused(tcv, cuda_ok):
    import torch

    from tconvolve import major
    from tconvolve._lib import TcvError

    g = torch.zeros(15 * 15, dtype=torch.complex64, device="cuda")
    with pytest.raises(TcvError) as e:
        major.fft_exec(g, 15, True)
    assert e.value.status == 8  # TCV_ERR_UNSUPPORTED, as the reference refuses odd sizes


def _close_uv(got, ref):
    peak = np.abs(ref[np.argmax(np.abs(ref))].real)
    return np.abs(got.real - ref.real).max() / peak <= THRESH


def _close(got, ref, psf_scale):
    d = np.abs(np.asarray(got) - np.asarray(ref)).max() * psf_scale
    return d <= THRESH, d


@pytest.mark.parametrize("cfg", [
    dict(n_samples=2000, w_size=9, cell_size=25.0, g_size=512, n_minor=20, cycles=3),
    dict(n_samples=1500, w_size=9, n_chan=3, cell_size=25.0, g_size=512, n_minor=20, cycles=2),
    dict(n_samples=160000, w_size=33, cell_size=5.0, g_size=4096, n_minor=100, cycles=1),
], ids=["512", "512-3chan", "4096"])
def test_major_cycle_against_oracle(tcv, orc, cuda_ok, cfg):
    """The small problem over three cycles; tMajorACC's own problem (160000 samples, 4096^2,
    100 minor iterations) over its first cycle."""
    from tconvolve._lib import IMG_DIRTY, IMG_MODEL, IMG_PSF, IMG_RESIDUAL
    from tconvolve.major import MajorCycle

    cycles = cfg.pop("cycles")
    m = MajorCycle(keep_stages=1, **cfg)
    m.init()
    st = orc.major_setup(cfg["n_samples"], cfg["w_size"], cfg.get("n_chan", 1), cfg["cell_size"], cfg["g_size"], 2000,
                         100)
    iu, iv, co = m.offsets()
    assert np.array_equal(iu, st["iu"]) and np.array_equal(iv, st["iv"]) and np.array_equal(co, st["coff"])
    assert m.info()["support"] == st["support"] and m.info()["scale"] == np.float32(st["scale"])
    psf_scale = None
    ok, d = _close(m.vis(0), st["vis"], 1.0)
    assert ok, ("true visibilities", d)
    data, psf = st["vis"], None
    for cyc in range(cycles):
        m.run_cycle()
        m.sync()
        o = orc.major_cycle(st, data, psf, cfg["n_minor"])
        if cyc == 0:
            assert _close_uv(m.grid(0), o["uv_psf"]), "psf uv grid"
            psf_scale = 1.0 / abs(float(o["psf"][np.argmax(np.abs(o["psf"]))]))
        assert _close_uv(m.grid(1), o["uv_data"]), ("uv grid", cyc)
        for name, which in (("psf", IMG_PSF), ("dirty", IMG_DIRTY), ("residual", IMG_RESIDUAL), ("model", IMG_MODEL)):
            ok, d = _close(m.image(which), o[name], psf_scale)
            assert ok, (name, cyc, d)
        for name, got in (("model_grid", m.grid(2)), ("model_vis", m.vis(1)), ("data", m.vis(0))):
            ok, d = _close(got, o[name], psf_scale)
            assert ok, (name, cyc, d)
        data, psf = o["data"], o["psf"]
    ms, n = m.stage_ms()
    assert n == cycles and all(v >= 0 for v in ms.values()) and ms["grid"] > 0 and ms["hogbom"] > 0
    m.close()
