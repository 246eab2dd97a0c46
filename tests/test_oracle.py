"""The oracle pinned against the reference (CPU only).

tconvolve_oracle.c restates attic/tConvolveMPI/Benchmark.cc; these tests check its outputs bit
for bit (sha256) against the reference's own outputs recorded in tests/golden/golden.json, plus
the known answers the reference prints (attic/tConvolveMPI/README.md:58-73).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import VIS_SEED, oracle_config, sha
from tconvolve.workload import PROBLEMS, normal_vis


@pytest.mark.parametrize("cfg", ["g1", "g2", "c1"])
@pytest.mark.parametrize("vis_kind", ["ones", "normal"])
def test_oracle_bit_exact_vs_reference(orc, golden, cfg, vis_kind):
    prob = PROBLEMS[cfg]
    vis = None if vis_kind == "ones" else normal_vis(prob.n_data(), VIS_SEED)
    r = orc.run_plain(oracle_config(orc, prob), vis=vis, threads=4)
    ref = golden["runs"][f"{cfg}_{vis_kind}"]
    assert r["support"] == ref["meta"]["support"]
    assert r["over_sample"] == ref["meta"]["overSample"]
    assert r["w_cell_size"] == pytest.approx(ref["meta"]["wCellSize"], rel=1e-15)
    for key in ("u", "v", "w", "iu", "iv", "coff", "C", "grid", "outdata", "data"):
        assert sha(r[key]) == ref["sha256"][key], f"{cfg}/{vis_kind}: {key} differs from the reference"


def test_oracle_small_arrays_match_fixture(orc):
    prob = PROBLEMS["g1"]
    r = orc.run_plain(oracle_config(orc, prob))
    fx = np.load("tests/golden/g1_ones.npz")
    assert np.array_equal(r["grid"], fx["grid"])
    assert np.array_equal(r["outdata"], fx["outdata"])


def test_oracle_threading_is_bit_identical(orc):
    prob = PROBLEMS["g2"]
    vis = normal_vis(prob.n_data(), 7)
    a = orc.run_plain(oracle_config(orc, prob), vis=vis, threads=1)
    b = orc.run_plain(oracle_config(orc, prob), vis=vis, threads=7)
    assert np.array_equal(a["grid"], b["grid"])
    assert np.array_equal(a["outdata"], b["outdata"])


def test_reference_known_answers_default_config(orc, golden):
    """attic/tConvolveMPI/README.md:58-73: Support = 64, W cellsize = 566.034, 268 MB, [129,129,8,8,33];
    and the float sumC of the 35 M entry table saturates at exactly 2^24."""
    cfg = oracle_config(orc, PROBLEMS["c2"])
    support, os_, wcs = orc.c_geometry(cfg)
    assert support == 64 and os_ == 8
    assert round(wcs, 3) == 566.034
    s = 2 * support + 1
    n = s * s * os_ * os_ * cfg.w_size
    assert n * 8 // (1024 * 1024) == 268
    c, _, _, _, _, sum_c = orc.init_c(cfg)
    assert sum_c == 16777216.0
    assert sha(c) == golden["runs"]["c2_ones"]["sha256"]["C"]
    u, v, w = orc.init_uvw(cfg)
    iu, iv, co = orc.init_offsets(cfg, u, v, w, wcs, support, os_)
    assert sha(co) == golden["runs"]["c2_ones"]["sha256"]["coff"]
    planes = np.unique(co // (s * s * os_ * os_))
    assert planes.min() == 8 and planes.max() == 24  # only the middle w-planes are touched
    # asymmetric footprint (Benchmark.cc:133): rows start at iv, columns at iu - support
    assert iu.min() - support >= 0 and iu.max() + support < cfg.g_size
    assert iv.min() >= 0 and iv.max() + 2 * support < cfg.g_size


def test_config1_arcsec_reading(orc, golden):
    """5 arcsec cells on a 1024 grid = 40.286 wavelengths: support 22, footprints in bounds
    (a literal 5-wavelength cell would put footprints up to 999 px from the centre)."""
    cfg = oracle_config(orc, PROBLEMS["c1"])
    support, _, wcs = orc.c_geometry(cfg)
    assert support == 22
    assert wcs == pytest.approx(2075.4577, rel=1e-7)
    u, v, w = orc.init_uvw(cfg)
    iu, iv, _ = orc.init_offsets(cfg, u, v, w, wcs, support, 8)
    assert iu.min() - support >= 0 and iu.max() + support < 1024
    assert iv.min() >= 0 and iv.max() + 2 * support < 1024


def test_fp64_oracle_close_to_fp32(orc):
    prob = PROBLEMS["g2"]
    vis = normal_vis(prob.n_data(), VIS_SEED)
    r = orc.run_plain(oracle_config(orc, prob), vis=vis, want_f64=True)
    assert orc.rel_l2(r["grid"], r["grid64"]) < 1e-6
    assert orc.rel_l2(r["outdata"], r["outdata64"]) < 1e-6


def test_oracle_detects_planted_error(orc):
    """A mistake planted in the oracle's inputs (one offset moved by one cell) must be caught by
    the same comparisons the GPU tests use."""
    prob = PROBLEMS["g1"]
    cfg = oracle_config(orc, prob)
    r = orc.run_plain(cfg)
    iu = r["iu"].copy()
    iu[17] += 1
    grid = np.zeros_like(r["grid"])
    orc.grid_f32(r["data"], r["support"], r["C"], r["coff"], iu, r["iv"], grid, prob.g_size)
    assert orc.rel_l2(grid, r["grid"]) > 1e-3
