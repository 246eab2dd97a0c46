"""The variable-support oracle pinned against the reference (CPU only).

tconvolve_oracle_current.c restates current/tConvolveMPI/Benchmark.cc; these tests check its
outputs bit for bit (sha256) against the reference's own outputs recorded in
tests/golden/current.json (generator: tests/golden/make_golden_current.py).
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR, sha


@pytest.fixture(scope="module")
def cur_golden():
    with open(os.path.join(GOLDEN_DIR, "current.json")) as f:
        return json.load(f)["runs"]


def _check(orc, ref, run_type, state=1, sort=False, kernels=True):
    g = orc.cur_geometry(run_type)
    m = ref["meta"]
    assert (g.n_samples, g.w_size, g.g_size, g.over_sample, g.support) == \
        (m["nSamples"], m["wSize"], m["gSize"], m["overSample"], m["support"])
    assert g.w_cell_size == m["wCellSize"] and g.uv_cell_size == m["uvCellSize"]
    u, v, w, after = orc.cur_init_uvw(run_type, state)
    assert after == m["next"]  # the generator state the reference object ends in
    c, s_size, off0 = orc.cur_init_c(run_type)
    iu, iv, wp, co = orc.cur_init_offsets(run_type, u, v, w, s_size, off0)
    if sort:
        iu, iv, wp, co = orc.cur_sort_by_plane(g.w_size, iu, iv, wp, co)
    arrays = dict(u=u, v=v, w=w, iu=iu, iv=iv, wplane=wp, coff=co, ssize=s_size, coff0=off0, C=c)
    # nPixelsGridded (Benchmark.cc:679-694): sum of sSize^2 over the samples
    assert int((s_size[wp].astype(np.int64) ** 2).sum()) == m["nPixelsGridded"]
    if kernels:
        grid = np.zeros(g.g_size * g.g_size, np.complex64)
        orc.cur_grid_f32(np.ones(iu.size, np.complex64), iu, iv, wp, co, s_size, c, grid, g.g_size, threads=8)
        arrays["grid"] = grid
        arrays["outdata"] = orc.cur_degrid_f32(grid, g.g_size, iu, iv, wp, co, s_size, c, threads=8)
    for key, a in arrays.items():
        assert sha(a) == ref["sha256"][key], f"run type {run_type}: {key} differs from the reference"


@pytest.mark.parametrize("name,run_type", [("rt1", 1), ("rt2", 2), ("rt3", 3), ("rt0", 0)])
def test_current_oracle_bit_exact(orc, cur_golden, name, run_type):
    _check(orc, cur_golden[name], run_type)


def test_current_oracle_wide_kernel_setup(orc, cur_golden):
    """87 x 87 kernels: set-up bit-exact (gridding, 4.1e10 updates per pass, is left to the GPU
    tests, which compare a subset against this oracle)."""
    _check(orc, cur_golden["rt4"], 4, kernels=False)


def test_current_oracle_run_sequence(orc, cur_golden):
    """tConvolveMPI runs the continuum type and then the spectral type on one object: the
    spectral samples continue the generator where the continuum samples left it."""
    _, _, _, state = orc.cur_init_uvw(0, 1)
    assert state == cur_golden["rt0"]["meta"]["next"]
    _check(orc, cur_golden["rt1_after_rt0"], 1, state=state)


def test_current_oracle_sorted(orc, cur_golden):
    """setSort(1): offsets ordered by w-plane (stable), data untouched."""
    _check(orc, cur_golden["rt1_sorted"], 1, sort=True)


def test_current_known_answers(orc):
    """Values the reference prints for its two tests (current/tConvolveMPI/Benchmark.cc:142-150,
    542-572): grid sizes, support, number of planes, kernel widths."""
    g0, g1 = orc.cur_geometry(0), orc.cur_geometry(1)
    assert (g0.g_size, g0.support, g0.w_size, g0.s_max, g0.over_sample) == (6440, 60, 483, 121, 4)
    assert (g1.g_size, g1.support, g1.w_size, g1.s_max, g1.over_sample) == (1034, 9, 135, 19, 8)
    _, s_size, _ = orc.cur_init_c(1)
    assert s_size.min() == 7 and s_size.max() == 19 and np.all(s_size % 2 == 1)
