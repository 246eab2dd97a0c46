"""Parity of the tuned plans at the reference default size (160 k samples, 4096^2 grid, 129^2
footprints, 33 w-planes): the plan shapes the autotuner picks for the timed workload, with the
real (r32) and complex64 (c64) tables, against the reference's FP32 result.

The reference result is the oracle's restatement of attic/tConvolveMPI/Benchmark.cc:125-195 run
here and pinned to the sha256 of the reference's own output (tests/golden/golden.json, c2_normal),
so every comparison below is against the reference's bits.

Bars (written here, used below):
  * grid and degridded samples: relative L2 <= 1e-5 (REL_L2_FP32) against the reference (the
    sample-parallel passes group each point's or sample's sum by warp: FP32 rounding only);
  * r32 and c64 with the same tuning: bit-identical (the attic table's imaginary parts are zero);
  * the same tuning run twice: bit-identical (no atomics; fixed summation order).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import REL_L2_FP32, VIS_SEED, oracle_config, sha
from tconvolve.workload import PROBLEMS, normal_vis

pytestmark = pytest.mark.gpu

# (tile rows, plane-group MiB, gridding work unit, degridding work unit[, sample-parallel passes]):
# the autotuner's pick for the timed r32 workload, the same with split gridding cells, a 64-sample
# gridding split, the whole table in one group, 8-row tiles with both passes split, and 8-row
# tiles with the sample-parallel degridding and with both passes sample-parallel
TUNINGS = [(16, 64, 0, 64), (16, 64, 256, 64), (16, 64, 64, 128), (16, -1, 0, 0), (8, 32, 512, 256),
           (8, 64, 0, 128, 2), (8, 64, 256, 128, 3)]


@pytest.fixture(scope="module")
def c2_reference(orc, golden):
    prob = PROBLEMS["c2"]
    ref = golden["runs"]["c2_normal"]
    cfg = oracle_config(orc, prob)
    vis = normal_vis(prob.n_data(), VIS_SEED)
    u, v, w = orc.init_uvw(cfg)
    c, _, support, os_, wcs, _ = orc.init_c(cfg)
    iu, iv, co = orc.init_offsets(cfg, u, v, w, wcs, support, os_)
    assert sha(c) == ref["sha256"]["C"] and sha(co) == ref["sha256"]["coff"]
    grid = np.zeros(prob.g_size * prob.g_size, np.complex64)
    orc.grid_f32(vis, support, c, co, iu, iv, grid, prob.g_size, threads=16)
    out = orc.degrid_f32(grid, prob.g_size, support, c, co, iu, iv, threads=16)
    assert sha(grid) == ref["sha256"]["grid"] and sha(out) == ref["sha256"]["outdata"]
    return vis, grid, out


@pytest.fixture(scope="module")
def c2_bench(tcv, cuda_ok):
    prob = PROBLEMS["c2"]
    b = tcv.Benchmark(**prob.kwargs())
    b.init()
    b.set_data(normal_vis(prob.n_data(), VIS_SEED))
    yield b
    b.close()


def _run(b, form, tuning):
    b.set_ctype(form)
    b.set_tuning(*tuning)
    b.zero_grid()
    b.runGrid()
    b.runDegrid()
    b.sync()
    return b.grid(), b.outdata()


@pytest.mark.parametrize("tuning", TUNINGS)
def test_tuned_plans_match_reference(c2_bench, c2_reference, orc, tuning):
    _, grid_ref, out_ref = c2_reference
    g32, o32 = _run(c2_bench, "r32", tuning)
    e_grid, e_out = orc.rel_l2(g32, grid_ref), orc.rel_l2(o32, out_ref)
    assert e_grid <= REL_L2_FP32 and e_out <= REL_L2_FP32, (tuning, e_grid, e_out)
    g64, o64 = _run(c2_bench, "c64", tuning)
    assert np.array_equal(g64, g32) and np.array_equal(o64, o32)
    g2, o2 = _run(c2_bench, "r32", tuning)
    assert np.array_equal(g2, g32) and np.array_equal(o2, o32)

