"""GPU parity of the variable-support path (current/tConvolveMPI) against the oracle and the
reference's recorded outputs.

Bars (written here, used below):
  * offsets (iu, iv, w-plane, cOffset), plane widths and plane offsets: bit-exact (sha256 of the
    reference's output);
  * u, v, w: within 4 ulp (relative 1e-15) of the reference: they pass through the device's
    double cos/sin of the hour angle, which may differ from the host libm in the last bit;
  * the table C: bit-exact but for last-bit differences where the device's exp and the double
    sin/cos rounded to float differ from the host libm's float sinf/cosf, and the per-plane
    normalisation sum carries them (measured: at most 0.1% of the words, at most 4 ulp; bound
    0.5% and 4 ulp);
  * grid and degridded samples, plain complex64 form, cells whole: relative L2 <= 1e-5
    (REL_L2_FP32) against the oracle (the reference's arithmetic and order, pinned bit-exact);
  * with busy cells split into work units, or with the sample-parallel kernels (which sum each
    point per warp, then the warps in order), the FP32 sums are grouped differently; the reference's
    own FP32 grid is then the yardstick: the relative L2 distance of our grid from the FP64 grid
    at most 1.5 x the reference's (both ~8e-6 on the spectral problem with unit data, where
    thousands of samples pile on each point), and degridding within 1e-6 of the FP64 degridding
    of the same grid (measured 5e-8; the reference's own is 1.3e-7);
  * bfloat16 / float16 tables: 6e-3 / 8e-4 against the same.
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR, REL_L2_FP32, sha

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cur_golden():
    with open(os.path.join(GOLDEN_DIR, "current.json")) as f:
        return json.load(f)["runs"]


def _table_close(gpu_c, ref_c):
    a, b = gpu_c.view(np.float32), ref_c.view(np.float32)
    diff = np.nonzero(a.view(np.uint32) != b.view(np.uint32))[0]
    ulps = np.abs(a[diff].view(np.int32).astype(np.int64) - b[diff].view(np.int32).astype(np.int64))
    print(f"table: {diff.size} of {a.size} words differ, max {ulps.max() if diff.size else 0} ulp")
    assert diff.size <= max(2, a.size // 200), f"{diff.size} table words differ"
    assert diff.size == 0 or ulps.max() <= 4


def _oracle_run(orc, run_type, iu, iv, wp, co, vis=None, threads=16):
    g = orc.cur_geometry(run_type)
    c, s_size, off0 = orc.cur_init_c(run_type)
    data = np.ones(iu.size, np.complex64) if vis is None else vis
    grid = np.zeros(g.g_size * g.g_size, np.complex64)
    orc.cur_grid_f32(data, iu, iv, wp, co, s_size, c, grid, g.g_size, threads=threads)
    out = orc.cur_degrid_f32(grid, g.g_size, iu, iv, wp, co, s_size, c, threads=threads)
    return c, grid, out


def _setup_checks(b, ref):
    u, v, w = b.uvw()
    iu, iv, wp, co = b.offsets()
    s_size, off0 = b.planes()
    for name, arr in (("iu", iu), ("iv", iv), ("wplane", wp), ("coff", co), ("ssize", s_size), ("coff0", off0)):
        assert sha(arr) == ref["sha256"][name], name
    assert b.nVisibilitiesGridded() == ref["meta"]["nSamples"]
    assert b.nPixelsGridded() == ref["meta"]["nPixelsGridded"]
    assert b.generator_state == ref["meta"]["next"]
    return u, v, w, iu, iv, wp, co


@pytest.mark.parametrize("run_type", [1, 2, 3, 0])
def test_current_parity(tcv, orc, cur_golden, cuda_ok, run_type):
    from tconvolve.current import Benchmark

    ref = cur_golden[f"rt{run_type}"]
    b = Benchmark()
    b.setSort(0)
    b.setRunType(run_type)
    b.init()
    assert b.getSupport() == ref["meta"]["support"]
    b.runGrid()
    b.runDegrid()
    b.sync()
    u, v, w, iu, iv, wp, co = _setup_checks(b, ref)
    ou, ov, ow, _ = orc.cur_init_uvw(run_type, 1)
    for a, r in ((u, ou), (v, ov), (w, ow)):
        assert np.allclose(a, r, rtol=1e-15, atol=1e-12)
    c_ref, grid_ref, out_ref = _oracle_run(orc, run_type, iu, iv, wp, co)
    assert sha(c_ref) == ref["sha256"]["C"]
    _table_close(b.C(), c_ref)
    assert orc.rel_l2(b.grid(), grid_ref) <= REL_L2_FP32
    assert orc.rel_l2(b.outdata(), out_ref) <= REL_L2_FP32
    # the footprints are the reference's: no grid point outside them was written
    assert np.count_nonzero(b.grid()) == ref["grid_nonzero"]
    b.close()


def test_current_run_sequence_and_sort(tcv, orc, cur_golden, cuda_ok):
    """tConvolveMPI's order (continuum, then spectral on the same object: the generator carries
    over), and setSort(1)."""
    from tconvolve.current import Benchmark

    b = Benchmark()
    b.setRunType(0)
    b.init()
    assert b.generator_state == cur_golden["rt0"]["meta"]["next"]
    b.setRunType(1)
    b.init()
    _setup_checks(b, cur_golden["rt1_after_rt0"])
    b.close()
    b = Benchmark()
    b.setSort(1)
    b.setRunType(1)
    b.init()
    b.runGrid()
    b.runDegrid()
    b.sync()
    _, _, _, iu, iv, wp, co = _setup_checks(b, cur_golden["rt1_sorted"])
    _, grid_ref, out_ref = _oracle_run(orc, 1, iu, iv, wp, co)
    assert orc.rel_l2(b.grid(), grid_ref) <= REL_L2_FP32
    assert orc.rel_l2(b.outdata(), out_ref) <= REL_L2_FP32
    b.close()


@pytest.mark.parametrize("tuning", [None, (8, 32, 256, 128, 3)], ids=["tile", "sample-parallel"])
def test_current_wide_kernels_subset(tcv, orc, cur_golden, cuda_ok, tuning):
    """87 x 87 kernels (4.1e10 updates per pass at full size): the full set-up against the
    reference, gridding and degridding of the first 150 k samples against the oracle, with the
    tile kernels and with the sample-parallel ones (87-wide rectangles: 32-column strips in
    degridding, tall steps of one row in each gridding half)."""
    import torch

    from tconvolve import raw
    from tconvolve.current import Benchmark

    b = Benchmark()
    b.setRunType(4)
    b.init()
    _, _, _, iu, iv, wp, co = _setup_checks(b, cur_golden["rt4"])
    c = b.C()
    s_size, off0 = b.planes()
    g = b.geometry()
    m = 150_000
    rng = np.random.default_rng(4)
    vis = (rng.standard_normal(m, dtype=np.float32) + 1j * rng.standard_normal(m, dtype=np.float32)).astype(np.complex64)
    d = {k: torch.from_numpy(np.ascontiguousarray(a[:m])).cuda() for k, a in (("iu", iu), ("iv", iv), ("wp", wp), ("co", co))}
    dc = torch.from_numpy(c).cuda()
    dv = torch.from_numpy(vis).cuda()
    grid = torch.zeros(g.g_size * g.g_size, dtype=torch.complex64, device="cuda")
    out = torch.empty(m, dtype=torch.complex64, device="cuda")
    plan = raw.VarPlan(d["iu"], d["iv"], d["co"], d["wp"], s_size, off0, g.g_size, c.size, tuning=tuning)
    plan.grid(dv, dc, tcv.C64, grid)
    plan.degrid(grid, dc, tcv.C64, out)
    torch.cuda.synchronize()
    ref = np.zeros(g.g_size * g.g_size, np.complex64)
    orc.cur_grid_f32(vis, iu[:m], iv[:m], wp[:m], co[:m], s_size, c, ref, g.g_size, threads=16)
    assert orc.rel_l2(grid.cpu().numpy(), ref) <= REL_L2_FP32
    ref_o = orc.cur_degrid_f32(ref, g.g_size, iu[:m], iv[:m], wp[:m], co[:m], s_size, c, threads=16)
    assert orc.rel_l2(out.cpu().numpy(), ref_o) <= REL_L2_FP32
    b.close()


@pytest.mark.parametrize("tuning", [None, (32, 512, 256, 8, 3)], ids=["tile", "sample-parallel"])
@pytest.mark.parametrize("form,bound", [("cbf16", 6e-3), ("cf16", 8e-4)])
def test_current_reduced_forms(tcv, orc, cuda_ok, form, bound, tuning):
    from tconvolve.current import Benchmark

    b = Benchmark()
    b.setRunType(1)
    if tuning:
        b.set_tuning(*tuning)
    b.init()
    iu, iv, wp, co = b.offsets()
    rng = np.random.default_rng(11)
    n = b.nVisibilitiesGridded()
    vis = (rng.standard_normal(n, dtype=np.float32) + 1j * rng.standard_normal(n, dtype=np.float32)).astype(np.complex64)
    b.set_data(vis)
    b.set_ctype(form)
    b.runGrid()
    b.runDegrid()
    b.sync()
    _, grid_ref, out_ref = _oracle_run(orc, 1, iu, iv, wp, co, vis=vis)
    e_grid, e_out = orc.rel_l2(b.grid(), grid_ref), orc.rel_l2(b.outdata(), out_ref)
    assert e_grid <= bound and e_out <= bound, (e_grid, e_out)
    assert e_grid > 1e-6
    b.close()


def _check_tuned(b, orc):
    """Grid + degrid twice (bit-identical), then the bars of the module docstring for the plan's
    tuning: cells whole -> the reference's order; split cells -> against FP64."""
    iu, iv, wp, co = b.offsets()
    b.zero_grid()
    b.runGrid()
    b.runDegrid()
    b.sync()
    g1, o1 = b.grid(), b.outdata()
    b.zero_grid()
    b.runGrid()
    b.runDegrid()
    b.sync()
    assert np.array_equal(b.grid(), g1) and np.array_equal(b.outdata(), o1)
    c, grid_ref, out_ref = _oracle_run(orc, 1, iu, iv, wp, co)
    s_size, _ = b.planes()
    g = b.geometry()
    split = b.tuning()[2]
    ref_order = split == 0 and not (len(b.tuning()) > 4 and b.tuning()[4] & 1)  # tile gridding, cells whole
    if ref_order:  # gridding cells whole: the reference's order at every point
        assert orc.rel_l2(g1, grid_ref) <= REL_L2_FP32
    else:
        g64 = orc.cur_grid_f64(np.ones(iu.size, np.complex64), iu, iv, wp, co, s_size, c, g.g_size, threads=16)
        assert orc.rel_l2(g1, g64) <= 1.5 * orc.rel_l2(grid_ref, g64) + 1e-7
    o64 = orc.cur_degrid_f64(g1, g.g_size, iu, iv, wp, co, s_size, c, threads=16)
    assert orc.rel_l2(o1, o64) <= 1e-6
    if ref_order:
        assert orc.rel_l2(o1, out_ref) <= REL_L2_FP32


@pytest.mark.parametrize("tuning", [(32, 0, 0, 16), (8, 0, 64, 16), (8, 64, 64, 16), (-1, 256, 128, 16),
                                    (32, 0, 0, 8), (-1, 128, 64, 8), (32, 256, 8, 8),
                                    (32, 0, 0, 8, 3), (-1, 256, 128, 8, 3), (8, 64, 16, 8, 2), (32, 0, 0, 8, 1),
                                    (32, 16, 64, 8, 1), (32, 40, 64, 8, 3), (8, 64, 64, 8, 3)])
def test_current_tunings_and_determinism(tcv, orc, cuda_ok, tuning):
    """Plane groups, work units, tile heights and the sample-parallel kernels (fifth entry: 1
    gridding, 2 degridding, 3 both) change the summation order only: every tuning within its bar
    (module docstring; sample-parallel gridding groups each point's sum by warp, so it is held to
    the split-cell bar), each bit-identical when rerun.  Work units of 16 and 40 samples leave some
    sample-parallel gridding warps without samples and others with a partial group of 32; 8 MiB
    plane groups run the sample-parallel passes once per group on the same pair records."""
    from tconvolve.current import Benchmark

    b = Benchmark()
    b.setRunType(1)
    b.init()
    b.set_tuning(*tuning)
    assert b.tuning() == (tuning[3],) + tuning[:3] + tuning[4:]
    _check_tuned(b, orc)
    b.close()


def test_current_autotune(tcv, orc, cuda_ok):
    """tcv_cur_tune keeps the fastest of the candidates it timed, leaves the object's grid alone,
    and the tuned plan meets the bars of its tuning."""
    from tconvolve.current import Benchmark

    b = Benchmark()
    b.setRunType(1)
    b.init()
    b.runGrid()
    b.sync()
    before = b.grid()
    best, ms, report = b.tune(reps=2)
    assert np.array_equal(b.grid(), before), "the tuner wrote into the object's grid"
    assert best == b.tuning() and ms > 0
    assert len(report) >= 9 and best in [t for t, _ in report]
    assert ms == min(m for _, m in report)
    assert {t[0] for t, _ in report} == {8, 16}
    _check_tuned(b, orc)
    b.close()


def _reference_check(a: np.ndarray, b: np.ndarray):
    """runGridCheck / runDegridCheck (current/tConvolveACC/Benchmark.cc:324-364): every point's
    |a - b| / |a| <= 1e-4 (a point where a == 0 must be 0 in b too: the quotient is inf otherwise,
    and 0/0 passes as the reference's NaN comparison does), and the null test: both sums of
    absolute values positive.  Returns (passed, worst relative error over a != 0)."""
    a64, b64 = a.astype(np.complex128), b.astype(np.complex128)
    d = np.abs(a64 - b64)
    nz = np.abs(a64) > 0
    if np.any(~nz & (d > 0)):
        return False, np.inf
    rel = d[nz] / np.abs(a64[nz])
    worst = float(rel.max()) if rel.size else 0.0
    return worst <= 1e-4 and np.abs(a64).sum() > 0 and np.abs(b64).sum() > 0, worst


@pytest.mark.parametrize("tuning", [None, (32, 512, 256, 8, 3)], ids=["default", "sample-parallel"])
def test_current_reference_point_checks(tcv, orc, cuda_ok, tuning):
    """The reference's own GPU-port check on the spectral-line run: grid and degridded samples
    against the CPU result (the oracle, pinned to the reference), point by point."""
    from tconvolve.current import Benchmark

    b = Benchmark()
    b.setRunType(1)
    if tuning:
        b.set_tuning(*tuning)
    b.init()
    b.runGrid()
    b.runDegrid()
    b.sync()
    iu, iv, wp, co = b.offsets()
    _, grid_ref, out_ref = _oracle_run(orc, 1, iu, iv, wp, co)
    ok_g, worst_g = _reference_check(grid_ref, b.grid())
    ok_d, worst_d = _reference_check(out_ref, b.outdata())
    print(f"\nper-point relative error: grid {worst_g:.2e}, degridded {worst_d:.2e}")
    assert ok_g and ok_d, (worst_g, worst_d)
    b.close()
