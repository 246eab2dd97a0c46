"""GPU parity: libtconvolve against the oracle and the reference's recorded outputs.

Bars (written here, used below):
  * set-up (u, v, w, iu, iv, cOffset): bit-exact (sha256 of the reference's output);
  * table C: bit-exact expected; at most 1 in 2^20 entries may differ, by at most 1 ulp
    (the FP64 cos/exp of CUDA and glibc may round a value differently near a float boundary);
  * grid and degridded samples, plain FP32 form: relative L2 <= 1e-5 against the reference
    (REL_L2_FP32), the parity bar of the path; the measured error is ~1e-7 (FP32 summation order).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import REL_L2_FP32, VIS_SEED, oracle_config, sha
from tconvolve.workload import PROBLEMS, normal_vis

pytestmark = pytest.mark.gpu


KERNELS = ["paired", "tma", "direct-tiles", "direct-anchor"]


def _use(b, kernels):
    """Select the kernel family: TMA pipeline, or direct with the tiles/anchor degridding kernel."""
    path, _, variant = kernels.partition("-")
    b.set_path(path)
    return variant


def _after_init(b, variant):
    if variant:
        b.set_degrid_variant(variant)


def _table_close(gpu_c, ref_c):
    a = gpu_c.view(np.float32)
    b = ref_c.view(np.float32)
    diff = np.nonzero(a.view(np.uint32) != b.view(np.uint32))[0]
    assert diff.size <= max(1, a.size >> 20), f"{diff.size} table entries differ"
    if diff.size:
        ulps = np.abs(a[diff].view(np.int32).astype(np.int64) - b[diff].view(np.int32).astype(np.int64))
        assert ulps.max() <= 1
    return diff.size


@pytest.mark.parametrize("kernels", KERNELS)
@pytest.mark.parametrize("cfg", ["g1", "g2", "c1"])
@pytest.mark.parametrize("vis_kind", ["ones", "normal"])
def test_benchmark_parity(tcv, orc, golden, cuda_ok, cfg, vis_kind, kernels):
    prob = PROBLEMS[cfg]
    ref = golden["runs"][f"{cfg}_{vis_kind}"]
    b = tcv.Benchmark(**prob.kwargs())
    variant = _use(b, kernels)
    b.init()
    _after_init(b, variant)
    if vis_kind == "normal":
        b.set_data(normal_vis(prob.n_data(), VIS_SEED))
    b.runGrid()
    b.runDegrid()
    b.sync()
    assert b.getSupport() == ref["meta"]["support"]
    assert b.wCellSize == ref["meta"]["wCellSize"]
    u, v, w = b.uvw()
    for name, arr in (("u", u), ("v", v), ("w", w)):
        assert sha(arr) == ref["sha256"][name], name
    iu, iv, co = b.offsets()
    for name, arr in (("iu", iu), ("iv", iv), ("coff", co)):
        assert sha(arr) == ref["sha256"][name], name
    r = orc.run_plain(oracle_config(orc, prob),
                      vis=None if vis_kind == "ones" else normal_vis(prob.n_data(), VIS_SEED), threads=8)
    assert sha(r["C"]) == ref["sha256"]["C"]
    _table_close(b.C(), r["C"])
    assert b.sumC == r["sum_c"]
    grid = b.grid()
    out = b.outdata()
    assert orc.rel_l2(grid, r["grid"]) <= REL_L2_FP32
    assert orc.rel_l2(out, r["outdata"]) <= REL_L2_FP32
    # the footprint is exactly the reference's: no grid point outside it was written
    assert np.count_nonzero(grid) == ref["grid_nonzero"]
    b.close()


@pytest.mark.parametrize("kernels", KERNELS)
def test_default_config_full_size(tcv, orc, golden, cuda_ok, kernels):
    """The reference default (160 k samples, 4096^2 grid, 129^2 footprints) at full size."""
    prob = PROBLEMS["c2"]
    ref = golden["runs"]["c2_normal"]
    b = tcv.Benchmark(**prob.kwargs())
    variant = _use(b, kernels)
    b.init()
    _after_init(b, variant)
    vis = normal_vis(prob.n_data(), VIS_SEED)
    b.set_data(vis)
    b.runGrid()
    b.runDegrid()
    b.sync()
    iu, iv, co = b.offsets()
    assert sha(iu) == ref["sha256"]["iu"] and sha(iv) == ref["sha256"]["iv"]
    assert sha(co) == ref["sha256"]["coff"]
    c = b.C()
    cfg = oracle_config(orc, prob)
    if sha(c) == ref["sha256"]["C"]:
        c_ref = c  # bit-identical to the reference's table: reuse it
    else:
        c_ref = orc.init_c(cfg)[0]
        _table_close(c, c_ref)
    assert b.sumC == 16777216.0
    grid_ref = np.zeros(prob.g_size * prob.g_size, np.complex64)
    orc.grid_f32(vis, b.getSupport(), c_ref, co, iu, iv, grid_ref, prob.g_size, threads=16)
    assert sha(grid_ref) == ref["sha256"]["grid"]
    out_ref = orc.degrid_f32(grid_ref, prob.g_size, b.getSupport(), c_ref, co, iu, iv, threads=16)
    assert sha(out_ref) == ref["sha256"]["outdata"]
    assert orc.rel_l2(b.grid(), grid_ref) <= REL_L2_FP32
    assert orc.rel_l2(b.outdata(), out_ref) <= REL_L2_FP32


def test_full_size_properties(tcv, cuda_ok):
    """Size-independent properties at the reference default size: determinism (bit-identical
    reruns), accumulation (two passes = 2 x one pass), linearity in the visibilities, and the
    adjoint identity <grid(x), g> == <x, degrid(g)> that ties the two kernels together."""
    prob = PROBLEMS["c2"]
    b = tcv.Benchmark(**prob.kwargs())
    b.init()
    x = normal_vis(prob.n_data(), 11)
    y = normal_vis(prob.n_data(), 12)
    b.set_data(x)
    b.runGrid()
    g1 = b.grid()
    b.zero_grid()
    b.runGrid()
    assert np.array_equal(b.grid(), g1)
    b.runGrid()
    g2 = b.grid()
    assert np.linalg.norm(g2 - 2 * g1) <= 1e-6 * np.linalg.norm(2 * g1)
    b.zero_grid()
    b.set_data(y)
    b.runGrid()
    gy = b.grid()
    b.zero_grid()
    b.set_data((2.5 * x + y).astype(np.complex64))
    b.runGrid()
    gl = b.grid()
    lin = (2.5 * g1.astype(np.complex128) + gy)
    assert np.linalg.norm(gl - lin) <= 1e-6 * np.linalg.norm(lin)
    # adjoint: degridding with the same table is the transpose of gridding (C real)
    b.set_grid(gy)
    b.runDegrid()
    dg = b.outdata().astype(np.complex128)
    # sum_p conj(gy_p) grid(x)_p == sum_k conj(degrid(gy)_k) x_k for a real table
    lhs = np.vdot(gy.astype(np.complex128), g1.astype(np.complex128))
    rhs = np.vdot(dg, x.astype(np.complex128))
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)
    b.runDegrid()
    assert np.array_equal(b.outdata(), dg.astype(np.complex64))


@pytest.mark.parametrize("kernels", KERNELS)
@pytest.mark.parametrize("form,bound", [("r32", 0.0), ("cbf16", 6e-3), ("rbf16", 6e-3),
                                         ("cf16", 8e-4), ("rf16", 8e-4)])
def test_reduced_table_forms(tcv, orc, cuda_ok, form, bound, kernels):
    """Table storage forms against the FP64 oracle.  r32 must equal the complex64 form bit for
    bit (the attic table is real); the 16-bit forms stay within the stated relative L2."""
    prob = PROBLEMS["c1"]
    vis = normal_vis(prob.n_data(), VIS_SEED)
    b = tcv.Benchmark(**prob.kwargs())
    variant = _use(b, kernels)
    b.init()
    _after_init(b, variant)
    b.set_data(vis)
    b.runGrid()
    b.runDegrid()
    g_plain, o_plain = b.grid(), b.outdata()
    b.set_ctype(form)
    b.zero_grid()
    b.runGrid()
    b.runDegrid()
    g, o = b.grid(), b.outdata()
    r = orc.run_plain(oracle_config(orc, prob), vis=vis, threads=8, want_f64=True)
    e_grid = orc.rel_l2(g, r["grid64"])
    e_out = orc.rel_l2(o, r["outdata64"])
    if form == "r32":
        assert np.array_equal(g, g_plain) and np.array_equal(o, o_plain)
    else:
        assert e_grid <= bound and e_out <= bound, (e_grid, e_out)
        assert e_grid > 1e-6  # it really used the reduced table


def test_table_form_rejects_complex_for_real(tcv, cuda_ok):
    import torch

    from tconvolve import raw

    c = torch.zeros(1000, dtype=torch.complex64, device="cuda")
    c.imag[5] = 1.0
    out, scale, nz = raw.convert_c(c, tcv.CBF16)
    assert nz == 1 and scale == 1.0


# ---------------------------------------------------------------------------------------------
# raw entry points (torch tensors through the C ABI) and edge cases
# ---------------------------------------------------------------------------------------------
def _setup(orc, prob):
    cfg = oracle_config(orc, prob)
    u, v, w = orc.init_uvw(cfg)
    c, c64, support, os_, wcs, _ = orc.init_c(cfg, want_f64=False)
    iu, iv, co = orc.init_offsets(cfg, u, v, w, wcs, support, os_)
    return c, support, iu, iv, co


def _dev(*arrs):
    import torch

    return [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrs]


def test_raw_empty_input(tcv, orc, cuda_ok):
    import torch

    from tconvolve import raw

    prob = PROBLEMS["g1"]
    c, support, iu, iv, co = _setup(orc, prob)
    dc, = _dev(c)
    z = torch.zeros(0, dtype=torch.int32, device="cuda")
    data = torch.zeros(0, dtype=torch.complex64, device="cuda")
    grid = torch.zeros(prob.g_size ** 2, dtype=torch.complex64, device="cuda")
    plan = raw.Plan(z, z, z, support, prob.g_size, c.size)
    plan.grid(data, dc, tcv.C64, grid)
    plan.degrid(grid, dc, tcv.C64, data)
    torch.cuda.synchronize()
    assert plan.rejected() == 0
    assert int(torch.count_nonzero(grid)) == 0


def test_raw_out_of_bounds_samples_are_rejected(tcv, orc, cuda_ok):
    import torch

    from tconvolve import raw

    prob = PROBLEMS["g2"]
    c, support, iu, iv, co = _setup(orc, prob)
    n = iu.size
    iu2, iv2, co2 = iu.copy(), iv.copy(), co.copy()
    bad = np.array([3, 50, 51, 777, n - 1])
    iu2[3] = support - 1                 # left edge one column out
    iu2[50] = prob.g_size - support      # right edge one column out
    iv2[51] = prob.g_size - 2 * support  # bottom edge one row out
    co2[777] = c.size - (2 * support + 1) ** 2 + 1  # table range overruns by one entry
    iv2[n - 1] = -1
    vis = normal_vis(n, 3)
    dvis, dc, diu, div, dco = _dev(vis, c, iu2, iv2, co2)
    grid = torch.zeros(prob.g_size ** 2, dtype=torch.complex64, device="cuda")
    plan = raw.Plan(diu, div, dco, support, prob.g_size, c.size)
    plan.grid(dvis, dc, tcv.C64, grid)
    out = torch.full((n,), 7 + 7j, dtype=torch.complex64, device="cuda")
    plan.degrid(grid, dc, tcv.C64, out)
    out_anchor = torch.full((n,), 7 + 7j, dtype=torch.complex64, device="cuda")
    plan.set_degrid_variant(1)
    plan.degrid(grid, dc, tcv.C64, out_anchor)
    torch.cuda.synchronize()
    assert plan.rejected() == bad.size
    assert np.all(out_anchor.cpu().numpy()[bad] == 0)
    assert orc.rel_l2(out_anchor.cpu().numpy(), out.cpu().numpy()) <= 1e-6
    keep = np.ones(n, bool)
    keep[bad] = False
    ref = np.zeros(prob.g_size ** 2, np.complex64)
    orc.grid_f32(vis[keep], support, c, co2[keep], iu2[keep], iv2[keep], ref, prob.g_size)
    assert orc.rel_l2(grid.cpu().numpy(), ref) <= REL_L2_FP32
    o = out.cpu().numpy()
    assert np.all(o[bad] == 0)
    ref_o = orc.degrid_f32(ref, prob.g_size, support, c, co2[keep], iu2[keep], iv2[keep])
    assert orc.rel_l2(o[keep], ref_o) <= REL_L2_FP32


def test_anchor_binning_made_when_needed(tcv, orc, cuda_ok):
    """A plan binned for the tile kernels has no anchor binning; the first anchor degridding makes
    it, and it follows new samples binned by a replayed graph."""
    import torch

    from tconvolve import raw
    from tconvolve._lib import PASS_BIN

    prob = PROBLEMS["g2"]
    c, support, iu, iv, co = _setup(orc, prob)
    g = prob.g_size
    vis = normal_vis(iu.size, 21)
    dvis, dc, diu, div, dco = _dev(vis, c, iu, iv, co)
    grid = torch.zeros(g * g, dtype=torch.complex64, device="cuda")
    plan = raw.Plan(diu, div, dco, support, g, c.size)
    plan.grid(dvis, dc, tcv.C64, grid)
    h_grid = grid.cpu().numpy()
    ref = orc.degrid_f32(h_grid, g, support, c, co, iu, iv)
    out_t = torch.empty(iu.size, dtype=torch.complex64, device="cuda")
    plan.degrid(grid, dc, tcv.C64, out_t)
    plan.set_degrid_variant(1)
    out_a = torch.empty_like(out_t)
    plan.degrid(grid, dc, tcv.C64, out_a)
    assert orc.rel_l2(out_t.cpu().numpy(), ref) <= REL_L2_FP32
    assert orc.rel_l2(out_a.cpu().numpy(), ref) <= REL_L2_FP32
    # a binning captured with the tile kernels' variant, replayed on other samples in the same
    # buffers (the reversed order of a different subset)
    plan.set_degrid_variant(0)
    graph = plan.capture(PASS_BIN, dvis, dc, tcv.C64, grid)
    sel = np.arange(iu.size)[::-1][: iu.size // 2].copy()
    iu2, iv2, co2 = (np.concatenate([a[sel], a[sel]]) for a in (iu, iv, co))
    for d, h in ((diu, iu2), (div, iv2), (dco, co2)):
        d.copy_(torch.from_numpy(h))
    graph.launch()
    plan.set_degrid_variant(1)
    plan.degrid(grid, dc, tcv.C64, out_a)
    ref2 = orc.degrid_f32(h_grid, g, support, c, co2, iu2, iv2)
    assert orc.rel_l2(out_a.cpu().numpy(), ref2) <= REL_L2_FP32
    plan.set_degrid_variant(0)
    plan.degrid(grid, dc, tcv.C64, out_t)
    assert orc.rel_l2(out_t.cpu().numpy(), ref2) <= REL_L2_FP32
    graph.close()


def test_raw_extreme_positions_and_collisions(tcv, orc, cuda_ok):
    """Footprints touching all four grid edges, and 3000 samples piled on one position (one tile
    list far longer than a staging chunk)."""
    import torch

    from tconvolve import raw

    prob = PROBLEMS["g1"]
    c, support, _, _, _ = _setup(orc, prob)
    s = 2 * support + 1
    g = prob.g_size
    rng = np.random.default_rng(5)
    corners_u = np.array([support, g - 1 - support, support, g - 1 - support], np.int32)
    corners_v = np.array([0, 0, g - s, g - s], np.int32)
    m = 3000
    iu = np.concatenate([corners_u, np.full(m, 61, np.int32)])
    iv = np.concatenate([corners_v, np.full(m, 40, np.int32)])
    nk = c.size // (s * s)
    co = (rng.integers(0, nk, iu.size) * s * s).astype(np.int32)
    vis = normal_vis(iu.size, 9)
    dvis, dc, diu, div, dco = _dev(vis, c, iu, iv, co)
    grid = torch.zeros(g * g, dtype=torch.complex64, device="cuda")
    raw.grid_raw(dvis, support, dc, tcv.C64, 1.0, dco, diu, div, grid, g)
    out = torch.empty(iu.size, dtype=torch.complex64, device="cuda")
    raw.degrid_raw(grid, g, support, dc, tcv.C64, 1.0, dco, diu, div, out)
    torch.cuda.synchronize()
    ref = np.zeros(g * g, np.complex64)
    orc.grid_f32(vis, support, c, co, iu, iv, ref, g)
    assert orc.rel_l2(grid.cpu().numpy(), ref) <= REL_L2_FP32
    ref_o = orc.degrid_f32(ref, g, support, c, co, iu, iv)
    assert orc.rel_l2(out.cpu().numpy(), ref_o) <= REL_L2_FP32


@pytest.mark.parametrize("g_size,cell,w_size", [(1023, 40.286094970136006, 5), (4096, 3.0, 3)])
def test_direct_degrid_path(tcv, orc, cuda_ok, g_size, cell, w_size):
    """Shapes the staged kernel does not take: an odd grid size (no TMA row pitch) and a
    167-wide footprint (too wide to stage); the direct kernel must give the same answers."""
    from tconvolve.workload import Problem

    prob = Problem("direct", 3000, w_size, 1, g_size, cell)
    b = tcv.Benchmark(**prob.kwargs())
    b.set_path("direct")
    b.init()
    b.set_degrid_variant("anchor")
    vis = normal_vis(prob.n_data(), 4)
    b.set_data(vis)
    b.runGrid()
    b.runDegrid()
    b.sync()
    assert b.plan_info()["degrid_mode"] == 1
    r = orc.run_plain(oracle_config(orc, prob), vis=vis, threads=8)
    assert orc.rel_l2(b.grid(), r["grid"]) <= REL_L2_FP32
    assert orc.rel_l2(b.outdata(), r["outdata"]) <= REL_L2_FP32


@pytest.mark.parametrize("layout", ["padded", "paired"])
@pytest.mark.parametrize("form", ["c64", "r32", "rbf16", "cf16"])
def test_raw_prepared_table(tcv, orc, cuda_ok, form, layout):
    """Prepared tables through the raw entry points: a table prepared by tcv_prepare_table, passed
    with its layout flag (TMA pipeline or paired tile kernels), gives the same grid and samples
    as the reference-layout kernels."""
    import ctypes

    import torch

    from tconvolve import raw
    from tconvolve._lib import PADDED, PAIRED, check, lib

    FLAG = PADDED if layout == "padded" else PAIRED
    prob = PROBLEMS["c1"]
    c, support, iu, iv, co = _setup(orc, prob)
    vis = normal_vis(iu.size, 31)
    dvis, dc, diu, div, dco = _dev(vis, c, iu, iv, co)
    t = tcv.CTYPE_BY_NAME[form]
    nbytes = lib().tcv_table_bytes(c.size, support, t | FLAG)
    assert nbytes > 0
    padded = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
    scale, nz = ctypes.c_float(), ctypes.c_int64()
    check(lib().tcv_prepare_table(ctypes.c_void_p(dc.data_ptr()), c.size, support, t | FLAG,
                                  ctypes.c_void_p(padded.data_ptr()), ctypes.byref(scale),
                                  ctypes.byref(nz), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)),
          "prepare")
    assert nz.value == 0
    if form == "c64":
        flat, fscale = dc, 1.0
    else:
        flat, fscale, _ = raw.convert_c(dc, t)
    plan = raw.Plan(diu, div, dco, support, prob.g_size, c.size)
    g_tma = torch.zeros(prob.g_size ** 2, dtype=torch.complex64, device="cuda")
    g_dir = torch.zeros_like(g_tma)
    plan.grid(dvis, padded, t | FLAG, g_tma, c_scale=scale.value)
    plan.grid(dvis, flat, t, g_dir, c_scale=fscale)
    o_tma = torch.empty_like(dvis)
    o_dir = torch.empty_like(dvis)
    plan.degrid(g_dir, padded, t | FLAG, o_tma, c_scale=scale.value)
    plan.degrid(g_dir, flat, t, o_dir, c_scale=fscale)
    torch.cuda.synchronize()
    assert plan.status() == 0
    a, b = g_tma.cpu().numpy(), g_dir.cpu().numpy()
    assert orc.rel_l2(a, b) <= 1e-6
    assert orc.rel_l2(o_tma.cpu().numpy(), o_dir.cpu().numpy()) <= 1e-6
    if form == "c64":
        ref = np.zeros(prob.g_size ** 2, np.complex64)
        orc.grid_f32(vis, support, c, co, iu, iv, ref, prob.g_size)
        assert orc.rel_l2(a, ref) <= REL_L2_FP32


def test_plan_reuse_and_streams(tcv, orc, cuda_ok):
    """One plan serves repeated passes on a caller's stream; results equal a fresh one-call run."""
    import torch

    from tconvolve import raw

    prob = PROBLEMS["g2"]
    c, support, iu, iv, co = _setup(orc, prob)
    vis = normal_vis(iu.size, 21)
    dvis, dc, diu, div, dco = _dev(vis, c, iu, iv, co)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        plan = raw.Plan(diu, div, dco, support, prob.g_size, c.size, stream=s)
        g_a = torch.zeros(prob.g_size ** 2, dtype=torch.complex64, device="cuda")
        for _ in range(3):
            plan.grid(dvis, dc, tcv.C64, g_a, stream=s)
    s.synchronize()
    g_b = torch.zeros_like(g_a)
    raw.grid_raw(dvis, support, dc, tcv.C64, 1.0, dco, diu, div, g_b, prob.g_size)
    torch.cuda.synchronize()
    a = g_a.cpu().numpy()
    bb = g_b.cpu().numpy()
    assert np.linalg.norm(a - 3 * bb) <= 1e-6 * np.linalg.norm(3 * bb)
    assert plan.status() == 0


def test_device_setup_functions(tcv, orc, cuda_ok):
    """initC, the generator and initCOffset through the raw entry points."""
    import torch

    from tconvolve import raw

    prob = PROBLEMS["g2"]
    cfg = oracle_config(orc, prob)
    c_gpu, sum_c = raw.init_c(prob.freq0, prob.cell_size, prob.baseline, prob.w_size)
    c_ref, _, support, os_, wcs, sum_ref = orc.init_c(cfg)
    assert sum_c == sum_ref
    _table_close(c_gpu.cpu().numpy(), c_ref)
    u, v, w = raw.init_uvw(prob.n_samples, prob.baseline, prob.seed + 1)
    u_ref, v_ref, w_ref = orc.init_uvw(cfg)
    assert np.array_equal(u.cpu().numpy(), u_ref) and np.array_equal(w.cpu().numpy(), w_ref)
    freq = torch.from_numpy(orc.init_freq(cfg)).cuda()
    iu, iv, co = raw.init_offsets(u, v, w, freq, prob.cell_size, wcs, prob.w_size, prob.g_size,
                                  support, os_)
    iu_r, iv_r, co_r = orc.init_offsets(cfg, u_ref, v_ref, w_ref, wcs, support, os_)
    assert np.array_equal(iu.cpu().numpy(), iu_r)
    assert np.array_equal(iv.cpu().numpy(), iv_r)
    assert np.array_equal(co.cpu().numpy(), co_r)


@pytest.mark.parametrize("form", ["c64", "r32"])
def test_specialised_tile_kernels_match_generic(tcv, orc, cuda_ok, form):
    """The tile kernels compiled at run time with the footprint width as a constant give the same
    results as the generic copies (and are really in use on the device)."""
    prob = PROBLEMS["c1"]
    vis = normal_vis(prob.n_data(), VIS_SEED)
    out = {}
    try:
        for jit in (True, False):
            tcv.jit_enable(jit)
            b = tcv.Benchmark(**prob.kwargs())
            b.set_path("direct")
            b.init()
            b.set_ctype(form)
            b.set_data(vis)
            b.runGrid()
            b.runDegrid()
            b.sync()
            out[jit] = (b.grid(), b.outdata())
            if jit:
                assert "specialised tile kernels in use" in tcv.jit_info(), tcv.jit_info()
            b.close()
    finally:
        tcv.jit_enable(True)
    assert orc.rel_l2(out[True][0], out[False][0]) <= 1e-6
    assert orc.rel_l2(out[True][1], out[False][1]) <= 1e-6
    r = orc.run_plain(oracle_config(orc, prob), vis=vis, threads=8)
    assert orc.rel_l2(out[True][0], r["grid"]) <= REL_L2_FP32
    assert orc.rel_l2(out[True][1], r["outdata"]) <= REL_L2_FP32
