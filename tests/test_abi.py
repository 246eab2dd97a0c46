"""The C ABI boundary, checked without a GPU: the library loads, exports every function that
include/tconvolve.h declares, the binding's table matches the header, host-only functions give
the reference's known answers, and calls that need a device fail loudly when there is none."""
from __future__ import annotations

import ctypes
import os
import re
import subprocess

import pytest

from conftest import REPO
from tconvolve.workload import PROBLEMS

HEADER = os.path.join(REPO, "include", "tconvolve.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tcv_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(tcv):
    from tconvolve._lib import LIB_PATH

    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], check=True, capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r" T (tcv_\w+)", out))
    declared = header_functions()
    assert len(declared) >= 50
    missing = [f for f in declared if f not in exported]
    assert not missing, f"declared but not exported: {missing}"


def test_probe_library_exports_its_header(tcv):
    """The L2 table-stream probe is a measurement tool in a library of its own (libtcvprobe.so,
    include/tcv_probe.h); libtconvolve.so does not export it."""
    from tconvolve._lib import LIB_PATH, PROBE_LIB_PATH, PROBE_SIGNATURES

    text = re.sub(r"/\*.*?\*/", "", open(os.path.join(REPO, "include", "tcv_probe.h")).read(), flags=re.S)
    declared = sorted(set(re.findall(r"\b(tcv_[a-z0-9_]+)\s*\(", text)))
    assert declared == sorted(PROBE_SIGNATURES)
    out = subprocess.run(["nm", "-D", "--defined-only", PROBE_LIB_PATH], check=True, capture_output=True,
                         text=True).stdout
    assert all(f" T {f}" in out for f in declared)
    main = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], check=True, capture_output=True, text=True).stdout
    assert "tcv_probe" not in main


def test_binding_covers_header(tcv):
    from tconvolve._lib import SIGNATURES

    assert sorted(SIGNATURES) == header_functions()


def test_cuda_gridder_shim_exports_reference_symbols(tcv):
    lib = os.path.join(tcv.BUILD_DIR, "libCudaGridder.so")
    out = subprocess.run(["nm", "-DC", "--defined-only", lib], check=True, capture_output=True,
                         text=True).stdout
    assert "gridKernelCuda(std::vector<std::complex<float>" in out
    assert "degridKernelCuda(std::vector<std::complex<float>" in out


@pytest.mark.parametrize("cfg", ["g1", "g2", "c1", "c2"])
def test_c_geometry_matches_reference(tcv, golden, cfg):
    prob = PROBLEMS[cfg]
    sup, os_, wcs, clen = ctypes.c_int(), ctypes.c_int(), ctypes.c_double(), ctypes.c_int64()
    st = tcv.lib().tcv_c_geometry(prob.freq0, prob.cell_size, prob.baseline, prob.w_size,
                                  ctypes.byref(sup), ctypes.byref(os_), ctypes.byref(wcs),
                                  ctypes.byref(clen))
    assert st == 0
    meta = golden["runs"][f"{cfg}_ones"]["meta"]
    assert sup.value == meta["support"] == prob.support()
    assert os_.value == meta["overSample"]
    assert wcs.value == meta["wCellSize"]
    assert clen.value == golden["runs"][f"{cfg}_ones"]["shape"]["C"][0]


def test_status_strings_and_type_sizes(tcv):
    L = tcv.lib()
    assert L.tcv_status_string(0) == b"ok"
    assert L.tcv_status_string(2) == b"sample outside grid or table"
    assert [L.tcv_ctype_bytes(t) for t in range(6)] == [8, 4, 4, 2, 4, 2]
    assert L.tcv_ctype_bytes(17) == 0
    assert b"sm_100a" in L.tcv_version()


def test_argument_validation_before_device_use(tcv):
    from tconvolve._lib import TcvConfig

    L = tcv.lib()
    bad = TcvConfig(n_samples=0, w_size=33, n_chan=1, g_size=4096, baseline=2000, cell_size=5.0)
    ctx = ctypes.c_void_p()
    assert L.tcv_create(ctypes.byref(bad), ctypes.byref(ctx)) == 1  # TCV_ERR_ARG
    assert L.tcv_plan_build(None, None, None, None, 10, 3, 64, 100, None, 0, None) == 1
    assert L.tcv_plan_workspace_bytes(-1, 3, 64, 100) == 0
    assert L.tcv_plan_workspace_bytes(1000, 22, 1024, 1166400) > 0
    assert L.tcv_run_grid(None) == 1
    assert L.tcv_convert_c(None, 10, 1, None, None, None, None) == 1


def test_no_silent_cpu_path(tcv):
    """Without a usable GPU the context cannot be created: the library has no CPU fallback."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is visible; the loud-failure path is for GPU-less hosts")
    from tconvolve import Benchmark, TcvError

    with pytest.raises(TcvError) as e:
        Benchmark(**PROBLEMS["g1"].kwargs())
    assert e.value.status == 4  # TCV_ERR_CUDA


def test_workspace_grows_with_samples(tcv):
    L = tcv.lib()
    a = L.tcv_plan_workspace_bytes(1000, 64, 4096, 35145792)
    b = L.tcv_plan_workspace_bytes(160000, 64, 4096, 35145792)
    assert b > a
    # 160 k samples x 9 tiles: keys + values, double-buffered, plus the anchor sort; < 64 MiB
    assert b < 64 << 20


def test_static_scratch_limit_is_the_documented_one(tcv):
    """The allocation-free entry's limit that the header states (n <= 269,745 samples of a 129 x 129
    footprint on a 4096 grid with the 33-plane table) is the one tcv_plan_workspace_bytes gives."""
    L = tcv.lib()
    limit = L.tcv_static_scratch_bytes()
    assert limit == 64 << 20
    assert L.tcv_plan_workspace_bytes(269745, 64, 4096, 35145792) <= limit
    assert L.tcv_plan_workspace_bytes(269746, 64, 4096, 35145792) > limit


def test_batch_argument_validation(tcv):
    """Batched plans, tuning and graphs: invalid arguments are refused on the host."""
    from tconvolve._lib import TcvJob, TcvTuning

    L = tcv.lib()
    jobs = (TcvJob * 3)()
    for j, (n, g) in enumerate([(1000, 2048), (0, 4096), (5000, 2048)]):
        jobs[j].n, jobs[j].g_size, jobs[j].d_grid = n, g, ctypes.c_void_p(256 * (j + 1))
    clen = 35145792
    ws = L.tcv_batch_workspace_bytes(jobs, 3, 64, clen, None)
    assert ws > 0
    # the workspace holds the cells of every job's tiles: it grows with each job
    assert ws > L.tcv_batch_workspace_bytes(jobs, 2, 64, clen, None) > 0
    for rows, mib in [(8, 32), (16, -1), (32, 8)]:
        t = TcvTuning(rows, mib)
        assert L.tcv_batch_workspace_bytes(jobs, 3, 64, clen, ctypes.byref(t)) > 0
    for rows, mib in [(7, 32), (64, 32), (16, -2)]:
        t = TcvTuning(rows, mib)
        assert L.tcv_batch_workspace_bytes(jobs, 3, 64, clen, ctypes.byref(t)) == 0
    assert L.tcv_batch_workspace_bytes(jobs, 0, 64, clen, None) == 0
    jobs[1].d_grid = None
    assert L.tcv_batch_workspace_bytes(jobs, 3, 64, clen, None) == 0  # every job needs a grid
    jobs[1].d_grid = ctypes.c_void_p(512)
    jobs[2].n = -1
    assert L.tcv_batch_workspace_bytes(jobs, 3, 64, clen, None) == 0
    plan = ctypes.c_void_p()
    assert L.tcv_batch_plan_create(ctypes.byref(plan), jobs, 3, 64, clen, None, None, 0, None) == 1
    assert L.tcv_plan_bin(None, None, None, None, None) == 1
    assert L.tcv_plan_tuning(None, None) == 1
    g = ctypes.c_void_p()
    assert L.tcv_graph_capture(ctypes.byref(g), None, 7, None, None, None, None, None, 0, 1.0, None, None) == 1
    assert L.tcv_graph_launch(None, None) == 1
    best = TcvTuning()
    assert L.tcv_autotune(jobs, 0, None, None, None, None, None, 0, 1.0, clen, 64, 3, ctypes.byref(best),
                          None, None) == 1
    n = ctypes.c_int()
    assert L.tcv_autotune_report(None, None, 0, ctypes.byref(n)) == 0 and n.value >= 0


def test_batch_geometry_limits(tcv):
    """More jobs than the tile record holds, or tiles per side beyond it, are refused as
    unsupported rather than mis-binned (no device work: the limits are host checks)."""
    from tconvolve._lib import TcvJob

    L = tcv.lib()
    many = (TcvJob * 1025)()
    for j in range(1025):
        many[j].n, many[j].g_size, many[j].d_grid = 1, 64, ctypes.c_void_p(256)
    plan = ctypes.c_void_p()
    work = ctypes.c_void_p(256)
    assert L.tcv_batch_plan_create(ctypes.byref(plan), many, 1025, 3, 7 * 7 * 64, None, work, 1 << 40,
                                   None) == 8  # TCV_ERR_UNSUPPORTED


def test_header_is_plain_c(tmp_path):
    """include/tconvolve.h compiles as C99 (the boundary is a C ABI, bindable from cgo/JNI/ctypes)."""
    src = tmp_path / "use.c"
    src.write_text('#include "tconvolve.h"\nint main(void) { tcv_server_config c; tcv_tuning t = {16, 32};\n'
                   '  c.tuning = t; return (int)sizeof(tcv_request) + c.tuning.tile_rows * 0; }\n')
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-I", os.path.join(REPO, "include"),
                    str(src)], check=True)


def test_server_argument_validation(tcv):
    import torch

    from tconvolve._lib import TcvRequest, TcvServerConfig

    L = tcv.lib()
    cfg = TcvServerConfig()
    L.tcv_server_config_default(ctypes.byref(cfg))
    assert (cfg.g_size, cfg.w_size, cfg.baseline, cfg.streams, cfg.max_batch) == (1024, 9, 2000, 2, 32)
    assert cfg.hbm_budget == int(150e9) and cfg.c_type == 1  # TCV_C_R32
    srv = ctypes.c_void_p()
    for field, value in [("streams", 9), ("max_batch", 129), ("g_size", 1), ("c_type", 0x100), ("batch_samples", -1)]:
        bad = TcvServerConfig()
        L.tcv_server_config_default(ctypes.byref(bad))
        setattr(bad, field, value)
        assert L.tcv_server_create(ctypes.byref(bad), ctypes.byref(srv)) == 1, field
    assert L.tcv_server_create(None, ctypes.byref(srv)) == 1
    req = TcvRequest()
    t = ctypes.c_uint64()
    assert L.tcv_server_submit(None, ctypes.byref(req), ctypes.byref(t)) == 1
    assert L.tcv_server_wait(None, 1, 0.0, None) == 1
    assert L.tcv_server_stats(None, None, None, None, None) == 1
    assert L.tcv_server_grid_alloc(None, None) == 1
    if not torch.cuda.is_available():
        # a valid configuration needs the GPU: no CPU fallback
        assert L.tcv_server_create(ctypes.byref(cfg), ctypes.byref(srv)) == 4  # TCV_ERR_CUDA


def test_current_geometry_matches_oracle(tcv, orc):
    """The library's host-side geometry of the variable-support run types equals the oracle's
    (itself pinned to the reference), and the plane tables match the reference's (sha256)."""
    import json

    from conftest import GOLDEN_DIR, sha
    from tconvolve._lib import TcvCurGeometry

    L = tcv.lib()
    with open(os.path.join(GOLDEN_DIR, "current.json")) as f:
        gold = json.load(f)["runs"]
    for rt in range(5):
        g = TcvCurGeometry()
        assert L.tcv_cur_geometry_of(rt, ctypes.byref(g)) == 0
        o = orc.cur_geometry(rt)
        assert (g.w_size, g.over_sample, g.support, g.g_size, g.n_baselines, g.n_samples, g.c_len, g.s_max) == \
            (o.w_size, o.over_sample, o.support, o.g_size, o.n_baselines, o.n_samples, o.c_len, o.s_max)
        assert g.w_cell_size == o.w_cell_size and g.uv_cell_size == o.uv_cell_size
        import numpy as np
        s = np.empty(g.w_size, np.int32)
        off = np.empty(g.w_size, np.int32)
        assert L.tcv_cur_planes(rt, s.ctypes.data_as(ctypes.c_void_p), off.ctypes.data_as(ctypes.c_void_p)) == 0
        assert sha(s) == gold[f"rt{rt}"]["sha256"]["ssize"] and sha(off) == gold[f"rt{rt}"]["sha256"]["coff0"]
    assert L.tcv_cur_geometry_of(5, ctypes.byref(TcvCurGeometry())) == 1
    rates = (ctypes.c_float * 2)()
    L.tcv_cur_required_rate(rates)
    # current/tConvolveMPI/Benchmark.cc:697-739 evaluated by hand
    assert rates[0] == np.float32(10 * 5443200 * 10 * 3 * 3 * 400 / 5250.0)
    assert rates[1] == np.float32(10 * 3758400 * 4 * 3 * 78 * 100 / 5500.0)


def test_hogbom_fft_major_argument_validation(tcv):
    """The minor-cycle, FFT and major-cycle entry points refuse bad arguments before any device
    use (so these run without a GPU)."""
    from tconvolve._lib import TcvMajorConfig, lib

    L = lib()
    P = ctypes.c_void_p
    fake = P(0x1000)  # never dereferenced: every call below fails its argument checks first
    f = ctypes.c_float
    # Hogbom: null images, bad widths, negative iterations, too small a workspace
    assert L.tcv_hogbom_workspace_bytes(0) == 0 and L.tcv_hogbom_workspace_bytes(4096) > 0
    assert L.tcv_hogbom_deconvolve(None, 64, fake, 64, fake, fake, 10, f(0.1), f(0.0), None, None, fake, 1 << 20,
                                   None) == 1
    assert L.tcv_hogbom_deconvolve(fake, 0, fake, 64, fake, fake, 10, f(0.1), f(0.0), None, None, fake, 1 << 20,
                                   None) == 1
    assert L.tcv_hogbom_deconvolve(fake, 64, fake, 64, fake, fake, -1, f(0.1), f(0.0), None, None, fake, 1 << 20,
                                   None) == 1
    assert L.tcv_hogbom_deconvolve(fake, 70000, fake, 64, fake, fake, 10, f(0.1), f(0.0), None, None, fake,
                                   1 << 20, None) == 8  # width^2 beyond 32-bit indices
    assert L.tcv_hogbom_deconvolve(fake, 64, fake, 64, fake, fake, 10, f(0.1), f(0.0), None, None, fake, 16,
                                   None) == 7  # workspace
    assert L.tcv_find_peak(None, 10, None, None, fake, 1 << 20, None) == 1
    # FFT steps: null grids, odd sizes (refused as the reference refuses them)
    assert L.tcv_fft_exec(None, 64, 1, None) == 1
    assert L.tcv_fft_exec(fake, 63, 1, None) == 8
    assert L.tcv_image_from_grid(fake, 63, f(1.0), fake, None) == 8
    assert L.tcv_grid_from_image(fake, 63, fake, None) == 8
    assert L.tcv_fft_fix(None, 10, f(1.0), None) == 1
    # major cycle: bad configurations
    cfg = TcvMajorConfig()
    L.tcv_major_config_default(ctypes.byref(cfg))
    assert (cfg.n_samples, cfg.w_size, cfg.g_size, cfg.n_major, cfg.n_minor, cfg.n_sources) == (160000, 33, 4096, 5,
                                                                                              100, 100)
    ctx = P()
    bad = TcvMajorConfig.from_buffer_copy(cfg)
    bad.g_size = 4095
    assert L.tcv_major_create(ctypes.byref(bad), ctypes.byref(ctx)) == 8
    bad = TcvMajorConfig.from_buffer_copy(cfg)
    bad.n_samples = 0
    assert L.tcv_major_create(ctypes.byref(bad), ctypes.byref(ctx)) == 1
    assert L.tcv_major_create(None, ctypes.byref(ctx)) == 1


def test_tuning_kernel_field_validation(tcv):
    """The sample-parallel kernels (tuning.kernel bits) need 8-row tiles; a plan workspace query
    with another tile height, or an unknown bit, is refused (0 bytes)."""
    import numpy as np

    from tconvolve._lib import TcvTuning, lib

    L = lib()
    s = np.array([7, 9, 11], np.int32)
    off0 = np.array([0, 49 * 64, (49 + 81) * 64], np.int32)
    c_len = int((49 + 81 + 121) * 64)
    args = (1000, s.ctypes.data_as(ctypes.c_void_p), off0.ctypes.data_as(ctypes.c_void_p), 3, 512, c_len)
    assert L.tcv_plan_workspace_bytes_var(*args, ctypes.byref(TcvTuning(8, 32, 0, 0, 3))) > 0
    assert L.tcv_plan_workspace_bytes_var(*args, ctypes.byref(TcvTuning(8, 32, 0, 0, 2))) > 0
    assert L.tcv_plan_workspace_bytes_var(*args, ctypes.byref(TcvTuning(16, 32, 0, 0, 1))) == 0
    assert L.tcv_plan_workspace_bytes_var(*args, ctypes.byref(TcvTuning(8, 32, 0, 0, 4))) == 0
    assert TcvTuning(8, 32, 0, 0, 3).as_tuple() == (8, 32, 0, 0, 3)
    assert TcvTuning(8, 32, 0, 0, 0).as_tuple() == (8, 32, 0, 0)


def test_band_split_argument_validation(tcv):
    """The row-band steps refuse bad arguments before any device work."""
    L = tcv.lib()
    P = ctypes.c_void_p
    one = P(16)  # never dereferenced: every call below fails its argument checks first
    rows = (ctypes.c_int32 * 3)(0, 100, 256)
    bad_rows = (ctypes.c_int32 * 3)(0, 300, 256)  # not ascending
    counts = P(32)
    assert L.tcv_band_histogram(None, 10, 4, 256, counts, None) == 1          # no iv
    assert L.tcv_band_histogram(one, 10, 4, 256, None, None) == 1             # no histogram
    assert L.tcv_band_histogram(one, -1, 4, 256, counts, None) == 1
    assert L.tcv_band_histogram(one, 0, 4, 256, counts, None) == 0            # nothing to count
    assert L.tcv_band_workspace_bytes(10, 0) == 0 and L.tcv_band_workspace_bytes(10, 65) == 0
    assert L.tcv_band_workspace_bytes(10, 2) > 0
    args = [one, one, one, one, 10, 4, 256, rows, 2, one, one, counts, one, 1 << 20, None]
    for i, bad in ((7, bad_rows), (8, 0), (8, 65), (4, -1), (11, None), (12, None)):
        a = list(args)
        a[i] = bad
        assert L.tcv_band_bucket(*a) == 1, i
    a = list(args)
    a[13] = 16  # workspace smaller than tcv_band_workspace_bytes
    assert L.tcv_band_bucket(*a) == 7
    assert L.tcv_band_unpack(None, 5, one, one, one, one, None) == 1
    assert L.tcv_band_unpack(one, 0, None, None, None, None, None) == 0
    assert L.tcv_band_scatter(one, None, 5, one, None) == 1
    assert L.tcv_rows_add(None, one, 5, None) == 1
    assert L.tcv_rows_add(one, one, -1, None) == 1
