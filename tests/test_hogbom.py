"""GPU Hogbom CLEAN (tcv_hogbom_*) against the reference and the oracle.

Bars (written here, used below): bit-exact.  The model, the residual, the peak picked at every
iteration, the iteration count and the PSF rows skipped equal the reference's HogbomGolden
(sha256 of its outputs in tests/golden/hogbom.json) and the oracle's at the full 4096^2 size; the
arithmetic is the reference's float roundings, so no tolerance applies.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN_DIR, sha

sys.path.insert(0, GOLDEN_DIR)
from make_golden_hogbom import cases  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hog_golden():
    with open(os.path.join(GOLDEN_DIR, "hogbom.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("name", ["w128", "w256", "w100", "w128_psf256", "stop"])
def test_hogbom_matches_reference(tcv, orc, hog_golden, cuda_ok, name):
    from tconvolve.hogbom import Hogbom

    dirty, psf = cases()[name]
    ref = hog_golden["cases"][name]
    p = hog_golden["params"]
    h = Hogbom(p["niters"], p["gain"], p["threshold"])
    model = np.zeros(dirty.size, np.float32)
    residual = h.deconvolve(dirty, ref["width"], psf, ref["psf_width"], model)
    assert sha(model) == ref["sha256"]["model"]
    assert sha(residual) == ref["sha256"]["residual"]
    o = orc.hogbom(dirty, psf, p["niters"], p["gain"], p["threshold"])
    assert h.last["done"] == o["done"] and h.last["stopped_at"] == o["stopped_at"]
    assert h.last["psf_peak_pos"] == o["psf_peak_pos"] and h.last["skipped_rows"] == 0


def _device_run(dirty, width, psf, psf_width, niters, gain, threshold):
    import torch

    from tconvolve.hogbom import deconvolve_device

    d = torch.from_numpy(dirty.ravel()).cuda()
    p = torch.from_numpy(psf.ravel()).cuda()
    m = torch.zeros_like(d)
    r = torch.empty_like(d)
    hv = torch.zeros(niters, dtype=torch.float32, device="cuda")
    hp = torch.zeros(niters, dtype=torch.int32, device="cuda")
    ws = deconvolve_device(d, width, p, psf_width, m, r, niters, gain, threshold, hist=(hv, hp))
    res = ws.result()
    return m.cpu().numpy(), r.cpu().numpy(), hv.cpu().numpy(), hp.cpu().numpy(), res


@pytest.mark.parametrize("width,niters,threshold", [(4096, 100, 0.0), (1024, 1000, 1e-5)])
def test_hogbom_full_size_against_oracle(tcv, orc, cuda_ok, width, niters, threshold):
    """tMajorACC's minor cycle at 4096^2 (100 iterations, no threshold) and tHogbomCleanOMP's at
    1024^2 (1000 iterations, threshold 1e-5): every iteration's peak and the final images."""
    from tconvolve.workload import synthetic_dirty, synthetic_psf

    dirty, psf = synthetic_dirty(width, 20, 1e-3, seed=7), synthetic_psf(width)
    m, r, hv, hp, res = _device_run(dirty, width, psf, width, niters, 0.1, threshold)
    o = orc.hogbom(dirty, psf, niters, 0.1, threshold)
    assert res["done"] == o["done"]
    assert np.array_equal(hp[:o["done"]], o["hist_pos"]) and np.array_equal(hv[:o["done"]], o["hist_val"])
    assert np.array_equal(m, o["model"]) and np.array_equal(r, o["residual"])


def test_hogbom_off_diagonal_psf(tcv, orc, cuda_ok):
    """A PSF whose peak is off the diagonal (px != py): the reference's row index y - (ry - px)
    leaves the PSF for some rows; both skip the same rows and agree elsewhere."""
    w = 256
    psf = np.roll(np.roll(__import__("tconvolve.workload", fromlist=["x"]).synthetic_psf(w), 40, axis=1), -30, axis=0)
    from tconvolve.workload import synthetic_dirty

    dirty = synthetic_dirty(w, 10, 1e-3, seed=9)
    m, r, hv, hp, res = _device_run(dirty, w, np.ascontiguousarray(psf), w, 200, 0.1, 0.0)
    o = orc.hogbom(dirty, psf, 200, 0.1, 0.0)
    assert o["skipped_rows"] > 0 and res["skipped_rows"] == o["skipped_rows"]
    assert np.array_equal(hp, o["hist_pos"]) and np.array_equal(m, o["model"]) and np.array_equal(r, o["residual"])


def test_find_peak_rules_on_gpu(tcv, orc, cuda_ok):
    import torch

    from tconvolve.hogbom import find_peak

    a = np.zeros(1 << 20, np.float32)
    assert find_peak(torch.from_numpy(a).cuda()) == (0.0, 0)
    a[[70000, 300000, 600001]] = [-2.0, 2.0, 1.5]
    assert find_peak(torch.from_numpy(a).cuda()) == (-2.0, 70000)
    a[3] = -2.0
    assert find_peak(torch.from_numpy(a).cuda()) == (-2.0, 3)
    rng = np.random.default_rng(0)
    b = rng.standard_normal(5_000_003).astype(np.float32)
    assert find_peak(torch.from_numpy(b).cuda()) == orc.find_peak(b)


def test_hogbom_deterministic(tcv, cuda_ok):
    from tconvolve.workload import synthetic_dirty, synthetic_psf

    dirty, psf = synthetic_dirty(512, 20, 1e-3, seed=11), synthetic_psf(512)
    a = _device_run(dirty, 512, psf, 512, 300, 0.1, 0.0)
    b = _device_run(dirty, 512, psf, 512, 300, 0.1, 0.0)
    assert all(np.array_equal(x, y) for x, y in zip(a[:4], b[:4]))


@pytest.mark.parametrize("width", [512, 100])
def test_persistent_and_per_launch_forms_agree(tcv, orc, cuda_ok, width):
    """The cooperative all-iterations launch and the launch-per-iteration form give the same bits
    (and the oracle's), on a float4-aligned width and an odd one."""
    from tconvolve._lib import lib
    from tconvolve.workload import synthetic_dirty, synthetic_psf

    dirty, psf = synthetic_dirty(width, 15, 1e-3, seed=13), synthetic_psf(width)
    runs = []
    try:
        for strategy in (1, 2):  # TCV_HOGBOM_PER_LAUNCH, TCV_HOGBOM_PERSISTENT
            lib().tcv_hogbom_set_strategy(strategy)
            runs.append(_device_run(dirty, width, psf, width, 400, 0.1, 1e-5))
    finally:
        lib().tcv_hogbom_set_strategy(0)
    (m1, r1, v1, p1, s1), (m2, r2, v2, p2, s2) = runs
    assert s1 == s2
    assert np.array_equal(m1, m2) and np.array_equal(r1, r2) and np.array_equal(p1, p2) and np.array_equal(v1, v2)
    o = orc.hogbom(dirty, psf, 400, 0.1, 1e-5)
    assert np.array_equal(m2, o["model"]) and np.array_equal(r2, o["residual"])


@pytest.mark.parametrize("limit_ns", [0, 1_000_000])
def test_barrier_timeout_path(tcv, orc, cuda_ok, limit_ns):
    """The cooperative loop's bounded grid-barrier wait, made to run out on purpose: the barrier
    is told to expect one CTA more than the launch has (an arrival nothing makes), with a short
    limit.  Every CTA must give up, flag the error and return (the launch ends), the loop must stop
    after its first iteration and tcv_hogbom_result must report TCV_ERR_TIMEOUT.  With the default
    wait restored, the next run on the same workspace is the oracle's bit for bit."""
    import ctypes

    import torch

    from tconvolve._lib import lib
    from tconvolve.hogbom import Workspace, deconvolve_device
    from tconvolve.workload import synthetic_dirty, synthetic_psf

    w = 1024
    dirty, psf = synthetic_dirty(w, 15, 1e-3, seed=21), synthetic_psf(w)
    d = torch.from_numpy(dirty.ravel()).cuda()
    p = torch.from_numpy(psf.ravel()).cuda()
    m = torch.zeros_like(d)
    r = torch.empty_like(d)
    ws = Workspace(w)
    L = lib()
    assert L.tcv_hogbom_set_wait(3_000_000_000, 0) == 1  # above the 2 s cap: TCV_ERR_ARG
    try:
        L.tcv_hogbom_set_strategy(2)  # TCV_HOGBOM_PERSISTENT
        assert L.tcv_hogbom_set_wait(limit_ns, 1) == 0
        deconvolve_device(d, w, p, w, m, r, 200, 0.1, 0.0, work=ws)
        torch.cuda.synchronize()  # returns: every CTA left the kernel
        done, stop = ctypes.c_int(), ctypes.c_int()
        st = L.tcv_hogbom_result(ctypes.c_void_p(ws.buf.data_ptr()), ctypes.byref(done), ctypes.byref(stop), None,
                                 None, None)
        assert st == 5  # TCV_ERR_TIMEOUT
        assert done.value == 1 and stop.value == -1
    finally:
        L.tcv_hogbom_set_wait(2_000_000_000, 0)
        L.tcv_hogbom_set_strategy(0)
    # the context is still usable and the next run is the reference's
    L.tcv_hogbom_set_strategy(2)
    try:
        m.zero_()
        deconvolve_device(d, w, p, w, m, r, 200, 0.1, 0.0, work=ws)
        res = ws.result()
    finally:
        L.tcv_hogbom_set_strategy(0)
    o = orc.hogbom(dirty, psf, 200, 0.1, 0.0)
    assert res["done"] == o["done"] == 200
    assert np.array_equal(m.cpu().numpy(), o["model"]) and np.array_equal(r.cpu().numpy(), o["residual"])
