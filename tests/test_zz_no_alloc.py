"""The allocation-free gridding entry point (tcv_grid_raw_static).

It exists for callers that cannot allocate device memory: a pipeline running latency-critical
work on other streams cannot accept the device-wide synchronisation of cudaMalloc/cudaFree, and
a host framework that owns all device memory forbids allocations it did not make.  Its scratch
is a fixed device array inside the library, shared by every call and keeping the previous
call's contents, so the test runs it twice in a row and compares both results with the ordinary
entry point (tcv_grid_raw with a caller workspace).  This file is collected last on purpose.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import REL_L2_FP32, VIS_SEED, oracle_config
from tconvolve.workload import PROBLEMS, normal_vis

pytestmark = pytest.mark.gpu


def _inputs(orc, prob):
    cfg = oracle_config(orc, prob)
    u, v, w = orc.init_uvw(cfg)
    c, _, support, os_, wcs, _ = orc.init_c(cfg)
    iu, iv, co = orc.init_offsets(cfg, u, v, w, wcs, support, os_)
    return c, support, iu, iv, co


@pytest.mark.parametrize("cfg", ["g2", "c1"])
def test_static_entry_matches_workspace_entry(tcv, orc, cuda_ok, cfg):
    import torch

    from tconvolve import raw
    from tconvolve._lib import check, lib

    prob = PROBLEMS[cfg]
    c, support, iu, iv, co = _inputs(orc, prob)
    vis = normal_vis(iu.size, VIS_SEED)
    dvis, dc, diu, div, dco = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (vis, c, iu, iv, co))
    g = prob.g_size
    ref = torch.zeros(g * g, dtype=torch.complex64, device="cuda")
    raw.grid_raw(dvis, support, dc, tcv.C64, 1.0, dco, diu, div, ref, g)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    P = ctypes.c_void_p
    for call in range(2):  # the second call starts from the first call's leftovers in the array
        out = torch.zeros(g * g, dtype=torch.complex64, device="cuda")
        check(lib().tcv_grid_raw_static(P(dvis.data_ptr()), iu.size, support, P(dc.data_ptr()), tcv.C64, 1.0,
                                        c.size, P(dco.data_ptr()), P(diu.data_ptr()), P(div.data_ptr()),
                                        P(out.data_ptr()), g, stream), f"tcv_grid_raw_static call {call}")
        torch.cuda.synchronize()
        a, b = out.cpu().numpy(), ref.cpu().numpy()
        assert orc.rel_l2(a, b) <= REL_L2_FP32
        assert np.array_equal(a, b)  # same plan and kernels: identical bits
    # and both agree with the oracle
    grid_o = np.zeros(g * g, np.complex64)
    orc.grid_f32(vis, support, c, co, iu, iv, grid_o, g)
    assert orc.rel_l2(ref.cpu().numpy(), grid_o) <= REL_L2_FP32


def test_static_entry_rejects_oversize(tcv, cuda_ok):
    """A problem whose plan exceeds the fixed array is refused before any device work."""
    from tconvolve._lib import lib

    L = lib()
    limit = L.tcv_static_scratch_bytes()
    n = 400000
    assert L.tcv_plan_workspace_bytes(n, 64, 4096, 35145792) > limit
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    st = L.tcv_grid_raw_static(dummy, n, 64, dummy, 0, 1.0, 35145792, dummy, dummy, dummy, dummy, 4096, None)
    assert st == 7  # TCV_ERR_WORKSPACE
