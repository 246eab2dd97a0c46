"""The L2 table-stream probe (tcv_probe_table_stream): argument checks on CPU, one measured launch
on the GPU (a positive, finite bandwidth, every output written)."""
from __future__ import annotations

import ctypes

import pytest


def test_probe_argument_validation(tcv):
    from tconvolve._lib import probe_lib as lib

    L = lib()
    fake = ctypes.c_void_p(0x1000)  # never dereferenced: the calls fail their argument checks first
    n = ctypes.c_int64()
    assert L.tcv_probe_table_stream(None, 1 << 20, 129, 4, fake, ctypes.byref(n), None) == 1
    assert L.tcv_probe_table_stream(fake, 1 << 20, 16, 4, fake, ctypes.byref(n), None) == 1  # stride < 32
    assert L.tcv_probe_table_stream(fake, 100, 129, 4, fake, ctypes.byref(n), None) == 1  # buffer < one window
    assert L.tcv_probe_table_stream(fake, 1 << 20, 129, 0, fake, ctypes.byref(n), None) == 1


@pytest.mark.gpu
def test_probe_measures(tcv, cuda_ok):
    import torch

    from tconvolve._lib import probe_lib as lib
    from tconvolve.raw import _ptr

    L = lib()
    buf = torch.rand(4 << 20, dtype=torch.float32, device="cuda")
    out = torch.full((int(L.tcv_probe_table_threads()),), float("nan"), dtype=torch.float32, device="cuda")
    n = ctypes.c_int64()
    assert L.tcv_probe_table_stream(_ptr(buf), buf.numel(), 129, 8, _ptr(out), ctypes.byref(n), None) == 0
    torch.cuda.synchronize()
    assert n.value == (out.numel() // 32) * 8 * 16 * 128
    assert bool(torch.isfinite(out).all()) and float(out.min()) >= 0.0
