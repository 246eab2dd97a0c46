"""The device header that the library compiles again at run time with NVRTC (tcv_jit.cu: the tile
kernels specialised on the footprint width and tile height) compiles here too, with the same
options, for every table form the specialisation serves.  NVRTC needs no GPU, so a source change
that would leave a GPU run on the generic kernels (or fail its first specialised launch) shows up
on the CPU."""
from __future__ import annotations

import ctypes
import os

import pytest

HDR = os.path.join(os.path.dirname(__file__), "..", "askap-benchmarks_b200", "csrc", "tcv_device.cuh")
OPTS = [b"--gpu-architecture=sm_100a", b"-std=c++17", b"-default-device", b"--fmad=true"]


def _nvrtc():
    try:
        return ctypes.CDLL("libnvrtc.so.12")
    except OSError:
        pytest.skip("libnvrtc.so.12 not found")


@pytest.mark.parametrize("kind", ["grid_tile_kernel", "degrid_tile_kernel"])
@pytest.mark.parametrize("tab", ["TabC64", "TabR32", "TabCBF16", "TabRBF16"])
def test_specialised_tile_kernels_compile(kind, tab):
    nv = _nvrtc()
    src = open(HDR, "rb").read()
    prog = ctypes.c_void_p()
    body = b'#include "tcv_device.cuh"\n'
    hs = (ctypes.c_char_p * 1)(src)
    hn = (ctypes.c_char_p * 1)(b"tcv_device.cuh")
    assert nv.nvrtcCreateProgram(ctypes.byref(prog), body, b"tcv_tile_specialised.cu", 1, hs, hn) == 0
    expr = f"tcv::{kind}<tcv::{tab}, 129, 16>".encode()
    assert nv.nvrtcAddNameExpression(prog, expr) == 0
    opts = (ctypes.c_char_p * len(OPTS))(*OPTS)
    rc = nv.nvrtcCompileProgram(prog, len(OPTS), opts)
    n = ctypes.c_size_t()
    nv.nvrtcGetProgramLogSize(prog, ctypes.byref(n))
    log = ctypes.create_string_buffer(n.value + 1)
    nv.nvrtcGetProgramLog(prog, log)
    try:
        assert rc == 0, log.value.decode(errors="replace")
        size = ctypes.c_size_t()
        assert nv.nvrtcGetCUBINSize(prog, ctypes.byref(size)) == 0 and size.value > 0
    finally:
        nv.nvrtcDestroyProgram(ctypes.byref(prog))
