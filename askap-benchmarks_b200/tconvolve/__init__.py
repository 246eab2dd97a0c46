"""tconvolve -- B200 (sm_100a) W-projection gridding and degridding behind the reference's
Benchmark interface (attic/tConvolveMPI/Benchmark.h).

The computation is in libtconvolve.so (C ABI: include/tconvolve.h); this package is the host-side
mirror of the reference interface plus thin torch wrappers of the raw entry points.
"""
from ._lib import (C64, R32, CBF16, RBF16, CF16, RF16, CTYPE_BY_NAME, CTYPE_NAMES, TcvError,
                   build, lib, LIB_PATH, BUILD_DIR)
from .benchmark import Benchmark


def jit_info() -> str:
    """State of the footprint-width specialisation of the tile kernels (tcv_jit_info)."""
    return lib().tcv_jit_info().decode()


def jit_enable(enabled: bool) -> None:
    lib().tcv_jit_enable(1 if enabled else 0)

__all__ = ["Benchmark", "jit_info", "jit_enable", "TcvError", "build", "lib", "C64", "R32", "CBF16", "RBF16", "CF16", "RF16",
           "CTYPE_BY_NAME", "CTYPE_NAMES", "LIB_PATH", "BUILD_DIR"]
