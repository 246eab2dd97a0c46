"""Shared test set-up.

Markers: `gpu` for tests that need a B200 (run with -m gpu); everything else runs on CPU.
The oracle (oracle/) is the checker; the product is askap-benchmarks_b200/ (libtconvolve.so).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "askap-benchmarks_b200")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN_DIR = os.path.join(REPO, "tests", "golden")
VIS_SEED = 1234

# relative L2 bound for the plain FP32 form against the reference output (the parity bar of the path)
REL_L2_FP32 = 1e-5


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN_DIR, "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def tcv():
    import tconvolve

    if not os.path.exists(tconvolve.LIB_PATH):
        tconvolve.build()
    tconvolve.lib()
    return tconvolve


@pytest.fixture(scope="session")
def cuda_ok():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    return True


def oracle_config(orc, prob):
    return orc.Config(prob.n_samples, prob.w_size, prob.n_chan, prob.g_size, prob.cell_size,
                      prob.baseline, prob.seed)
