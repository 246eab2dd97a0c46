"""The C++ drivers of the reference programs beyond tConvolve (built by the csrc Makefile):
tHogbomClean (current/tHogbomCleanOMP) must reproduce the reference's HogbomGolden bit for bit on
the golden images; tConvolveCurrent (current/tConvolveMPI) and tMajor (current/tMajorACC) run their
flows and print the reference's report lines; current::Benchmark's std::vector kernel forms equal
the object's own passes."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import GOLDEN_DIR, PKG, REPO, sha

sys.path.insert(0, GOLDEN_DIR)
from make_golden_hogbom import cases  # noqa: E402

pytestmark = pytest.mark.gpu
BUILD = os.path.join(PKG, "_build")


@pytest.mark.parametrize("name", ["w128", "stop"])
def test_thogbomclean_matches_reference(tcv, cuda_ok, tmp_path, name):
    with open(os.path.join(GOLDEN_DIR, "hogbom.json")) as f:
        ref = json.load(f)["cases"][name]
    dirty, psf = cases()[name]
    dirty.astype(np.float32).tofile(tmp_path / "dirty.img")
    psf.astype(np.float32).tofile(tmp_path / "psf.img")
    out = subprocess.run([os.path.join(BUILD, "tHogbomClean"), str(tmp_path / "dirty.img"), str(tmp_path / "psf.img"),
                          str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert "Cleaning rate" in out.stdout and "Done" in out.stdout
    assert sha(np.fromfile(tmp_path / "model.img", np.float32)) == ref["sha256"]["model"]
    assert sha(np.fromfile(tmp_path / "residual.img", np.float32)) == ref["sha256"]["residual"]


def test_tconvolvecurrent_runs(tcv, cuda_ok):
    out = subprocess.run([os.path.join(BUILD, "tConvolveCurrent")], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    for line in ("+++++ Test 0 +++++", "+++++ Test 1 +++++", "Continuum gridding performance (per process)",
                 "Spectral degridding performance (per process)"):
        assert line in out.stdout
    assert out.stdout.count("Done") == 2


def test_tmajor_runs(tcv, cuda_ok):
    out = subprocess.run([os.path.join(BUILD, "tMajor"), "-n", "2000", "-w", "9", "-f", "5", "-g", "512", "-M", "2",
                          "-m", "20"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    for line in ("cycle 1", "Gridding PSF", "Hogbom clean", "Cleaning rate", "Degridding rate"):
        assert line in out.stdout


def test_current_benchmark_vector_forms(tcv, cuda_ok, tmp_path):
    exe = tmp_path / "cpp_current_check"
    csrc = os.path.join(PKG, "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{REPO}/include", f"-I{csrc}", "-I/usr/local/cuda/include", "-o",
                    str(exe), os.path.join(REPO, "tests", "cpp_current_check.cc"), os.path.join(csrc, "CurrentBenchmark.cc"),
                    f"-L{BUILD}", "-ltconvolve", "-L/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{BUILD}"],
                   check=True, capture_output=True, timeout=300)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.split() == ["grid_equal", "1", "degrid_equal", "1", "c_equal", "1"], out.stdout
