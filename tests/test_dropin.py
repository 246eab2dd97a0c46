"""The drop-in seams run on the GPU, as a maintainer would use them.

* The reference's own attic/tConvolveCuda/tConvolveCuda.cc main, compiled unmodified and linked
  against this project's libCudaGridder.so (oracle/Makefile target `cudaref`), runs its CPU gridding
  and degridding and the GPU forms through gridKernelCuda/degridKernelCuda (tcv_grid_host_raw /
  tcv_degrid_host_raw) and checks every grid point and sample itself (tConvolveCuda.cc:362-389,
  :420-448: |real(cpu) - real(gpu)| <= 1e-5).  Both of its "Verifying result...Pass" lines must
  appear.
* The tConvolve driver (csrc/tConvolve.cc, the flow of attic/tConvolveMPI/tConvolveMPI.cc:78-121)
  prints the reference's report lines with positive rates.
* The C++ Benchmark class's std::vector forms (initC, gridKernel, degridKernel; csrc/Benchmark.cc,
  interface of attic/tConvolveMPI/Benchmark.h:55-99) against the oracle pinned to the reference's
  output: the table bit for bit (up to the 1-ulp allowance of the FP64 cos/exp), grid and degridded
  samples within relative L2 1e-5 (REL_L2_FP32).
"""
from __future__ import annotations

import os
import re
import subprocess

import numpy as np
import pytest

from conftest import PKG, REL_L2_FP32, REPO, oracle_config, sha
from tconvolve.workload import PROBLEMS

pytestmark = pytest.mark.gpu
BUILD = os.path.join(PKG, "_build")
CUDA_REF = os.path.join(REPO, "oracle", "_ref", "tConvolveCuda")


@pytest.mark.skipif(not os.path.exists(CUDA_REF), reason="the reference's tConvolveCuda was not built (no reference tree)")
def test_reference_tconvolvecuda_passes_on_libcudagridder(tcv, cuda_ok):
    out = subprocess.run([CUDA_REF], capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    assert out.stdout.count("Verifying result...Pass") == 2, out.stdout[-2000:]
    assert "Support = 64 pixels" in out.stdout
    for line in ("+++++ Forward processing (GPU) +++++", "+++++ Reverse processing (GPU) +++++"):
        assert line in out.stdout
    rates = [float(x) for x in re.findall(r"rate\s+([0-9.eE+-]+) \(million grid points per second\)", out.stdout)]
    assert len(rates) == 4 and min(rates) > 0


def test_tconvolve_driver_report_lines(tcv, cuda_ok):
    prob = PROBLEMS["c1"]
    out = subprocess.run([os.path.join(BUILD, "tConvolve"), "-n", str(prob.n_samples), "-w", str(prob.w_size),
                          "-g", str(prob.g_size), "-s", repr(prob.cell_size), "-r", "3"],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    s = out.stdout
    for line in ("Initializing W projection convolution function", "Support = 22 pixels",
                 "Shape of convolution function = [45, 45, 8, 8, 9]", "+++++ Forward processing (B200) +++++",
                 "+++++ Reverse processing (B200) +++++", "Number of processes: 1", "Done"):
        assert line in s, line
    g = re.search(r"Gridding rate\s+([0-9.eE+-]+) \(million grid points per second\)", s)
    d = re.search(r"Degridding rate\s+([0-9.eE+-]+) \(million grid points per second\)", s)
    assert g and d and float(g.group(1)) > 0 and float(d.group(1)) > 0
    assert re.search(r"Time per visibility spectral sample [0-9.eE+-]+ \(us\)", s)


@pytest.mark.parametrize("cfg", ["g2", "c1"])
def test_cpp_benchmark_vector_forms(tcv, orc, golden, cuda_ok, tmp_path, cfg):
    exe = tmp_path / "cpp_attic_check"
    csrc = os.path.join(PKG, "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{REPO}/include", f"-I{csrc}", "-o", str(exe),
                    os.path.join(REPO, "tests", "cpp_attic_check.cc"), os.path.join(csrc, "Benchmark.cc"),
                    f"-L{BUILD}", "-ltconvolve", f"-Wl,-rpath,{BUILD}"], check=True, capture_output=True, timeout=300)
    prob = PROBLEMS[cfg]
    out = subprocess.run([str(exe), str(prob.n_samples), str(prob.w_size), str(prob.n_chan), str(prob.g_size),
                          repr(prob.cell_size), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    ref = golden["runs"][f"{cfg}_ones"]
    support, os_, wcs, obj_support = open(tmp_path / "meta.txt").read().split()
    assert int(support) == ref["meta"]["support"] == int(obj_support) and int(os_) == ref["meta"]["overSample"]
    assert float(wcs) == ref["meta"]["wCellSize"]
    rd = lambda n: np.fromfile(tmp_path / n, np.complex64)  # noqa: E731
    c = rd("C.c64")
    r = orc.run_plain(oracle_config(orc, prob), vis=None, threads=8)  # the reference's data = 1+0i
    assert sha(r["C"]) == ref["sha256"]["C"] and sha(r["grid"]) == ref["sha256"]["grid"]
    diff = np.count_nonzero(c.view(np.uint32) != r["C"].view(np.uint32))
    assert diff <= max(1, c.size * 2 >> 20)
    for grid, outdata in ((rd("grid.c64"), rd("outdata.c64")), (rd("obj_grid.c64"), rd("obj_outdata.c64"))):
        assert orc.rel_l2(grid, r["grid"]) <= REL_L2_FP32
        assert orc.rel_l2(outdata, r["outdata"]) <= REL_L2_FP32
        assert np.count_nonzero(grid) == ref["grid_nonzero"]
