"""Generate the golden fixtures of Hogbom CLEAN from the reference's own code.

Runs oracle/_ref/hogbom/ref_driver_hogbom (current/tHogbomCleanOMP/HogbomGolden.cc compiled
unmodified by `make -C oracle ref-hogbom` from the reference tree; the reference's Parameters.h:
1000 iterations, gain 0.1, threshold 1e-5) on synthetic images from tconvolve.workload and records,
per case, the sha256 of the inputs and of the model and residual it returns, with their float64
norms, in hogbom.json.  The reference's own input images (data/dirty_*.img, data/psf_*.img) are
not in its tree.

Cases: square images of 128, 256 and 100 (odd-sized rows) pixels with a PSF of the same size; a
128-pixel image with a 256-pixel PSF; a faint single source that meets the 1e-5 threshold and
stops early.

Usage: python tests/golden/make_golden_hogbom.py   (needs the reference tree)
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "askap-benchmarks_b200"))
from tconvolve.workload import synthetic_dirty, synthetic_psf  # noqa: E402

DRIVER = os.path.join(REPO, "oracle", "_ref", "hogbom", "ref_driver_hogbom")


def cases():
    """name -> (dirty, psf) float32 arrays; the tests rebuild them with the same calls."""
    return {
        "w128": (synthetic_dirty(128, 20, 1e-3, seed=1), synthetic_psf(128)),
        "w256": (synthetic_dirty(256, 20, 1e-3, seed=2), synthetic_psf(256)),
        "w100": (synthetic_dirty(100, 10, 1e-3, seed=5), synthetic_psf(100)),
        "w128_psf256": (synthetic_dirty(128, 20, 1e-3, seed=3), synthetic_psf(256, scale=2.0)),
        "stop": (synthetic_dirty(128, 1, 0.0, seed=4) * np.float32(1e-4), synthetic_psf(128)),
    }


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run(dirty: np.ndarray, psf: np.ndarray) -> dict:
    with tempfile.TemporaryDirectory() as td:
        paths = [os.path.join(td, n) for n in ("dirty.img", "psf.img", "model.out", "residual.out")]
        dirty.astype(np.float32).tofile(paths[0])
        psf.astype(np.float32).tofile(paths[1])
        subprocess.run([DRIVER] + paths, check=True, capture_output=True)
        model = np.fromfile(paths[2], np.float32)
        residual = np.fromfile(paths[3], np.float32)
    return {"width": int(round(np.sqrt(dirty.size))), "psf_width": int(round(np.sqrt(psf.size))),
            "sha256": {"dirty": sha(dirty), "psf": sha(psf), "model": sha(model), "residual": sha(residual)},
            "norm": {"model": float(np.linalg.norm(model.astype(np.float64))),
                     "residual": float(np.linalg.norm(residual.astype(np.float64)))},
            "model_nonzero": int(np.count_nonzero(model))}


def main():
    out = {"params": {"niters": 1000, "gain": 0.1, "threshold": 1e-5}, "cases": {}}
    for name, (d, p) in cases().items():
        print("running", name, flush=True)
        out["cases"][name] = run(d, p)
    with open(os.path.join(HERE, "hogbom.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
