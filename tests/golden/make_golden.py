"""Generate the golden fixtures from the reference's own code.

Runs oracle/_ref/<cfg>/ref_driver (attic/tConvolveMPI/Benchmark.cc compiled unmodified by
oracle/Makefile from the reference tree) for every configuration, once with the reference's
visibilities (1+0i) and once with N(0,1) visibilities (tconvolve.workload.normal_vis(n, 1234)),
and records:

  golden.json   per run: support, overSample, wCellSize, array shapes, sha256 of every output
                (u, v, w, iu, iv, cOffset, C, grid, outdata), and float64 norms
  <cfg>_<vis>.npz  full grid and outdata for the small configurations g1 and g2, and outdata for c1

The sha256 values pin bit-exact agreement; the arrays support tolerance checks.
Usage: python tests/golden/make_golden.py   (needs the reference tree; run `make -C oracle ref`)
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
from tconvolve.workload import PROBLEMS, normal_vis  # noqa: E402

VIS_SEED = 1234
FILES = [("u", "f64", np.float64), ("v", "f64", np.float64), ("w", "f64", np.float64),
         ("iu", "i32", np.int32), ("iv", "i32", np.int32), ("coff", "i32", np.int32),
         ("C", "c64", np.complex64), ("grid", "c64", np.complex64),
         ("outdata", "c64", np.complex64), ("data", "c64", np.complex64)]


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run(cfg: str, vis_kind: str) -> dict:
    drv = os.path.join(REPO, "oracle", "_ref", cfg, "ref_driver")
    prob = PROBLEMS[cfg]
    with tempfile.TemporaryDirectory() as td:
        args = [drv, "dump", td]
        if vis_kind == "normal":
            vp = os.path.join(td, "vis.c64")
            normal_vis(prob.n_data(), VIS_SEED).tofile(vp)
            args.append(vp)
        subprocess.run(args, check=True, capture_output=True)
        meta = {}
        for line in open(os.path.join(td, "meta.txt")):
            k, v = line.split()
            meta[k] = float(v) if "." in v or "e" in v else int(v)
        arrs = {name: np.fromfile(os.path.join(td, f"{name}.{ext}"), dtype=dt)
                for name, ext, dt in FILES}
    rec = {"meta": meta, "sha256": {k: sha(a) for k, a in arrs.items()},
           "shape": {k: list(a.shape) for k, a in arrs.items()},
           "norm": {k: float(np.linalg.norm(a.astype(np.complex128))) for k, a in arrs.items()
                    if a.dtype == np.complex64}}
    # nonzero footprint of the grid, as a cheap structural pin
    g = arrs["grid"]
    rec["grid_nonzero"] = int(np.count_nonzero(g))
    if cfg in ("g1", "g2"):
        np.savez_compressed(os.path.join(HERE, f"{cfg}_{vis_kind}.npz"), grid=g,
                            outdata=arrs["outdata"])
    elif cfg == "c1":
        np.savez_compressed(os.path.join(HERE, f"{cfg}_{vis_kind}.npz"), outdata=arrs["outdata"])
    return rec


def main():
    out = {"vis_seed": VIS_SEED, "runs": {}}
    for cfg in ("g1", "g2", "c1", "c2"):
        for vis_kind in ("ones", "normal"):
            print("running", cfg, vis_kind, flush=True)
            out["runs"][f"{cfg}_{vis_kind}"] = run(cfg, vis_kind)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
