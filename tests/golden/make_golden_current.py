"""Generate the golden fixtures of the variable-support path from the reference's own code.

Runs oracle/_ref/current/ref_driver_current (current/tConvolveMPI/Benchmark.cc compiled unmodified
by `make -C oracle ref-current` from the reference tree) and records, per run, the scalars of
meta.txt and the sha256, shape and float64 norm of every array (u, v, w, iu, iv, wplane, coff,
ssize, coff0, C, grid, outdata) in current.json.  The sha256 values pin bit-exact agreement.

Runs: every run type (0 continuum, 1 spectral, 2 nearest neighbour, 3 7x7, 4 87x87) on a fresh
object; run type 1 after run type 0 on the same object (tConvolveMPI's order,
current/tConvolveMPI/tConvolveMPI.cc:85-92: the generator state carries over); run type 1 with
setSort(1).  The reference visibilities are 1+0i (current/tConvolveMPI/Benchmark.cc:258-262).

Usage: python tests/golden/make_golden_current.py   (needs the reference tree)
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
DRIVER = os.path.join(REPO, "oracle", "_ref", "current", "ref_driver_current")
FILES = [("u", np.float64), ("v", np.float64), ("w", np.float64), ("iu", np.int32), ("iv", np.int32),
         ("wplane", np.int32), ("coff", np.int32), ("ssize", np.int32), ("coff0", np.int32),
         ("C", np.complex64), ("grid", np.complex64), ("outdata", np.complex64)]
RUNS = {"rt0": (0, 0, []), "rt1": (1, 0, []), "rt2": (2, 0, []), "rt3": (3, 0, []), "rt4": (4, 0, []),
        "rt1_after_rt0": (1, 0, [0]), "rt1_sorted": (1, 1, [])}


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run(run_type: int, sort: int, earlier: list) -> dict:
    with tempfile.TemporaryDirectory() as td:
        subprocess.run([DRIVER, "dump", str(run_type), str(sort), td] + [str(e) for e in earlier], check=True,
                       capture_output=True)
        meta = {}
        for line in open(os.path.join(td, "meta.txt")):
            k, v = line.split()
            meta[k] = float(v) if ("." in v or "e" in v) else int(v)
        arrs = {n: np.fromfile(os.path.join(td, f"{n}.bin"), dtype=t) for n, t in FILES}
    return {"run_type": run_type, "sort": sort, "earlier": earlier, "meta": meta,
            "sha256": {k: sha(a) for k, a in arrs.items()}, "shape": {k: list(a.shape) for k, a in arrs.items()},
            "norm": {k: float(np.linalg.norm(a.astype(np.complex128))) for k, a in arrs.items()
                     if a.dtype == np.complex64},
            "grid_nonzero": int(np.count_nonzero(arrs["grid"]))}


def main():
    out = {"runs": {}}
    for name, (rt, sort, earlier) in RUNS.items():
        print("running", name, flush=True)
        out["runs"][name] = run(rt, sort, earlier)
    with open(os.path.join(HERE, "current.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
