"""The bench's reference arm on CPU: one JSON line with the keys its contract names, timed from
the reference's own gridKernel/degridKernel built from source (oracle/_ref; skipped where that
build is absent)."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

from conftest import REPO

REF_DRIVER = os.path.join(REPO, "oracle", "_ref", "c2", "ref_driver")


@pytest.mark.skipif(not os.path.exists(REF_DRIVER), reason="the reference's CPU path is not built here")
def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=REPO, check=True).stdout
    lines = [ln for ln in out.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("c2: 160000 samples x 1 chan, gSize 4096, wSize 33, support 64")


def test_warmup_below_three_is_refused():
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--warmup", "2"],
                       capture_output=True, text=True, timeout=120, cwd=REPO)
    assert r.returncode == 2
