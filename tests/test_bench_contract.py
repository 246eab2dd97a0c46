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


def _bench():
    import importlib.util

    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(REPO, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_gpus_flag_starts_one_rank_per_gpu():
    """--gpus N runs N ranks: in this process for N = 1 or under torchrun with WORLD_SIZE = N,
    as N torchrun ranks when started plainly with N GPUs visible, and refuses what it cannot
    meet (more GPUs than visible, a WORLD_SIZE that disagrees)."""
    b = _bench()
    assert b.world_plan(1, {}, 0) == ("run", None)
    assert b.world_plan(1, {}, 8) == ("run", None)
    assert b.world_plan(4, {"WORLD_SIZE": "4"}, 0) == ("run", None)
    assert b.world_plan(2, {}, 8) == ("spawn", None)
    assert b.world_plan(8, {}, 8) == ("spawn", None)
    act, why = b.world_plan(2, {}, 1)
    assert act == "error" and "only 1 GPU" in why
    act, why = b.world_plan(2, {"WORLD_SIZE": "1"}, 0)
    assert act == "error" and "WORLD_SIZE=1" in why
    assert b.world_plan(0, {}, 8)[0] == "error"
    argv = b.spawn_argv(4, ["--gpus", "4", "--steps", "10", "--warmup", "3"], 29512)
    assert argv[1:4] == ["-m", "torch.distributed.run", "--nnodes=1"]
    assert "--nproc-per-node=4" in argv and "--master-addr=127.0.0.1" in argv and "--master-port=29512" in argv
    assert argv[argv.index(os.path.join(REPO, "bench.py")) + 1:] == ["--gpus", "4", "--steps", "10", "--warmup", "3"]


def test_gpus_beyond_visible_fails_loudly():
    """On a machine without enough GPUs (here: none), --gpus 2 exits non-zero with a message
    instead of running one rank and reporting n_gpus 1."""
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    env["CUDA_VISIBLE_DEVICES"] = ""
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--gpus", "2", "--steps", "1", "--warmup", "3"],
                       capture_output=True, text=True, timeout=300, cwd=REPO, env=env)
    assert r.returncode == 2
    assert "--gpus 2 but only 0 GPU(s) visible" in r.stderr
    assert r.stdout.strip() == ""
