#!/usr/bin/env python
"""Benchmark: tConvolve W-projection gridding + degridding on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--form c64|r32|...]

Workload: the reference's default problem (attic/tConvolveMPI/Benchmark.h:39-46): 160000 samples,
33 w-planes, 4096^2 grid, 5-wavelength cells, support 64 (129^2 footprints), u,v,w from the
reference generator, N(0,1) complex64 visibilities.  One step = one binning plan (device sort of
this batch's samples) + one gridding pass + one degridding pass (2 x 2.66e9 updates).

Multi-GPU: one process per GPU, each an independent replica of the workload (the reference's MPI
ranks are replicas that only meet at barriers); value = all ranks' updates / max-over-ranks time.

Prints one JSON line (rank 0).  The `reference` arm times the reference's own CPU code
(attic/tConvolveMPI/Benchmark.cc compiled from source into oracle/_ref) on the host's cores.
"""
from __future__ import annotations

import argparse
import ctypes
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "askap-benchmarks_b200"))

from tconvolve.workload import PROBLEMS, normal_vis  # noqa: E402

METRIC = "grid+degrid updates/s at rel-L2<=1e-5"
UNIT = "updates/s"
VIS_SEED = 1234
ALG_BYTES = {"grid": 24, "degrid": 16}  # per update: C 8 + grid read 8 (+ grid write 8)
FALLBACK_HBM_GBS = 6650.0
L2_FLUSH_BYTES = 512 << 20
REL_L2_BAR = 1e-5  # the metric's bar: relative L2 against the reference's FP32 result (and FP64)
REF_DRIVER = os.path.join(REPO, "oracle", "_ref", "c2", "ref_driver")
REF_DRIVER_CURRENT = os.path.join(REPO, "oracle", "_ref", "current", "ref_driver_current")
REF_DRIVER_HOGBOM = os.path.join(REPO, "oracle", "_ref", "hogbom", "ref_driver_hogbom")


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--workload", default="c2", choices=sorted(PROBLEMS))
    p.add_argument("--form", default="r32",
                   help="table storage form of the headline: r32 (default; the attic table is real, "
                        "so this is the plain FP32 result bit for bit) or c64 (the plain complex64 "
                        "table), or a reduced form for study; c64 is always measured beside it")
    p.add_argument("--path", default="direct", choices=["direct", "paired", "tma"], help="kernel family")
    p.add_argument("--degrid", default="tiles", choices=["tiles", "anchor"],
                   help="degridding kernel on the direct path")
    p.add_argument("--no-tune", action="store_true", help="default tile shape and plane groups, no autotuning")
    p.add_argument("--tuning", default=None,
                   help="tile rows,group MiB,grid split,degrid split for every measured form instead of "
                        "autotuning (e.g. 16,64,0,128)")
    p.add_argument("--no-batched", action="store_true", help="skip the 64-job batched measurement")
    p.add_argument("--no-serving", action="store_true", help="skip the serving (Poisson arrivals) measurement")
    p.add_argument("--serve-seconds", type=float, default=2.0, help="arrival window per serving rate")
    p.add_argument("--no-hogbom", action="store_true", help="skip the Hogbom CLEAN (minor cycle) measurement")
    p.add_argument("--no-major", action="store_true", help="skip the imaging major cycle measurement")
    p.add_argument("--no-current", action="store_true",
                   help="skip the variable-support (current/tConvolveMPI) continuum and spectral measurement")
    p.add_argument("--bands", action="store_true",
                   help="also time the headline job split into row bands over the ranks (tconvolve.bands: "
                        "halo rows exchanged over NCCL; strong scaling)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-precision", action="store_true",
                   help="skip the parity gate of the headline (the line then states no precision)")
    p.add_argument("--cpu-seconds", type=float, default=4.0, help="target wall time of the CPU sample")
    return p.parse_args()


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ------------------------------------------------------------------------------------------------
# CPU reference timing (oracle/_ref: the reference's Benchmark.cc built from source)
# ------------------------------------------------------------------------------------------------
def run_reference_cpu(threads: int, per_thread: int, steps: int, warmup: int):
    if not os.path.exists(REF_DRIVER):
        raise RuntimeError(f"reference build missing: {REF_DRIVER}")
    out = subprocess.run([REF_DRIVER, "time", str(threads), str(per_thread), str(steps), str(warmup)],
                         check=True, capture_output=True, text=True).stdout
    rates, step_s = [], []
    for line in out.splitlines():
        if line.startswith("step "):
            f = line.split()
            g, d, u = float(f[3]), float(f[5]), float(f[7])
            rates.append(2 * u / (g + d))
            step_s.append(g + d)
    return rates, step_s


def run_reference_cpu_current(run_type: int, threads: int, steps: int, max_samples: int):
    """The reference's current/tConvolveMPI Benchmark (oracle/_ref/current) on the host cores: one
    object per thread (as one per MPI rank), each over the first max_samples samples."""
    if not os.path.exists(REF_DRIVER_CURRENT):
        raise RuntimeError(f"reference build missing: {REF_DRIVER_CURRENT}")
    out = subprocess.run([REF_DRIVER_CURRENT, "time", str(run_type), str(threads), str(steps), str(max_samples)],
                         check=True, capture_output=True, text=True, timeout=600).stdout
    rates = []
    for line in out.splitlines():
        if line.startswith("step "):
            f = line.split()
            g, d, px = float(f[3]), float(f[5]), float(f[7])
            rates.append({"grid_px_s": px / g, "degrid_px_s": px / d, "updates_per_s": 2 * px / (g + d)})
    return rates


def cpu_sample_size(threads: int, seconds: float) -> int:
    # about 3e8 updates/s per core for the reference loop; 16641 updates per sample per pass, 2 passes
    per = int(seconds * 3e8 / (2 * 16641))
    return max(200, min(per, 160000))


def workload_name(name: str, prob, support: int) -> str:
    """The workload as both arms name it in config.workload."""
    return (f"{name}: {prob.n_samples} samples x {prob.n_chan} chan, gSize {prob.g_size}, wSize {prob.w_size}, "
            f"support {support} ({2 * support + 1}^2 footprint), cellSize {prob.cell_size}")


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = host_threads()
    per_thread = cpu_sample_size(threads, 1.0)
    rates, step_s = run_reference_cpu(threads, per_thread, args.steps, args.warmup)
    value = statistics.mean(rates)
    prob = PROBLEMS[args.workload]
    sample = (f"{threads} thread replicas x first {per_thread} samples of the {args.workload} workload, "
              f"reference gridKernel then degridKernel per step (tConvolveMT-style)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * statistics.mean(step_s), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (reference generator, vis = 1+0i)",
        "config": {"workload": workload_name(args.workload, prob, prob.support()),
                   "form": "reference CPU (std::complex<float>)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------------------------
# clocks during the timed region
# ------------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        # the first sample is written once nvidia-smi is up: start timing after its start-up, which
        # would otherwise compete with the host thread that enqueues the timed launches
        t0 = time.time()
        while time.time() - t0 < 5.0 and os.path.getsize(self.path) == 0 and self.proc.poll() is None:
            time.sleep(0.02)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait(timeout=10)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                smax.append(float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_hbm_peak():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def ncu_l2_bytes_per_update(kernel: str):
    """L2-to-SM bytes per update of one pass from the committed ncu summary (profiles/), or None."""
    path = os.path.join(REPO, "profiles", f"{kernel}_c2_traffic.txt")
    try:
        for line in open(path):
            if line.startswith("l2_to_sm_bytes_per_update:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def ncu_traffic(kernel: str):
    """DRAM bytes per launch from the committed ncu summary (profiles/), or None."""
    path = os.path.join(REPO, "profiles", f"{kernel}_c2_traffic.txt")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


# ------------------------------------------------------------------------------------------------
# B200 arm
# ------------------------------------------------------------------------------------------------
def b200_arm(args):
    import torch
    import torch.distributed as dist

    import tconvolve
    from tconvolve import replicas
    from tconvolve._lib import check, lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180),
                                device_id=torch.device("cuda", local))
    prob = PROBLEMS[args.workload]
    form = tconvolve.CTYPE_BY_NAME[args.form]
    n = prob.n_data()
    stream = torch.cuda.Stream()  # a non-default stream: every launch and event below goes to it
    torch.cuda.set_stream(stream)

    b = tconvolve.Benchmark(**prob.kwargs(), device=local)
    b.set_stream(stream.cuda_stream)
    b.set_path(args.path)
    b.init()
    vis = normal_vis(n, VIS_SEED)
    b.set_data(vis)
    tunings = {}
    if args.tuning and args.path == "direct":
        fixed = (tuple(int(x) for x in args.tuning.split(",")) + (0, 0, 0, 0))[:4]
        for name in dict.fromkeys([args.form, "c64"]):
            tunings[name] = (fixed, None)
        b.set_ctype(form)
        b.set_tuning(*fixed)
    elif not args.no_tune and args.path == "direct":
        # autotuned tile shape and plane groups for each form measured (tcv_tune on this problem)
        if args.form != "c64":
            b.set_ctype("c64")
            tunings["c64"] = b.tune(3)
        b.set_ctype(form)
        tunings[args.form] = b.tune(3)
    elif form != tconvolve.C64:
        b.set_ctype(form)
    if world > 1 and tunings:
        # every replica takes rank 0's choices: a different gridding split would change the order
        # of the sums, and the replicas' results are compared bit for bit
        tunings = replicas.rank0_tunings(tunings, device="cuda")
        b.set_tuning(*tunings[args.form][0][:4])
    b.sync()
    bufs = b.device_buffers()
    support = b.getSupport()
    updates = b.updates_per_pass()
    c_len = b.c_len
    L = lib()
    TcvTuning = tconvolve._lib.TcvTuning
    tuning = {"t": TcvTuning(*(tunings[args.form][0] if args.form in tunings else (16, 32)))}
    # one workspace for every plan the bench builds (each measured form's tuning)
    wbytes = max(L.tcv_plan_workspace_bytes_tuned(n, support, prob.g_size, c_len, ctypes.byref(TcvTuning(*t)))
                 for t in [(16, 32, 0, 0)] + [v[0] for v in tunings.values()])
    work = torch.empty(wbytes, dtype=torch.uint8, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    sp = ctypes.c_void_p(stream.cuda_stream)
    P = ctypes.c_void_p

    dvariant = {"tiles": tconvolve._lib.DEGRID_TILES, "anchor": tconvolve._lib.DEGRID_ANCHOR}[args.degrid]

    PASS_BIN, PASS_GRID, PASS_DEGRID = tconvolve._lib.PASS_BIN, tconvolve._lib.PASS_GRID, tconvolve._lib.PASS_DEGRID

    def make_step(tab, iu, iv, coff, data, grid, out, passes_list):
        """A persistent plan over the arrays (device pointers) with table `tab`, and its passes
        captured as CUDA graphs (tcv_graph_capture), one graph per entry of passes_list: the
        binning, gridding and degridding all run at every launch.  Returns (run(evs), eager(),
        close()): run launches the graphs in order, recording evs[0] before and evs[k+1] after
        graph k; eager makes the same passes as plain calls (for counting their kernels)."""
        plan = ctypes.c_void_p()
        check(L.tcv_plan_build_tuned(ctypes.byref(plan), P(iu), P(iv), P(coff), n, support, prob.g_size, c_len,
                                     ctypes.byref(tuning["t"]), P(work.data_ptr()), wbytes, sp), "plan")
        check(L.tcv_plan_set_degrid_variant(plan, dvariant), "degrid variant")
        graphs = []
        for passes in passes_list:
            gph = ctypes.c_void_p()
            check(L.tcv_graph_capture(ctypes.byref(gph), plan, passes, P(iu), P(iv), P(coff), P(data),
                                      P(tab.c_active), tab.c_type, tab.c_scale, P(grid), P(out)), "capture")
            graphs.append(gph)

        def run(evs=None):
            if evs:
                evs[0].record(stream)
            for k, gph in enumerate(graphs):
                check(L.tcv_graph_launch(gph, sp), "graph launch")
                if evs:
                    evs[k + 1].record(stream)

        def eager():
            cs = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)  # the capture stream too
            check(L.tcv_plan_bin(plan, P(iu), P(iv), P(coff), cs), "bin")
            check(L.tcv_plan_grid(plan, P(data), P(tab.c_active), tab.c_type, tab.c_scale, P(grid), cs), "grid")
            check(L.tcv_plan_degrid(plan, P(grid), P(tab.c_active), tab.c_type, tab.c_scale, P(out), cs), "degrid")

        def close():
            for gph in graphs:
                L.tcv_graph_destroy(gph)
            L.tcv_plan_destroy(plan)

        return run, eager, close

    def timed(tab, steps, count=False):
        """Timed steps with table `tab` (a tcv_device_buffers): binning, gridding and degridding
        passes, each one graph launch, events between them."""
        run, eager, close = make_step(tab, tab.iu, tab.iv, tab.coff, tab.data, tab.grid, tab.outdata,
                                      (PASS_BIN, PASS_GRID, PASS_DEGRID))
        counted = None
        if count:
            eager()
            torch.cuda.synchronize()
            counted = count_step_kernels(torch, eager)  # kernels of one step, from a capture of it
        for _ in range(args.warmup):
            run()
            flush.zero_()
        torch.cuda.synchronize()
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(steps)]
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(steps):
            run(evs[k])
            flush.zero_()  # L2 flush between timed steps (outside the events)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        wall = time.perf_counter() - t0
        close()
        return ([e[0].elapsed_time(e[1]) for e in evs], [e[1].elapsed_time(e[2]) for e in evs],
                [e[2].elapsed_time(e[3]) for e in evs], [e[0].elapsed_time(e[3]) for e in evs], wall, counted)

    gpu_uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    clocks = ClockSampler(gpu_uuid)
    clocks.start()
    plan_ms, grid_ms, degrid_ms, step_ms, t_wall, launches_per_step = timed(bufs, args.steps, count=True)
    plain = None
    if args.form != "c64":
        # the plain form (complex64 table, the reference's storage) measured beside the chosen one
        b.set_ctype("c64")
        chosen_t = tuning["t"]
        if "c64" in tunings:
            tuning["t"] = TcvTuning(*tunings["c64"][0])
        p_plan, p_grid, p_degrid, p_step, _, _ = timed(b.device_buffers(), args.steps)
        tuning["t"] = chosen_t
        b.set_ctype(form)
        bufs = b.device_buffers()
        plain = {"form": "c64", "value": world * 2 * updates / (statistics.mean(p_step) * 1e-3),
                 "grid_ms": statistics.mean(p_grid), "degrid_ms": statistics.mean(p_degrid),
                 "plan_ms": statistics.mean(p_plan),
                 "tuning": tunings["c64"][0] if "c64" in tunings else (16, 32)}

    # e2e: the same step through the C ABI with host buffers: H2D of the batch's samples from
    # pinned memory, plan, grid, degrid, D2H of the degridded visibilities, every step
    iu_h, iv_h, co_h = b.offsets()
    h_vis = torch.from_numpy(vis).pin_memory()
    h_iu = torch.from_numpy(iu_h).pin_memory()
    h_iv = torch.from_numpy(iv_h).pin_memory()
    h_co = torch.from_numpy(co_h).pin_memory()
    h_out = torch.empty(n, dtype=torch.complex64).pin_memory()
    d_vis = torch.empty(n, dtype=torch.complex64, device="cuda")
    d_iu = torch.empty(n, dtype=torch.int32, device="cuda")
    d_iv = torch.empty_like(d_iu)
    d_co = torch.empty_like(d_iu)
    d_out = torch.empty(n, dtype=torch.complex64, device="cuda")

    d_vis.copy_(h_vis)
    d_iu.copy_(h_iu)
    d_iv.copy_(h_iv)
    d_co.copy_(h_co)
    e2e_run, _, e2e_close = make_step(bufs, d_iu.data_ptr(), d_iv.data_ptr(), d_co.data_ptr(), d_vis.data_ptr(),
                                      bufs.grid, d_out.data_ptr(), (PASS_BIN | PASS_GRID | PASS_DEGRID,))

    def e2e_step():
        d_vis.copy_(h_vis, non_blocking=True)
        d_iu.copy_(h_iu, non_blocking=True)
        d_iv.copy_(h_iv, non_blocking=True)
        d_co.copy_(h_co, non_blocking=True)
        e2e_run()
        h_out.copy_(d_out, non_blocking=True)

    for _ in range(args.warmup):
        e2e_step()
        flush.zero_()
    torch.cuda.synchronize()
    e2e_ms = []
    for _ in range(max(args.steps // 4, 3)):
        a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        e2e_step()
        z.record(stream)
        z.synchronize()  # the result is on the host when the step ends
        e2e_ms.append(a.elapsed_time(z))
        flush.zero_()
    torch.cuda.synchronize()
    e2e_close()
    clk = clocks.stop()
    if int(torch.count_nonzero(torch.isnan(torch.view_as_real(h_out)))) != 0:
        raise RuntimeError("non-finite degridded output")

    # Parity gate of the headline: one more pass of each timed plan (same graphs, table form and
    # tuning) into a zeroed grid, compared on rank 0 with the reference's FP32 result and the
    # FP64 oracle; the line carries no value when either measured form is off by more than 1e-5.
    def one_pass(tab, t):
        saved = tuning["t"]
        tuning["t"] = t
        run, _, close = make_step(tab, tab.iu, tab.iv, tab.coff, tab.data, tab.grid, tab.outdata,
                                  (PASS_BIN, PASS_GRID, PASS_DEGRID))
        tuning["t"] = saved
        b.zero_grid()
        run()
        torch.cuda.synchronize()
        res = (b.grid(), b.outdata())
        close()
        return res

    results = {args.form: one_pass(bufs, tuning["t"])}
    if plain is not None:
        b.set_ctype("c64")
        results["c64"] = one_pass(b.device_buffers(), TcvTuning(*plain["tuning"]))
        b.set_ctype(form)
        bufs = b.device_buffers()
    precision = None
    if rank == 0 and not args.no_precision:
        t0 = time.perf_counter()
        grid32, out32, grid64, out64, pins, rel_l2, threads = oracle_reference(prob, vis, args.workload)
        precision = {"bar": REL_L2_BAR, "reference": "oracle restatement of the reference's FP32 gridKernel/degridKernel "
                                                      "on the same samples" +
                                                      (", sha256-identical to the reference's own output"
                                                       if pins and all(pins.values()) else ""),
                     "reference_pinned": pins, "forms": {}, "check_s": None, "threads": threads}
        for name, (g_res, o_res) in results.items():
            precision["forms"][name] = {
                "grid_rel_l2": rel_l2(g_res, grid32), "degrid_rel_l2": rel_l2(o_res, out32),
                "grid_rel_l2_fp64": rel_l2(g_res, grid64), "degrid_rel_l2_fp64": rel_l2(o_res, out64)}
        precision["reference_vs_fp64"] = {"grid_rel_l2": rel_l2(grid32, grid64), "degrid_rel_l2": rel_l2(out32, out64)}
        precision["check_s"] = time.perf_counter() - t0
        worst = max(max(f.values()) for f in precision["forms"].values())
        precision["pass"] = bool(worst <= REL_L2_BAR and (not pins or all(pins.values())))
    del results

    # max over ranks of the device time; replicas of one problem must agree bit for bit
    mean_step = statistics.mean(step_ms)
    e2e_mean = statistics.mean(e2e_ms)
    replicas_agree = True
    if world > 1:
        mean_step, e2e_mean, t_wall = replicas.max_over_ranks([mean_step, e2e_mean, t_wall], device="cuda")
        replicas_agree = replicas.cross_check(replicas.checksum(h_out.numpy()), device="cuda")
    value = world * 2 * updates / (mean_step * 1e-3)
    e2e_value = world * 2 * updates / (e2e_mean * 1e-3)

    g_ms, d_ms = statistics.mean(grid_ms), statistics.mean(degrid_ms)
    dom = "grid" if g_ms >= d_ms else "degrid"
    dom_ms = max(g_ms, d_ms)
    peak, peak_kind = measured_hbm_peak()
    achieved = ALG_BYTES[dom] * updates / (dom_ms * 1e-3) / 1e9
    traffic = ncu_traffic(dom)
    kname = {("grid", "tma"): "pipe_kernel<gridding> (TMA pipeline)",
             ("degrid", "tma"): "pipe_kernel<degridding> + slot_reduce_kernel (TMA pipeline)",
             ("grid", "paired"): "pair_tile_kernel<gridding>",
             ("degrid", "paired"): "pair_tile_kernel<degridding> + slot_reduce_kernel",
             ("grid", "direct"): "grid_tile_kernel",
             ("degrid", "direct"): ("degrid_tile_kernel + slot_reduce_kernel" if args.degrid == "tiles"
                                    else "degrid_staged_kernel")}[(dom, args.path)]

    l2_ceiling = l2_table_ceiling(torch, stream, updates, g_ms, d_ms, args.form) if args.path == "direct" else None
    bands = None
    if args.bands and args.path == "direct":
        t = tuning["t"]
        bands = bands_section(args, torch, stream, world, rank, prob, support, c_len, (iu_h, iv_h, co_h), vis,
                              b.C(), form, (t.tile_rows, t.group_mib, t.split, t.degrid_split), updates, flush)

    # the other workloads run after the headline's context is released
    batched = serving = current = hogbom = major = None
    if not (args.no_batched and args.no_serving and args.no_current and args.no_hogbom and args.no_major):
        b.close()
        torch.cuda.empty_cache()
    if not args.no_batched:
        batched = batched_section(args, torch, stream, world)
        torch.cuda.empty_cache()
    if not args.no_serving:
        serving = serving_section(args, local)
    if not args.no_current:
        current = current_section(args, torch, world)
        torch.cuda.empty_cache()
    if not args.no_hogbom and world == 1:
        hogbom = hogbom_section(args, torch)
        torch.cuda.empty_cache()
    if not args.no_major and world == 1:
        major = major_section(args, torch)
        torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args)

    rc = 0
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mean_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": f"synthetic: reference generator u,v,w (seed 0); N(0,1) complex64 visibilities "
                    f"(PCG64 seed {VIS_SEED})",
            "config": {"workload": workload_name(args.workload, prob, support),
                       "form": (f"{args.form} (chosen form: real parts of the reference's table, whose "
                                "imaginary parts are zero; bit-identical to the plain c64 result)"
                                if args.form == "r32" else args.form),
                       "path": args.path, "degrid": args.degrid,
                       "tuning": {"tile_rows": tuning["t"].tile_rows, "group_mib": tuning["t"].group_mib,
                                  "split": tuning["t"].split, "degrid_split": tuning["t"].degrid_split,
                                  "chosen_by": ("fixed (--tuning)" if args.tuning else "autotuner (tcv_tune)")
                                  if tunings else "default"},
                       "parallelism": f"replicas x{world}",
                       "l2": f"{L2_FLUSH_BYTES >> 20} MiB buffer written between timed steps",
                       "step": ("binning + gridding pass + degridding pass, every step; each pass one CUDA "
                                "graph launch (tcv_graph_capture) on a persistent plan, events between them"),
                       "e2e_step": ("H2D of the samples (data, iu, iv, cOffset) from pinned memory, one graph "
                                    "launch of the three passes, D2H of the degridded samples")},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": kname,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback 6650 GB/s",
                         "alg_bytes_per_update": ALG_BYTES[dom], "launch_ms": dom_ms,
                         "achieved_basis": ("model bytes, not DRAM: the reference loop's bytes per update "
                                            "(table entry, grid point read and written) x updates / launch time"),
                         "traffic_source": ("static: dram__bytes_read.sum + dram__bytes_write.sum of one pass from "
                                            "the ncu capture summarised in profiles/, not measured in this run"),
                         "reading": ("frac above 1: the reference loop's bytes per update are served from "
                                     "registers (the grid tile) and L2 (the table's plane group); DRAM moves "
                                     "`traffic` bytes per launch, so HBM does not bind; the binding resource is "
                                     "the L2-to-SM table stream (`binding`, `l2_table_ceiling`)"),
                         "binding": "l2_table_stream",
                         "l2_to_sm_bytes_per_update": ncu_l2_bytes_per_update(dom),
                         "l2_table_ceiling": l2_ceiling},
            "kernels": {"plan_ms": statistics.mean(plan_ms), "grid_ms": g_ms, "degrid_ms": d_ms,
                        "grid_alg_GBps": ALG_BYTES["grid"] * updates / (g_ms * 1e-3) / 1e9,
                        "degrid_alg_GBps": ALG_BYTES["degrid"] * updates / (d_ms * 1e-3) / 1e9,
                        "grid_updates_per_s": updates / (g_ms * 1e-3),
                        "degrid_updates_per_s": updates / (d_ms * 1e-3)},
            "precision": precision,
            "plain_form": plain,
            "batched": batched,
            "serving": serving,
            "current": current,
            "hogbom": hogbom,
            "major": major,
            "bands": bands,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": n * (8 + 4 * 3),
                    "d2h_bytes_per_step": n * 8, "ms_per_step": e2e_mean,
                    "note": ("the grid stays resident on the device between passes (the degridded samples "
                             "come back each step); a caller that also needs the gridded image on the host "
                             f"adds a D2H of {prob.g_size * prob.g_size * 8} bytes per step")},
            "gpu_launches": launches_per_step * args.steps if launches_per_step else None,
            "launches_per_step": launches_per_step,
            "wall_s_timed_loop": t_wall,
            "replicas_agree": replicas_agree,
            "clocks": clk,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        if precision is not None and not precision["pass"]:
            # the metric is quoted at rel-L2 <= 1e-5: a result outside it has no value
            line["value"] = None
            line["e2e"]["value"] = None
            line["parity_failed"] = "a measured form is off the reference by more than 1e-5 (see precision)"
            rc = 3
        print(json.dumps(line), flush=True)
    if args.no_batched and args.no_serving and args.no_current and args.no_hogbom and args.no_major:
        b.close()  # not released above
    if world > 1:
        dist.destroy_process_group()
    return rc


def bands_section(args, torch, stream, world, rank, prob, support, c_len, offsets, vis, c64_h, form, tuning, updates,
                  flush):
    """The headline job split into row bands over the ranks (tconvolve.bands): rank r starts with
    the r-th contiguous share of the samples, the set-up moves each sample to the rank that owns
    its footprint's centre row, and a step is one gridding pass (halo rows added into their
    owners') and one degridding pass (halo rows fetched, values returned to the ranks that hold
    those samples) of the whole job.  Device time of a step, max over ranks; the job is the same at
    every N (strong scaling).  Checked once against one GPU's plan over all samples."""
    import torch.distributed as dist

    import tconvolve
    from tconvolve import raw, replicas
    from tconvolve.bands import BandJob, CudaBandOps, DistComm, SoloComm

    iu_h, iv_h, co_h = offsets
    n, g = iu_h.size, prob.g_size
    a, e = rank * n // world, (rank + 1) * n // world

    def dev(x):
        return torch.from_numpy(np.ascontiguousarray(x)).cuda()

    c64 = dev(c64_h)
    tab, scale = (c64, 1.0) if form == tconvolve.C64 else raw.convert_c(c64, form)[:2]
    t0 = time.perf_counter()
    job = BandJob(dev(vis[a:e]), dev(iu_h[a:e]), dev(iv_h[a:e]), dev(co_h[a:e]), support, g, c_len,
                  comm=DistComm() if world > 1 else SoloComm(), ops=CudaBandOps(), tuning=tuning)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    grid = torch.zeros(g * g, dtype=torch.complex64, device="cuda")
    out = torch.empty(e - a, dtype=torch.complex64, device="cuda")

    # one pass of each against one GPU's plan over every sample (the band rows of the grid; the
    # degridded values of this rank's share)
    job.grid(grid, tab, form, scale)
    job.degrid(grid, tab, form, out, scale)
    plan = raw.Plan(dev(iu_h), dev(iv_h), dev(co_h), support, g, c_len, tuning=tuning)
    one = torch.zeros(g * g, dtype=torch.complex64, device="cuda")
    plan.grid(dev(vis), tab, form, one, scale)
    one_out = torch.empty(n, dtype=torch.complex64, device="cuda")
    plan.degrid(one, tab, form, one_out, scale)
    r0, r1 = job.band
    sums = torch.stack([(grid[r0 * g:r1 * g] - one[r0 * g:r1 * g]).abs().double().pow(2).sum(),
                        one[r0 * g:r1 * g].abs().double().pow(2).sum(),
                        (out - one_out[a:e]).abs().double().pow(2).sum(),
                        one_out[a:e].abs().double().pow(2).sum()])
    if world > 1:
        dist.all_reduce(sums)
    sums = sums.cpu().tolist()
    del plan, one, one_out

    steps = max(args.steps // 2, 5)
    for _ in range(args.warmup):
        job.grid(grid, tab, form, scale)
        job.degrid(grid, tab, form, out, scale)
        flush.zero_()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = []
    for _ in range(steps):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record(stream)
        job.grid(grid, tab, form, scale)
        ev[1].record(stream)
        job.degrid(grid, tab, form, out, scale)
        ev[2].record(stream)
        flush.zero_()
        ms.append((ev[0], ev[1], ev[2]))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    g_ms = statistics.mean(x[0].elapsed_time(x[1]) for x in ms)
    d_ms = statistics.mean(x[1].elapsed_time(x[2]) for x in ms)
    step_ms = statistics.mean(x[0].elapsed_time(x[2]) for x in ms)
    mine = [float(job.n_band), float(r1 - r0)]
    if world > 1:
        step_ms, g_ms, d_ms, setup_s = replicas.max_over_ranks([step_ms, g_ms, d_ms, setup_s], device="cuda")
        every = torch.zeros(2 * world, dtype=torch.float64, device="cuda")
        every[2 * rank:2 * rank + 2] = torch.tensor(mine, dtype=torch.float64)
        dist.all_reduce(every)
        every = every.cpu().tolist()
    else:
        every = mine
    return {"value": 2 * updates / (step_ms * 1e-3), "unit": UNIT, "ranks": world, "scaling": "strong",
            "ms_per_step": step_ms, "grid_ms": g_ms, "degrid_ms": d_ms, "steps": steps,
            "rows": job.rows, "samples_per_rank": [int(x) for x in every[0::2]],
            "setup_s": setup_s, "tuning": list(tuning),
            "grid_rel_l2_vs_one_gpu": (sums[0] / sums[1]) ** 0.5 if sums[1] else None,
            "degrid_rel_l2_vs_one_gpu": (sums[2] / sums[3]) ** 0.5 if sums[3] else None,
            # halo rows: each interior band edge, both ways, after gridding and before degridding;
            # the degridded values of samples that changed rank (at most all of them)
            "exchange_bytes_per_step_at_most": 2 * 2 * (world - 1) * support * g * 8 + n * 8,
            "setup_exchange_bytes_at_most": n * 20}


def batched_section(args, torch, stream, world):
    """The batched workload: 64 jobs (channels / Taylor terms) with sample counts log-uniform in
    [1e4, 4e5] and grids of 2048^2 or 4096^2 sharing the 33-plane table, binned by one plan and run
    as one captured CUDA graph (bin + grid + degrid of every job) per step, with the tile shape and
    plane groups from the autotuner.  The grids (5 GB) are far larger than L2.  Measured for the
    chosen form, the plain c64 form and the bf16 form; the bf16 result's relative L2 distance from
    the plain result, and every form's distance from the FP64 oracle on three of the jobs (the
    smallest of each grid size and the median job), are measured here."""
    import tconvolve
    from tconvolve import raw
    from tconvolve._lib import PASS_BIN, PASS_DEGRID, PASS_GRID
    from tconvolve.batch import Batch, autotune, make_problem
    from tconvolve.workload import batch_sizes

    sizes = batch_sizes(64, seed=0)
    p = make_problem(sizes, vis_seed=VIS_SEED)
    s2 = (2 * p["support"] + 1) ** 2
    torch.cuda.synchronize()
    res = {"workload": "64 jobs, n log-uniform in [1e4, 4e5] (PCG64 seed 0), gSize 2048 or 4096, wSize 33, "
                       "support 64, one shared table",
           "samples": p["total"], "step": "one CUDA graph launch: bin + grid + degrid of all jobs",
           "forms": {}}
    outs = {}
    rejected = None
    # the FP64 oracle on a few jobs (the smallest of each grid size and the median job): every form's
    # grid and degridded samples there against it
    fp64 = {}
    first = np.concatenate([[0], np.cumsum([n for n, _ in sizes])]).astype(np.int64)
    check_jobs = None
    if not args.no_precision:
        order_n = sorted(range(len(sizes)), key=lambda j: sizes[j][0])
        check_jobs = sorted({min((j for j in order_n if sizes[j][1] == 2048), key=lambda j: sizes[j][0]),
                             min((j for j in order_n if sizes[j][1] == 4096), key=lambda j: sizes[j][0]),
                             order_n[len(order_n) // 2]})
    for name in dict.fromkeys([args.form, "c64", "rbf16"]):
        ct = tconvolve.CTYPE_BY_NAME[name]
        c, scale, _ = (p["c64"], 1.0, 0) if ct == tconvolve.C64 else raw.convert_c(p["c64"], ct)
        t0 = time.perf_counter()
        best, best_ms, report = autotune(sizes, p["iu"], p["iv"], p["coff"], p["data"], c, ct, p["support"], scale,
                                         reps=3, stream=stream)
        tune_s = time.perf_counter() - t0
        grids = [torch.zeros(g * g, dtype=torch.complex64, device="cuda") for _, g in sizes]
        bt = Batch(sizes, grids, p["iu"], p["iv"], p["coff"], p["support"], p["c_len"], tuning=best, stream=stream)
        if rejected is None:
            rejected = bt.rejected(stream)
        out = torch.empty(p["total"], dtype=torch.complex64, device="cuda")
        graph = bt.capture(PASS_BIN | PASS_GRID | PASS_DEGRID, p["data"], c, ct, vis=out, c_scale=scale)
        for _ in range(max(args.warmup, 3)):
            graph.launch(stream)
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        k = 5
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(k + 1)]
        ev[0].record(stream)
        for i in range(k):
            graph.launch(stream)
            ev[i + 1].record(stream)
        torch.cuda.synchronize()
        ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(k)]
        step_ms = statistics.mean(ms)
        if world > 1:
            from tconvolve import replicas
            step_ms = replicas.max_over_ranks([step_ms], device="cuda")[0]
        # one more pass into zeroed grids for the comparison of forms
        for gr in grids:
            gr.zero_()
        graph.launch(stream)
        torch.cuda.synchronize()
        outs[name] = out.clone()
        if check_jobs is not None:
            fp64[name] = [(grids[j].cpu().numpy(), out[first[j]:first[j] + sizes[j][0]].cpu().numpy())
                          for j in check_jobs]
        upd = (p["total"] - rejected) * s2
        res["forms"][name] = {"value": world * 2 * upd / (step_ms * 1e-3), "unit": UNIT, "ms_per_step": step_ms,
                              "steps": k, "tuning": list(best), "autotune_s": tune_s,
                              "candidates": [[list(t), m] for t, m in report]}
        graph.close()
        bt.close()
        del grids, out
        torch.cuda.empty_cache()
    if "rbf16" in outs and "c64" in outs:
        a, r = outs["rbf16"], outs["c64"]
        res["forms"]["rbf16"]["rel_l2_vs_plain"] = float(torch.linalg.vector_norm(a - r) /
                                                         torch.linalg.vector_norm(r))
    if check_jobs is not None:
        res["precision_vs_fp64"] = batched_fp64_errors(p, sizes, first, check_jobs, fp64)
    res["rejected_samples"] = rejected
    res["rejected_note"] = ("samples whose footprint (rows iv..iv+128) leaves a 2048 grid; skipped and counted, "
                            "not in the update count")
    return res


def batched_fp64_errors(p, sizes, first, jobs, results):
    """Relative L2 of each form's grid and degridded samples against the FP64 oracle, on the
    given jobs (their in-bounds samples; the reference would write out of bounds for the others):
    the oracle's double gridding and degridding with the real double table of the same geometry
    and the reference's normalisation."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as orc

    threads = host_threads()
    cfg = orc.Config(160000, 33, 1, 4096, 5.0)
    _, c_f64, support, _, _, _ = orc.init_c(cfg, want_f64=True)
    s = 2 * support + 1
    iu, iv, co, data = (p[k].cpu().numpy() for k in ("iu", "iv", "coff", "data"))
    out = {"jobs": [{"job": int(j), "samples": int(sizes[j][0]), "g_size": int(sizes[j][1])} for j in jobs],
           "forms": {name: {"grid_rel_l2": [], "degrid_rel_l2": []} for name in results}}
    for k, j in enumerate(jobs):
        g = int(sizes[j][1])
        sl = slice(int(first[j]), int(first[j] + sizes[j][0]))
        keep = (iu[sl] - support >= 0) & (iu[sl] - support + s <= g) & (iv[sl] >= 0) & (iv[sl] + s <= g)
        a = [np.ascontiguousarray(x[sl][keep]) for x in (iu, iv, co)]
        ref = np.zeros(g * g, np.complex128)
        orc.grid_f64(data[sl][keep].astype(np.complex128), support, c_f64, a[2], a[0], a[1], ref, g, threads)
        ref_o = orc.degrid_f64(ref, g, support, c_f64, a[2], a[0], a[1], threads)
        for name, per_job in results.items():
            grid_j, out_j = per_job[k]
            out["forms"][name]["grid_rel_l2"].append(orc.rel_l2(grid_j, ref))
            out["forms"][name]["degrid_rel_l2"].append(orc.rel_l2(out_j[keep], ref_o))
    for e in out["forms"].values():
        e["grid_rel_l2_max"] = max(e["grid_rel_l2"])
        e["degrid_rel_l2_max"] = max(e["degrid_rel_l2"])
    return out


def serving_section(args, device):
    """Serving: Poisson arrivals of gridding and degridding requests (half each) of 16000 samples
    on the 1024^2-grid, 9-plane, 5 arcsec problem (32.4e6 updates each) over 64 resident grids,
    under a 150 GB device-memory budget; latency is submission to result-ready, measured by the
    server.  The chosen form runs at 50, 100, 200 and 500 requests/s (light load: batches of about
    one request) and at a saturating open-loop rate and a burst of 256 requests (continuous
    batching: batches of many requests); the bf16 form runs the saturating load and the burst
    beside it.  Each form's served results are checked against the FP64 oracle: one gridding
    request into a fresh grid, then one degridding request of that grid."""
    from tconvolve.serve import Server, poisson_run, request_pool

    chosen = args.form if args.form in ("r32", "c64", "rbf16", "cbf16") else "r32"
    pool = request_pool(32, 16000, seed=7)
    upd = 16000 * 45 * 45
    out = {"workload": "Poisson arrivals, half gridding / half degridding requests of 16000 samples "
                       "(1024^2 grid, 9 w-planes, support 22: 32.4e6 updates each), 64 resident grids",
           "form": chosen, "hbm_budget_bytes": int(150e9), "slots": 2, "max_batch": 32,
           "latency": "submission to result-ready (server clock)", "forms": {}}
    for form in dict.fromkeys([chosen, "rbf16"]):
        srv = Server(c_type=form, streams=2, max_batch=32, batch_samples=32 * 16000, hbm_budget=150e9, device=device)
        grids = [srv.grid_alloc() for _ in range(64)]
        poisson_run(srv, rate=200, duration=0.3, pool=pool, grids=grids, seed=99)  # warm-up
        rates = []
        loads = ([("poisson", r, args.serve_seconds) for r in (50, 100, 200, 500)] if form == chosen else [])
        loads += [("poisson", 20000, 1.0), ("burst", 256, None)]
        for kind, rate, dur in loads:
            if kind == "poisson":
                r = poisson_run(srv, rate=rate, duration=dur, pool=pool, grids=grids, seed=rate)
            else:
                r = burst_run(srv, rate, pool, grids, seed=5)
            r["load"] = kind
            r["updates_per_s"] = r["throughput_req_s"] * upd if r["throughput_req_s"] else None
            rates.append(r)
        entry = {"rates": rates, "bytes_held": srv.stats()["bytes_held"]}
        if not args.no_precision:
            entry["precision_vs_fp64"] = served_precision(srv, pool[0])
        srv.close()
        out["forms"][form] = entry
    out["rates"] = out["forms"][chosen]["rates"]
    return out


def burst_run(server, n: int, pool, grids, seed: int = 0) -> dict:
    """n requests submitted back to back (half gridding, half degridding, random resident grids):
    the server batches them as slots free up; latency and throughput as poisson_run reports."""
    from tconvolve import _lib

    rng = np.random.default_rng(seed)
    kinds = rng.random(n) < 0.5
    picks = rng.integers(0, len(pool), n)
    gsel = rng.integers(0, len(grids), n)
    t0 = time.perf_counter()
    reqs = []
    for i in range(n):
        u, v, w, vis = pool[picks[i]]
        kind = _lib.REQ_DEGRID if kinds[i] else _lib.REQ_GRID
        reqs.append(server.submit(kind, grids[gsel[i]], u, v, w, vis if kind == _lib.REQ_GRID else None))
    submit_s = time.perf_counter() - t0
    infos = [r.wait() for r in reqs]
    lat = np.array([i.t_done - i.t_submit for i in infos]) * 1e3
    span = max(i.t_done for i in infos) - min(i.t_submit for i in infos)
    return {"requests": n, "submit_span_s": submit_s, "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
            "throughput_req_s": n / span if span > 0 else None,
            "mean_batch": float(np.mean([i.batch_requests for i in infos])),
            "errors": int(sum(1 for i in infos if i.status != 0))}


def served_precision(srv, inputs) -> dict:
    """One gridding request into a fresh resident grid and one degridding request of that grid,
    through the server, against the FP64 oracle of the same samples (the 1024^2, 9-plane, 5 arcsec
    problem's real double table with the reference's normalisation)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as orc
    from tconvolve import _lib

    u, v, w, vis = inputs
    g = srv.grid_alloc()
    srv.submit(_lib.REQ_GRID, g, u, v, w, vis).wait()
    grid = srv.grid_read(g)
    r = srv.submit(_lib.REQ_DEGRID, g, u, v, w)
    r.wait()
    srv.grid_free(g)
    cfg = orc.CONFIGS["c1"]
    _, c_f64, support, os_, wcs, _ = orc.init_c(cfg, want_f64=True)
    iu, iv, co = orc.init_offsets(orc.Config(u.size, cfg.w_size, 1, cfg.g_size, cfg.cell_size), u, v, w, wcs,
                                  support, os_)
    gs = cfg.g_size
    grid64 = np.zeros(gs * gs, np.complex128)
    orc.grid_f64(vis.astype(np.complex128), support, c_f64, co, iu, iv, grid64, gs, host_threads())
    out64 = orc.degrid_f64(grid64, gs, support, c_f64, co, iu, iv, host_threads())
    # the degridding request read the served grid: its FP64 reference degrids that same grid
    served64 = orc.degrid_f64(grid.astype(np.complex128), gs, support, c_f64, co, iu, iv, host_threads())
    return {"grid_rel_l2": orc.rel_l2(grid, grid64), "degrid_rel_l2_same_grid": orc.rel_l2(r.vis_out, served64),
            "degrid_rel_l2_end_to_end": orc.rel_l2(r.vis_out, out64), "samples": int(u.size)}


def current_section(args, torch, world):
    """The variable-support benchmark of current/tConvolveMPI (tConvolveMPI.cc:85-186): the
    continuum run (6440^2 grid, 483 w-planes, kernels 7^2..121^2) and then the spectral-line run
    (1034^2, 135 planes, 7^2..19^2) on one Benchmark object, unit visibilities as in the reference.
    A step is runGrid + runDegrid; updates are nPixelsGridded per pass.  Each run is measured with
    the default plan and with the plan tcv_cur_tune picks; the reference's own code is timed on the
    host cores beside it (bounded sample)."""
    from tconvolve.current import RUN_TYPES, Benchmark, required_rate

    b = Benchmark()
    b.setSort(0)
    stream = torch.cuda.ExternalStream(b.stream) if b.stream else torch.cuda.current_stream()
    res = {"workload": "current/tConvolveMPI: continuum then spectral line on one object (the generator "
                       "continues), data 1+0i, wide-field 36-antenna track",
           "step": "runGrid + runDegrid", "required_rate_px_s": dict(zip(("continuum", "spectral"), required_rate())),
           "runs": {}}

    def timed(k):
        for _ in range(3):
            b.runGrid()
            b.runDegrid()
        b.sync()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * k + 1)]
        ev[0].record(stream)
        for i in range(k):
            b.runGrid()
            ev[2 * i + 1].record(stream)
            b.runDegrid()
            ev[2 * i + 2].record(stream)
        b.sync()
        torch.cuda.synchronize()
        g = [ev[2 * i].elapsed_time(ev[2 * i + 1]) for i in range(k)]
        d = [ev[2 * i + 1].elapsed_time(ev[2 * i + 2]) for i in range(k)]
        gm, dm = statistics.median(g), statistics.median(d)
        if world > 1:
            from tconvolve import replicas
            gm, dm = replicas.max_over_ranks([gm, dm], device="cuda")
        return gm, dm

    for rt in (0, 1):
        b.setRunType(rt)
        b.set_tuning()  # the default plan first (a tuning stays with the object across init calls)
        t0 = time.perf_counter()
        b.init()
        b.sync()
        init_s = time.perf_counter() - t0
        px = b.nPixelsGridded()
        g = b.geometry()
        entry = {"gSize": g.g_size, "wSize": g.w_size, "support": g.support, "samples": b.nVisibilitiesGridded(),
                 "pixels_per_pass": px, "init_s": init_s}
        gm, dm = timed(5)
        entry["default"] = {"tuning": list(b.tuning()), "grid_ms": gm, "degrid_ms": dm,
                            "value": world * 2 * px / ((gm + dm) * 1e-3)}
        t0 = time.perf_counter()
        best, _, report = b.tune(reps=3)
        tune_s = time.perf_counter() - t0
        gm, dm = timed(5)
        entry["tuned"] = {"tuning": list(best), "autotune_s": tune_s, "grid_ms": gm, "degrid_ms": dm,
                          "grid_px_s": px / (gm * 1e-3), "degrid_px_s": px / (dm * 1e-3),
                          "value": world * 2 * px / ((gm + dm) * 1e-3), "unit": UNIT,
                          "candidates": [[list(t), m] for t, m in report]}
        if not args.no_cpu_baseline and world == 1:
            threads = host_threads() if rt == 1 else min(host_threads(), 8)
            sample = 400_000 if rt == 0 else 0  # continuum: a prefix; spectral: every sample
            try:
                r = run_reference_cpu_current(rt, threads, 2, sample)
                best_r = max(r, key=lambda x: x["updates_per_s"])
                what = f"first {sample} samples" if sample else "all samples"
                entry["cpu_reference"] = dict(best_r, cores=threads, kind="reference",
                                              sample=f"{threads} objects (one per thread) x {what}, "
                                                     f"runGrid + runDegrid of current/tConvolveMPI/Benchmark.cc, "
                                                     f"best of 2")
            except (RuntimeError, subprocess.CalledProcessError, subprocess.TimeoutExpired, OSError) as e:
                entry["cpu_reference"] = {"value": None, "sample": f"unavailable: {e}"}
        res["runs"][RUN_TYPES[rt]] = entry
    b.close()
    return res


def hogbom_section(args, torch):
    """Hogbom CLEAN as current/tHogbomCleanOMP runs it (Parameters.h: 1000 iterations, gain 0.1,
    threshold 1e-5) on synthetic 4096^2 and 1024^2 dirty images and PSFs (tconvolve.workload; the
    reference's data/*.img inputs are not in its tree).  Metric: iterations per second (the
    reference's "Cleaning rate").  Algorithmic bytes per iteration: the residual read once
    (4 B/pixel) plus the PSF overlap read and the residual overlap written (8 B/pixel of overlap)."""
    from tconvolve.hogbom import Workspace, deconvolve_device
    from tconvolve.workload import synthetic_dirty, synthetic_psf

    res = {"workload": "synthetic dirty image (20 point sources x PSF + 1e-3 uniform noise) and PSF, "
                       "1000 iterations, gain 0.1, threshold 1e-5", "sizes": {}}
    peak, peak_kind = measured_hbm_peak()
    for w in (4096, 1024):
        dirty, psf = synthetic_dirty(w, 20, 1e-3, seed=7), synthetic_psf(w)
        d = torch.from_numpy(dirty.ravel()).cuda()
        p = torch.from_numpy(psf.ravel()).cuda()
        m = torch.zeros_like(d)
        r = torch.empty_like(d)
        hv = torch.zeros(1000, dtype=torch.float32, device="cuda")
        hp = torch.zeros(1000, dtype=torch.int32, device="cuda")
        ws = Workspace(w)
        times = []
        for rep in range(4):  # the first run is the warm-up
            m.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            deconvolve_device(d, w, p, w, m, r, 1000, 0.1, 1e-5, hist=(hv, hp), work=ws)
            e1.record()
            torch.cuda.synchronize()
            if rep:
                times.append(e0.elapsed_time(e1))
        out = ws.result()
        ms = statistics.median(times)
        pos = hp[:out["done"]].cpu().numpy().astype(np.int64)
        rx, ry, c = pos % w, pos // w, w // 2  # PSF peak at the centre: overlap = (w - |rx - c|)(w - |ry - c|)
        overlap = ((w - np.abs(rx - c)) * (w - np.abs(ry - c))).astype(np.float64)
        alg_bytes = 4.0 * w * w * out["done"] + 8.0 * overlap.sum()
        achieved = alg_bytes / (ms * 1e-3) / 1e9
        res["sizes"][str(w)] = {"iterations": out["done"], "ms": ms, "us_per_iteration": 1e3 * ms / out["done"],
                                "iterations_per_s": out["done"] / (ms * 1e-3),
                                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                             "frac": achieved / peak, "peak_source": peak_kind,
                                             "alg_bytes_per_iteration": alg_bytes / out["done"]}}
        del d, p, m, r
    if not args.no_cpu_baseline:
        res["cpu_reference"] = hogbom_cpu_reference()
    return res


def hogbom_cpu_reference():
    """The reference's HogbomGolden (current/tHogbomCleanOMP/HogbomGolden.cc, compiled from its
    source) on the 1024^2 synthetic images: one core, 1000 iterations."""
    import tempfile

    from tconvolve.workload import synthetic_dirty, synthetic_psf

    if not os.path.exists(REF_DRIVER_HOGBOM):
        return {"value": None, "sample": f"unavailable: reference build missing: {REF_DRIVER_HOGBOM}"}
    with tempfile.TemporaryDirectory() as td:
        paths = [os.path.join(td, n) for n in ("dirty.img", "psf.img", "model.out", "residual.out")]
        synthetic_dirty(1024, 20, 1e-3, seed=7).tofile(paths[0])
        synthetic_psf(1024).tofile(paths[1])
        t0 = time.perf_counter()
        subprocess.run([REF_DRIVER_HOGBOM] + paths, check=True, capture_output=True, timeout=600)
        s = time.perf_counter() - t0
    return {"value": 1000 / s, "unit": "iterations/s", "cores": 1, "kind": "reference",
            "sample": "1024^2 synthetic images, 1000 iterations of HogbomGolden::deconvolve (wall time of the "
                      "driver, image reads included)"}


def major_section(args, torch):
    """The imaging major cycle of current/tMajorACC with its own constants (160000 samples, 33
    w-planes, 4096^2, cell 5 wavelengths, 100 sources, 100 minor iterations): 5 cycles, device time
    per stage as the reference's timers.  A first object is run once to warm up (the first
    gridding launch compiles the tile kernels for the footprint width)."""
    from tconvolve.major import MajorCycle

    warm = MajorCycle()
    warm.init()
    warm.run_cycle()
    warm.sync()
    warm.close()
    torch.cuda.empty_cache()
    m = MajorCycle()
    t0 = time.perf_counter()
    m.init()
    init_s = time.perf_counter() - t0
    cycles = m.config.n_major
    for _ in range(cycles):
        m.run_cycle()
    m.sync()
    ms, n = m.stage_ms()
    info = m.info()
    m.close()
    s = 2 * info["support"] + 1
    updates = info["n_vis"] * s * s
    per_cycle = {k: v / n for k, v in ms.items() if k not in ("psf_grid", "psf_ifft")}
    cycle_ms = sum(ms.values()) / n
    res = {"workload": "tMajorACC: 160000 samples, wSize 33, 4096^2, support 64, 100 sources, 5 major x 100 minor",
           "cycles": n, "init_s": init_s, "ms_per_cycle": cycle_ms, "stage_ms_per_cycle": per_cycle,
           "psf_ms": {"psf_grid": ms["psf_grid"], "psf_ifft": ms["psf_ifft"]},
           "grid_updates_per_s": updates / (per_cycle["grid"] * 1e-3),
           "degrid_updates_per_s": updates / (per_cycle["degrid"] * 1e-3),
           "minor_iterations_per_s": m.config.n_minor / (per_cycle["hogbom"] * 1e-3)}
    if not args.no_cpu_baseline:
        res["cpu_port"] = major_cpu_port()
    return res


def major_cpu_port():
    """One major cycle of the oracle's restatement of tMajorACC's CPU path at full size (its
    gridding and degridding in C on all host threads, numpy's FFT, the C Hogbom on one core).
    tMajorACC itself needs FFTW, OpenACC and the PGI compiler and is not built here."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as orc

    threads = host_threads()
    t0 = time.perf_counter()
    st = orc.major_setup(threads=threads)
    setup_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    orc.major_cycle(st, st["vis"], None, 100, threads=threads)
    s = time.perf_counter() - t0
    return {"value": s * 1e3, "unit": "ms per major cycle (first cycle, PSF included)", "cores": threads,
            "kind": "port", "setup_s": setup_s,
            "sample": "one full-size major cycle of the oracle restatement (C gridding/degridding on all threads, "
                      "numpy FFT, C Hogbom)"}


def oracle_reference(prob, vis, workload: str):
    """The checker of the headline: the reference's FP32 grid and degridded samples for this
    workload (the oracle's restatement of attic/tConvolveMPI/Benchmark.cc:125-195, on all host
    threads), pinned to the sha256 of the reference's own output recorded in
    tests/golden/golden.json, and the FP64 oracle of the same samples (real double table, the
    reference's normalisation constant).  Returns (grid32, out32, grid64, out64, pins)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import hashlib

    import oracle as orc

    def sha(a):
        return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()

    threads = host_threads()
    cfg = orc.Config(prob.n_samples, prob.w_size, prob.n_chan, prob.g_size, prob.cell_size, prob.baseline, prob.seed)
    u, v, w = orc.init_uvw(cfg)
    c, c_f64, support, os_, wcs, _ = orc.init_c(cfg, want_f64=True)
    iu, iv, co = orc.init_offsets(cfg, u, v, w, wcs, support, os_)
    g = prob.g_size
    grid32 = np.zeros(g * g, np.complex64)
    orc.grid_f32(vis, support, c, co, iu, iv, grid32, g, threads)
    out32 = orc.degrid_f32(grid32, g, support, c, co, iu, iv, threads)
    grid64 = np.zeros(g * g, np.complex128)
    orc.grid_f64(vis.astype(np.complex128), support, c_f64, co, iu, iv, grid64, g, threads)
    out64 = orc.degrid_f64(grid64, g, support, c_f64, co, iu, iv, threads)
    pins = {}
    try:
        with open(os.path.join(REPO, "tests", "golden", "golden.json")) as f:
            rec = json.load(f)["runs"].get(f"{workload}_normal")
    except (OSError, ValueError, KeyError):
        rec = None
    if rec:
        for name, arr in (("C", c), ("coff", co), ("iu", iu), ("iv", iv), ("grid", grid32), ("outdata", out32)):
            pins[name] = sha(arr) == rec["sha256"][name]
    return grid32, out32, grid64, out64, pins, orc.rel_l2, threads


def l2_table_ceiling(torch, stream, updates, g_ms, d_ms, form):
    """The tile kernels' own ceiling, measured live: the L2-to-SM bandwidth of random 128-byte
    row segments (16 rows at the 129-entry table stride, from a 64 MiB buffer that stays in L2,
    tcv_probe_table_stream), against which their table stream (table bytes per update x updates
    / pass time) is set.  The HBM roofline above counts the reference's per-update grid traffic,
    which these kernels keep on chip."""
    import tconvolve
    from tconvolve.raw import _ptr

    L = tconvolve.lib()
    P = tconvolve._lib.probe_lib()
    buf = torch.rand(16 << 20, dtype=torch.float32, device="cuda")
    out = torch.empty(int(P.tcv_probe_table_threads()), dtype=torch.float32, device="cuda")
    nbytes = ctypes.c_int64()
    launch = lambda: P.tcv_probe_table_stream(_ptr(buf), buf.numel(), 129, 256, _ptr(out), ctypes.byref(nbytes),
                                              ctypes.c_void_p(stream.cuda_stream))
    for _ in range(3):
        if launch() != 0:
            return None
    ms = []
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        launch()
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    probe = nbytes.value / (statistics.median(ms) * 1e-3) / 1e9
    tb = L.tcv_ctype_bytes(tconvolve.CTYPE_BY_NAME[form])
    grid_gbs = tb * updates / (g_ms * 1e-3) / 1e9
    degrid_gbs = tb * updates / (d_ms * 1e-3) / 1e9
    return {"unit": "GB/s", "probe": probe, "table_bytes_per_update": tb,
            "grid": grid_gbs, "grid_frac": grid_gbs / probe, "degrid": degrid_gbs, "degrid_frac": degrid_gbs / probe,
            "probe_shape": "random 128-byte row segments, 16 rows at a 129-entry stride, 64 MiB L2-resident buffer"}


def count_step_kernels(torch, step):
    """Kernel nodes in a CUDA-graph capture of one step (0 if capture is unavailable)."""
    try:
        import cuda.bindings.runtime as rt
    except ImportError:
        return 0
    g = torch.cuda.CUDAGraph(keep_graph=True)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.graph(g, stream=s):
        step()
    torch.cuda.synchronize()
    handle = g.raw_cuda_graph()
    err, _, count = rt.cudaGraphGetNodes(handle, 0)
    err, nodes, count = rt.cudaGraphGetNodes(handle, count)
    kernels = 0
    for nd in nodes:
        err, t = rt.cudaGraphNodeGetType(nd)
        if t == rt.cudaGraphNodeType.cudaGraphNodeTypeKernel:
            kernels += 1
    del g
    return kernels


def cpu_baseline(args):
    threads = host_threads()
    per_thread = cpu_sample_size(threads, args.cpu_seconds)
    try:
        rates, _ = run_reference_cpu(threads, per_thread, 1, 0)
        return {"value": rates[0], "unit": UNIT, "cores": threads, "kind": "reference",
                "sample": f"{threads} thread replicas x first {per_thread} samples of the workload, "
                          f"one gridKernel + degridKernel pass of the reference's Benchmark.cc"}
    except (RuntimeError, subprocess.CalledProcessError, OSError) as e:
        return {"value": None, "unit": UNIT, "cores": threads, "kind": "reference",
                "sample": f"unavailable: {e}"}


def visible_gpus() -> int:
    try:
        import torch

        return torch.cuda.device_count()
    except Exception:  # noqa: BLE001 - no usable CUDA runtime: no GPU
        return 0


def world_plan(gpus: int, env, visible: int):
    """How a B200 run with --gpus N starts: ("run", None) in this process (N = 1, or already one
    rank of N under torchrun), ("spawn", None) as N ranks under torchrun (N > 1 and not a rank
    yet), or ("error", why) for a request that cannot be met.  One rank per GPU, as the
    reference's MPI replicas run one process per core (attic/tConvolveMPI/tConvolveMPI.cc:65-111)."""
    if gpus < 1:
        return "error", f"--gpus {gpus}: at least one GPU"
    ws = env.get("WORLD_SIZE")
    if ws is not None:
        if int(ws) != gpus:
            return "error", f"--gpus {gpus} but WORLD_SIZE={ws}: launch one rank per GPU"
        return "run", None
    if gpus == 1:
        return "run", None
    if visible < gpus:
        return "error", f"--gpus {gpus} but only {visible} GPU(s) visible"
    return "spawn", None


def spawn_argv(gpus: int, argv, port: int):
    """The torchrun command that runs this bench as `gpus` ranks on one node."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
            "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + list(argv)


def free_port() -> int:
    import socket

    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def main():
    args = parse_args()
    if args.warmup < 3:
        print("warmup must be >= 3", file=sys.stderr)
        return 2
    if args.impl == "reference":
        return reference_arm(args)
    action, why = world_plan(args.gpus, os.environ, visible_gpus() if "WORLD_SIZE" not in os.environ else 0)
    if action == "error":
        print(f"bench.py: {why}", file=sys.stderr)
        return 2
    if action == "spawn":
        # one process per GPU; the ranks' own barriers and process-group timeout bound the run
        r = subprocess.run(spawn_argv(args.gpus, sys.argv[1:], free_port()), timeout=3600)
        return r.returncode
    return b200_arm(args)


if __name__ == "__main__":
    sys.exit(main())
