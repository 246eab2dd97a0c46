"""Burn-in soak test of the gridder over many GPUs (attic/tConvolveBurnIn).

Every rank runs the same problem (attic/tConvolveBurnIn/Benchmark.h:39-46: 160000 samples, 33
planes, 4096^2, unit visibilities) cycle after cycle: gridding accumulates into the grid (the
reference never clears it, Benchmark.cc:91-99), degridding reads it.  After each pass a rank sends
its result to rank (r + n/2) mod n and compares the one it receives, element by element, with the
reference's test: |real part difference| > FLT_EPSILON is an error (Benchmark.cc:343-374).  Error
counts are summed and the pass times gathered as min/avg/max (tConvolveBurnIn.cc:62-97, 140-175).

B200 form: one process per GPU (torch.distributed, NCCL over NVLink; gloo on CPU for the host
logic), results exchanged device to device with send/recv of the whole array, compared on the
device; pass times from CUDA events.  The kernels are deterministic, so healthy replicas agree bit
for bit.

    torchrun --nproc-per-node N -m tconvolve.burnin [cycles]
"""
from __future__ import annotations

import numpy as np

FLT_EPSILON = float(np.finfo(np.float32).eps)


def partners(rank: int, n: int):
    """(destination, source) of the exchange: send to (r + n/2) mod n, receive from the rank that
    sends here, (r - n/2) mod n (the reference receives from MPI_ANY_SOURCE; this is that rank)."""
    return (rank + n // 2) % n, (rank - n // 2) % n


def share_and_compare(data, eps: float = FLT_EPSILON):
    """Benchmark::shareAndCompare (attic/tConvolveBurnIn/Benchmark.cc:343-374) on a complex
    tensor: exchange with the partner ranks and count the elements whose real parts differ by more
    than eps.  Returns (ok, mismatches, first mismatching index or -1, source rank)."""
    import torch
    import torch.distributed as dist

    from .replicas import world

    rank, n = world()
    dest, src = partners(rank, n)
    if n == 1 or dest == rank:
        other = data.clone()
    else:
        other = torch.empty_like(data)
        ops = [dist.P2POp(dist.isend, data, dest), dist.P2POp(dist.irecv, other, src)]
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    a = torch.view_as_real(data)[..., 0] if data.is_complex() else data
    b = torch.view_as_real(other)[..., 0] if other.is_complex() else other
    bad = (a - b).abs() > eps
    count = int(bad.sum().item())
    first = int(torch.nonzero(bad.flatten())[0].item()) if count else -1
    return count == 0, count, first, src


def accumulate_errors(success: bool, device="cpu") -> int:
    """Number of ranks that reported a failure (tConvolveBurnIn.cc:62-77; every rank gets it)."""
    import torch
    import torch.distributed as dist

    from .replicas import world

    t = torch.tensor([0 if success else 1], dtype=torch.int64, device=device)
    if world()[1] > 1:
        dist.all_reduce(t)
    return int(t.item())


def gather_times(seconds: float, device="cpu"):
    """(min, avg, max) of a time over the ranks (tConvolveBurnIn.cc:79-97)."""
    import torch
    import torch.distributed as dist

    from .replicas import world

    _, n = world()
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    if n > 1:
        allt = [torch.empty_like(t) for _ in range(n)]
        dist.all_gather(allt, t)
        vals = [float(x.item()) for x in allt]
    else:
        vals = [float(t.item())]
    return min(vals), sum(vals) / len(vals), max(vals)


class BurnIn:
    """The burn-in Benchmark (attic/tConvolveBurnIn/Benchmark.h:55-99) on one GPU."""

    def __init__(self, n_samples: int = 160000, w_size: int = 33, n_chan: int = 1, g_size: int = 4096,
                 cell_size: float = 5.0, baseline: int = 2000, device="cuda"):
        import torch

        from . import raw
        from ._lib import C64

        self.c_type = C64
        self.g_size = g_size
        freq = torch.tensor([(1.4e9 - 2.0e5 * i / n_chan) / 2.998e8 for i in range(n_chan)], dtype=torch.float64,
                            device=device)
        u, v, w = raw.init_uvw(n_samples, baseline, 1, device=device)
        self.support, os_, wcs, c_len = raw.c_geometry(float(freq[0].item()), cell_size, baseline, w_size)
        self.c, _ = raw.init_c(float(freq[0].item()), cell_size, baseline, w_size, device=device)
        self.iu, self.iv, self.coff = raw.init_offsets(u, v, w, freq, cell_size, wcs, w_size, g_size, self.support,
                                                       os_)
        self.plan = raw.Plan(self.iu, self.iv, self.coff, self.support, g_size, c_len)
        n = n_samples * n_chan
        self.data = torch.ones(n, dtype=torch.complex64, device=device)  # Benchmark.cc:75-78
        self.outdata = torch.zeros(n, dtype=torch.complex64, device=device)
        self.grid = torch.zeros(g_size * g_size, dtype=torch.complex64, device=device)
        self.updates = n * (2 * self.support + 1) ** 2

    def _timed(self, fn):
        import torch

        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) * 1e-3

    def run_grid(self):
        """runGrid (Benchmark.cc:91-99): grid += gridding, then the cross-rank comparison."""
        t = self._timed(lambda: self.plan.grid(self.data, self.c, self.c_type, self.grid))
        return share_and_compare(self.grid), t

    def run_degrid(self):
        t = self._timed(lambda: self.plan.degrid(self.grid, self.c, self.c_type, self.outdata))
        return share_and_compare(self.outdata), t


def run(cycles: int = 1, device="cuda", printer=print, **problem) -> dict:
    """tConvolveBurnIn's main loop (tConvolveBurnIn.cc:100-195).  Returns the error counts and the
    per-cycle time statistics; rank 0 prints the reference's report lines."""
    from .replicas import world

    rank, n = world()
    b = BurnIn(device=device, **problem)
    grid_err = degrid_err = 0
    stats = []
    for cycle in range(1, cycles + 1):
        if rank == 0:
            printer(f"+++++ Cycle {cycle} of {cycles} +++++")
        (ok, _, _, _), tg = b.run_grid()
        grid_err += accumulate_errors(ok, device)
        gs = gather_times(tg, device)
        (ok, _, _, _), td = b.run_degrid()
        degrid_err += accumulate_errors(ok, device)
        ds = gather_times(td, device)
        stats.append({"grid_s": gs, "degrid_s": ds})
        if rank == 0:
            printer(f"    Number of processes:            {n}")
            printer(f"    Gridding error count:           {grid_err}")
            printer(f"    Degridding error count:         {degrid_err}")
            printer(f"    Gridding times (min/avg/max):   {gs[0]} / {gs[1]} / {gs[2]} seconds")
            printer(f"    Degridding times (min/avg/max): {ds[0]} / {ds[1]} / {ds[2]} seconds")
    return {"ranks": n, "cycles": cycles, "grid_errors": grid_err, "degrid_errors": degrid_err, "times": stats,
            "updates_per_pass": b.updates}


def main(argv=None) -> int:
    import datetime
    import os
    import sys

    import torch
    import torch.distributed as dist

    args = sys.argv[1:] if argv is None else argv
    if len(args) > 1:
        print("usage: python -m tconvolve.burnin [# of cycles]", file=sys.stderr)
        return 1
    cycles = int(args[0]) if args else 1
    if "RANK" in os.environ:
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        r = run(cycles)
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()
    return 0 if r["grid_errors"] == 0 and r["degrid_errors"] == 0 else 2


if __name__ == "__main__":
    raise SystemExit(main())
