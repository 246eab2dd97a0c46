"""Row-band split of one gridding job over the ranks of a process group (one process per GPU).

The reference's ranks are independent replicas (attic/tConvolveMPI/tConvolveMPI.cc:78-119: every
MPI rank grids its own copy of the problem).  Here the ranks share ONE grid: rank b owns the
rows [rows[b], rows[b+1]) (tcv_band_bounds balances the samples' centre rows over the ranks),
grids the samples whose footprint's centre row lies in its band into a full-size local grid, and
exchanges the `support` rows that those footprints reach past each edge of its band with the
neighbour that owns them (the footprint of Benchmark.cc:137-150 covers rows iv .. iv + 2*support).

Steps, and what crosses between ranks:

  set-up  centre-row histogram of this rank's samples (tcv_band_histogram), summed over the ranks
          (gSize int64); the bounds (tcv_band_bounds); a stable partition of this rank's samples
          by band (tcv_band_bucket) and one all-to-all of 20-byte records (data, iu, iv,
          cOffset); a plan over the samples received
  grid    zero the halo rows; tcv_plan_grid; send each halo (support rows) to the neighbour that
          owns it; add what the neighbours sent into the band's edge rows (tcv_rows_add), the
          lower neighbour's first
  degrid  receive the neighbours' edge rows into the halo rows; tcv_plan_degrid; all-to-all of
          the degridded values back to the ranks that hold those samples; tcv_band_scatter into
          their input order

After grid(), the band's own rows of the local grid hold the sums of every rank's samples there
(added to what they held, as the reference's gridding adds); the rows outside the band are
scratch.  degrid() reads the band's rows plus the halo rows it receives and overwrites `out`.

DistComm runs the exchanges through torch.distributed (NCCL between GPUs, gloo on CPU);
CudaBandOps does every computation through libtconvolve.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check, lib
from .raw import Plan, _ptr, _stream


class DistComm:
    """The exchanges of a band split over a torch.distributed process group (the default one)."""

    def __init__(self):
        import torch.distributed as dist

        self.dist = dist
        self.rank = dist.get_rank()
        self.size = dist.get_world_size()

    def all_reduce_sum(self, t):
        self.dist.all_reduce(t)

    def all_to_all(self, out, inp, out_splits, in_splits):
        self.dist.all_to_all_single(out, inp, list(out_splits), list(in_splits))

    def exchange(self, sends, recvs):
        """Point-to-point: sends and recvs are lists of (peer rank, tensor)."""
        d = self.dist
        ops = [d.P2POp(d.isend, t, p) for p, t in sends] + [d.P2POp(d.irecv, t, p) for p, t in recvs]
        if ops:
            for r in d.batch_isend_irecv(ops):
                r.wait()


class SoloComm:
    """The exchanges of a one-rank split (one band: nothing crosses)."""

    rank, size = 0, 1

    def all_reduce_sum(self, t):
        pass

    def all_to_all(self, out, inp, out_splits, in_splits):
        out.copy_(inp)

    def exchange(self, sends, recvs):
        assert not sends and not recvs


class CudaBandOps:
    """The device steps, each one libtconvolve call on torch CUDA tensors (include/tconvolve.h)."""

    def __init__(self, device="cuda", stream=None):
        self.device = device
        self.stream = stream

    def _s(self):
        return _stream(self.stream)

    def histogram(self, iv, support: int, g_size: int):
        import torch

        hist = torch.zeros(g_size, dtype=torch.int64, device=self.device)
        check(lib().tcv_band_histogram(_ptr(iv), iv.numel(), support, g_size, _ptr(hist), self._s()),
              "tcv_band_histogram")
        return hist

    def bucket(self, data, iu, iv, coff, support: int, g_size: int, rows):
        """(records [n, 5] int32, perm [n] int32, per-band counts as a host list)."""
        import torch

        n = iu.numel()
        nb = len(rows) - 1
        rows_h = np.ascontiguousarray(rows, np.int32)
        rec = torch.empty((n, 5), dtype=torch.int32, device=self.device)
        perm = torch.empty(n, dtype=torch.int32, device=self.device)
        counts = torch.empty(nb, dtype=torch.int64, device=self.device)
        wbytes = lib().tcv_band_workspace_bytes(n, nb)
        if wbytes == 0:
            raise _lib.TcvError(1, "tcv_band_workspace_bytes")
        work = torch.empty(wbytes, dtype=torch.uint8, device=self.device)
        check(lib().tcv_band_bucket(_ptr(data), _ptr(iu), _ptr(iv), _ptr(coff), n, support, g_size,
                                    ctypes.c_void_p(rows_h.ctypes.data), nb, _ptr(rec), _ptr(perm),
                                    _ptr(counts), _ptr(work), wbytes, self._s()), "tcv_band_bucket")
        return rec, perm, [int(x) for x in counts.cpu().tolist()]

    def unpack(self, rec):
        import torch

        m = rec.shape[0]
        data = torch.empty(m, dtype=torch.complex64, device=self.device)
        iu, iv, coff = (torch.empty(m, dtype=torch.int32, device=self.device) for _ in range(3))
        check(lib().tcv_band_unpack(_ptr(rec), m, _ptr(data), _ptr(iu), _ptr(iv), _ptr(coff), self._s()),
              "tcv_band_unpack")
        return data, iu, iv, coff

    def scatter(self, src, perm, dst):
        check(lib().tcv_band_scatter(_ptr(src), _ptr(perm), src.numel(), _ptr(dst), self._s()), "tcv_band_scatter")

    def rows_add(self, dst, src):
        check(lib().tcv_rows_add(_ptr(dst), _ptr(src), dst.numel(), self._s()), "tcv_rows_add")

    def zero(self, t):
        import torch

        with torch.cuda.stream(self.stream or torch.cuda.current_stream()):
            t.zero_()

    def plan(self, iu, iv, coff, support: int, g_size: int, c_len: int, tuning=None):
        return _CudaPlan(Plan(iu, iv, coff, support, g_size, c_len, stream=self.stream, tuning=tuning), self.stream)

    # torch.distributed orders its NCCL work after the current stream and makes the current
    # stream wait for it; a separate stream of these ops is joined to the current one both ways.
    def before_comm(self):
        import torch

        cur = torch.cuda.current_stream()
        if self.stream is not None and self.stream != cur:
            cur.wait_stream(self.stream)

    def after_comm(self):
        import torch

        cur = torch.cuda.current_stream()
        if self.stream is not None and self.stream != cur:
            self.stream.wait_stream(cur)


class _CudaPlan:
    def __init__(self, plan: Plan, stream):
        self.plan, self.stream = plan, stream

    def grid(self, data, c, c_type, c_scale, grid):
        self.plan.grid(data, c, c_type, grid, c_scale, stream=self.stream)

    def degrid(self, grid, c, c_type, c_scale, out):
        self.plan.degrid(grid, c, c_type, out, c_scale, stream=self.stream)

    def rejected(self) -> int:
        return self.plan.rejected(stream=self.stream)


def band_bounds(hist, g_size: int, support: int, n_bands: int) -> list:
    """tcv_band_bounds on a host histogram (host arithmetic): the n_bands + 1 row bounds."""
    h = np.ascontiguousarray(hist, np.int64)
    if h.size != g_size:
        raise ValueError("histogram must hold g_size counts")
    rows = np.empty(n_bands + 1, np.int32)
    check(lib().tcv_band_bounds(ctypes.c_void_p(h.ctypes.data), g_size, support, n_bands,
                                ctypes.c_void_p(rows.ctypes.data)), "tcv_band_bounds")
    return [int(r) for r in rows]


def halo_plan(rows, b: int, support: int):
    """Row ranges of band b's exchanges, as (peer, first row, end row) lists:
    grid_send  - this rank's halo rows, added by their owner
    grid_recv  - the owner's rows a neighbour's halo is added into
    fetch_send - this rank's edge rows a neighbour degrids from
    fetch_recv - the halo rows received for degridding
    Every interior band edge moves `support` rows each way; the grid's outer edges move none."""
    n = len(rows) - 1
    r0, r1, s = rows[b], rows[b + 1], support
    out = {"grid_send": [], "grid_recv": [], "fetch_send": [], "fetch_recv": []}
    if s == 0:
        return out
    if b > 0:
        out["grid_send"].append((b - 1, r0 - s, r0))
        out["grid_recv"].append((b - 1, r0, r0 + s))
        out["fetch_send"].append((b - 1, r0, r0 + s))
        out["fetch_recv"].append((b - 1, r0 - s, r0))
    if b < n - 1:
        out["grid_send"].append((b + 1, r1, r1 + s))
        out["grid_recv"].append((b + 1, r1 - s, r1))
        out["fetch_send"].append((b + 1, r1 - s, r1))
        out["fetch_recv"].append((b + 1, r1, r1 + s))
    return out


class BandJob:
    """One job's samples split into row bands over the ranks of `comm` (set-up in the constructor).

    data, iu, iv, coff: this rank's share of the samples (any share: an all-to-all moves each to
    the rank that owns its band), on the ops' device.  grid(), degrid(): one pass each, the same
    arguments on every rank (every rank takes the same exchange steps in the same order)."""

    def __init__(self, data, iu, iv, coff, support: int, g_size: int, c_len: int, comm=None, ops=None,
                 tuning=None):
        import torch

        self.comm = comm if comm is not None else DistComm()
        self.ops = ops if ops is not None else CudaBandOps()
        self.support, self.g_size, self.c_len = support, g_size, c_len
        self.rank, self.size = self.comm.rank, self.comm.size
        self.n_local = iu.numel()
        dev = self.ops.device
        hist = self.ops.histogram(iv, support, g_size)
        self.ops.before_comm()
        self.comm.all_reduce_sum(hist)
        self.rows = band_bounds(hist.cpu().numpy(), g_size, support, self.size)
        rec, self.perm, self.send_counts = self.ops.bucket(data, iu, iv, coff, support, g_size, self.rows)
        sc = torch.tensor(self.send_counts, dtype=torch.int64, device=dev)
        rc = torch.empty_like(sc)
        self.comm.all_to_all(rc, sc, [1] * self.size, [1] * self.size)
        self.recv_counts = [int(x) for x in rc.cpu().tolist()]
        self.n_band = sum(self.recv_counts)
        recv = torch.empty((self.n_band, 5), dtype=torch.int32, device=dev)
        self.ops.before_comm()
        self.comm.all_to_all(recv, rec, self.recv_counts, self.send_counts)
        self.ops.after_comm()
        self.data, self.iu, self.iv, self.coff = self.ops.unpack(recv)
        self.plan = (self.ops.plan(self.iu, self.iv, self.coff, support, g_size, c_len, tuning)
                     if self.n_band > 0 else None)
        self.halo = halo_plan(self.rows, self.rank, support)
        self._band_out = torch.empty(self.n_band, dtype=torch.complex64, device=dev)
        self._back = torch.empty(self.n_local, dtype=torch.complex64, device=dev)
        self._recv_bufs = [torch.empty((e - a) * g_size, dtype=torch.complex64, device=dev)
                           for _, a, e in self.halo["grid_recv"]]

    @property
    def band(self):
        """(first row, end row) of this rank's band."""
        return self.rows[self.rank], self.rows[self.rank + 1]

    def _rows(self, grid, a: int, e: int):
        return grid[a * self.g_size:e * self.g_size]

    @staticmethod
    def _real(t):
        import torch

        return torch.view_as_real(t)

    def grid(self, grid, c, c_type: int, c_scale: float = 1.0):
        """Grid this band's samples into `grid` (g_size^2 complex64), then add the neighbours'
        halos into the band's edge rows."""
        for _, a, e in self.halo["grid_send"]:
            self.ops.zero(self._rows(grid, a, e))
        if self.plan is not None:
            self.plan.grid(self.data, c, c_type, c_scale, grid)
        sends = [(p, self._real(self._rows(grid, a, e))) for p, a, e in self.halo["grid_send"]]
        recvs = [(p, self._real(buf)) for (p, _, _), buf in zip(self.halo["grid_recv"], self._recv_bufs)]
        self.ops.before_comm()
        self.comm.exchange(sends, recvs)
        self.ops.after_comm()
        for (_, a, e), buf in zip(self.halo["grid_recv"], self._recv_bufs):
            self.ops.rows_add(self._rows(grid, a, e), buf)

    def degrid(self, grid, c, c_type: int, out, c_scale: float = 1.0):
        """Degrid this rank's own samples (the n_local it passed in, in that order) into `out`
        from the band rows of `grid` and the neighbours' edge rows."""
        sends = [(p, self._real(self._rows(grid, a, e))) for p, a, e in self.halo["fetch_send"]]
        recvs = [(p, self._real(self._rows(grid, a, e))) for p, a, e in self.halo["fetch_recv"]]
        self.ops.before_comm()
        self.comm.exchange(sends, recvs)
        self.ops.after_comm()
        if self.plan is not None:
            self.plan.degrid(grid, c, c_type, c_scale, self._band_out)
        self.ops.before_comm()
        self.comm.all_to_all(self._real(self._back), self._real(self._band_out), self.send_counts,
                             self.recv_counts)
        self.ops.after_comm()
        self.ops.scatter(self._back, self.perm, out)

    def rejected(self) -> int:
        return self.plan.rejected() if self.plan is not None else 0


def run(steps: int = 5, device="cuda", printer=print, problem: str = "c2", tuning=(16, 64, 0, 64)) -> dict:
    """tConvolveMPI's flow (attic/tConvolveMPI/tConvolveMPI.cc:78-121) for ONE job split into row
    bands over the ranks: every rank makes the reference's samples (u, v, w from its generator,
    data 1+0i, attic/tConvolveMPI/Benchmark.cc:46-80), keeps its contiguous share and hands the
    rest to their bands' ranks; then `steps` gridding passes and `steps` degridding passes of the
    whole job, each timed on the device (the slowest rank's time); rank 0 prints the reference's
    report lines with the job's rates."""
    import torch

    from . import raw
    from .replicas import max_over_ranks, world
    from .workload import PROBLEMS

    rank, n = world()
    prob = PROBLEMS[problem]
    freq = torch.tensor([(1.4e9 - 2.0e5 * i / prob.n_chan) / 2.998e8 for i in range(prob.n_chan)],
                        dtype=torch.float64, device=device)  # Benchmark.cc:86-90
    u, v, w = raw.init_uvw(prob.n_samples, prob.baseline, 1, device=device)
    support, os_, wcs, c_len = raw.c_geometry(float(freq[0].item()), prob.cell_size, prob.baseline, prob.w_size)
    c64, _ = raw.init_c(float(freq[0].item()), prob.cell_size, prob.baseline, prob.w_size, device=device)
    # the real form of the table: the attic table's imaginary parts are zero, so it gives the
    # complex64 table's results bit for bit at half the table bytes
    c, scale, _ = raw.convert_c(c64, _lib.R32)
    iu, iv, coff = raw.init_offsets(u, v, w, freq, prob.cell_size, wcs, prob.w_size, prob.g_size, support, os_)
    total = iu.numel()
    a, e = rank * total // n, (rank + 1) * total // n
    data = torch.ones(e - a, dtype=torch.complex64, device=device)  # Benchmark.cc:75-78
    job = BandJob(data, iu[a:e].contiguous(), iv[a:e].contiguous(), coff[a:e].contiguous(), support, prob.g_size,
                  c_len, comm=DistComm() if n > 1 else SoloComm(), ops=CudaBandOps(device), tuning=tuning)
    grid = torch.zeros(prob.g_size * prob.g_size, dtype=torch.complex64, device=device)
    out = torch.empty(e - a, dtype=torch.complex64, device=device)
    R32 = _lib.R32

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) * 1e-3

    job.grid(grid, c, R32, scale)  # warm-up: the specialised kernels are built at the first pass
    job.degrid(grid, c, R32, out, scale)
    torch.cuda.synchronize()
    t_grid, t_degrid = max_over_ranks([timed(lambda: job.grid(grid, c, R32, scale)),
                                       timed(lambda: job.degrid(grid, c, R32, out, scale))], device=device)
    updates = float(total) * (2 * support + 1) ** 2 * steps
    if rank == 0:
        for title, t, what in (("Forward", t_grid, "Gridding"), ("Reverse", t_degrid, "Degridding")):
            printer(f"+++++ {title} processing (row bands) +++++")
            printer(f"    Number of processes: {n}")
            printer(f"    Time {t} (s) ")
            printer(f"    Time per visibility spectral sample {1e6 * t / (total * steps)} (us) ")
            printer(f"    Time per {what.lower()}   {1e9 * t / updates} (ns) ")
            printer(f"    {what} rate   {updates / t / 1e6} (million grid points per second)")
        printer("Done")
    return {"ranks": n, "rows": job.rows, "grid_s": t_grid, "degrid_s": t_degrid, "updates": updates,
            "samples_per_rank": job.n_band, "rejected": job.rejected()}


def main(argv=None) -> int:
    """torchrun --nproc-per-node N -m tconvolve.bands [passes]"""
    import datetime
    import os
    import sys

    import torch
    import torch.distributed as dist

    args = sys.argv[1:] if argv is None else argv
    if len(args) > 1 or (args and not args[0].isdigit()):
        print("usage: python -m tconvolve.bands [# of passes]", file=sys.stderr)
        return 1
    steps = int(args[0]) if args else 5
    if "RANK" in os.environ:
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0"))))
    try:
        run(steps)
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
