"""Multi-process replica plumbing (one process per GPU).

The reference scales by independent replicas that meet only at barriers
(attic/tConvolveMPI/tConvolveMPI.cc:89-111, MPI_Barrier around each timed pass) and, in the
burn-in variant, compare their results across ranks (attic/tConvolveBurnIn/Benchmark.cc:343-374).
Here the replicas are torch.distributed processes: NCCL on GPUs, gloo on CPU (tests).

* max_over_ranks  - device time of a step = the slowest rank's, as the benchmark reports it
* checksum        - order-independent 64-bit digest of a result array (bit pattern based)
* cross_check     - every rank's digest must equal rank 0's (replicas of one problem are
                    bit-identical because the kernels are deterministic)
* rank0_tunings   - every rank takes rank 0's plan tunings (each rank's autotuner may pick a
                    different one, and a different gridding split changes the order of the sums)
"""
from __future__ import annotations

import hashlib

import numpy as np


def world():
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def max_over_ranks(values, device="cpu"):
    """Element-wise maximum of a list of floats over all ranks."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    _, n = world()
    if n > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu().tolist()]


def checksum(arr: np.ndarray) -> int:
    """64-bit digest of the exact bytes of an array (equal iff the bits are equal, w.h.p.)."""
    h = hashlib.blake2b(np.ascontiguousarray(arr).tobytes(), digest_size=8).digest()
    return int.from_bytes(h, "little") & 0x7FFFFFFFFFFFFFFF


def cross_check(digest: int, device="cpu") -> bool:
    """True on every rank iff all ranks hold the same digest (a MIN and a MAX all-reduce)."""
    import torch
    import torch.distributed as dist

    _, n = world()
    if n == 1:
        return True
    lo = torch.tensor([digest], dtype=torch.int64, device=device)
    hi = lo.clone()
    dist.all_reduce(lo, op=dist.ReduceOp.MIN)
    dist.all_reduce(hi, op=dist.ReduceOp.MAX)
    return int(lo.item()) == int(hi.item())


def rank0_tunings(tunings: dict, device="cpu") -> dict:
    """{name: (tuning tuple of up to five ints, extra)} with every tuple replaced by rank 0's; the
    same names on every rank.  A fifth entry of 0 is dropped (the kernel-bits field unset)."""
    import torch
    import torch.distributed as dist

    _, n = world()
    if n == 1:
        return dict(tunings)
    out = {}
    for name in sorted(tunings):
        t = torch.tensor((list(tunings[name][0]) + [0] * 5)[:5], dtype=torch.int64, device=device)
        dist.broadcast(t, 0)
        vals = [int(x) for x in t.cpu().tolist()]
        out[name] = (tuple(vals[:4]) + ((vals[4],) if vals[4] else ()), tunings[name][1])
    return out
