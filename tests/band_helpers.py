"""Test helpers for the row-band split (tconvolve.bands).

* NumpyBandOps  - the device steps restated in numpy, with the oracle's gridding and degridding
                  (oracle/tconvolve_oracle.c) as the plan: the stand-in that lets the band split's
                  exchanges run as gloo ranks on CPU.
* ThreadComm    - the exchanges between ranks that are threads of one process on one GPU.  Each
                  rank's kernels run on its own stream and never wait on another rank's: every
                  exchange synchronises the sender's stream, copies on the host's orders and
                  meets at a barrier with a time limit.
* run_threads   - runs fn(rank, comm) for every rank of such a group and returns the results.
"""
from __future__ import annotations

import threading

import numpy as np


def centre_rows(iv, support: int, g_size: int):
    return np.clip(np.asarray(iv, np.int64) + support, 0, g_size - 1)


def band_index(iv, support: int, g_size: int, rows):
    """Band of each sample: the band that holds its footprint's centre row."""
    return np.searchsorted(np.asarray(rows[1:-1], np.int64), centre_rows(iv, support, g_size), side="right")


def bucket_numpy(data, iu, iv, coff, support: int, g_size: int, rows):
    """Stable partition by band: (records [n, 5] int32, perm int32, counts)."""
    data = np.ascontiguousarray(data, np.complex64)
    b = band_index(iv, support, g_size, rows)
    order = np.argsort(b, kind="stable")
    parts = np.empty((data.size, 5), np.int32)
    parts[:, 0] = data.real.view(np.int32)
    parts[:, 1] = data.imag.view(np.int32)
    parts[:, 2] = iu
    parts[:, 3] = iv
    parts[:, 4] = coff
    counts = np.bincount(b, minlength=len(rows) - 1).astype(np.int64)
    return parts[order], order.astype(np.int32), counts


class _OraclePlan:
    def __init__(self, orc, c, iu, iv, coff, support, g_size):
        self.orc, self.c = orc, c
        self.iu, self.iv, self.coff = (np.ascontiguousarray(a.numpy()) for a in (iu, iv, coff))
        self.support, self.g_size = support, g_size

    def grid(self, data, c, c_type, c_scale, grid):
        self.orc.grid_f32(data.numpy(), self.support, self.c, self.coff, self.iu, self.iv, grid.numpy(),
                          self.g_size)

    def degrid(self, grid, c, c_type, c_scale, out):
        out.numpy()[:] = self.orc.degrid_f32(grid.numpy(), self.g_size, self.support, self.c, self.coff, self.iu,
                                             self.iv)

    def rejected(self) -> int:
        return 0


class NumpyBandOps:
    """CPU stand-in of tconvolve.bands.CudaBandOps on torch CPU tensors."""

    device = "cpu"

    def __init__(self, orc, c):
        self.orc, self.c = orc, c

    def histogram(self, iv, support, g_size):
        import torch

        h = np.bincount(centre_rows(iv.numpy(), support, g_size), minlength=g_size).astype(np.int64)
        return torch.from_numpy(h)

    def bucket(self, data, iu, iv, coff, support, g_size, rows):
        import torch

        rec, perm, counts = bucket_numpy(data.numpy(), iu.numpy(), iv.numpy(), coff.numpy(), support, g_size, rows)
        return torch.from_numpy(rec), torch.from_numpy(perm), [int(x) for x in counts]

    def unpack(self, rec):
        import torch

        r = rec.numpy()
        data = np.empty(r.shape[0], np.complex64)
        data.real = r[:, 0].view(np.float32)
        data.imag = r[:, 1].view(np.float32)
        return (torch.from_numpy(data), torch.from_numpy(r[:, 2].copy()), torch.from_numpy(r[:, 3].copy()),
                torch.from_numpy(r[:, 4].copy()))

    def scatter(self, src, perm, dst):
        dst.numpy()[perm.numpy()] = src.numpy()

    def rows_add(self, dst, src):
        dst += src

    def zero(self, t):
        t.zero_()

    def plan(self, iu, iv, coff, support, g_size, c_len, tuning=None):
        return _OraclePlan(self.orc, self.c, iu, iv, coff, support, g_size)

    def before_comm(self):
        pass

    def after_comm(self):
        pass


class _Board:
    def __init__(self, size: int, timeout: float):
        self.size = size
        self.barrier = threading.Barrier(size, timeout=timeout)
        self.slots = {}
        self.lock = threading.Lock()


class ThreadComm:
    """Exchanges between ranks that are threads of one process (one GPU)."""

    def __init__(self, board: _Board, rank: int):
        self.board, self.rank, self.size = board, rank, board.size
        self.seq = 0

    def _sync(self):
        import torch

        torch.cuda.current_stream().synchronize()

    def _post(self, key, value):
        with self.board.lock:
            self.board.slots[(self.seq,) + key] = value

    def _get(self, key):
        with self.board.lock:
            return self.board.slots[(self.seq,) + key]

    def _end(self):
        self._sync()
        self.board.barrier.wait()  # every rank has copied what it needed
        if self.rank == 0:
            with self.board.lock:
                for k in [k for k in self.board.slots if k[0] == self.seq]:
                    del self.board.slots[k]
        self.seq += 1

    def all_reduce_sum(self, t):
        self._sync()
        self._post(("ar", self.rank), t.clone())
        self.board.barrier.wait()
        acc = self._get(("ar", 0)).clone()
        for r in range(1, self.size):
            acc += self._get(("ar", r))
        t.copy_(acc)
        self._end()

    def all_to_all(self, out, inp, out_splits, in_splits):
        self._sync()
        self._post(("a2a", self.rank), (inp, list(in_splits)))
        self.board.barrier.wait()
        o = 0
        for r in range(self.size):
            src, splits = self._get(("a2a", r))
            a = sum(splits[:self.rank])
            k = splits[self.rank]
            assert k == out_splits[r], "all-to-all split sizes disagree"
            if k:
                out[o:o + k].copy_(src[a:a + k])
            o += k
        self._end()

    def exchange(self, sends, recvs):
        self._sync()
        for p, t in sends:
            self._post(("p2p", self.rank, p), t)
        self.board.barrier.wait()
        for p, t in recvs:
            t.copy_(self._get(("p2p", p, self.rank)))
        self._end()


def run_threads(size: int, fn, timeout: float = 120.0):
    """fn(rank, comm) on `size` threads, each with its own CUDA stream; returns the results by
    rank, or raises the first exception (the others' barriers are broken so that they end)."""
    import torch

    board = _Board(size, timeout)
    out = [None] * size
    errs = []

    def body(rank):
        try:
            s = torch.cuda.Stream()
            with torch.cuda.stream(s):
                out[rank] = fn(rank, ThreadComm(board, rank))
                s.synchronize()
        except BaseException as e:  # noqa: BLE001 - reported to the caller below
            errs.append(e)
            board.barrier.abort()

    threads = [threading.Thread(target=body, args=(r,)) for r in range(size)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout + 30)
    if errs:
        raise errs[0]
    if any(t.is_alive() for t in threads):
        raise TimeoutError("a rank thread did not finish")
    return out
