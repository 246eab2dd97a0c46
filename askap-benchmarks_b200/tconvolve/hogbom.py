"""Hogbom CLEAN on the GPU (libtconvolve tcv_hogbom_*), mirroring the reference's class
HogbomGolden / HogbomCuda (current/tHogbomCleanOMP/HogbomGolden.h, attic/tHogbomCleanCuda/HogbomCuda.h):

    h = Hogbom()                       # Parameters.h: 1000 iterations, gain 0.1, threshold 1e-5
    h.deconvolve(dirty, dirtyWidth, psf, psfWidth, model, residual)

dirty, psf, model are numpy float32 arrays (host, as the reference's std::vector<float>); model is
accumulated into and residual receives the result.  deconvolve_device runs on torch tensors that
are already on the GPU, asynchronously on a stream.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, lib
from .raw import _ptr, _stream

NITERS, GAIN, THRESHOLD = 1000, 0.1, 1e-5  # current/tHogbomCleanOMP/Parameters.h


class Workspace:
    """Device workspace of one deconvolution (state word and per-block peak candidates)."""

    def __init__(self, width: int, device="cuda"):
        import torch

        self.bytes = int(lib().tcv_hogbom_workspace_bytes(int(width)))
        self.buf = torch.empty(self.bytes, dtype=torch.uint8, device=device)

    def result(self, stream=None) -> dict:
        done, stop = ctypes.c_int(), ctypes.c_int()
        skipped, ppos = ctypes.c_int64(), ctypes.c_int64()
        check(lib().tcv_hogbom_result(_ptr(self.buf), ctypes.byref(done), ctypes.byref(stop), ctypes.byref(skipped),
                                      ctypes.byref(ppos), _stream(stream)), "tcv_hogbom_result")
        return {"done": done.value, "stopped_at": stop.value, "skipped_rows": skipped.value,
                "psf_peak_pos": ppos.value}


def deconvolve_device(dirty, width: int, psf, psf_width: int, model, residual, niters: int = NITERS,
                      gain: float = GAIN, threshold: float = THRESHOLD, hist=None, work: Workspace | None = None,
                      stream=None) -> Workspace:
    """tcv_hogbom_deconvolve on float32 CUDA tensors (model accumulated into, residual written).
    hist: optional (values float32[niters], positions int32[niters]) CUDA tensors.  Returns the
    workspace, whose result() reads the iteration count after the stream finishes."""
    ws = work or Workspace(width, device=dirty.device)
    hv = _ptr(hist[0]) if hist is not None else None
    hp = _ptr(hist[1]) if hist is not None else None
    check(lib().tcv_hogbom_deconvolve(_ptr(dirty), int(width), _ptr(psf), int(psf_width), _ptr(model), _ptr(residual),
                                      int(niters), ctypes.c_float(gain), ctypes.c_float(threshold), hv, hp,
                                      _ptr(ws.buf), ws.bytes, _stream(stream)), "tcv_hogbom_deconvolve")
    return ws


def find_peak(image, work: Workspace | None = None, stream=None):
    """findPeak on a float32 CUDA tensor: (value, first index of the largest |value|)."""
    ws = work or Workspace(1, device=image.device)
    v, p = ctypes.c_float(), ctypes.c_int64()
    check(lib().tcv_find_peak(_ptr(image), int(image.numel()), ctypes.byref(v), ctypes.byref(p), _ptr(ws.buf),
                              ws.bytes, _stream(stream)), "tcv_find_peak")
    return float(v.value), int(p.value)


class Hogbom:
    """HogbomGolden's interface (HogbomGolden.h) on the GPU."""

    def __init__(self, niters: int = NITERS, gain: float = GAIN, threshold: float = THRESHOLD, device="cuda"):
        self.niters, self.gain, self.threshold, self.device = niters, gain, threshold, device
        self.last = None

    def deconvolve(self, dirty: np.ndarray, dirtyWidth: int, psf: np.ndarray, psfWidth: int, model: np.ndarray,
                   residual: np.ndarray | None = None) -> np.ndarray:
        """residual = dirty cleaned by niters iterations (fewer at the threshold); model += the
        components.  Returns the residual (also written into `residual` when given)."""
        import torch

        d = torch.from_numpy(np.ascontiguousarray(dirty, dtype=np.float32).ravel()).to(self.device)
        p = torch.from_numpy(np.ascontiguousarray(psf, dtype=np.float32).ravel()).to(self.device)
        m = torch.from_numpy(np.ascontiguousarray(model, dtype=np.float32).ravel()).to(self.device)
        r = torch.empty_like(d)
        ws = deconvolve_device(d, dirtyWidth, p, psfWidth, m, r, self.niters, self.gain, self.threshold)
        self.last = ws.result()
        out = r.cpu().numpy()
        model.reshape(-1)[:] = m.cpu().numpy()
        if residual is not None:
            residual.reshape(-1)[:] = out
        return out


def main(argv=None) -> int:
    """tHogbomCleanOMP's driver (current/tHogbomCleanOMP/tHogbomCleanOMP.cc:81-124) on the GPU:
    raw float32 dirty and PSF images (--dirty/--psf, the reference's .img format) or synthetic ones
    (--width), the reference's parameters unless overridden, and its report lines."""
    import argparse

    import torch

    from .workload import synthetic_dirty, synthetic_psf

    ap = argparse.ArgumentParser(prog="python -m tconvolve.hogbom")
    ap.add_argument("--dirty")
    ap.add_argument("--psf")
    ap.add_argument("--width", type=int, default=4096, help="synthetic images of this size when no files are given")
    ap.add_argument("--niters", type=int, default=NITERS)
    ap.add_argument("--gain", type=float, default=GAIN)
    ap.add_argument("--threshold", type=float, default=THRESHOLD)
    ap.add_argument("--repeat", type=int, default=1)
    a = ap.parse_args(argv)
    if a.dirty and a.psf:
        dirty, psf = np.fromfile(a.dirty, np.float32), np.fromfile(a.psf, np.float32)
    else:
        dirty, psf = synthetic_dirty(a.width, 20, 1e-3, seed=7).ravel(), synthetic_psf(a.width).ravel()
    dim, pdim = int(round(np.sqrt(dirty.size))), int(round(np.sqrt(psf.size)))
    if dim * dim != dirty.size or pdim * pdim != psf.size:
        print("Error: Image is not square")
        return 1
    print(f"Iterations = {a.niters}")
    print(f"Image dimensions = {dim}x{dim}")
    d, p = torch.from_numpy(dirty).cuda(), torch.from_numpy(psf).cuda()
    m, r = torch.zeros_like(d), torch.empty_like(d)
    ws = Workspace(dim)
    print("+++++ Forward processing (B200) +++++")
    for _ in range(a.repeat):
        m.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        deconvolve_device(d, dim, p, pdim, m, r, a.niters, a.gain, a.threshold, work=ws)
        e1.record()
        torch.cuda.synchronize()
        s = e0.elapsed_time(e1) * 1e-3
        done = ws.result()["done"]
        print(f"    Time {s} (s) ")
        print(f"    Time per cycle {s / max(done, 1) * 1000} (ms)")
        print(f"    Cleaning rate  {done / s} (iterations per second)")
    print("Done")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
