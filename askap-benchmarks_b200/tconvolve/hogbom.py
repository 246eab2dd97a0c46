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
