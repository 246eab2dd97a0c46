"""ctypes binding of libtconvolve.so (the C ABI declared in include/tconvolve.h).

The library is the only implementation: if it is missing or fails to load, every call raises.
There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD_DIR = os.path.join(PKG_ROOT, "_build")
CSRC_DIR = os.path.join(PKG_ROOT, "csrc")
LIB_PATH = os.path.join(BUILD_DIR, "libtconvolve.so")
PROBE_LIB_PATH = os.path.join(BUILD_DIR, "libtcvprobe.so")

TCV_OK = 0
STATUS_NAMES = {
    0: "TCV_OK", 1: "TCV_ERR_ARG", 2: "TCV_ERR_BOUNDS", 3: "TCV_ERR_OOM", 4: "TCV_ERR_CUDA",
    5: "TCV_ERR_TIMEOUT", 6: "TCV_ERR_STATE", 7: "TCV_ERR_WORKSPACE", 8: "TCV_ERR_UNSUPPORTED",
}

# table storage types (tcv_ctype)
C64, R32, CBF16, RBF16, CF16, RF16 = range(6)
CTYPE_NAMES = {C64: "c64", R32: "r32", CBF16: "cbf16", RBF16: "rbf16", CF16: "cf16", RF16: "rf16"}
CTYPE_BY_NAME = {v: k for k, v in CTYPE_NAMES.items()}
PADDED = 0x100          # TCV_C_PADDED: prepared (TMA) table layout
PAIRED = 0x200          # TCV_C_PAIRED: paired table layout (two columns per lane)
PATH_TMA, PATH_DIRECT, PATH_PAIRED = 0, 1, 2
DEGRID_TILES, DEGRID_ANCHOR = 0, 1
PASS_BIN, PASS_GRID, PASS_DEGRID = 1, 2, 4


class TcvError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(f"{what}: {STATUS_NAMES.get(status, status)}")


class TcvConfig(ctypes.Structure):
    _fields_ = [
        ("n_samples", ctypes.c_int64),
        ("w_size", ctypes.c_int32),
        ("n_chan", ctypes.c_int32),
        ("g_size", ctypes.c_int32),
        ("baseline", ctypes.c_int32),
        ("cell_size", ctypes.c_double),
        ("seed", ctypes.c_uint64),
        ("c_type", ctypes.c_int32),
        ("device", ctypes.c_int32),
    ]


class TcvDeviceBuffers(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p), ("outdata", ctypes.c_void_p), ("grid", ctypes.c_void_p),
        ("c64", ctypes.c_void_p), ("c_active", ctypes.c_void_p), ("iu", ctypes.c_void_p),
        ("iv", ctypes.c_void_p), ("coff", ctypes.c_void_p), ("u", ctypes.c_void_p),
        ("v", ctypes.c_void_p), ("w", ctypes.c_void_p), ("plan", ctypes.c_void_p),
        ("c_scale", ctypes.c_float), ("c_type", ctypes.c_int32),
    ]


class TcvJob(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("g_size", ctypes.c_int32), ("d_grid", ctypes.c_void_p)]


class TcvTuning(ctypes.Structure):
    _fields_ = [("tile_rows", ctypes.c_int32), ("group_mib", ctypes.c_int32), ("split", ctypes.c_int32),
                ("degrid_split", ctypes.c_int32), ("kernel", ctypes.c_int32)]

    def as_tuple(self):
        """(tile_rows, group_mib, split, degrid_split), with a fifth entry, kernel, when a pass uses
        the sample-parallel kernels (bit mask: 1 gridding, 2 degridding)."""
        t = (int(self.tile_rows), int(self.group_mib), int(self.split), int(self.degrid_split))
        return t + (int(self.kernel),) if self.kernel else t


class TcvServerConfig(ctypes.Structure):
    _fields_ = [
        ("g_size", ctypes.c_int32), ("w_size", ctypes.c_int32), ("cell_size", ctypes.c_double),
        ("baseline", ctypes.c_int32), ("c_type", ctypes.c_int32), ("streams", ctypes.c_int32),
        ("max_batch", ctypes.c_int32), ("batch_samples", ctypes.c_int64), ("hbm_budget", ctypes.c_size_t),
        ("tuning", TcvTuning), ("device", ctypes.c_int32), ("graphs", ctypes.c_int32),
    ]


class TcvRequest(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32), ("grid", ctypes.c_int32), ("n", ctypes.c_int64),
        ("u", ctypes.c_void_p), ("v", ctypes.c_void_p), ("w", ctypes.c_void_p),
        ("vis", ctypes.c_void_p), ("vis_out", ctypes.c_void_p),
    ]


class TcvRequestInfo(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32), ("batch_requests", ctypes.c_int32), ("rejected", ctypes.c_int64),
        ("t_submit", ctypes.c_double), ("t_start", ctypes.c_double), ("t_done", ctypes.c_double),
    ]


REQ_GRID, REQ_DEGRID = 0, 1


class TcvMajorConfig(ctypes.Structure):
    _fields_ = [
        ("n_samples", ctypes.c_int64), ("w_size", ctypes.c_int32), ("n_chan", ctypes.c_int32),
        ("cell_size", ctypes.c_double), ("g_size", ctypes.c_int32), ("baseline", ctypes.c_int32),
        ("n_major", ctypes.c_int32), ("n_minor", ctypes.c_int32), ("gain", ctypes.c_float),
        ("n_sources", ctypes.c_int32), ("device", ctypes.c_int32), ("keep_stages", ctypes.c_int32),
        ("tuning", TcvTuning),
    ]


MAJOR_STAGES = ("psf_grid", "psf_ifft", "grid", "ifft", "hogbom", "fft", "degrid", "subtract")
IMG_PSF, IMG_DIRTY, IMG_RESIDUAL, IMG_MODEL = 0, 1, 2, 3


class TcvCurGeometry(ctypes.Structure):
    _fields_ = [
        ("run_type", ctypes.c_int32), ("w_size", ctypes.c_int32), ("over_sample", ctypes.c_int32),
        ("support", ctypes.c_int32), ("g_size", ctypes.c_int32), ("n_baselines", ctypes.c_int32),
        ("n_samples", ctypes.c_int64), ("c_len", ctypes.c_int64), ("s_min", ctypes.c_int32),
        ("s_max", ctypes.c_int32), ("w_cell_size", ctypes.c_double), ("uv_cell_size", ctypes.c_double),
    ]

_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_D = ctypes.c_double
_F = ctypes.c_float
_S = ctypes.c_size_t
_PP = ctypes.POINTER(ctypes.c_void_p)

# name -> (restype, argtypes); every symbol declared in include/tconvolve.h
SIGNATURES = {
    "tcv_status_string": (ctypes.c_char_p, [_I]),
    "tcv_ctype_bytes": (_S, [_I]),
    "tcv_version": (ctypes.c_char_p, []),
    "tcv_c_geometry": (_I, [_D, _D, _I, _I, _P, _P, _P, _P]),
    "tcv_init_c_scratch_bytes": (_S, []),
    "tcv_init_c_raw": (_I, [_D, _D, _I, _I, _P, _P, _P, _P]),
    "tcv_convert_c": (_I, [_P, _I64, _I, _P, _P, _P, _P]),
    "tcv_table_bytes": (_S, [_I64, _I, _I]),
    "tcv_prepare_table": (_I, [_P, _I64, _I, _I, _P, _P, _P, _P]),
    "tcv_init_uvw_raw": (_I, [_I64, _I, ctypes.c_uint64, _P, _P, _P, _P]),
    "tcv_init_offsets_raw": (_I, [_P, _P, _P, _I64, _P, _I, _D, _D, _I, _I, _I, _I, _P, _P, _P, _P]),
    "tcv_plan_workspace_bytes": (_S, [_I64, _I, _I, _I64]),
    "tcv_plan_build": (_I, [_PP, _P, _P, _P, _I64, _I, _I, _I64, _P, _S, _P]),
    "tcv_plan_grid": (_I, [_P, _P, _P, _I, _F, _P, _P]),
    "tcv_plan_degrid": (_I, [_P, _P, _P, _I, _F, _P, _P]),
    "tcv_plan_rejected": (_I, [_P, _P, _P]),
    "tcv_plan_status": (_I, [_P, _P]),
    "tcv_plan_set_degrid_variant": (_I, [_P, _I]),
    "tcv_plan_info": (_I, [_P, _P, _P, _P, _P, _P]),
    "tcv_plan_destroy": (None, [_P]),
    "tcv_plan_workspace_bytes_tuned": (_S, [_I64, _I, _I, _I64, _P]),
    "tcv_plan_build_tuned": (_I, [_PP, _P, _P, _P, _I64, _I, _I, _I64, _P, _P, _S, _P]),
    "tcv_batch_workspace_bytes": (_S, [_P, _I, _I, _I64, _P]),
    "tcv_batch_plan_create": (_I, [_PP, _P, _I, _I, _I64, _P, _P, _S, _P]),
    "tcv_plan_bin": (_I, [_P, _P, _P, _P, _P]),
    "tcv_plan_tuning": (_I, [_P, _P]),
    "tcv_autotune": (_I, [_P, _I, _P, _P, _P, _P, _P, _I, _F, _I64, _I, _I, _P, _P, _P]),
    "tcv_autotune_report": (_I, [_P, _P, _I, _P]),
    "tcv_graph_capture": (_I, [_PP, _P, _I, _P, _P, _P, _P, _P, _I, _F, _P, _P]),
    "tcv_graph_launch": (_I, [_P, _P]),
    "tcv_graph_destroy": (None, [_P]),
    "tcv_server_config_default": (None, [_P]),
    "tcv_server_create": (_I, [_P, _PP]),
    "tcv_server_destroy": (None, [_P]),
    "tcv_server_grid_alloc": (_I, [_P, _P]),
    "tcv_server_grid_free": (_I, [_P, _I]),
    "tcv_server_grid_read": (_I, [_P, _I, _P]),
    "tcv_server_grid_write": (_I, [_P, _I, _P]),
    "tcv_server_submit": (_I, [_P, _P, _P]),
    "tcv_server_wait": (_I, [_P, ctypes.c_uint64, _D, _P]),
    "tcv_server_stats": (_I, [_P, _P, _P, _P, _P]),
    "tcv_cur_geometry_of": (_I, [_I, _P]),
    "tcv_cur_planes": (_I, [_I, _P, _P]),
    "tcv_cur_init_uvw_raw": (_I, [_I, ctypes.c_uint64, _P, _P, _P, _P, _P]),
    "tcv_cur_init_c_raw": (_I, [_I, _P, _P]),
    "tcv_cur_init_offsets_raw": (_I, [_I, _P, _P, _P, _I64, _P, _P, _P, _P, _P, _P, _P]),
    "tcv_cur_required_rate": (None, [_P]),
    "tcv_cur_create": (_I, [_I, _PP]),
    "tcv_cur_destroy": (None, [_P]),
    "tcv_cur_last_error": (ctypes.c_char_p, [_P]),
    "tcv_cur_set_sort": (_I, [_P, _I]),
    "tcv_cur_set_run_type": (_I, [_P, _I]),
    "tcv_cur_get_run_type": (_I, [_P]),
    "tcv_cur_set_ctype": (_I, [_P, _I]),
    "tcv_cur_set_tuning": (_I, [_P, _P]),
    "tcv_cur_tune": (_I, [_P, _I, _P, _P]),
    "tcv_hogbom_workspace_bytes": (_S, [_I]),
    "tcv_hogbom_deconvolve": (_I, [_P, _I, _P, _I, _P, _P, _I, _F, _F, _P, _P, _P, _S, _P]),
    "tcv_hogbom_result": (_I, [_P, _P, _P, _P, _P, _P]),
    "tcv_hogbom_set_strategy": (None, [_I]),
    "tcv_hogbom_set_wait": (_I, [ctypes.c_uint64, ctypes.c_uint32]),
    "tcv_find_peak": (_I, [_P, _I64, _P, _P, _P, _S, _P]),
    "tcv_fft_exec": (_I, [_P, _I, _I, _P]),
    "tcv_band_histogram": (_I, [_P, _I64, _I, _I, _P, _P]),
    "tcv_band_bounds": (_I, [_P, _I, _I, _I, _P]),
    "tcv_band_workspace_bytes": (_S, [_I64, _I]),
    "tcv_band_bucket": (_I, [_P, _P, _P, _P, _I64, _I, _I, _P, _I, _P, _P, _P, _P, _S, _P]),
    "tcv_band_unpack": (_I, [_P, _I64, _P, _P, _P, _P, _P]),
    "tcv_band_scatter": (_I, [_P, _P, _I64, _P, _P]),
    "tcv_rows_add": (_I, [_P, _P, _I64, _P]),
    "tcv_fft_fix": (_I, [_P, _I64, _F, _P]),
    "tcv_image_from_grid": (_I, [_P, _I, _F, _P, _P]),
    "tcv_grid_from_image": (_I, [_P, _I, _P, _P]),
    "tcv_major_config_default": (None, [_P]),
    "tcv_major_create": (_I, [_P, _P]),
    "tcv_major_destroy": (None, [_P]),
    "tcv_major_last_error": (ctypes.c_char_p, [_P]),
    "tcv_major_get_stream": (_P, [_P]),
    "tcv_major_init": (_I, [_P]),
    "tcv_major_run_cycle": (_I, [_P]),
    "tcv_major_sync": (_I, [_P]),
    "tcv_major_stage_ms": (_I, [_P, _P, _P]),
    "tcv_major_info": (_I, [_P, _P, _P, _P, _P]),
    "tcv_major_get_image": (_I, [_P, _I, _P]),
    "tcv_major_get_grid": (_I, [_P, _I, _P]),
    "tcv_major_get_vis": (_I, [_P, _I, _P]),
    "tcv_major_get_offsets": (_I, [_P, _P, _P, _P]),
    "tcv_cur_init": (_I, [_P]),
    "tcv_cur_run_grid": (_I, [_P]),
    "tcv_cur_run_degrid": (_I, [_P]),
    "tcv_cur_sync": (_I, [_P]),
    "tcv_cur_get_stream": (_P, [_P]),
    "tcv_cur_support": (_I, [_P]),
    "tcv_cur_n_visibilities": (_I64, [_P]),
    "tcv_cur_n_pixels": (_I64, [_P]),
    "tcv_cur_generator_state": (ctypes.c_uint64, [_P]),
    "tcv_cur_info": (_I, [_P, _P]),
    "tcv_cur_set_data": (_I, [_P, _P, _I64]),
    "tcv_cur_zero_grid": (_I, [_P]),
    "tcv_cur_get_grid": (_I, [_P, _P]),
    "tcv_cur_get_outdata": (_I, [_P, _P, _I64]),
    "tcv_cur_get_c": (_I, [_P, _P, _I64]),
    "tcv_cur_get_uvw": (_I, [_P, _P, _P, _P]),
    "tcv_cur_get_offsets": (_I, [_P, _P, _P, _P, _P]),
    "tcv_cur_get_planes": (_I, [_P, _P, _P]),
    "tcv_plan_workspace_bytes_var": (_S, [_I64, _P, _P, _I, _I, _I64, _P]),
    "tcv_plan_build_var": (_I, [_PP, _P, _P, _P, _P, _I64, _P, _P, _I, _I, _I64, _P, _P, _S, _P]),
    "tcv_jit_prepare": (_I, [_I, _I]),
    "tcv_jit_enable": (None, [_I]),
    "tcv_jit_info": (ctypes.c_char_p, []),
    "tcv_grid_raw": (_I, [_P, _I64, _I, _P, _I, _F, _I64, _P, _P, _P, _P, _I, _P, _S, _P]),
    "tcv_degrid_raw": (_I, [_P, _I, _I, _P, _I, _F, _I64, _P, _P, _P, _P, _I64, _P, _S, _P]),
    "tcv_static_scratch_bytes": (_S, []),
    "tcv_grid_raw_static": (_I, [_P, _I64, _I, _P, _I, _F, _I64, _P, _P, _P, _P, _I, _P]),
    "tcv_grid_host_raw": (_I, [_P, _I64, _I, _P, _I64, _P, _P, _P, _P, _I, _I, _P]),
    "tcv_degrid_host_raw": (_I, [_P, _I, _I, _P, _I64, _P, _P, _P, _P, _I64, _I, _P]),
    "tcv_init_c_host": (_I, [_D, _D, _I, _I, _P, _I64, _I, _P, _P, _P, _P]),
    "tcv_config_default": (None, [_P]),
    "tcv_create": (_I, [_P, _PP]),
    "tcv_destroy": (None, [_P]),
    "tcv_last_error": (ctypes.c_char_p, [_P]),
    "tcv_set_stream": (_I, [_P, _P]),
    "tcv_get_stream": (_P, [_P]),
    "tcv_sync": (_I, [_P]),
    "tcv_init": (_I, [_P]),
    "tcv_run_grid": (_I, [_P]),
    "tcv_run_degrid": (_I, [_P]),
    "tcv_support": (_I, [_P]),
    "tcv_over_sample": (_I, [_P]),
    "tcv_w_cell_size": (_D, [_P]),
    "tcv_sum_c": (_F, [_P]),
    "tcv_c_len": (_I64, [_P]),
    "tcv_n_data": (_I64, [_P]),
    "tcv_updates_per_pass": (_D, [_P]),
    "tcv_set_ctype": (_I, [_P, _I]),
    "tcv_set_path": (_I, [_P, _I]),
    "tcv_get_path": (_I, [_P]),
    "tcv_set_tuning": (_I, [_P, _P]),
    "tcv_get_tuning": (_I, [_P, _P]),
    "tcv_tune": (_I, [_P, _I, _P, _P]),
    "tcv_set_data": (_I, [_P, _P, _I64]),
    "tcv_get_data": (_I, [_P, _P, _I64]),
    "tcv_get_outdata": (_I, [_P, _P, _I64]),
    "tcv_set_grid": (_I, [_P, _P]),
    "tcv_get_grid": (_I, [_P, _P]),
    "tcv_zero_grid": (_I, [_P]),
    "tcv_get_c": (_I, [_P, _P, _I64]),
    "tcv_get_offsets": (_I, [_P, _P, _P, _P]),
    "tcv_get_uvw": (_I, [_P, _P, _P, _P]),
    "tcv_set_uvw": (_I, [_P, _P, _P, _P]),
    "tcv_get_device_buffers": (_I, [_P, _P]),
}

_lib = None


def build(quiet: bool = True) -> str:
    """Compile the CUDA library and host programs for sm_100a (make in csrc/)."""
    cmd = ["make", "-C", CSRC_DIR, f"-j{min(8, os.cpu_count() or 1)}"]
    if quiet:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    """The loaded library.  Raises if it has not been built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libtconvolve.so not built ({LIB_PATH}); run build() first")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


# the L2 table-stream probe (include/tcv_probe.h): a measurement tool in a library of its own
PROBE_SIGNATURES = {
    "tcv_probe_table_threads": (_I64, []),
    "tcv_probe_table_stream": (_I, [_P, _I64, _I, _I, _P, _P, _P]),
}
_probe = None


def probe_lib() -> ctypes.CDLL:
    """libtcvprobe.so, loaded with its signatures (built beside libtconvolve.so)."""
    global _probe
    if _probe is None:
        if not os.path.exists(PROBE_LIB_PATH):
            raise RuntimeError(f"libtcvprobe.so not built ({PROBE_LIB_PATH}); run build() first")
        P = ctypes.CDLL(PROBE_LIB_PATH)
        for name, (res, args) in PROBE_SIGNATURES.items():
            fn = getattr(P, name)
            fn.restype = res
            fn.argtypes = args
        _probe = P
    return _probe


def check(status: int, what: str, ctx=None) -> None:
    if status != TCV_OK:
        extra = ""
        if ctx:
            msg = lib().tcv_last_error(ctx)
            extra = f" ({msg.decode()})" if msg else ""
        raise TcvError(status, what + extra)


def autotune_report(cap: int = 64):
    """Candidates and median ms of the last tuning run (tcv_autotune or tcv_cur_tune):
    [((tile_rows, group_mib, split, degrid_split), ms), ...]."""
    cands = (TcvTuning * cap)()
    times = (ctypes.c_float * cap)()
    n = ctypes.c_int()
    check(lib().tcv_autotune_report(cands, times, cap, ctypes.byref(n)), "tcv_autotune_report")
    return [(cands[i].as_tuple(), float(times[i])) for i in range(min(n.value, cap))]
