"""ctypes binding of the engine's C-ABI (include/umpalumpa_fr.h, include/umpalumpa_fr_server.h).

The shared library is built in-tree (``umpalumpa_b200/lib/libfr_b200.so``).  There is no
fallback: if the library is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_float, c_int, c_int32, c_uint32, c_uint64, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libfr_b200.so")

FR_OK = 0
FR_E_INVALID = -1
FR_E_NOT_INIT = -2
FR_E_MISMATCH = -3
FR_E_NO_TABLE = -4
FR_E_CUDA = -5
FR_E_CAPACITY = -6
FR_E_UNSUPPORTED = -7

STATUS_NAMES = {
    FR_E_INVALID: "FR_E_INVALID", FR_E_NOT_INIT: "FR_E_NOT_INIT", FR_E_MISMATCH: "FR_E_MISMATCH",
    FR_E_NO_TABLE: "FR_E_NO_TABLE", FR_E_CUDA: "FR_E_CUDA", FR_E_CAPACITY: "FR_E_CAPACITY",
    FR_E_UNSUPPORTED: "FR_E_UNSUPPORTED",
}


class FrSettings(ctypes.Structure):
    _fields_ = [("interpolation", c_int32), ("blob_order", c_int32), ("type", c_int32),
                ("alpha", c_float), ("blob_radius", c_float), ("max_resolution", c_float),
                ("storage", c_int32), ("accumulation", c_int32), ("layout", c_int32)]


FR_LAYOUT_AUTO, FR_LAYOUT_ROWS, FR_LAYOUT_BANDED = 0, 1, 2


class FrDims(ctypes.Structure):
    _fields_ = [("fft_x", c_uint64), ("fft_y", c_uint64), ("n_projections", c_uint64),
                ("volume_x", c_uint64), ("volume_y", c_uint64), ("volume_z", c_uint64),
                ("n_spaces", c_uint64), ("table_elems", c_uint64)]


class FrConstants(ctypes.Structure):
    _fields_ = [("cMaxVolumeIndexX", c_int32), ("cMaxVolumeIndexYZ", c_int32),
                ("cBlobRadius", c_float), ("cOneOverBlobRadiusSqr", c_float),
                ("cBlobAlpha", c_float), ("cIw0", c_float), ("cIDeltaSqrt", c_float),
                ("cOneOverBessiOrderAlpha", c_float)]


class FrLaunchParams(ctypes.Structure):
    _fields_ = [("brick", c_int32), ("item_capacity", c_int32), ("ctas_per_sm", c_int32),
                ("groups", c_int32)]


class FrExecStats(ctypes.Structure):
    _fields_ = [("pairs", c_uint64), ("items", c_uint64), ("chunks", c_uint64), ("launches", c_uint64)]


class FrPhaseTimes(ctypes.Structure):
    _fields_ = [("binning_ms", ctypes.c_double), ("insert_ms", ctypes.c_double),
                ("insert_launches", c_uint64), ("insert_spaces", c_uint64)]


class FrJob(ctypes.Structure):
    _fields_ = [("fft", c_void_p), ("scales", c_void_p), ("n_projections", c_uint64), ("volume", c_void_p),
                ("weight", c_void_p), ("spaces", c_void_p), ("n_spaces", c_uint64), ("fft_x", c_uint64),
                ("fft_y", c_uint64), ("volume_x", c_uint64), ("volume_y", c_uint64), ("volume_z", c_uint64)]


class FrBatchLimits(ctypes.Structure):
    _fields_ = [("max_jobs", c_uint64), ("max_spaces", c_uint64), ("max_bricks", c_uint64),
                ("max_volume_side", c_uint64), ("table_elems", c_uint64)]


FR_BATCH_GRAPH = 1

FR_TUNING_OFF, FR_TUNING_CACHED, FR_TUNING_ON_EXECUTE = 0, 1, 2

FR_PREP_FFT_AUTO, FR_PREP_FFT_CUFFT, FR_PREP_FFT_FUSED = 0, 1, 2


class FrPrepSettings(ctypes.Structure):
    _fields_ = [("size_x", c_uint32), ("size_y", c_uint32), ("out_x", c_uint32), ("out_y", c_uint32),
                ("normalize", c_int32), ("center", c_int32), ("shift", c_int32), ("crop_freq", c_int32),
                ("max_freq", c_float), ("storage", c_int32), ("chunk", c_uint32), ("fft", c_uint32),
                ("out_layout", c_uint32)]


class FrTuneReport(ctypes.Structure):
    _fields_ = [("best", FrLaunchParams), ("best_ms", ctypes.c_double), ("default_ms", ctypes.c_double),
                ("trials", c_uint32), ("sample_spaces", c_uint32), ("key", ctypes.c_char * 256)]


class FrServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget", c_uint64), ("staging_bytes", c_uint64), ("max_jobs", c_uint32),
                ("max_step_projections", c_uint32), ("max_step_entries", c_uint32), ("max_volume_side", c_uint32),
                ("table_elems", c_uint32), ("pipeline_depth", c_uint32), ("reserve_bytes", c_uint64)]


class FrServerJobDesc(ctypes.Structure):
    _fields_ = [("fft_x", c_uint32), ("fft_y", c_uint32), ("volume_x", c_uint32), ("volume_y", c_uint32),
                ("volume_z", c_uint32), ("image_x", c_uint32), ("image_y", c_uint32), ("space_weight", c_float)]


class FrServerBatch(ctypes.Structure):
    _fields_ = [("fft", c_void_p), ("scales", c_void_p), ("rotations", c_void_p), ("spaces", c_void_p),
                ("n_projections", c_uint64), ("n_spaces", c_uint64)]


class FrServerJobInfo(ctypes.Structure):
    _fields_ = [("state", c_int32), ("pad", c_int32), ("batches_submitted", c_uint64),
                ("batches_done", c_uint64), ("spaces_done", c_uint64), ("volume", c_void_p), ("weight", c_void_p),
                ("t_open", ctypes.c_double), ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double)]


class FrServerStats(ctypes.Structure):
    _fields_ = [("steps", c_uint64), ("entries", c_uint64), ("spaces", c_uint64), ("jobs_done", c_uint64),
                ("bytes_admitted", c_uint64), ("peak_bytes_admitted", c_uint64), ("jobs_active", c_uint32),
                ("jobs_queued", c_uint32), ("peak_jobs_active", c_uint32), ("pad", c_uint32),
                ("busy_ms", ctypes.c_double), ("max_admit_ms", ctypes.c_double)]


class FrServerStepRecord(ctypes.Structure):
    _fields_ = [("t_formed", ctypes.c_double), ("t_enqueued", ctypes.c_double), ("t_launched", ctypes.c_double),
                ("t_retired", ctypes.c_double),
                ("gpu_ms", c_float), ("slices", c_uint32), ("spaces", c_uint64), ("jobs", c_uint32),
                ("gpu_span_ms", c_float)]


FR_JOB_QUEUED, FR_JOB_ACTIVE, FR_JOB_DONE, FR_JOB_FAILED = 0, 1, 2, 3

# name -> (restype, argtypes); every symbol the public headers declare
SIGNATURES = {
    "fr_settings_default": (None, [POINTER(FrSettings)]),
    "fr_last_error": (c_char_p, []),
    "fr_create": (c_int, [c_int, c_void_p, POINTER(c_void_p)]),
    "fr_destroy": (c_int, [c_void_p]),
    "fr_init": (c_int, [c_void_p, POINTER(FrDims), POINTER(FrSettings)]),
    "fr_execute": (c_int, [c_void_p, c_void_p, c_void_p, c_uint64, c_void_p, c_void_p, c_void_p,
                           c_uint64, c_void_p]),
    "fr_synchronize": (c_int, [c_void_p]),
    "fr_cleanup": (c_int, [c_void_p]),
    "fr_used_bytes": (c_uint64, [c_void_p]),
    "fr_make_constants": (c_int, [POINTER(FrDims), POINTER(FrSettings), POINTER(FrConstants)]),
    "fr_fill_blob_table": (c_int, [c_void_p, c_uint64, POINTER(FrSettings), c_void_p]),
    "fr_compute_traverse_spaces": (c_int, [c_void_p, c_uint64, c_uint32, c_uint32, c_uint32, c_uint32,
                                           c_int, c_float, c_float, c_int32, c_void_p, c_void_p]),
    "fr_quantize_projections": (c_int, [c_void_p, c_uint64, c_uint64, c_uint64, c_int, c_void_p, c_void_p,
                                        c_void_p]),
    "fr_band_plane_elems": (c_uint64, [c_uint64, c_uint64]),
    "fr_band_projections": (c_int, [c_void_p, c_uint64, c_uint64, c_uint64, c_int, c_void_p, c_void_p]),
    "fr_get_launch_params": (c_int, [c_void_p, POINTER(FrLaunchParams)]),
    "fr_set_launch_params": (c_int, [c_void_p, POINTER(FrLaunchParams)]),
    "fr_get_exec_stats": (c_int, [c_void_p, POINTER(FrExecStats)]),
    "fr_set_profiling": (c_int, [c_void_p, c_int]),
    "fr_get_phase_times": (c_int, [c_void_p, POINTER(FrPhaseTimes), c_int]),
    "fr_batch_init": (c_int, [c_void_p, POINTER(FrBatchLimits), POINTER(FrSettings)]),
    "fr_batch_execute": (c_int, [c_void_p, POINTER(FrJob), c_uint64, c_void_p, c_int]),
    "fr_insert_noalloc": (c_int, [c_int, c_void_p, POINTER(FrDims), POINTER(FrSettings), c_void_p, c_void_p,
                                  c_uint64, c_void_p, c_void_p, c_void_p, c_uint64, c_void_p]),
    "fr_compute_traverse_spaces_sym": (c_int, [c_void_p, c_uint64, c_void_p, c_uint32, c_uint32, c_uint32, c_uint32,
                                               c_uint32, c_int, c_float, c_float, c_int32, c_void_p, c_void_p]),
    "fr_prep_create": (c_int, [c_int, c_void_p, POINTER(FrPrepSettings), POINTER(c_void_p)]),
    "fr_prep_destroy": (c_int, [c_void_p]),
    "fr_prep_execute": (c_int, [c_void_p, c_void_p, c_uint64, c_void_p, c_void_p]),
    "fr_set_tuning": (c_int, [c_void_p, c_int, c_char_p]),
    "fr_autotune": (c_int, [c_void_p, c_void_p, c_void_p, c_uint64, c_void_p, c_uint64, c_void_p,
                            POINTER(FrTuneReport)]),
    "fr_batch_autotune": (c_int, [c_void_p, POINTER(FrJob), c_uint64, c_void_p, POINTER(FrTuneReport)]),
    "fr_tuning_key": (c_int, [c_void_p, c_char_p, c_uint64, c_char_p, c_uint64]),
    "fr_server_config_default": (None, [POINTER(FrServerConfig)]),
    "fr_server_create": (c_int, [c_int, POINTER(FrServerConfig), POINTER(FrSettings), POINTER(c_void_p)]),
    "fr_server_destroy": (c_int, [c_void_p]),
    "fr_server_clock": (ctypes.c_double, [c_void_p]),
    "fr_server_open_job": (c_int, [c_void_p, POINTER(FrServerJobDesc), POINTER(c_uint64)]),
    "fr_server_submit": (c_int, [c_void_p, c_uint64, POINTER(FrServerBatch)]),
    "fr_server_close_job": (c_int, [c_void_p, c_uint64]),
    "fr_server_wait_job": (c_int, [c_void_p, c_uint64, ctypes.c_double, POINTER(FrServerJobInfo)]),
    "fr_server_query_job": (c_int, [c_void_p, c_uint64, POINTER(FrServerJobInfo)]),
    "fr_server_read_job": (c_int, [c_void_p, c_uint64, c_void_p, c_void_p]),
    "fr_server_release_job": (c_int, [c_void_p, c_uint64]),
    "fr_server_get_stats": (c_int, [c_void_p, POINTER(FrServerStats)]),
    "fr_server_step_log": (c_int, [c_void_p, POINTER(FrServerStepRecord), c_uint64, POINTER(c_uint64)]),
}

_lib = None


class FRError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def lib():
    """Load the engine library (raises if it is missing: no CPU fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"engine library not built: {LIB_PATH} (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return lib().fr_last_error().decode(errors="replace")


def check(status: int):
    if status != FR_OK:
        raise FRError(status, last_error())
    return status
